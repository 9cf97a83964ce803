"""The CPU oracle against the reference's own golden vectors and known answers.

Fixtures come from tests/golden/make_golden.py, which evaluates the
reference's Python reference functions (RGB9E5 pack/unpack of
test_mesh_colors_rgb9e5.py:15-50, hemi-oct of surface_probes.py:45-110,
lattice addressing of mesh_colors.py:32-61, FP64 brute-force any-hit of
vertex_baker/visibility_baker.py:348-402).
"""

import numpy as np


def test_rgb9e5_pack_matches_reference_bit_exact(golden, oracle_mod):
    packed = oracle_mod.pack_rgb9e5(golden["rgb9e5_values"])
    np.testing.assert_array_equal(packed, golden["rgb9e5_packed"])
    # the seven values of test_mesh_colors_rgb9e5.py:62-72 come first
    np.testing.assert_array_equal(packed[:7], golden["rgb9e5_packed"][:7])


def test_rgb9e5_unpack_matches_reference_bit_exact(golden, oracle_mod):
    np.testing.assert_array_equal(oracle_mod.unpack_rgb9e5(golden["rgb9e5_packed"]), golden["rgb9e5_decoded"])


def test_rgb9e5_quantization_within_half_step(oracle_mod):
    # test_mesh_colors_rgb9e5.py:130-146
    values = np.asarray([[0.1, 0.2, 0.3], [1.0, 2.0, 3.0], [10.0, 100.0, 1000.0], [0.001, 0.5, 12.0]], np.float32)
    packed = oracle_mod.pack_rgb9e5(values)
    decoded = oracle_mod.unpack_rgb9e5(packed)
    step = np.exp2((packed >> 27).astype(np.float64) - 24.0)
    assert np.all(np.abs(decoded - values) < step[:, None] * 0.501)


def test_hemi_oct_matches_reference(golden, oracle_mod):
    uv = oracle_mod.hemi_oct_encode(golden["hemi_dirs"])
    np.testing.assert_allclose(uv, golden["hemi_uv"], atol=1e-6)
    # canonical directions of test_surface_probes.py:95-116
    np.testing.assert_allclose(uv[:5], [[0.5, 0.5], [1, 1], [0, 0], [1, 0], [0, 1]], atol=1e-6)
    np.testing.assert_allclose(oracle_mod.hemi_oct_decode(golden["hemi_uv"]), golden["hemi_decoded"], atol=2e-6)
    np.testing.assert_allclose(oracle_mod.hemi_oct_decode(uv), golden["hemi_dirs"], atol=2e-6)


def test_lattice_address_to_ij_matches_reference(golden, oracle_mod):
    ij = oracle_mod.address_to_ij(golden["mc_address"], golden["mc_resolution"])
    np.testing.assert_array_equal(ij, golden["mc_ij"])


def test_rng_is_the_reference_lcg(oracle_mod):
    # common.slang:164-210, restated with Python integers
    x, y, s = 17, 23, 5
    state = ((x * 100591) ^ (y * 102191) ^ (s * 103643)) & 0xFFFFFFFF
    expect = []
    for _ in range(64):
        state = (1664525 * state + 1013904223) & 0xFFFFFFFF
        expect.append(np.float32((state >> 8) * 2.0**-24))
    np.testing.assert_array_equal(oracle_mod.rng_sequence(x, y, s, 64), np.asarray(expect, np.float32))


def test_own_sincos_is_within_two_ulp(oracle_mod):
    a = np.linspace(0.0, 2.0 * np.pi, 400001, dtype=np.float32)
    s, c = oracle_mod.sincos(a)
    ref_s, ref_c = np.sin(a.astype(np.float64)), np.cos(a.astype(np.float64))
    assert np.max(np.abs(s - ref_s)) < 1.2e-7
    assert np.max(np.abs(c - ref_c)) < 1.2e-7


def test_f16_conversion_rounds_to_nearest_even(oracle_mod):
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.normal(size=20000).astype(np.float32) * 100,
                        np.float32([0.0, -0.0, 65504, 65519, 65520, 1e-8, 2.9802322e-08, 5.9604645e-08,
                                    6.1035156e-05, 4.0, 2.0, np.inf])])
    np.testing.assert_array_equal(oracle_mod.f32_to_f16(x), x.astype(np.float16).view(np.uint16))


def test_any_hit_agrees_with_reference_bruteforce(golden, oracle_mod):
    """Watertight FP32/FP64 any-hit vs the reference's FP64 Moller-Trumbore."""
    tris = golden["vis_triangles"]
    verts = np.zeros((tris.shape[0] * 3, 8), np.float32)
    verts[:, 0:3] = tris.reshape(-1, 3)
    idx = np.arange(tris.shape[0] * 3, dtype=np.uint32).reshape(-1, 3)
    eye = np.eye(4, dtype=np.float32).reshape(1, 16)
    scene = oracle_mod.OracleScene(verts, idx, np.array([[verts.shape[0], idx.size, 0, 0]], np.uint32),
                                   np.array([[0, 0, 0, 0]], np.uint32), eye, eye, np.zeros((1, 8), np.float32))
    o, d = golden["vis_origins"], golden["vis_directions"]
    rays = np.zeros((o.shape[0], 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 1e-6
    rays[:, 4:7] = d
    rays[:, 7] = golden["vis_max_distance"][0]
    expect = golden["vis_occluded"].astype(bool)
    for mode in (0, 1, 2):
        vis, _ = scene.visibility(rays, mode=mode)
        agree = np.mean((vis == 0.0) == expect)
        assert agree >= 0.999, (mode, agree)
