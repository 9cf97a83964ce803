"""Surface-probe PRT L2: the host math the reference's tests pin
(test_surface_probe_prt.py: basis orthonormality under sphere sampling, a
constant environment gives pi * color, static source kept and negative
ringing clamped), and the baker and evaluator on the oracle: on an
unoccluded plane the Y00 transport is pi * Y00 for every sample, the
lighting projection of a constant sky is sky * sqrt(4 pi) in coefficient 0,
and the evaluated field is pi * sky."""

import math

import numpy as np
import pytest


def test_basis_is_orthonormal_under_sphere_sampling():
    from nan_b200.surface_probe_prt import surface_probe_sh_l2_basis

    n = 20000
    i = np.arange(n, dtype=np.float64)
    y = 1.0 - 2.0 * (i + 0.5) / n
    phi = 2.0 * math.pi * np.mod(i * 0.6180339887498949, 1.0)
    r = np.sqrt(np.maximum(1.0 - y * y, 0.0))
    dirs = np.stack((r * np.cos(phi), y, r * np.sin(phi)), axis=1)
    basis = np.stack([surface_probe_sh_l2_basis(d) for d in dirs])
    gram = (4.0 * math.pi / n) * basis.T @ basis
    np.testing.assert_allclose(gram, np.eye(9), atol=2.0e-3)


def test_constant_environment_gives_pi_times_color():
    from nan_b200.surface_probe_prt import constant_environment_sh, evaluate_prt_l2_rgb

    color = np.array([1.25, 0.5, 2.0])
    transport = np.zeros((9, 3))
    transport[0] = math.pi * 0.2820947918  # integral of max(n.w, 0) Y00 over the sphere
    np.testing.assert_allclose(evaluate_prt_l2_rgb(transport, constant_environment_sh(color)), math.pi * color,
                               rtol=2.0e-9)


def test_static_source_kept_and_negative_ringing_clamped():
    from nan_b200.surface_probe_prt import evaluate_prt_l2_rgb

    transport = np.zeros((9, 3))
    lighting = np.zeros((9, 3))
    transport[0] = (1.0, -2.0, 0.5)
    lighting[0] = (2.0, 2.0, 2.0)
    np.testing.assert_allclose(evaluate_prt_l2_rgb(transport, lighting, static_source=(0.25, 0.5, 0.75)),
                               (2.25, 0.0, 1.75))
    with pytest.raises(ValueError):
        evaluate_prt_l2_rgb(np.zeros((4, 3)), lighting)


def _plane():
    from nan_b200.scene_node import Material, Mesh, SceneNode

    v = np.zeros((4, 8), np.float32)
    v[:, :3] = [(-5, 0, -5), (5, 0, -5), (5, 0, 5), (-5, 0, 5)]
    v[:, 4] = 1.0
    node = SceneNode(name="plane")
    mesh = node.add_mesh(Mesh(v, np.array([[0, 2, 1], [0, 3, 2]], np.uint32)))
    node.add_instance(mesh, node.add_material(Material()), node.add_transform(np.eye(4, dtype=np.float32)))
    return node


def test_oracle_unoccluded_plane_transport_and_evaluation():
    from nan_b200 import scenes
    from nan_b200.scene import Lighting
    from oracle.oracle import OracleScene, prt_evaluate, prt_project_lighting

    node = _plane()
    orc = OracleScene(**node.pack())
    probes, pinst = scenes.surface_sites(node, 64, seed=2, radius=0.25)
    n = probes.shape[0]
    sky = np.array([0.5, 1.0, 2.0])
    light = Lighting(sun_intensity=0.0, sky_radiance=tuple(sky), sun_disk=False)
    values = np.zeros((n, 27), np.float32)
    counts = np.zeros(n, np.uint32)
    self_hits = np.zeros(n, np.uint32)
    radial = np.zeros((n, 16), np.uint32)
    static = np.zeros((n, 3), np.float32)
    for it in range(3):
        orc.trace_probes_prt(light, values, counts, self_hits, radial, static, probes, pinst,
                             np.arange(n, dtype=np.uint32), it, 8, 3, it == 0)
    np.testing.assert_array_equal(counts, 3)
    np.testing.assert_array_equal(self_hits, 0)
    np.testing.assert_array_equal(static, 0.0)
    t = values.reshape(n, 9, 3)
    np.testing.assert_allclose(t[:, 0, :], math.pi * 0.2820947918, rtol=1e-6)
    sh = prt_project_lighting(light, 2048)
    np.testing.assert_allclose(sh[0, :3], sky * math.sqrt(4.0 * math.pi), rtol=5e-5)  # float sum of 2048 terms
    assert np.abs(sh[1:, :3]).max() < 1e-3 * sky.max()
    np.testing.assert_array_equal(sh[:, 3], 0.0)
    out, out_counts = prt_evaluate(values, counts, static, sh)
    np.testing.assert_array_equal(out_counts, counts)
    np.testing.assert_allclose(out, np.broadcast_to(math.pi * sky, out.shape), rtol=2e-3)
    # probes without samples evaluate to the static source alone, clamped at 0
    static2 = np.full((n, 3), -1.0, np.float32)
    static2[0] = (0.25, 0.5, 0.75)
    out0, _ = prt_evaluate(values, np.zeros(n, np.uint32), static2, sh)
    np.testing.assert_array_equal(out0[0], np.float32([0.25, 0.5, 0.75]))
    np.testing.assert_array_equal(out0[1:], 0.0)
