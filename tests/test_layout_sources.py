"""Host-side audit sources of the probe layout: boundary-edge points
(_boundary_edge_candidates, surface_probes.py:658-779) lie on the edges used
by a single triangle, evenly spaced, with barycentrics that rebuild them; a
closed mesh has none; render vertices (_instance_vertex_anchors,
surface_probes.py:375-442) are the transformed vertices with normalised
transformed normals, each on an incident triangle."""

import numpy as np


def _instance_triangles(node, i):
    mesh_id, _, transform_id = node.instances[i]
    mesh = node.meshes[mesh_id]
    m = node.transforms[transform_id].astype(np.float64)
    p = mesh.vertices[:, :3].astype(np.float64) @ m[:3, :3].T + m[:3, 3]
    return mesh, p[mesh.indices.astype(np.int64).reshape(-1, 3)].astype(np.float32)


def test_boundary_points_of_an_open_quad():
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import _boundary_edges

    node = scenes.reference_demo()
    mesh, t = _instance_triangles(node, 0)  # the 2 x 2 floor quad
    pos, nrm, tri, b1, b2 = _boundary_edges(t, mesh.indices, 0.3)
    assert pos.shape[0] == 4 * 7  # ceil(2 / 0.3) segments on each of the 4 outer edges
    on_border = np.isclose(np.abs(pos[:, 0]), 1.0) | np.isclose(np.abs(pos[:, 2]), 1.0)
    assert on_border.all()
    np.testing.assert_allclose(nrm, np.tile([0, 1, 0], (pos.shape[0], 1)), atol=1e-6)
    rebuilt = t[tri, 0] * (1 - b1 - b2)[:, None] + t[tri, 1] * b1[:, None] + t[tri, 2] * b2[:, None]
    np.testing.assert_allclose(rebuilt, pos, atol=1e-5)


def test_closed_mesh_has_no_boundary():
    """Edges are keyed by vertex index, as in the reference: a tetrahedron
    with shared vertices is closed; a box with per-face vertices is not."""
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import _boundary_edges

    v = np.float32([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    idx = np.uint32([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]])
    assert _boundary_edges(v[idx.astype(np.int64)], idx, 0.1)[0].shape[0] == 0
    node = scenes.reference_demo()
    mesh, t = _instance_triangles(node, 6)  # the tall box
    # each face's 4 outer edges (its diagonal is shared by its two triangles)
    assert _boundary_edges(t, mesh.indices, 10.0)[0].shape[0] == 4 * 6


def test_render_vertices_follow_the_transform():
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import _render_vertices

    node = scenes.reference_demo()
    mesh_id, _, transform_id = node.instances[6]
    mesh = node.meshes[mesh_id]
    pos, nrm, tri, b1, b2 = _render_vertices(mesh, node.transforms[transform_id], 10 ** 6, np.random.default_rng(0))
    assert pos.shape[0] == np.unique(mesh.indices).shape[0]
    np.testing.assert_allclose(np.linalg.norm(nrm, axis=1), 1.0, atol=1e-6)
    _, t = _instance_triangles(node, 6)
    rebuilt = t[tri, 0] * (1 - b1 - b2)[:, None] + t[tri, 1] * b1[:, None] + t[tri, 2] * b2[:, None]
    np.testing.assert_allclose(rebuilt, pos, atol=1e-5)


def test_group_surface_sampling():
    """Instances of one mesh sampled together: exact per-instance counts,
    points on their own triangles, triangles drawn in proportion to area x
    density."""
    from nan_b200.surface_probe_layout import _surface_points_group

    base = np.float32([[[0, 0, 0], [1, 0, 0], [0, 0, 1]], [[1, 0, 0], [3, 0, 0], [1, 0, 2]]])  # areas 0.5, 2
    t = np.stack([base, base * 2.0, base + np.float32([5, 1, 0])])
    areas = 0.5 * np.linalg.norm(np.cross(t[:, :, 1] - t[:, :, 0], t[:, :, 2] - t[:, :, 0]), axis=2)
    dens = np.array([[1.0, 1.0], [1.0, 1.0], [4.0, 1.0]])
    counts = [20000, 5, 20000]
    out = _surface_points_group(t, areas, counts, np.random.default_rng(3), dens)
    for j, (pos, nrm, tri, b1, b2) in enumerate(out):
        assert pos.shape[0] == counts[j]
        rebuilt = (t[j, tri, 0] * (1 - b1 - b2)[:, None] + t[j, tri, 1] * b1[:, None] + t[j, tri, 2] * b2[:, None])
        np.testing.assert_allclose(rebuilt, pos, atol=1e-5)
        np.testing.assert_allclose(np.abs(nrm[:, 1]), 1.0)
    assert abs((out[0][2] == 0).mean() - 0.2) < 0.02  # 0.5 / 2.5
    assert abs((out[2][2] == 0).mean() - 0.5) < 0.02  # 4 x 0.5 / (2 + 2)


def test_group_audit_sources_equal_per_instance_helpers():
    """With caps above every count (nothing drawn at random) the grouped
    sources equal the per-instance helpers, instance by instance."""
    from nan_b200.scene_node import Mesh
    from nan_b200.scenes import make_transform
    from nan_b200.surface_probe_layout import (_audit_sources_group, _boundary_edge_list, _boundary_edges,
                                               _centroids, _inset_corners, _render_vertices, _vertex_list)

    mesh = Mesh.cube((1.0, 2.0, 0.5))
    mats = np.stack([make_transform((1.0, 0.0, 2.0), (0.0, 0.3, 0.0), (1.0, 1.0, 1.0)),
                     make_transform((-3.0, 1.0, 0.0), (0.2, 0.0, 0.1), (0.5, 2.0, 1.5)),
                     make_transform((0.0, 0.0, 0.0))]).astype(np.float64)
    p = np.einsum("vk,gjk->gvj", mesh.vertices[:, :3].astype(np.float64), mats[:, :3, :3]) + mats[:, None, :3, 3]
    t = p[:, mesh.indices.astype(np.int64)].astype(np.float32)
    kernels = np.float32([0.3, 0.7, 0.2])
    caps = np.full(3, 10 ** 6)
    parts = _audit_sources_group(t, mesh, mats, kernels, caps, _boundary_edge_list(mesh.indices), _vertex_list(mesh),
                                 np.random.default_rng(0))
    for j in range(3):
        expect = [_boundary_edges(t[j], mesh.indices, float(kernels[j]) * 0.5),
                  _inset_corners(t[j], float(kernels[j]) * 0.05, 10 ** 6, None),
                  _centroids(t[j], 10 ** 6, None),
                  _render_vertices(mesh, mats[j], 10 ** 6, None)]
        for got, ref in zip(parts[j], expect):
            for a, b in zip(got, ref):
                np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-6)
