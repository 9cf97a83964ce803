"""nan_scene_build_noalloc: the BVH build for callers that cannot allocate.

Some callers may not call cudaMalloc at all -- code living inside another
framework's memory pool, or a real-time loop with an allocation ban. This
entry point builds an LBVH (binary nodes, whatever the context's tuning asks)
from a fixed scratch array in device memory and writes it into buffers the
caller already owns. Its tree differs from nan_scene_build's default
binned-SAH tree, but the hits do not: the closest hit is chosen by (t, flat index) in
any tree. The test calls it through the C ABI twice in a row on one context
(a larger scene first, then a smaller one, so the second call starts from the
first call's leftover scratch) and checks each result against
nan_scene_build's with the same exact comparisons the parity tests use; then
it checks the error paths, which return before the build touches the
caller's buffers. This file is collected last.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_scene(device, scene, ctx):
    import torch

    from nan_b200 import _native

    n = int(scene.info()["triangle_count"])
    nodes = torch.empty((max(n - 1, 1) * 16,), dtype=torch.float32, device=device.torch_device)
    tris = torch.empty((n * 12,), dtype=torch.float32, device=device.torch_device)
    refs = torch.empty((n * 2,), dtype=torch.int32, device=device.torch_device)
    torch.cuda.synchronize()
    rc = _native.lib().nan_scene_build_noalloc(
        ctx.handle, ctypes.byref(scene._desc), nodes.data_ptr(), nodes.numel() * 4, tris.data_ptr(),
        tris.numel() * 4, refs.data_ptr(), refs.numel() * 4, _native.stream_handle(None))
    _native.check(rc)
    return nodes, tris, refs


def _compare(device, scene, ctx, seed):
    import torch

    from nan_b200 import _native

    n = int(scene.info()["triangle_count"])
    # world triangles
    a = scene.world_triangles()
    b = torch.empty_like(a)
    _native.check(_native.lib().nan_scene_world_triangles(ctx.handle, b.data_ptr(), _native.stream_handle(None)))
    torch.testing.assert_close(b, a, rtol=0, atol=0)
    # closest and any hits on seeded rays
    tri = a.cpu().numpy().reshape(n, 3, 3)
    lo, hi = tri.reshape(-1, 3).min(0), tri.reshape(-1, 3).max(0)
    rng = np.random.default_rng(seed)
    rays = np.zeros((8192, 8), np.float32)
    rays[:, 0:3] = rng.uniform(lo, hi, size=(8192, 3))
    d = rng.normal(size=(8192, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 7] = 1e30
    rt = torch.from_numpy(rays).to(device.torch_device)
    ids_a, tb_a = scene.intersect(rt)
    ids_b = torch.empty_like(ids_a)
    tb_b = torch.empty_like(tb_a)
    _native.check(_native.lib().nan_intersect(ctx.handle, rt.data_ptr(), 8192, ids_b.data_ptr(), tb_b.data_ptr(),
                                              _native.stream_handle(None)))
    torch.testing.assert_close(ids_b, ids_a, rtol=0, atol=0)
    torch.testing.assert_close(tb_b, tb_a, rtol=0, atol=0)
    vis_a = scene.occluded(rt)
    vis_b = torch.empty_like(vis_a)
    _native.check(_native.lib().nan_occluded(ctx.handle, rt.data_ptr(), 8192, vis_b.data_ptr(),
                                             _native.stream_handle(None)))
    torch.testing.assert_close(vis_b, vis_a, rtol=0, atol=0)
    ctx.check()
    assert (ids_a[:, 0] == 1).float().mean().item() > 0.2


def test_noalloc_build_matches_allocating_build_twice(device):
    import nan_b200
    from nan_b200 import scenes

    large = nan_b200.Scene(device, scenes.terrain_boxes(seed=4, grid=161, boxes=200))
    small = nan_b200.Scene(device, scenes.cornell_box(32, 32))
    ctx = device.new_context()
    keep = []
    for k, scene in enumerate((large, small)):
        keep.append(_noalloc_scene(device, scene, ctx))
        _compare(device, scene, ctx, seed=100 + k)
    ctx.close()


def _call(ctx, scene, nodes, nodes_bytes, tris, tris_bytes, refs, refs_bytes):
    from nan_b200 import _native

    return _native.lib().nan_scene_build_noalloc(ctx.handle, ctypes.byref(scene._desc), nodes, nodes_bytes, tris,
                                                 tris_bytes, refs, refs_bytes, _native.stream_handle(None))


def _last_error():
    from nan_b200 import _native

    return _native.lib().nan_last_error().decode()


def test_noalloc_build_error_paths(device):
    import torch

    import nan_b200
    from nan_b200 import _native, scenes

    scene = nan_b200.Scene(device, scenes.cornell_box(32, 32))
    n = int(scene.info()["triangle_count"])
    buf = torch.empty((max(n - 1, 1) * 16 + n * 12 + n * 2 + 64,), dtype=torch.float32, device=device.torch_device)
    base = buf.data_ptr()
    nodes, tris, refs = base, base + max(n - 1, 1) * 64, base + max(n - 1, 1) * 64 + n * 48
    nb, tb, rb = max(n - 1, 1) * 64, n * 48, n * 8
    ctx = device.new_context()
    # output buffers too small
    assert _call(ctx, scene, nodes, nb - 64, tris, tb, refs, rb) == _native.NAN_ERR_INVALID_ARGUMENT
    assert "too small" in _last_error()
    assert _call(ctx, scene, nodes, nb, tris, tb, refs, rb - 8) == _native.NAN_ERR_INVALID_ARGUMENT
    # misaligned outputs
    assert _call(ctx, scene, nodes + 4, nb, tris, tb, refs, rb) == _native.NAN_ERR_INVALID_ARGUMENT
    assert "aligned" in _last_error()
    assert _call(ctx, scene, nodes, nb, tris, tb, refs + 4, rb) == _native.NAN_ERR_INVALID_ARGUMENT
    # nothing was built by the failed calls
    info = _native.NanSceneInfo()
    assert _native.lib().nan_scene_info(ctx.handle, ctypes.byref(info)) == _native.NAN_ERR_NO_SCENE
    # the same buffers, right-sized and aligned, build
    _native.check(_call(ctx, scene, nodes, nb, tris, tb, refs, rb))
    _native.check(_native.lib().nan_scene_info(ctx.handle, ctypes.byref(info)))
    assert info.triangle_count == n
    ctx.close()
    # a context that holds a BVH allocated by nan_scene_build is refused
    assert _call(scene.context, scene, nodes, nb, tris, tb, refs, rb) == _native.NAN_ERR_INVALID_ARGUMENT
    assert "nan_scene_build" in _last_error()
    # a scene beyond the 64 MiB scratch (about 400k triangles) hits the limit
    big = nan_b200.Scene(device, scenes.terrain_boxes(seed=2, grid=451, boxes=0))
    m = int(big.info()["triangle_count"])
    assert m > 350_000
    ctx2 = device.new_context()
    big_buf = torch.empty((max(m - 1, 1) * 16 + m * 12 + m * 2,), dtype=torch.float32, device=device.torch_device)
    bn, bt = big_buf.data_ptr(), big_buf.data_ptr() + max(m - 1, 1) * 64
    br = bt + m * 48
    rc = _call(ctx2, big, bn, max(m - 1, 1) * 64, bt, m * 48, br, m * 8)
    assert rc == _native.NAN_ERR_LIMIT, (rc, _last_error())
    assert "64 MiB" in _last_error()
    ctx2.close()
    torch.cuda.synchronize()
