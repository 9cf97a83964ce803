"""Rebuilding a context's scene: nan_scene_build keeps the context's BVH
storage when the new scene fits in it, and grows it otherwise. Rebuilds in
both directions trace exactly like fresh builds, and an LBVH rebuild after a
PLOC build (which also wrote 8-wide nodes) never traverses the old wide
nodes, even when the tuning asks for width 8."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rays(scene, n, seed):
    import torch

    tris = scene.world_triangles().cpu().numpy().reshape(-1, 3)
    lo, hi = tris.min(0), tris.max(0)
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 7] = 1e30
    return torch.from_numpy(r).cuda()


def _intersect(ctx, rays):
    import torch

    from nan_b200 import _native

    n = rays.shape[0]
    ids = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    tb = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    _native.check(_native.lib().nan_intersect(ctx.handle, rays.data_ptr(), n, ids.data_ptr(), tb.data_ptr(),
                                              _native.stream_handle(None)))
    return ids, tb


def test_rebuild_reuses_storage_and_matches_fresh_builds(device):
    import torch

    import nan_b200
    from nan_b200 import _native, scenes

    mid = nan_b200.Scene(device, scenes.terrain_boxes(seed=2, grid=97, boxes=40))
    small = nan_b200.Scene(device, scenes.cornell_box(32, 32))
    large = nan_b200.Scene(device, scenes.terrain_boxes(seed=3, grid=161, boxes=120))
    ctx = device.new_context()
    for scene, builder, width in ((mid, "sah", 8), (small, "sah", 2), (large, "sah", 2), (mid, "ploc", 8),
                                  (small, "ploc", 2), (large, "ploc", 8), (mid, "lbvh", 8), (large, "lbvh", 2)):
        ctx.configure(bvh_builder=builder, bvh_width=width)
        _native.check(_native.lib().nan_scene_build(ctx.handle, ctypes.byref(scene._desc),
                                                    _native.stream_handle(None)))
        scene.configure(bvh_width=2)
        rays = _rays(scene, 4096, seed=len(builder) + width)
        ids, tb = _intersect(ctx, rays)
        ref_ids, ref_tb = scene.intersect(rays)
        torch.testing.assert_close(ids, ref_ids, rtol=0, atol=0)
        torch.testing.assert_close(tb, ref_tb, rtol=0, atol=0)
        assert (ids[:, 0] == 1).float().mean().item() > 0.2
    ctx.check()
    ctx.close()
