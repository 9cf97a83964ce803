"""Mesh Colors resolve on the GPU against the oracle: the accumulated slot
cache and its RGB9E5-packed (frozen) form, drawn through the camera, equal
the oracle's resolve bit for bit (>= 99.9 % of pixels exact, all within 1e-4
relative), on the Cornell box (double-sided walls, back sides) and on the
terrain."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["cornell", "terrain"])
def test_resolve_matches_oracle(which, device):
    import torch

    import nan_b200
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MeshColorsLayout
    from oracle.oracle import OracleScene

    if which == "cornell":
        node = scenes.cornell_box(64, 64)
        node.lighting.sun_disk = True
    else:
        node = scenes.terrain_boxes(seed=1, grid=129, boxes=120)
    scene = nan_b200.Scene(device, node)
    orc = OracleScene(**scene.host)
    layout = MeshColorsLayout.build(node, texels_per_unit=8.0, min_resolution=2, max_resolution=16)
    tracer = nan_b200.TextureSpacePathTracer(device, scene, layout, samples_per_texel=1, max_bounces=2)
    slots = torch.zeros((layout.total_payload_count, 4), dtype=torch.int32, device="cuda")
    for it in range(4):
        tracer.execute(None, slots, it, reset=(it == 0))
    packed = torch.zeros(layout.total_payload_count, dtype=torch.int32, device="cuda")
    nan_b200.MeshColorsRGB9E5Packer(device).execute(None, slots, packed, layout.total_payload_count)
    resolve = nan_b200.MeshColorsResolve(device, scene, layout, tracer)
    w, h = 96, 64
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    px = np.stack(np.meshgrid(np.arange(w), np.arange(h), indexing="xy"), -1).reshape(-1, 2)
    host_slots = slots.cpu().numpy().view(np.uint32)
    host_packed = packed.cpu().numpy().view(np.uint32)
    for frozen in (False, True):
        node.camera.begin_frame(w, h)
        (resolve.execute_frozen if frozen else resolve.execute)(None, packed if frozen else slots, out)
        gpu = out.cpu().numpy().reshape(-1, 4)
        ref = orc.resolve_mesh_colors(scene.lighting, node.camera, w, h, px, layout.face_array,
                                      layout.instance_array, layout.side_array,
                                      host_packed if frozen else host_slots, packed=frozen)
        exact = np.all(gpu == ref, axis=1)
        rel = np.max(np.abs(gpu - ref) / np.maximum(np.abs(ref), 1e-3), axis=1)
        print(which, "frozen" if frozen else "slots", "exact", exact.mean(), "lit pixels", (gpu[:, :3].sum(1) > 0).mean())
        assert exact.mean() >= 0.999, exact.mean()
        assert (rel <= 1e-4).mean() >= 0.999
    device.check()
