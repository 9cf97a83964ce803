"""TextureSpacePathTracer.execute_host (payload in pinned host memory,
copied in and out per texel chunk on two copy streams around the tracing)
gives the same slots as execute on a device buffer, bit for bit."""

import pytest

pytestmark = pytest.mark.gpu


def test_execute_host_matches_device_execute(device):
    import torch

    import nan_b200
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MeshColorsLayout

    node = scenes.terrain_boxes(seed=4, grid=97, boxes=40)
    scene = nan_b200.Scene(device, node)
    layout = MeshColorsLayout.build(node, texels_per_unit=8.0, min_resolution=2, max_resolution=16)
    tracer = nan_b200.TextureSpacePathTracer(device, scene, layout)
    ref = torch.zeros((layout.total_payload_count, 4), dtype=torch.int32, device="cuda")
    staging = torch.zeros_like(ref)
    host = torch.zeros_like(ref, device="cpu").pin_memory()
    for it in range(3):
        tracer.execute(None, ref, it, reset=(it == 0))
        tracer.execute_host(host, staging, it, reset=(it == 0), chunks=3)
    tracer.host_ready()
    torch.cuda.synchronize()
    assert len(tracer._spans[1]) == 3
    torch.testing.assert_close(host, ref.cpu(), rtol=0, atol=0)
    with pytest.raises(ValueError):
        tracer.execute_host(torch.zeros_like(host), staging, 0)
    device.check()
