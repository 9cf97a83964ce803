"""Timing of surface-probe placement on the GPU, for profiling.

`layout` mode builds SurfaceProbeSiteLayout.build_wse on the seeded
terrain + boxes scene (the reference's default path: density prepass,
adaptive elimination of 5x oversampled candidates, audit/repair filter,
budgeted repair, protected closure, support estimate, packing) `repeats`
times and prints each build's stage profile.

`wse` mode eliminates one set of area-weighted candidates on the terrain
without boxes (90 per m^2, about 206k on grid 313) down to a fifth,
`repeats` times, plain and adaptive (densities varying 6:1 across the
terrain), and prints the CUDA-synchronised wall time of each call.
"""

from __future__ import annotations

import json
import time


def _wse(device, grid: int, repeats: int) -> dict:
    import numpy as np
    import torch

    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import _surface_points
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler

    node = scenes.terrain_boxes(seed=2, grid=grid, boxes=0)
    mesh_id, _, transform_id = node.instances[0]
    mesh = node.meshes[mesh_id]
    m = node.transforms[transform_id].astype(np.float64)
    p = mesh.vertices[:, :3].astype(np.float64) @ m[:3, :3].T + m[:3, 3]
    t = p[mesh.indices.astype(np.int64).reshape(-1, 3)].astype(np.float32)
    areas = 0.5 * np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]).astype(np.float64), axis=1)
    n = int(areas.sum() * 90.0)
    pos, nrm, _, _, _ = _surface_points(t, areas, n, np.random.default_rng(5))
    dens = (0.4 + 2.0 * (0.5 + 0.5 * np.sin(pos[:, 0] * 0.7 + pos[:, 2] * 0.3))).astype(np.float32)
    sampler = SurfaceProbeSampler(device)
    pt, nt, dt = (torch.as_tensor(x, device=device.torch_device) for x in (pos, nrm, dens))
    out = {"candidates": n, "output": n // 5, "plain_ms": [], "adaptive_ms": []}
    for key, d in (("plain_ms", None), ("adaptive_ms", dt)):
        for _ in range(repeats):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sampler.eliminate(pt, nt, [0, n], [n // 5], [float(areas.sum())], relative_densities=d)
            torch.cuda.synchronize()
            out[key].append((time.perf_counter() - t0) * 1e3)
        out[key.replace("_ms", "_rounds")] = sampler.last_rounds
    return out


def main(argv=None) -> None:
    import argparse

    from nan_b200 import scenes
    from nan_b200.scene import Device
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler

    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", choices=("layout", "wse"), default="layout")
    ap.add_argument("--grid", type=int, default=313)
    ap.add_argument("--boxes", type=int, default=500)
    ap.add_argument("--sites", type=int, default=20480)
    ap.add_argument("--repeats", type=int, default=3)
    args = ap.parse_args(argv)
    device = Device(0)
    if args.mode == "wse":
        print(json.dumps(_wse(device, args.grid, args.repeats)))
        return
    node = scenes.terrain_boxes(seed=1, grid=args.grid, boxes=args.boxes)
    sampler = SurfaceProbeSampler(device)
    builds = []
    for r in range(args.repeats):
        prof: dict = {}
        t0 = time.perf_counter()
        layout = SurfaceProbeSiteLayout.build_wse(node, args.sites, sampler=sampler, seed=1, profile=prof)
        prof["total_s"] = time.perf_counter() - t0
        prof["probe_records"] = int(layout.total_probe_count)
        builds.append(prof)
    device.check()
    print(json.dumps({"scene": node.name, "sites": args.sites, "builds": builds}))


if __name__ == "__main__":
    main()
