"""Surface-probe site selection on the GPU: weighted sample elimination
(surface_probe_sampler.py / surface_probe_sampler.h:120-130 and
weighted_sample_elimination, surface_probes.py:1091-1123 of the reference)
and deficit repair (deficit_repair, surface_probes.py:1201-1253;
deficit_repair_python, surface_probe_sampler.py:990-1103).

SurfaceProbeSampler.deficit_repair adds repair candidates where audit
points gather fewer than min_gather_count probes: candidates are chosen one
at a time by their summed deficit score (highest first, lowest index on
ties), computed as parallel rounds that give the same choices.

SurfaceProbeSampler.estimate_support gives each site its support f (the
area-weighted kernel mass of the surface around it, relative to a flat
disc) and density multiplier m.

SurfaceProbeSampler.filter_audit_repair_candidates keeps one audit point per
cell and normal cone and drops repair candidates that duplicate a selected
base site or an earlier candidate bit for bit
(filter_audit_repair_candidates_cpp, surface_probe_sampler.py:721-800).

SurfaceProbeSampler.eliminate thins many candidate sets in one call (one
persistent set of launches for all instances of a scene); with
relative_densities it runs the adaptive elimination
(adaptive_weighted_sample_elimination, surface_probes.py:988-1166), each
candidate compared within its own d_max / sqrt(density);
weighted_sample_elimination keeps the reference's single-set signature and
returns (selected indices ascending, Poisson radius). The elimination is the
reference's: largest weight first (lowest index on ties), weights
sum_j (1 - d_ij / d_max)^8 over compatible neighbours, run as parallel
rounds that remove every local maximum at once and give the same survivors.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np

from ._native import Context, NanRepairOptions, NanSupportOptions, NanWseOptions, check, lib, ptr, stream_handle

WSE_NORMAL_COSINE_THRESHOLD = 0.5
WSE_PLANE_DISTANCE_SCALE = 0.35


def _points(dev, positions, normals, instances, name):
    import torch

    p = torch.as_tensor(np.asarray(positions, dtype=np.float32).reshape(-1, 3) if not hasattr(positions, "device")
                        else positions, dtype=torch.float32, device=dev).reshape(-1, 3).contiguous()
    n = torch.as_tensor(np.asarray(normals, dtype=np.float32).reshape(-1, 3) if not hasattr(normals, "device")
                        else normals, dtype=torch.float32, device=dev).reshape(-1, 3).contiguous()
    i = torch.as_tensor(np.asarray(instances, dtype=np.int64).astype(np.uint32).view(np.int32)
                        if not hasattr(instances, "device") else instances, device=dev).reshape(-1).contiguous()
    if p.shape[0] != n.shape[0] or p.shape[0] != i.shape[0]:
        raise ValueError(f"{name} positions, normals and instances must have the same length")
    return p, n, i


class SupportEstimateResult(NamedTuple):
    """As the reference's SupportEstimateResult (support_f, density_m); unpacks
    as a pair."""
    support_f: np.ndarray
    density_m: np.ndarray


@dataclass(frozen=True)
class CandidateFilterResult:
    """As the reference's CandidateFilterResult (surface_probe_sampler.py:211-215),
    without its CPU timing profile."""
    audit_indices: np.ndarray
    repair_indices: np.ndarray


@dataclass(frozen=True)
class DeficitRepairResult:
    """As the reference's DeficitRepairResult (surface_probe_sampler.py:219-229)."""
    selected_candidate_indices: np.ndarray
    counts_before: np.ndarray
    counts_after: np.ndarray
    weight_sums_before: np.ndarray
    weight_sums_after: np.ndarray
    ess_before: np.ndarray
    ess_after: np.ndarray
    rounds: int = 0


class SurfaceProbeSampler:
    """Owns the context the elimination and the repair run in."""

    def __init__(self, device):
        self.device = device
        index = getattr(device, "index", 0)
        self.context = Context(int(index))
        self.last_rounds = 0

    def eliminate(self, positions, normals, set_offsets, output_counts, surface_areas, *,
                  normal_cosine_threshold: float = WSE_NORMAL_COSINE_THRESHOLD,
                  plane_distance_scale: float = WSE_PLANE_DISTANCE_SCALE, relative_densities=None, stream=None):
        """positions, normals: float32 [N, 3] (CUDA tensors or arrays), the sets
        contiguous with boundaries set_offsets [S+1]. Returns (keep uint8 CUDA
        tensor [N], Poisson radius per set). relative_densities (float32 [N],
        finite and positive) selects the adaptive elimination; its Poisson
        radius is the base one, sqrt(area / (2 sqrt(3) count))."""
        import torch

        dev = self.device.torch_device if hasattr(self.device, "torch_device") else torch.device("cuda")
        pos = torch.as_tensor(positions, dtype=torch.float32, device=dev).reshape(-1, 3).contiguous()
        nrm = torch.as_tensor(normals, dtype=torch.float32, device=dev).reshape(-1, 3).contiguous()
        dens = None
        if relative_densities is not None:
            dens = torch.as_tensor(relative_densities, dtype=torch.float32, device=dev).reshape(-1).contiguous()
            if dens.shape[0] != pos.shape[0]:
                raise ValueError("relative_densities must have one value per candidate")
        off = np.ascontiguousarray(set_offsets, dtype=np.uint32).reshape(-1)
        outs = np.ascontiguousarray(output_counts, dtype=np.uint32).reshape(-1)
        areas = np.ascontiguousarray(surface_areas, dtype=np.float32).reshape(-1)
        sets = off.shape[0] - 1
        if sets < 0 or outs.shape[0] != sets or areas.shape[0] != sets or int(off[-1]) != pos.shape[0]:
            raise ValueError("set_offsets, output_counts and surface_areas must describe the candidate sets")
        keep = torch.zeros(pos.shape[0], dtype=torch.uint8, device=dev)
        radii = np.zeros(max(sets, 1), np.float32)
        rounds = ctypes.c_uint32(0)
        opt = NanWseOptions(float(normal_cosine_threshold), float(plane_distance_scale))
        if dens is None:
            check(lib().nan_wse_eliminate(self.context.handle, ptr(pos), ptr(nrm), off.ctypes.data, sets,
                                          outs.ctypes.data, areas.ctypes.data, ctypes.byref(opt), ptr(keep),
                                          radii.ctypes.data, ctypes.byref(rounds), stream_handle(stream)))
        else:
            check(lib().nan_wse_eliminate_adaptive(self.context.handle, ptr(pos), ptr(nrm), ptr(dens),
                                                   off.ctypes.data, sets, outs.ctypes.data, areas.ctypes.data,
                                                   ctypes.byref(opt), ptr(keep), radii.ctypes.data,
                                                   ctypes.byref(rounds), stream_handle(stream)))
        self.last_rounds = int(rounds.value)
        return keep, radii[:sets]

    def filter_audit_repair_candidates(self, candidate_positions, candidate_normals, base_positions, base_normals,
                                       base_selected_indices, *, audit_cell_size, normal_cosine_threshold: float,
                                       candidate_sets=None, base_sets=None, stream=None) -> CandidateFilterResult:
        """The reference's audit/repair candidate filter on the GPU. One set
        by default; with candidate_sets and base_sets (per point set
        indices) audit_cell_size is a per-set sequence. Result indices are
        host int64 arrays, ascending."""
        import torch

        dev = self.device.torch_device if hasattr(self.device, "torch_device") else torch.device("cuda")
        f3 = lambda a: torch.as_tensor(a if hasattr(a, "device") else np.asarray(a, dtype=np.float32),
                                       dtype=torch.float32, device=dev).reshape(-1, 3).contiguous()
        u32 = lambda a: torch.as_tensor(a if hasattr(a, "device") else np.asarray(a, dtype=np.int64).astype(
            np.uint32).view(np.int32), device=dev).reshape(-1).contiguous()
        cp, cn, bp, bn = f3(candidate_positions), f3(candidate_normals), f3(base_positions), f3(base_normals)
        if cn.shape != cp.shape or bn.shape != bp.shape:
            raise ValueError("normals must match positions")
        if cp.shape[0] == 0 or bp.shape[0] == 0:
            raise ValueError("candidate and base arrays must be non-empty")
        sel = u32(base_selected_indices)
        cells = np.ascontiguousarray(np.atleast_1d(np.asarray(audit_cell_size, dtype=np.float64)))
        sets = int(cells.shape[0])
        cs = bs = None
        if candidate_sets is not None or base_sets is not None:
            if candidate_sets is None or base_sets is None:
                raise ValueError("candidate_sets and base_sets go together")
            cs, bs = u32(candidate_sets), u32(base_sets)
            if cs.shape[0] != cp.shape[0] or bs.shape[0] != bp.shape[0]:
                raise ValueError("set indices must cover every point")
        elif sets != 1:
            raise ValueError("several cell sizes need candidate_sets and base_sets")
        n = cp.shape[0]
        audit = torch.empty(n, dtype=torch.int32, device=dev)
        repair = torch.empty(n, dtype=torch.int32, device=dev)
        na, nr = ctypes.c_uint32(0), ctypes.c_uint32(0)
        check(lib().nan_filter_audit_repair(self.context.handle, ptr(cp), ptr(cn), ptr(cs) if cs is not None else None,
                                            n, ptr(bp), ptr(bn), ptr(bs) if bs is not None else None, bp.shape[0],
                                            ptr(sel) if sel.numel() else None, sel.shape[0], sets, cells.ctypes.data,
                                            float(normal_cosine_threshold), ptr(audit), ctypes.byref(na), ptr(repair),
                                            ctypes.byref(nr), stream_handle(stream)))
        host = lambda t, k: t[:k].cpu().numpy().view(np.uint32).astype(np.int64)
        return CandidateFilterResult(host(audit, na.value), host(repair, nr.value))

    def build_point_octrees(self, position_sets, *, leaf_capacity: int = 8, max_depth: int = 16, stream=None):
        """Point octrees of several position sets (each f32 [n, 3]) in one
        GPU call, as build_point_octree builds each: per set (nodes u32
        [M, 4], order i64 [n], root centre, root half extent), or None for an
        empty set."""
        sets = [np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3) for x in position_sets]
        offsets = np.concatenate([[0], np.cumsum([x.shape[0] for x in sets])]).astype(np.uint32)
        if int(offsets[-1]) == 0:
            return [None] * len(sets)
        nodes_h, node_offsets, order_h, roots = self.build_point_octrees_flat(
            np.concatenate(sets), offsets, leaf_capacity=leaf_capacity, max_depth=max_depth, stream=stream)
        out = []
        for k in range(len(sets)):
            if offsets[k + 1] == offsets[k]:
                out.append(None)
                continue
            out.append((nodes_h[node_offsets[k]:node_offsets[k + 1]].copy(), order_h[offsets[k]:offsets[k + 1]],
                        tuple(float(v) for v in roots[k, :3]), float(roots[k, 3])))
        return out

    def build_point_octrees_flat(self, positions, set_offsets, *, leaf_capacity: int = 8, max_depth: int = 16,
                                 stream=None):
        """build_point_octrees over sets stored back to back (positions f32
        [N, 3], set k at set_offsets[k]:set_offsets[k + 1]): (nodes u32 [M,
        4] with set k's nodes at node_offsets[k]:node_offsets[k + 1], child
        and probe indices local to the set; node_offsets u32 [S + 1]; order
        i64 [N], set k's permutation of its own points at its offsets; roots
        f64 [S, 4], centre and half extent). An empty set has no nodes."""
        import torch

        dev = self.device.torch_device if hasattr(self.device, "torch_device") else torch.device("cuda")
        offsets = np.ascontiguousarray(set_offsets, dtype=np.uint32).reshape(-1)
        sets = offsets.shape[0] - 1
        n = int(offsets[-1])
        pos = torch.as_tensor(np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3), device=dev)
        if pos.shape[0] != n:
            raise ValueError("set_offsets must end at the number of positions")
        order = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
        node_offsets = np.zeros(sets + 1, np.uint32)
        roots = np.zeros((max(sets, 1), 4), np.float64)
        capacity = max(64, n // max(int(leaf_capacity), 1) * 3 + 2 * sets)
        for _ in range(2):
            nodes = torch.empty((capacity, 4), dtype=torch.int32, device=dev)
            rc = lib().nan_build_point_octrees(self.context.handle, ptr(pos), offsets.ctypes.data, sets,
                                               int(leaf_capacity), int(max_depth), ptr(nodes), capacity,
                                               node_offsets.ctypes.data, ptr(order), roots.ctypes.data,
                                               stream_handle(stream))
            if rc == 3 and int(node_offsets[-1]) > capacity:  # NAN_ERR_LIMIT: retry at the needed size
                capacity = int(node_offsets[-1])
                continue
            check(rc)
            break
        nodes_h = nodes[:int(node_offsets[-1])].cpu().numpy().view(np.uint32)
        return nodes_h, node_offsets, order[:n].cpu().numpy().astype(np.int64), roots[:sets]

    def deficit_repair(self, base_positions, base_normals, base_instances, candidate_positions, candidate_normals,
                       candidate_instances, audit_positions, audit_normals, audit_instances, instance_radii, *,
                       min_gather_count: int = 4, max_repair_count: int, normal_cosine_threshold: float = 0.5,
                       weight_epsilon: float = 1e-6, stream=None) -> DeficitRepairResult:
        """The reference's deficit_repair on the GPU (arrays or CUDA tensors;
        instance_radii per instance). Result arrays are on the host."""
        import torch

        dev = self.device.torch_device if hasattr(self.device, "torch_device") else torch.device("cuda")
        bp, bn, bi = _points(dev, base_positions, base_normals, base_instances, "base")
        cp, cn, ci = _points(dev, candidate_positions, candidate_normals, candidate_instances, "candidate")
        ap, an, ai = _points(dev, audit_positions, audit_normals, audit_instances, "audit")
        radii = np.ascontiguousarray(instance_radii, dtype=np.float32).reshape(-1)
        na = ap.shape[0]
        budget = max(0, min(int(max_repair_count), cp.shape[0]))
        selected = torch.zeros(max(budget, 1), dtype=torch.int32, device=dev)
        counts = [torch.zeros(na, dtype=torch.int32, device=dev) for _ in range(2)]
        floats = [torch.zeros(na, dtype=torch.float32, device=dev) for _ in range(4)]
        opt = NanRepairOptions(max(1, min(32, int(min_gather_count))), budget, float(normal_cosine_threshold),
                               float(weight_epsilon))
        count = ctypes.c_uint32(0)
        rounds = ctypes.c_uint32(0)
        check(lib().nan_deficit_repair(self.context.handle, ptr(bp), ptr(bn), ptr(bi), bp.shape[0], ptr(cp), ptr(cn),
                                       ptr(ci), cp.shape[0], ptr(ap), ptr(an), ptr(ai), na, radii.ctypes.data,
                                       radii.shape[0], ctypes.byref(opt), ptr(selected), ctypes.byref(count),
                                       ptr(counts[0]), ptr(counts[1]), ptr(floats[0]), ptr(floats[1]), ptr(floats[2]),
                                       ptr(floats[3]), ctypes.byref(rounds), stream_handle(stream)))
        host = lambda t: t.cpu().numpy()
        return DeficitRepairResult(host(selected)[:count.value].astype(np.int64), host(counts[0]).view(np.uint32),
                                   host(counts[1]).view(np.uint32), host(floats[0]), host(floats[1]), host(floats[2]),
                                   host(floats[3]), int(rounds.value))


    def estimate_support(self, reference_positions, reference_normals, reference_instances, reference_area_weights,
                         query_positions, query_normals, query_instances, instance_radii, *,
                         normal_cosine_threshold: float = 0.5, weight_epsilon: float = 1e-6,
                         max_density_multiplier: float = 8.0, stream=None):
        """The reference's estimate_surface_support on the GPU: support_f and
        density_m per query site (host float32 arrays), as a
        SupportEstimateResult that also unpacks as a pair."""
        import torch

        dev = self.device.torch_device if hasattr(self.device, "torch_device") else torch.device("cuda")
        rp, rn, ri = _points(dev, reference_positions, reference_normals, reference_instances, "reference")
        qp, qn, qi = _points(dev, query_positions, query_normals, query_instances, "query")
        ra = torch.as_tensor(np.asarray(reference_area_weights, dtype=np.float32).reshape(-1)
                             if not hasattr(reference_area_weights, "device") else reference_area_weights,
                             dtype=torch.float32, device=dev).reshape(-1).contiguous()
        if ra.shape[0] != rp.shape[0]:
            raise ValueError("reference_area_weights must have one weight per reference point")
        radii = np.ascontiguousarray(instance_radii, dtype=np.float32).reshape(-1)
        f = torch.zeros(qp.shape[0], dtype=torch.float32, device=dev)
        m = torch.zeros(qp.shape[0], dtype=torch.float32, device=dev)
        opt = NanSupportOptions(float(normal_cosine_threshold), float(weight_epsilon), float(max_density_multiplier),
                                0.0)
        check(lib().nan_estimate_support(self.context.handle, ptr(rp), ptr(rn), ptr(ri), ptr(ra), rp.shape[0],
                                         ptr(qp), ptr(qn), ptr(qi), qp.shape[0], radii.ctypes.data, radii.shape[0],
                                         ctypes.byref(opt), ptr(f), ptr(m), stream_handle(stream)))
        return SupportEstimateResult(f.cpu().numpy(), m.cpu().numpy())


def adaptive_weighted_sample_elimination(positions, normals, relative_densities, output_count: int, *,
                                         surface_area: float, partition_masses=None,
                                         normal_cosine_threshold: float = WSE_NORMAL_COSINE_THRESHOLD,
                                         plane_distance_scale: float = WSE_PLANE_DISTANCE_SCALE, device=None):
    """Single-set adaptive form: (selected candidate indices ascending, base
    Poisson radius). partition_masses only shape the reference's CPU
    partitioning; they are checked for shape and otherwise unused."""
    from .scene import Device

    n = int(np.asarray(positions).reshape(-1, 3).shape[0]) if not hasattr(positions, "shape") else int(
        positions.shape[0])
    if n == 0:
        raise ValueError("weighted sample elimination needs at least one candidate")
    if partition_masses is not None and np.asarray(partition_masses).reshape(-1).shape[0] != n:
        raise ValueError("partition_masses must have one value per candidate")
    sampler = SurfaceProbeSampler(device if device is not None else Device(0))
    keep, radii = sampler.eliminate(positions, normals, [0, n], [max(1, min(int(output_count), n))],
                                    [float(surface_area)], normal_cosine_threshold=normal_cosine_threshold,
                                    plane_distance_scale=plane_distance_scale, relative_densities=relative_densities)
    return np.flatnonzero(keep.cpu().numpy()).astype(np.int64), float(radii[0])


def weighted_sample_elimination(positions, normals, output_count: int, *, surface_area: float,
                                normal_cosine_threshold: float = WSE_NORMAL_COSINE_THRESHOLD,
                                plane_distance_scale: float = WSE_PLANE_DISTANCE_SCALE, device=None):
    """Single-set form: (selected candidate indices ascending, Poisson radius)."""
    from .scene import Device

    n = int(np.asarray(positions).reshape(-1, 3).shape[0]) if not hasattr(positions, "shape") else int(
        positions.shape[0])
    if n == 0:
        raise ValueError("weighted sample elimination needs at least one candidate")
    sampler = SurfaceProbeSampler(device if device is not None else Device(0))
    keep, radii = sampler.eliminate(positions, normals, [0, n], [max(1, min(int(output_count), n))],
                                    [float(surface_area)], normal_cosine_threshold=normal_cosine_threshold,
                                    plane_distance_scale=plane_distance_scale)
    return np.flatnonzero(keep.cpu().numpy()).astype(np.int64), float(radii[0])

