// nan_octree.cu -- per-instance point octrees of surface-probe sites on the
// GPU, for many point sets in one call (_build_point_octree_python,
// surface_probes.py:1348-1438; C ABI surface_probe_build_point_octree,
// surface_probe_sampler.h:120-223).
//
// The reference walks the tree depth first: a node holding more than
// leaf_capacity points (and above max_depth) splits into its present
// octants (bit o set where the point is > float32(centre) on that axis),
// numbers them contiguously at the moment it splits, and pushes them so that
// octant 0 is walked first; a leaf names its points, in ascending input
// order, at the next free place of the output order.
//
// Here every point first computes its whole octant path (16 levels of 3 bits,
// the centres stepped in float64 exactly as the walk steps them) and the
// points are sorted by (set, path): the runs of equal path prefixes are then
// the nodes, their order is the walk's order, and a run's length is its point
// count. A point that starts a run at some depth emits the nodes of all the
// depths from there down to its leaf, ancestors first, which lists the nodes
// in walk (pre)order. Node numbers follow from that list: a node's children
// are numbered 1 + (the children of the branches before it in the list) on.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "nan_internal.h"

namespace {

constexpr int kPathLevels = 16;  // 48 bits of path under 16 bits of set index

__device__ __forceinline__ unsigned int ordered_bits(float f) {
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float from_ordered(unsigned int u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_oct_bounds(const float* pos, const uint32_t* set_of, uint32_t n, unsigned int* lo, unsigned int* hi,
                             int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t s = set_of[i];
    for (int a = 0; a < 3; ++a) {
        const float v = pos[3 * i + a];
        if (!isfinite(v)) {
            atomicOr(status, 1);
            return;
        }
        atomicMin(lo + 3 * s + a, ordered_bits(v));
        atomicMax(hi + 3 * s + a, ordered_bits(v));
    }
}

// Root cube per set: centre (lo + hi) / 2, half extent max(max axis span / 2,
// 1e-5) x 1.0001, in float64 from the float32 bounds.
__global__ void k_oct_roots(uint32_t sets, const unsigned int* lo, const unsigned int* hi, double4* roots) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= sets) return;
    double c[3], span = 0.0;
    for (int a = 0; a < 3; ++a) {
        const double l = (double)from_ordered(lo[3 * s + a]), h = (double)from_ordered(hi[3 * s + a]);
        c[a] = (l + h) * 0.5;
        span = fmax(span, h - l);
    }
    roots[s] = make_double4(c[0], c[1], c[2], fmax(span * 0.5, 1e-5) * 1.0001);
}

__global__ void k_oct_paths(const float* pos, const uint32_t* set_of, uint32_t n, const double4* roots, int depth,
                            unsigned long long* keys, uint32_t* idx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t s = set_of[i];
    const double4 r = roots[s];
    double c[3] = {r.x, r.y, r.z}, e = r.w;
    const float p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    unsigned long long path = 0;
    for (int l = 0; l < depth; ++l) {
        uint32_t o = 0;
        for (int a = 0; a < 3; ++a)
            if (p[a] > __double2float_rn(c[a])) o |= 1u << a;
        path |= (unsigned long long)o << (3 * (kPathLevels - 1 - l));
        const double half = e * 0.5;
        for (int a = 0; a < 3; ++a) c[a] = c[a] + ((o >> a) & 1u ? half : -half);
        e = half;
    }
    keys[i] = ((unsigned long long)s << 48) | path;
    idx[i] = i;
}

// All keys sharing the first l path levels (and the set).
__device__ __forceinline__ unsigned long long prefix_mask(int l) {
    return ~((1ull << (3 * (kPathLevels - l))) - 1ull);  // l = 0 keeps the set bits only
}

__device__ __forceinline__ uint32_t lower_bound64(const unsigned long long* k, uint32_t n, unsigned long long v) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (k[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

struct RunInfo {
    uint32_t begin, count;
};

__device__ __forceinline__ RunInfo run_at(const unsigned long long* keys, uint32_t n, unsigned long long key, int l) {
    const unsigned long long p = key & prefix_mask(l);
    const unsigned long long next = p + (1ull << (3 * (kPathLevels - l)));
    const uint32_t b = lower_bound64(keys, n, p);
    const uint32_t e = lower_bound64(keys, n, next);
    return {b, e - b};
}

// Per sorted point: its leaf depth L (the first depth whose run holds at most
// `capacity` points, or `depth`), the first depth l0 at which it starts a run,
// and the number of nodes it emits (depths l0..L).
__global__ void k_oct_levels(const unsigned long long* keys, uint32_t n, uint32_t capacity, int depth, uint8_t* leaf_l,
                             uint8_t* first_l, uint32_t* emit) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const unsigned long long k = keys[q];
    int L = depth;
    for (int l = 0; l < depth; ++l)
        if (run_at(keys, n, k, l).count <= capacity) {
            L = l;
            break;
        }
    int l0 = 0;
    if (q > 0) {
        const unsigned long long prev = keys[q - 1];
        if ((prev >> 48) == (k >> 48)) {
            l0 = kPathLevels + 1;  // the same path: no new run at any depth
            for (int l = 1; l <= kPathLevels; ++l)
                if ((prev & prefix_mask(l)) != (k & prefix_mask(l))) {
                    l0 = l;
                    break;
                }
        }
    }
    leaf_l[q] = (uint8_t)L;
    first_l[q] = (uint8_t)min(l0, 255);
    emit[q] = l0 <= L ? (uint32_t)(L - l0 + 1) : 0u;
}

struct NodeEntries {
    uint32_t* start;   // sorted position of the node's first point
    uint32_t* count;   // its points
    int* parent;       // entry index of the parent, -1 for a root
    uint32_t* mask;    // present child octants (branches)
    uint8_t* level;
    uint8_t* octant;   // its octant in the parent
    uint8_t* leaf;
};

__global__ void k_oct_emit(const unsigned long long* keys, uint32_t n, const uint8_t* leaf_l, const uint8_t* first_l,
                           const uint32_t* emit_off, NodeEntries ne) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int L = leaf_l[q], l0 = first_l[q];
    if (l0 > L) return;
    const unsigned long long k = keys[q];
    for (int l = l0; l <= L; ++l) {
        const uint32_t e = emit_off[q] + (uint32_t)(l - l0);
        ne.start[e] = q;
        ne.count[e] = run_at(keys, n, k, l).count;
        ne.level[e] = (uint8_t)l;
        ne.leaf[e] = l == L ? 1u : 0u;
        ne.mask[e] = 0u;
        const uint32_t oct = l > 0 ? (uint32_t)((k >> (3 * (kPathLevels - l))) & 7ull) : 0u;
        ne.octant[e] = (uint8_t)oct;
        if (l == 0) {
            ne.parent[e] = -1;
        } else if (l - 1 >= l0) {
            ne.parent[e] = (int)e - 1;
        } else {
            const uint32_t qp = run_at(keys, n, k, l - 1).begin;
            ne.parent[e] = (int)(emit_off[qp] + (uint32_t)(l - 1 - first_l[qp]));
        }
    }
}

__global__ void k_oct_masks(uint32_t m, NodeEntries ne) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m || ne.parent[e] < 0) return;
    atomicOr(ne.mask + ne.parent[e], 1u << ne.octant[e]);
}

__global__ void k_oct_children(uint32_t m, NodeEntries ne, uint32_t* nchild) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < m) nchild[e] = ne.leaf[e] ? 0u : (uint32_t)__popc(ne.mask[e]);
}

// Node numbers local to each set: the set's root (its first entry) is 0; a
// branch's children start at 1 + the children of the branches before it.
__global__ void k_oct_write(uint32_t m, NodeEntries ne, const uint32_t* child_scan, const uint32_t* set_first,
                            const uint32_t* entry_set, const uint32_t* point_set_begin, uint32_t* local_id,
                            uint4* nodes, int* status) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const uint32_t s = entry_set[e];
    const uint32_t f = set_first[s];
    uint32_t id = 0;
    if (e != f) {
        const int p = ne.parent[e];
        const uint32_t base = 1u + child_scan[p] - child_scan[f];
        id = base + (uint32_t)__popc(ne.mask[p] & ((1u << ne.octant[e]) - 1u));
    }
    local_id[e] = id;
    if (f + id >= set_first[s + 1]) {  // a numbering outside the set's nodes: reported, not written
        atomicOr(status, 4);
        return;
    }
    uint4 out;
    if (ne.leaf[e]) {
        out = make_uint4(0u, 0u, ne.start[e] - point_set_begin[entry_set[e]], ne.count[e]);
    } else {
        out = make_uint4(1u + child_scan[e] - child_scan[f], ne.mask[e], 0u, 0u);
    }
    nodes[f + id] = out;
}

__global__ void k_oct_entry_sets(uint32_t m, const NodeEntries ne, const unsigned long long* keys,
                                 uint32_t* entry_set) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < m) entry_set[e] = (uint32_t)(keys[ne.start[e]] >> 48);
}

// Leaf key per point (its path cut at its leaf depth), scattered to input
// order so a stable sort lists each leaf's points in ascending input order.
__global__ void k_oct_leaf_keys(const unsigned long long* keys, const uint32_t* idx, uint32_t n,
                                const uint8_t* leaf_l, unsigned long long* leaf_key) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) leaf_key[idx[q]] = keys[q] & prefix_mask(leaf_l[q]);
}

// The emit offset at each set's first point (the set's first node entry),
// gathered so the host reads all of them in one copy.
__global__ void k_oct_set_firsts(uint32_t sets, const uint32_t* set_offsets, const uint32_t* emit_off,
                                 uint32_t* out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k <= sets) out[k] = emit_off[set_offsets[k]];
}

__global__ void k_oct_iota(uint32_t n, uint32_t* v) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

__global__ void k_oct_order(uint32_t n, const uint32_t* sorted_idx, const uint32_t* set_of,
                            const uint32_t* point_set_begin, uint32_t* order) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const uint32_t i = sorted_idx[q];
    order[q] = i - point_set_begin[set_of[i]];
}

uint32_t blocks(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

}  // namespace

namespace nan_host {

int launch_build_point_octrees(NanContext* ctx, const float* positions, const uint32_t* set_offsets,
                               uint32_t set_count, uint32_t leaf_capacity, uint32_t max_depth, uint32_t* nodes,
                               uint32_t node_capacity, uint32_t* node_offsets, uint32_t* order, double* roots,
                               cudaStream_t st) {
    const uint32_t n = set_offsets[set_count];
    std::vector<uint32_t> set_of_host(n);
    for (uint32_t k = 0; k < set_count; ++k)
        for (uint32_t i = set_offsets[k]; i < set_offsets[k + 1]; ++i) set_of_host[i] = k;
    std::vector<void*> owned;
    cudaError_t e = cudaSuccess;
    auto get = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (e == cudaSuccess) e = nan_host::scratch_alloc(&p, std::max<size_t>(bytes, 16), st);
        if (e == cudaSuccess) owned.push_back(p);
        return p;
    };
    auto release = [&]() {
        for (void* p : owned) cudaFreeAsync(p, st);
        owned.clear();
    };
    uint32_t* set_of = (uint32_t*)get(n * 4ull);
    uint32_t* set_begin = (uint32_t*)get((set_count + 1) * 4ull);  // set_offsets on the device
    uint32_t* firsts = (uint32_t*)get((set_count + 1) * 4ull);
    unsigned int* lo = (unsigned int*)get(set_count * 12ull);
    unsigned int* hi = (unsigned int*)get(set_count * 12ull);
    double4* root_dev = (double4*)get(set_count * sizeof(double4));
    int* status = (int*)get(sizeof(int));
    unsigned long long* keys = (unsigned long long*)get(n * 8ull);
    unsigned long long* keys_sorted = (unsigned long long*)get(n * 8ull);
    uint32_t* idx = (uint32_t*)get(n * 4ull);
    uint32_t* idx_sorted = (uint32_t*)get(n * 4ull);
    uint8_t* leaf_l = (uint8_t*)get(n);
    uint8_t* first_l = (uint8_t*)get(n);
    uint32_t* emit_off = (uint32_t*)get((n + 1) * 4ull);
    size_t tmp_bytes = 0, need = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, need, keys, keys_sorted, idx, idx_sorted, (int)n, 0, 64, st);
    tmp_bytes = std::max(tmp_bytes, need);
    cub::DeviceScan::ExclusiveSum(nullptr, need, emit_off, emit_off, (int)(n + 1), st);
    tmp_bytes = std::max(tmp_bytes, need);
    void* tmp = get(tmp_bytes);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "octree scratch");
    }
    cudaMemcpyAsync(set_of, set_of_host.data(), n * 4ull, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(set_begin, set_offsets, (set_count + 1) * 4ull, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(lo, 0xff, set_count * 12ull, st);
    cudaMemsetAsync(hi, 0x00, set_count * 12ull, st);
    cudaMemsetAsync(status, 0, sizeof(int), st);
    const int depth = (int)max_depth;
    k_oct_bounds<<<blocks(n, 256), 256, 0, st>>>(positions, set_of, n, lo, hi, status);
    k_oct_roots<<<blocks(set_count, 128), 128, 0, st>>>(set_count, lo, hi, root_dev);
    k_oct_paths<<<blocks(n, 256), 256, 0, st>>>(positions, set_of, n, root_dev, depth, keys, idx);
    cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys_sorted, idx, idx_sorted, (int)n, 0, 64, st);
    k_oct_levels<<<blocks(n, 128), 128, 0, st>>>(keys_sorted, n, leaf_capacity, depth, leaf_l, first_l, emit_off);
    cudaMemsetAsync(emit_off + n, 0, 4, st);
    cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, emit_off, emit_off, (int)(n + 1), st);
    ctx->launches += 6;
    // node counts: the total and, per set, the first entry (the emit offset of its first point)
    std::vector<uint32_t> emit_host(set_count + 1);
    int host_status = 0;
    k_oct_set_firsts<<<blocks(set_count + 1, 256), 256, 0, st>>>(set_count, set_begin, emit_off, firsts);
    cudaMemcpyAsync(emit_host.data(), firsts, (set_count + 1) * 4ull, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess || host_status) {
        release();
        if (e != cudaSuccess) return cuda_fail(e, "octree paths");
        set_error("point positions must be finite");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    const uint32_t m = emit_host[set_count];
    for (uint32_t k = 0; k <= set_count; ++k) node_offsets[k] = emit_host[k];
    if (m > node_capacity) {
        release();
        set_error("the octrees need more nodes than node_capacity (node_offsets[set_count] holds the count)");
        return NAN_ERR_LIMIT;
    }
    NodeEntries ne{(uint32_t*)get(m * 4ull), (uint32_t*)get(m * 4ull), (int*)get(m * 4ull), (uint32_t*)get(m * 4ull),
                   (uint8_t*)get(m), (uint8_t*)get(m), (uint8_t*)get(m)};
    uint32_t* nchild = (uint32_t*)get((m + 1) * 4ull);
    uint32_t* child_scan = (uint32_t*)get((m + 1) * 4ull);
    uint32_t* entry_set = (uint32_t*)get(m * 4ull);
    uint32_t* set_first = (uint32_t*)get((set_count + 1) * 4ull);
    uint32_t* local_id = (uint32_t*)get(m * 4ull);
    unsigned long long* leaf_key = (unsigned long long*)get(n * 8ull);
    size_t need2 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need2, nchild, child_scan, (int)(m + 1), st);
    void* tmp2 = get(need2);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "octree node scratch");
    }
    cudaMemcpyAsync(set_first, emit_host.data(), (set_count + 1) * 4ull, cudaMemcpyHostToDevice, st);
    k_oct_emit<<<blocks(n, 128), 128, 0, st>>>(keys_sorted, n, leaf_l, first_l, emit_off, ne);
    k_oct_masks<<<blocks(m, 256), 256, 0, st>>>(m, ne);
    k_oct_children<<<blocks(m, 256), 256, 0, st>>>(m, ne, nchild);
    cudaMemsetAsync(nchild + m, 0, 4, st);
    cub::DeviceScan::ExclusiveSum(tmp2, need2, nchild, child_scan, (int)(m + 1), st);
    k_oct_entry_sets<<<blocks(m, 256), 256, 0, st>>>(m, ne, keys_sorted, entry_set);
    k_oct_write<<<blocks(m, 256), 256, 0, st>>>(m, ne, child_scan, set_first, entry_set, set_begin, local_id,
                                               reinterpret_cast<uint4*>(nodes), status);
    // the output order: leaves in walk order, each leaf's points ascending
    k_oct_leaf_keys<<<blocks(n, 256), 256, 0, st>>>(keys_sorted, idx_sorted, n, leaf_l, leaf_key);
    k_oct_iota<<<blocks(n, 256), 256, 0, st>>>(n, idx);
    cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, leaf_key, keys, idx, idx_sorted, (int)n, 0, 64, st);
    k_oct_order<<<blocks(n, 256), 256, 0, st>>>(n, idx_sorted, set_of, set_begin, order);
    ctx->launches += 10;
    std::vector<double4> roots_host(set_count);
    cudaMemcpyAsync(roots_host.data(), root_dev, set_count * sizeof(double4), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    release();
    if (e != cudaSuccess) return cuda_fail(e, "point octree");
    if (host_status) {
        set_error("point octree: a node number fell outside its set");
        return NAN_ERR_LIMIT;
    }
    for (uint32_t k = 0; k < set_count; ++k) {
        roots[4 * k] = roots_host[k].x;
        roots[4 * k + 1] = roots_host[k].y;
        roots[4 * k + 2] = roots_host[k].z;
        roots[4 * k + 3] = roots_host[k].w;
    }
    return NAN_OK;
}

}  // namespace nan_host
