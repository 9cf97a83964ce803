// nan_wse.cu -- weighted sample elimination (Yuksel 2015) of surface-probe
// candidates on the GPU, for many candidate sets in one call
// (weighted_sample_elimination, surface_probes.py:897-985; C ABI
// surface_probe_wse_eliminate, surface_probe_sampler.h:120-223).
//
// Per set: d_max = max(2 sqrt(A / (2 sqrt(3) n_out)), 1e-6). Two candidates
// of a set are neighbours when 1e-20 < |d|^2 < d_max^2, their normals' dot is
// at least the cosine threshold and both plane distances |d . n| are at most
// max(d_max * plane_scale, 1e-8); the neighbour contributes (1 - |d|/d_max)^8
// to the other's weight (float64, rounded to integer units of 2^-50 so that
// every sum is exact and order-free). The reference removes the candidate of
// largest weight (lowest index on ties) and subtracts its contributions from
// its neighbours until n_out remain.
//
// The same elimination in parallel: every round removes, at once, each
// candidate whose (weight, -index) exceeds that of all its remaining
// neighbours. Such a candidate is removed before all of its neighbours in the
// sequential order too, and with exact sums its weight at removal is the one
// the sequential process sees; the sequential order is then (removal weight
// descending, index ascending), so the survivors are the last n_out of that
// order within each set.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "nan_internal.h"

namespace {

constexpr double kWseUnit = 1125899906842624.0;  // 2^50 units per unit of weight
constexpr uint32_t kWseMaxDegree = 8000;       // keeps every weight below 2^63 units
constexpr uint32_t kCellBits = 16;
constexpr int kCellLimit = 1 << kCellBits;

struct WseSet {
    double d_max, inv_cell, plane_limit;
    int cmin[3];
};

struct WseArgs {
    const float* pos;  // f32[N][3]
    const float* nrm;  // f32[N][3]
    const uint32_t* set_of;
    const WseSet* sets;
    double ncos;
    uint32_t n;
};

__device__ __forceinline__ void cell_of(const WseArgs& a, uint32_t i, const WseSet& s, int c[3]) {
    for (int k = 0; k < 3; ++k) c[k] = (int)floor((double)a.pos[3 * i + k] * s.inv_cell);
}

// Per set the smallest cell coordinate on each axis; lanes of one warp that
// share a set reduce first, so each warp issues one atomic per set and axis.
__global__ void k_wse_cells(WseArgs a, WseSet* sets, int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const uint32_t si = a.set_of[i];
    const double inv = sets[si].inv_cell;
    const unsigned group = __match_any_sync(__activemask(), si);
    const bool leader = (threadIdx.x & 31u) == (uint32_t)(__ffs(group) - 1);
    for (int k = 0; k < 3; ++k) {
        const double f = floor((double)a.pos[3 * i + k] * inv);
        int v = 0x7fffffff;
        if (f > -1.0e9 && f < 1.0e9) v = (int)f;
        else atomicOr(status, 1);
        const int m = __reduce_min_sync(group, v);
        if (leader) atomicMin(&sets[si].cmin[k], m);
    }
}

__global__ void k_wse_keys(WseArgs a, unsigned long long* keys, uint32_t* idx, int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const uint32_t si = a.set_of[i];
    const WseSet s = a.sets[si];
    int c[3];
    cell_of(a, i, s, c);
    unsigned long long key = (unsigned long long)si << 48;
    for (int k = 0; k < 3; ++k) {
        const int r = c[k] - s.cmin[k];
        if (r < 0 || r >= kCellLimit - 1) {
            atomicOr(status, 2);
            return;
        }
        key |= (unsigned long long)r << (32 - 16 * k);
    }
    keys[i] = key;
    idx[i] = i;
}

__device__ __forceinline__ uint32_t lower_bound_key(const unsigned long long* keys, uint32_t n,
                                                    unsigned long long k) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (keys[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Contribution of candidate j to candidate i in 2^-50 units (0: not neighbours).
__device__ __forceinline__ long long wse_contribution(const WseArgs& a, const WseSet& s, uint32_t i, uint32_t j) {
    const double dx = (double)a.pos[3 * j] - (double)a.pos[3 * i];
    const double dy = (double)a.pos[3 * j + 1] - (double)a.pos[3 * i + 1];
    const double dz = (double)a.pos[3 * j + 2] - (double)a.pos[3 * i + 2];
    const double d2 = (dx * dx + dy * dy) + dz * dz;
    if (!(d2 > 1e-20) || !(d2 < s.d_max * s.d_max)) return 0;
    const double nix = a.nrm[3 * i], niy = a.nrm[3 * i + 1], niz = a.nrm[3 * i + 2];
    const double njx = a.nrm[3 * j], njy = a.nrm[3 * j + 1], njz = a.nrm[3 * j + 2];
    const double ndot = (njx * nix + njy * niy) + njz * niz;
    if (!(ndot >= a.ncos)) return 0;
    const double pa = fabs((dx * nix + dy * niy) + dz * niz);
    const double pb = fabs((dx * njx + dy * njy) + dz * njz);
    if (!(pa <= s.plane_limit) || !(pb <= s.plane_limit)) return 0;
    const double base = fmax(1.0 - sqrt(d2) / s.d_max, 0.0);
    const double b2 = base * base;
    const double b4 = b2 * b2;
    return __double2ll_rn((b4 * b4) * kWseUnit);
}

// Walks the 3x3x3 cells around candidate i; kFill = false counts neighbours,
// kFill = true writes them and the initial weight.
template <bool kFill>
__global__ void k_wse_neighbors(WseArgs a, const unsigned long long* keys, const uint32_t* sorted_idx,
                                const uint32_t* offsets, uint32_t* degree, uint32_t* nbr, long long* contrib,
                                long long* weight, int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const uint32_t si = a.set_of[i];
    const WseSet s = a.sets[si];
    int c[3];
    cell_of(a, i, s, c);
    uint32_t count = 0;
    uint32_t out = kFill ? offsets[i] : 0u;
    long long w = 0;
    // keys order cells by (set, x, y, z): the three z-neighbours of one (x, y)
    // column are one contiguous key range, found by one search
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy) {
            const int r0 = c[0] + dx - s.cmin[0], r1 = c[1] + dy - s.cmin[1], rz = c[2] - s.cmin[2];
            if (r0 < 0 || r1 < 0) continue;
            const unsigned long long column = ((unsigned long long)si << 48) | ((unsigned long long)r0 << 32) |
                                              ((unsigned long long)r1 << 16);
            const unsigned long long lo = column | (unsigned long long)max(rz - 1, 0);
            const unsigned long long hi = column | (unsigned long long)(rz + 1);
            for (uint32_t k = lower_bound_key(keys, a.n, lo); k < a.n && keys[k] <= hi; ++k) {
                const uint32_t j = sorted_idx[k];
                if (j == i) continue;
                const long long q = wse_contribution(a, s, i, j);
                if (q <= 0) continue;
                if (kFill) {
                    nbr[out] = j;
                    contrib[out] = q;
                    ++out;
                    w += q;
                } else {
                    ++count;
                }
            }
        }
    if (kFill) {
        weight[i] = w;
    } else {
        if (count > kWseMaxDegree) {
            atomicOr(status, 4);
            count = 0;
        }
        degree[i] = count;
    }
}

__global__ void k_wse_mark(uint32_t n, const uint32_t* offsets, const uint32_t* nbr, const long long* weight,
                           const uint8_t* active, uint8_t* mark) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!active[i]) {
        mark[i] = 0;
        return;
    }
    const long long wi = weight[i];
    bool top = true;
    for (uint32_t e = offsets[i]; e < offsets[i + 1]; ++e) {
        const uint32_t j = nbr[e];
        if (!active[j]) continue;
        const long long wj = weight[j];
        if (!(wi > wj || (wi == wj && i < j))) {
            top = false;
            break;
        }
    }
    mark[i] = top ? 1 : 0;
}

__global__ void k_wse_remove(uint32_t n, const uint32_t* offsets, const uint32_t* nbr, const long long* contrib,
                             long long* weight, uint8_t* active, const uint8_t* mark, long long* key,
                             unsigned int* removed) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !mark[i]) return;
    active[i] = 0;
    key[i] = weight[i];
    atomicAdd(removed, 1u);
    for (uint32_t e = offsets[i]; e < offsets[i + 1]; ++e) {
        const uint32_t j = nbr[e];
        // a neighbour of a removed candidate is never removed in the same round
        if (active[j]) atomicAdd(reinterpret_cast<unsigned long long*>(weight + j),
                                 (unsigned long long)(-contrib[e]));
    }
}

__global__ void k_wse_order_keys(uint32_t n, const long long* key, const uint32_t* set_of,
                                 unsigned long long* order_key, uint32_t* idx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    order_key[i] = (unsigned long long)(0x7fffffffffffffffLL - key[i]);  // removal weight, descending
    idx[i] = i;
    (void)set_of;
}

__global__ void k_wse_set_of_sorted(uint32_t n, const uint32_t* idx, const uint32_t* set_of, uint32_t* out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) out[r] = set_of[idx[r]];
}

// Sorted by (set, removal weight desc, index asc): position r of set s is
// eliminated while r - begin(s) < count(s) - n_out(s).
__global__ void k_wse_keep(uint32_t n, const uint32_t* idx, const uint32_t* set_sorted, const uint32_t* set_begin,
                           const uint32_t* set_eliminate, uint8_t* keep) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint32_t s = set_sorted[r];
    keep[idx[r]] = (r - set_begin[s]) >= set_eliminate[s] ? 1 : 0;
}

template <class T>
cudaError_t alloc(T** p, size_t count, cudaStream_t s) {
    return cudaMallocAsync(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T), s);
}

uint32_t blocks(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

}  // namespace

namespace nan_host {

int launch_wse_eliminate(NanContext* ctx, const float* positions, const float* normals, const uint32_t* set_offsets,
                         uint32_t set_count, const uint32_t* output_counts, const float* surface_areas,
                         const NanWseOptions* opt, uint8_t* keep, float* poisson_radii, uint32_t* rounds_out,
                         cudaStream_t st) {
    const uint32_t n = set_offsets[set_count];
    std::vector<WseSet> host_sets(set_count);
    std::vector<uint32_t> set_of_host(n), begin_host(set_count), elim_host(set_count);
    for (uint32_t k = 0; k < set_count; ++k) {
        const uint32_t count = set_offsets[k + 1] - set_offsets[k];
        const uint32_t out = std::max(1u, std::min(output_counts[k], std::max(count, 1u)));
        const double r = std::sqrt(std::max((double)surface_areas[k], 1e-20) / (2.0 * std::sqrt(3.0) * (double)out));
        WseSet& s = host_sets[k];
        s.d_max = std::max(2.0 * r, 1e-6);
        s.inv_cell = 1.0 / std::max(s.d_max, 1e-8);
        s.plane_limit = std::max(s.d_max * (double)opt->plane_distance_scale, 1e-8);
        s.cmin[0] = s.cmin[1] = s.cmin[2] = 0x7fffffff;
        begin_host[k] = set_offsets[k];
        elim_host[k] = count > out ? count - out : 0u;
        if (poisson_radii)
            poisson_radii[k] = count == out ? (float)std::sqrt(std::max((double)surface_areas[k], 1e-20) / out)
                                            : (float)(s.d_max * 0.5);
        for (uint32_t i = set_offsets[k]; i < set_offsets[k + 1]; ++i) set_of_host[i] = k;
    }
    if (rounds_out) *rounds_out = 0;
    if (n == 0) return NAN_OK;

    WseSet* sets = nullptr;
    uint32_t *set_of = nullptr, *idx = nullptr, *idx_sorted = nullptr, *degree = nullptr, *offsets = nullptr;
    uint32_t *nbr = nullptr, *set_begin = nullptr, *set_elim = nullptr, *set_sorted = nullptr;
    unsigned long long *keys = nullptr, *keys_sorted = nullptr;
    long long *contrib = nullptr, *weight = nullptr, *rkey = nullptr;
    uint8_t *active = nullptr, *mark = nullptr;
    int* status = nullptr;
    unsigned int* removed = nullptr;
    void* tmp = nullptr;
    auto release = [&]() {
        for (void* p : {(void*)sets, (void*)set_of, (void*)idx, (void*)idx_sorted, (void*)degree, (void*)offsets,
                        (void*)nbr, (void*)set_begin, (void*)set_elim, (void*)set_sorted, (void*)keys,
                        (void*)keys_sorted, (void*)contrib, (void*)weight, (void*)rkey, (void*)active, (void*)mark,
                        (void*)status, (void*)removed, tmp})
            if (p) cudaFreeAsync(p, st);
    };
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
        return e == cudaSuccess;
    };
    ok(alloc(&sets, set_count, st));
    ok(alloc(&set_of, n, st));
    ok(alloc(&idx, n, st));
    ok(alloc(&idx_sorted, n, st));
    ok(alloc(&degree, n + 1, st));
    ok(alloc(&offsets, n + 1, st));
    ok(alloc(&keys, n, st));
    ok(alloc(&keys_sorted, n, st));
    ok(alloc(&weight, n, st));
    ok(alloc(&rkey, n, st));
    ok(alloc(&active, n, st));
    ok(alloc(&mark, n, st));
    ok(alloc(&status, 1, st));
    ok(alloc(&removed, 1, st));
    ok(alloc(&set_begin, set_count, st));
    ok(alloc(&set_elim, set_count, st));
    ok(alloc(&set_sorted, n, st));
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "wse scratch");
    }
    ok(cudaMemcpyAsync(sets, host_sets.data(), set_count * sizeof(WseSet), cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(set_of, set_of_host.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(set_begin, begin_host.data(), set_count * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(set_elim, elim_host.data(), set_count * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    ok(cudaMemsetAsync(status, 0, sizeof(int), st));
    WseArgs a{positions, normals, set_of, sets, (double)opt->normal_cosine_threshold, n};
    const uint32_t g = blocks(n, 256);
    k_wse_cells<<<g, 256, 0, st>>>(a, sets, status);
    k_wse_keys<<<g, 256, 0, st>>>(a, keys, idx, status);
    ctx->launches += 2;
    int host_status = 0;
    ok(cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    ok(cudaStreamSynchronize(st));
    if (e != cudaSuccess || host_status) {
        release();
        if (e != cudaSuccess) return cuda_fail(e, "wse cells");
        set_error(host_status & 2 ? "a candidate set spans more than 65535 cells of d_max on an axis"
                                  : "candidate positions must be finite");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    // sort candidates by (set, cell)
    size_t tmp_bytes = 0, need = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, need, keys, keys_sorted, idx, idx_sorted, (int)n, 0, 64, st);
    tmp_bytes = std::max(tmp_bytes, need);
    cub::DeviceScan::ExclusiveSum(nullptr, need, degree, offsets, (int)(n + 1), st);
    tmp_bytes = std::max(tmp_bytes, need);
    cub::DeviceRadixSort::SortPairs(nullptr, need, keys, keys_sorted, idx, idx_sorted, (int)n, 0, 64, st);
    tmp_bytes = std::max(tmp_bytes, need);
    uint32_t *tmp_u = nullptr;
    cub::DeviceRadixSort::SortPairs(nullptr, need, set_of, set_sorted, idx, tmp_u, (int)n, 0, 32, st);
    tmp_bytes = std::max(tmp_bytes, need);
    if (!ok(cudaMallocAsync(&tmp, std::max<size_t>(tmp_bytes, 1), st))) {
        release();
        return cuda_fail(e, "wse sort scratch");
    }
    cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys_sorted, idx, idx_sorted, (int)n, 0, 64, st);
    // neighbour lists
    k_wse_neighbors<false><<<g, 256, 0, st>>>(a, keys_sorted, idx_sorted, nullptr, degree, nullptr, nullptr, nullptr,
                                              status);
    ok(cudaMemsetAsync(degree + n, 0, sizeof(uint32_t), st));
    cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, degree, offsets, (int)(n + 1), st);
    uint32_t edges = 0;
    ok(cudaMemcpyAsync(&edges, offsets + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ok(cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    ok(cudaStreamSynchronize(st));
    if (e == cudaSuccess && host_status) {
        release();
        set_error("a candidate has more than 8000 neighbours within d_max");
        return NAN_ERR_LIMIT;
    }
    if (!ok(alloc(&nbr, edges, st)) || !ok(alloc(&contrib, edges, st))) {
        release();
        return cuda_fail(e, "wse neighbour lists");
    }
    k_wse_neighbors<true><<<g, 256, 0, st>>>(a, keys_sorted, idx_sorted, offsets, nullptr, nbr, contrib, weight,
                                             status);
    ok(cudaMemsetAsync(active, 1, n, st));
    ctx->launches += 2;
    // elimination rounds, until every candidate has its removal weight
    uint32_t rounds = 0, done = 0;
    ok(cudaMemsetAsync(removed, 0, sizeof(unsigned int), st));
    while (e == cudaSuccess && done < n) {
        for (int k = 0; k < 8; ++k) {
            k_wse_mark<<<g, 256, 0, st>>>(n, offsets, nbr, weight, active, mark);
            k_wse_remove<<<g, 256, 0, st>>>(n, offsets, nbr, contrib, weight, active, mark, rkey, removed);
            ctx->launches += 2;
            ++rounds;
        }
        ok(cudaMemcpyAsync(&done, removed, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
        ok(cudaStreamSynchronize(st));
        if (rounds > 4u * n + 64u) break;  // each round removes at least the global maximum
    }
    if (e == cudaSuccess && done < n) {
        release();
        set_error("weighted sample elimination did not finish");
        return NAN_ERR_LIMIT;
    }
    // order by (set, removal weight desc, index asc); stable sorts keep the index order
    k_wse_order_keys<<<g, 256, 0, st>>>(n, rkey, set_of, keys, idx);
    cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys_sorted, idx, idx_sorted, (int)n, 0, 64, st);
    k_wse_set_of_sorted<<<g, 256, 0, st>>>(n, idx_sorted, set_of, degree);
    cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, degree, set_sorted, idx_sorted, idx, (int)n, 0, 32, st);
    k_wse_keep<<<g, 256, 0, st>>>(n, idx, set_sorted, set_begin, set_elim, keep);
    ctx->launches += 3;
    ok(cudaGetLastError());
    release();
    if (rounds_out) *rounds_out = rounds;
    return e == cudaSuccess ? NAN_OK : cuda_fail(e, "wse");
}

}  // namespace nan_host
