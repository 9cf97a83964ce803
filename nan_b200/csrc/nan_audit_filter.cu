// nan_audit_filter.cu -- the audit/repair candidate filter of surface-probe
// placement on the GPU (surface_probe_filter_audit_repair_candidates,
// surface_probe_sampler.cpp:1736-1997; the Python form
// _deduplicate_audit_candidates and _exclude_selected_duplicates,
// surface_probes.py:782-832), for many candidate sets in one call.
//
// Audit points: candidates are bucketed by the cell floor(p / cell_size) of
// their set; within a cell, in index order, a candidate is kept unless its
// normal's dot with an already kept one of the cell reaches the cosine
// threshold. Stable-sorting (set, cell) keys of the index-ordered candidates
// gives each cell its members in index order, and one thread walks a cell.
//
// Repair candidates: a candidate is kept when no selected base site and no
// lower-indexed candidate of its set has the same position and normal bits.
// Entries (the selected base sites first, then the candidates by index) are
// stable-sorted by a 64-bit hash of (set, position bits, normal bits), so an
// entry's exact duplicates before it in that order sit before it in its hash
// run; a candidate scans back through its run and is kept when it finds none.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "nan_internal.h"

namespace {

struct FilterSets {
    const double* inv_cell;  // per set 1 / max(cell_size, 1e-8)
    int* cmin;               // per set smallest cell coordinate on each axis [S][3]
    uint32_t count;
    uint32_t axis_bits;      // bits of each axis in a cell key
};

struct FilterPoints {
    const float* pos;
    const float* nrm;
    const uint32_t* set;  // null: every point in set 0
    uint32_t n;
};

__device__ __forceinline__ uint32_t set_of(const FilterPoints& p, uint32_t i) { return p.set ? p.set[i] : 0u; }

__device__ __forceinline__ bool finite3(const float* v) {
    return isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]);
}

__global__ void k_flt_cmin(FilterPoints c, FilterSets s, int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const uint32_t k = set_of(c, i);
    if (k >= s.count) {
        atomicOr(status, 8);
        return;
    }
    if (!finite3(c.pos + 3 * i) || !finite3(c.nrm + 3 * i)) {
        atomicOr(status, 1);
        return;
    }
    const double inv = s.inv_cell[k];
    for (int a = 0; a < 3; ++a) {
        const double f = floor((double)c.pos[3 * i + a] * inv);
        if (!(f > -1.0e9 && f < 1.0e9)) {
            atomicOr(status, 2);
            return;
        }
        atomicMin(&s.cmin[3 * k + a], (int)f);
    }
}

__global__ void k_flt_cell_keys(FilterPoints c, FilterSets s, unsigned long long* keys, uint32_t* idx, int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    idx[i] = i;
    keys[i] = ~0ull;
    const uint32_t k = set_of(c, i);
    if (k >= s.count || !finite3(c.pos + 3 * i)) return;  // reported by k_flt_cmin
    const double inv = s.inv_cell[k];
    unsigned long long key = (unsigned long long)k;
    for (int a = 0; a < 3; ++a) {
        const long long r = (long long)floor((double)c.pos[3 * i + a] * inv) - s.cmin[3 * k + a];
        if (r < 0 || r >= (1ll << s.axis_bits) - 1) {  // the all-ones key marks a skipped candidate
            atomicOr(status, 2);
            return;
        }
        key = (key << s.axis_bits) | (unsigned long long)r;
    }
    keys[i] = key;
}

// One thread per cell: its members are sorted[q0 .. q1) in index order; the
// kept ones (the cell's representatives) are listed from reps[q0].
__global__ void k_flt_dedup(const unsigned long long* keys, const uint32_t* sorted, uint32_t n, const float* nrm,
                            double ncos, uint32_t* reps, uint8_t* audit) {
    const uint32_t q0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (q0 >= n || keys[q0] == ~0ull || (q0 > 0 && keys[q0 - 1] == keys[q0])) return;
    uint32_t kept = 0;
    for (uint32_t q = q0; q < n && keys[q] == keys[q0]; ++q) {
        const uint32_t i = sorted[q];
        const float* a = nrm + 3 * i;
        bool duplicate = false;
        for (uint32_t r = 0; r < kept && !duplicate; ++r) {
            const float* b = nrm + 3 * reps[q0 + r];
            const float d = (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
            duplicate = (double)d >= ncos;
        }
        if (!duplicate) {
            reps[q0 + kept++] = i;
            audit[i] = 1;
        }
    }
}

// Entry e < M is the selected base site base_selected[e]; entry M + i is
// candidate i.
struct FilterEntries {
    FilterPoints base, cand;
    const uint32_t* base_selected;
    uint32_t m;
};

// False for a selected base index out of range (reported, never read).
__device__ __forceinline__ bool entry_words(const FilterEntries& f, uint32_t e, uint32_t w[7]) {
    const FilterPoints& p = e < f.m ? f.base : f.cand;
    const uint32_t i = e < f.m ? f.base_selected[e] : e - f.m;
    if (e < f.m && i >= f.base.n) return false;
    w[0] = set_of(p, i);
    for (int a = 0; a < 3; ++a) {
        w[1 + a] = __float_as_uint(p.pos[3 * i + a]);
        w[4 + a] = __float_as_uint(p.nrm[3 * i + a]);
    }
    return true;
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x ^= x >> 31;
    x *= 0x7fb5d329728ea185ull;
    x ^= x >> 27;
    x *= 0x81dadef4bc2dd44dull;
    x ^= x >> 33;
    return x;
}

__global__ void k_flt_hash(FilterEntries f, unsigned long long* keys, uint32_t* idx, int* status) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= f.m + f.cand.n) return;
    idx[e] = e;
    uint32_t w[7];
    if (!entry_words(f, e, w)) {
        atomicOr(status, 4);
        keys[e] = 0;
        return;
    }
    unsigned long long h = 0x243f6a8885a308d3ull;
    for (int k = 0; k < 7; ++k) h = mix64(h ^ (w[k] + 0x9e3779b97f4a7c15ull * (unsigned long long)(k + 1)));
    keys[e] = h;
}

__global__ void k_flt_exclude(FilterEntries f, const unsigned long long* keys, const uint32_t* sorted,
                              uint8_t* repair) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= f.m + f.cand.n) return;
    const uint32_t e = sorted[q];
    if (e < f.m) return;
    uint32_t w[7], v[7];
    entry_words(f, e, w);
    for (uint32_t r = q; r > 0 && keys[r - 1] == keys[q]; --r) {
        if (!entry_words(f, sorted[r - 1], v)) continue;
        bool same = true;
        for (int k = 0; k < 7; ++k) same = same && v[k] == w[k];
        if (same) return;
    }
    repair[e - f.m] = 1;
}

uint32_t blocks(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

}  // namespace

namespace nan_host {

int launch_filter_audit_repair(NanContext* ctx, const float* cand_pos, const float* cand_nrm, const uint32_t* cand_set,
                               uint32_t cand_count, const float* base_pos, const float* base_nrm,
                               const uint32_t* base_set, uint32_t base_count, const uint32_t* base_selected,
                               uint32_t base_selected_count, uint32_t set_count, const double* cell_sizes,
                               double ncos, uint32_t* audit_indices, uint32_t* audit_count, uint32_t* repair_indices,
                               uint32_t* repair_count, cudaStream_t st) {
    std::vector<double> inv(set_count);
    for (uint32_t k = 0; k < set_count; ++k) inv[k] = 1.0 / std::max(cell_sizes[k], 1e-8);
    uint32_t set_bits = 0;
    while ((1ull << set_bits) < set_count) ++set_bits;
    const uint32_t axis_bits = std::min(21u, (64u - set_bits) / 3u);
    const uint32_t n = cand_count, m = base_selected_count, entries = m + n;

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
    double* inv_dev = (double*)get(set_count * sizeof(double));
    int* cmin = (int*)get(set_count * 3ull * sizeof(int));
    int* status = (int*)get(sizeof(int));
    unsigned long long* keys = (unsigned long long*)get(entries * 8ull);
    unsigned long long* keys_sorted = (unsigned long long*)get(entries * 8ull);
    uint32_t* idx = (uint32_t*)get(entries * 4ull);
    uint32_t* idx_sorted = (uint32_t*)get(entries * 4ull);
    uint32_t* reps = (uint32_t*)get(n * 4ull);
    uint8_t* audit = (uint8_t*)get(n);
    uint8_t* repair = (uint8_t*)get(n);
    uint32_t* counts = (uint32_t*)get(2 * sizeof(uint32_t));
    size_t tmp_bytes = 0, need = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, need, keys, keys_sorted, idx, idx_sorted, (int)entries, 0, 64, st);
    tmp_bytes = std::max(tmp_bytes, need);
    cub::DeviceSelect::Flagged(nullptr, need, thrust::counting_iterator<uint32_t>(0), audit, audit_indices, counts,
                               (int)n, st);
    tmp_bytes = std::max(tmp_bytes, need);
    void* tmp = get(tmp_bytes);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "candidate filter scratch");
    }
    cudaMemcpyAsync(inv_dev, inv.data(), set_count * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(cmin, 0x7f, set_count * 3ull * sizeof(int), st);
    cudaMemsetAsync(status, 0, sizeof(int), st);
    cudaMemsetAsync(audit, 0, n, st);
    cudaMemsetAsync(repair, 0, n, st);
    const FilterSets sets{inv_dev, cmin, set_count, axis_bits};
    const FilterPoints cand{cand_pos, cand_nrm, cand_set, n};
    const FilterPoints base{base_pos, base_nrm, base_set, base_count};
    const FilterEntries fe{base, cand, base_selected, m};

    // audit points: (set, cell) buckets walked in index order
    k_flt_cmin<<<blocks(n, 256), 256, 0, st>>>(cand, sets, status);
    k_flt_cell_keys<<<blocks(n, 256), 256, 0, st>>>(cand, sets, keys, idx, status);
    cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys_sorted, idx, idx_sorted, (int)n, 0, 64, st);
    k_flt_dedup<<<blocks(n, 128), 128, 0, st>>>(keys_sorted, idx_sorted, n, cand_nrm, ncos, reps, audit);
    // repair candidates: exact duplicates of a selected base site or of a
    // lower-indexed candidate are dropped
    k_flt_hash<<<blocks(entries, 256), 256, 0, st>>>(fe, keys, idx, status);
    cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys_sorted, idx, idx_sorted, (int)entries, 0, 64, st);
    k_flt_exclude<<<blocks(entries, 256), 256, 0, st>>>(fe, keys_sorted, idx_sorted, repair);
    cub::DeviceSelect::Flagged(tmp, tmp_bytes, thrust::counting_iterator<uint32_t>(0), audit, audit_indices, counts,
                               (int)n, st);
    cub::DeviceSelect::Flagged(tmp, tmp_bytes, thrust::counting_iterator<uint32_t>(0), repair, repair_indices,
                               counts + 1, (int)n, st);
    ctx->launches += 9;
    uint32_t host_counts[2] = {0, 0};
    int host_status = 0;
    cudaMemcpyAsync(host_counts, counts, sizeof(host_counts), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    release();
    if (e != cudaSuccess) return cuda_fail(e, "candidate filter");
    if (host_status) {
        set_error(host_status & 8   ? "a candidate set index is out of range"
                  : host_status & 4 ? "base_selected_indices contains an invalid index"
                  : host_status & 1 ? "candidate positions and normals must be finite"
                                    : "a candidate set spans too many audit cells on an axis");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    *audit_count = host_counts[0];
    *repair_count = host_counts[1];
    return NAN_OK;
}

}  // namespace nan_host
