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
//
// The adaptive elimination (_adaptive_weighted_sample_elimination_python,
// surface_probes.py:988-1088; C ABI surface_probe_wse_eliminate_adaptive)
// gives candidate i its own d_max_i = max(d_max / sqrt(density_i), 1e-6) and
// plane limit; j contributes to i under i's d_max, so "j is in i's list" is
// one-sided. The rounds then hold when a removed candidate lowers the
// candidates whose lists hold it (its out-list, the transposed lists) and a
// candidate is taken only when it tops both its lists.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "nan_internal.h"
#include "nan_math.cuh"
#include "nan_pairwise.h"

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
    const float* density;  // f32[N] relative densities (adaptive) or null
    double plane_scale;
};

// Candidate i's d_max and plane limit.
__device__ __forceinline__ void wse_radius(const WseArgs& a, const WseSet& s, uint32_t i, double* d_max,
                                           double* plane_limit) {
    if (!a.density) {
        *d_max = s.d_max;
        *plane_limit = s.plane_limit;
        return;
    }
    *d_max = fmax(s.d_max / sqrt((double)a.density[i]), 1e-6);
    *plane_limit = fmax(*d_max * a.plane_scale, 1e-8);
}

// Adaptive sets: the smallest density of each set (its largest d_max sizes
// the cells); densities must be finite and positive.
__global__ void k_wse_density_min(WseArgs a, unsigned int* min_bits, int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float d = a.density[i];
    if (!(d > 0.0f) || !(d <= 3.4028235e38f)) {
        atomicOr(status, 32);
        return;
    }
    atomicMin(min_bits + a.set_of[i], __float_as_uint(d));  // positive floats order as their bits
}

__global__ void k_wse_set_cells(uint32_t set_count, const unsigned int* min_bits, WseSet* sets) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= set_count || min_bits[k] == 0xffffffffu) return;
    const double cell = fmax(sets[k].d_max / sqrt((double)__uint_as_float(min_bits[k])), 1e-6);
    sets[k].inv_cell = 1.0 / fmax(cell, 1e-8);
}

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

// Contribution of candidate j to candidate i in 2^-50 units (0: not
// neighbours), under i's d_max and plane limit.
__device__ __forceinline__ long long wse_contribution(const WseArgs& a, double d_max, double plane_limit, uint32_t i,
                                                      uint32_t j) {
    const double dx = (double)a.pos[3 * j] - (double)a.pos[3 * i];
    const double dy = (double)a.pos[3 * j + 1] - (double)a.pos[3 * i + 1];
    const double dz = (double)a.pos[3 * j + 2] - (double)a.pos[3 * i + 2];
    const double d2 = (dx * dx + dy * dy) + dz * dz;
    if (!(d2 > 1e-20) || !(d2 < d_max * d_max)) return 0;
    const double nix = a.nrm[3 * i], niy = a.nrm[3 * i + 1], niz = a.nrm[3 * i + 2];
    const double njx = a.nrm[3 * j], njy = a.nrm[3 * j + 1], njz = a.nrm[3 * j + 2];
    const double ndot = (njx * nix + njy * niy) + njz * niz;
    if (!(ndot >= a.ncos)) return 0;
    const double pa = fabs((dx * nix + dy * niy) + dz * niz);
    const double pb = fabs((dx * njx + dy * njy) + dz * njz);
    if (!(pa <= plane_limit) || !(pb <= plane_limit)) return 0;
    const double base = fmax(1.0 - sqrt(d2) / d_max, 0.0);
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
    double d_max, plane_limit;
    wse_radius(a, s, i, &d_max, &plane_limit);
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
                const long long q = wse_contribution(a, d_max, plane_limit, i, j);
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

__device__ __forceinline__ bool wse_tops(uint32_t i, long long wi, const uint32_t* offsets, const uint32_t* nbr,
                                         const long long* weight, const uint8_t* active) {
    for (uint32_t e = offsets[i]; e < offsets[i + 1]; ++e) {
        const uint32_t j = nbr[e];
        if (!active[j]) continue;
        const long long wj = weight[j];
        if (!(wi > wj || (wi == wj && i < j))) return false;
    }
    return true;
}

// out_offsets / out_nbr: the transposed lists of the adaptive elimination
// (null when the relation is symmetric).
__global__ void k_wse_mark(uint32_t n, const uint32_t* offsets, const uint32_t* nbr, const uint32_t* out_offsets,
                           const uint32_t* out_nbr, const long long* weight, const uint8_t* active, uint8_t* mark) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!active[i]) {
        mark[i] = 0;
        return;
    }
    const long long wi = weight[i];
    bool top = wse_tops(i, wi, offsets, nbr, weight, active);
    if (top && out_offsets) top = wse_tops(i, wi, out_offsets, out_nbr, weight, active);
    mark[i] = top ? 1 : 0;
}

// A removed candidate lowers every remaining candidate whose list holds it
// (lose_offsets / lose_nbr / lose_contrib: the lists themselves when the
// relation is symmetric, else their transpose).
__global__ void k_wse_remove(uint32_t n, const uint32_t* lose_offsets, const uint32_t* lose_nbr,
                             const long long* lose_contrib, long long* weight, uint8_t* active, const uint8_t* mark,
                             long long* key, unsigned int* removed) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !mark[i]) return;
    active[i] = 0;
    key[i] = weight[i];
    atomicAdd(removed, 1u);
    for (uint32_t e = lose_offsets[i]; e < lose_offsets[i + 1]; ++e) {
        const uint32_t j = lose_nbr[e];
        // a candidate related to a removed one is never removed in the same round
        if (active[j]) atomicAdd(reinterpret_cast<unsigned long long*>(weight + j),
                                 (unsigned long long)(-lose_contrib[e]));
    }
}

__global__ void k_wse_out_degree(uint32_t n, const uint32_t* offsets, const uint32_t* nbr, uint32_t* out_degree) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (uint32_t e = offsets[i]; e < offsets[i + 1]; ++e) atomicAdd(out_degree + nbr[e], 1u);
}

__global__ void k_wse_out_fill(uint32_t n, const uint32_t* offsets, const uint32_t* nbr, const long long* contrib,
                               const uint32_t* out_offsets, uint32_t* cursor, uint32_t* out_nbr,
                               long long* out_contrib) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (uint32_t e = offsets[i]; e < offsets[i + 1]; ++e) {
        const uint32_t j = nbr[e];
        const uint32_t at = out_offsets[j] + atomicAdd(cursor + j, 1u);
        out_nbr[at] = i;
        out_contrib[at] = contrib[e];
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
    return nan_host::scratch_alloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T), s);
}

uint32_t blocks(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

// ---------------------------------------------------------------------------
// Deficit repair (deficit_repair_python, surface_probe_sampler.py:990-1103;
// C ABI surface_probe_deficit_repair, surface_probe_sampler.h:120-223).
// An audit point gathers probes of its own instance as the resolve does
// (_gather_weights_reference, :949-987: weight (1 - d^2/R^2)^2 x plane
// Gaussian x soft normal gate, kept above epsilon, the 32 largest); its
// deficit is min_gather - count. Repair candidates are then chosen one at a
// time by score = sum over the deficient audits a candidate reaches of
// (2 deficit - 1), highest first (lowest index on ties), each choice
// lowering the deficits it reaches by one, until the budget is spent or no
// score is positive. A score only falls when a candidate sharing one of its
// audits is chosen, so the same parallel rounds as the elimination give the
// sequential choices: every candidate whose (score, -index) tops those of
// all candidates sharing an audit with it is chosen at once.
// ---------------------------------------------------------------------------
constexpr float kRepairHardCos = 0.17364818f;

struct RepairSet {
    const float* pos;
    const float* nrm;
    const uint32_t* inst;
    uint32_t n;
};

struct RepairInst {
    double inv_cell;
    float r2;           // float32(R * R)
    float plane_sigma;  // float32(max(R / 4, 1e-6))
    int cmin[3];
};

struct RepairParams {
    const RepairInst* inst;
    uint32_t inst_count;
    float ncos_span;  // float32(max(threshold, hard + 1e-3) - hard)
    float eps;
    uint32_t min_gather;
};

__device__ __forceinline__ float rep_weight(const RepairParams& rp, const RepairInst& ri, const float* q,
                                            const float* qn, const float* p, const float* pn) {
    const float dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
    const float d2 = (dx * dx + dy * dy) + dz * dz;
    const float nc = (pn[0] * qn[0] + pn[1] * qn[1]) + pn[2] * qn[2];
    if (!(d2 <= ri.r2) || !(nc >= kRepairHardCos)) return 0.0f;
    const float pd = fabsf((dx * qn[0] + dy * qn[1]) + dz * qn[2]);
    const float t = pd / ri.plane_sigma;
    const float pw = nbd::nan_exp(-0.5f * (t * t));
    const float sp = fmaxf(1.0f - d2 / ri.r2, 0.0f);
    const float g = fminf(fmaxf((nc - kRepairHardCos) / rp.ncos_span, 0.0f), 1.0f);
    const float soft = ((g * g) * (3.0f - 2.0f * g)) * fmaxf(nc, 0.0f);
    const float w = ((sp * sp) * pw) * soft;
    return w > rp.eps ? w : 0.0f;
}

// numpy's float64 pairwise sum of float32 values (n <= 128: eight running
// partial sums, combined pairwise, then the remainder in order).
__device__ __forceinline__ double pairwise_sum(const float* v, uint32_t n, bool square) {
    auto at = [&](uint32_t i) { return square ? (double)(v[i] * v[i]) : (double)v[i]; };
    if (n < 8u) {
        double r = 0.0;
        for (uint32_t i = 0; i < n; ++i) r += at(i);
        return r;
    }
    double r[8];
    for (int j = 0; j < 8; ++j) r[j] = at(j);
    uint32_t i = 8;
    for (; i < n - (n % 8u); i += 8)
        for (int j = 0; j < 8; ++j) r[j] += at(i + j);
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; ++i) res += at(i);
    return res;
}

__global__ void k_rep_cmin(RepairSet set, RepairInst* inst, uint32_t inst_count, int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= set.n) return;
    const uint32_t k = set.inst[i];
    if (k >= inst_count) {
        atomicOr(status, 8);
        return;
    }
    const double inv = inst[k].inv_cell;
    const unsigned group = __match_any_sync(__activemask(), k);
    const bool leader = (threadIdx.x & 31u) == (uint32_t)(__ffs(group) - 1);
    for (int a = 0; a < 3; ++a) {
        const double f = floor((double)set.pos[3 * i + a] * inv);
        int v = 0x7fffffff;
        if (f > -1.0e9 && f < 1.0e9) v = (int)f;
        else atomicOr(status, 1);
        const int m = __reduce_min_sync(group, v);
        if (leader) atomicMin(&inst[k].cmin[a], m);
    }
}

__device__ __forceinline__ bool rep_cell(const RepairInst& ri, const float* p, int r[3]) {
    for (int a = 0; a < 3; ++a) {
        r[a] = (int)floor((double)p[a] * ri.inv_cell) - ri.cmin[a];
        if (r[a] < 0 || r[a] >= kCellLimit - 1) return false;
    }
    return true;
}

__global__ void k_rep_keys(RepairSet set, const RepairInst* inst, uint32_t inst_count, unsigned long long* keys,
                           uint32_t* idx, int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= set.n) return;
    const uint32_t k = set.inst[i];
    if (k >= inst_count) {
        atomicOr(status, 8);
        keys[i] = ~0ull;
        idx[i] = i;
        return;
    }
    int r[3];
    if (!rep_cell(inst[k], set.pos + 3 * i, r)) {
        atomicOr(status, 2);
        keys[i] = ~0ull;
        idx[i] = i;
        return;
    }
    keys[i] = ((unsigned long long)k << 48) | ((unsigned long long)r[0] << 32) | ((unsigned long long)r[1] << 16) |
              (unsigned long long)r[2];
    idx[i] = i;
}

struct RepairGrid {
    const unsigned long long* keys;  // sorted
    const uint32_t* idx;
    uint32_t n;
};

// Calls f(j) for every point of `g` in the 3x3x3 cells around the cell `c`
// of instance k.
template <class F>
__device__ __forceinline__ void rep_neighbourhood(const RepairGrid& g, uint32_t k, const int c[3], F f) {
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy) {
            const int r0 = c[0] + dx, r1 = c[1] + dy;
            if (r0 < 0 || r1 < 0) continue;
            const unsigned long long column = ((unsigned long long)k << 48) | ((unsigned long long)r0 << 32) |
                                              ((unsigned long long)r1 << 16);
            const unsigned long long lo = column | (unsigned long long)max(c[2] - 1, 0);
            const unsigned long long hi = column | (unsigned long long)(c[2] + 1);
            for (uint32_t q = lower_bound_key(g.keys, g.n, lo); q < g.n && g.keys[q] <= hi; ++q) f(g.idx[q]);
        }
}

// Per audit: the 32 largest weights over the base probes and, when given,
// the chosen repair candidates; count, float64 pairwise sum and ESS.
__global__ void k_rep_gather(RepairParams rp, RepairSet audits, RepairSet base, RepairGrid base_grid,
                             RepairSet extra, RepairGrid extra_grid, const uint8_t* extra_on, uint32_t* counts,
                             float* sums, float* ess) {
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= audits.n) return;
    const uint32_t k = audits.inst[a];
    const RepairInst ri = rp.inst[k];
    int c[3];
    float top[32];
    uint32_t n = 0;
    const float* q = audits.pos + 3 * a;
    const float* qn = audits.nrm + 3 * a;
    auto offer = [&](float w) {
        if (w <= 0.0f) return;
        if (n < 32u) {
            uint32_t j = n++;
            while (j > 0 && top[j - 1] < w) {
                top[j] = top[j - 1];
                --j;
            }
            top[j] = w;
        } else if (w > top[31]) {
            uint32_t j = 31;
            while (j > 0 && top[j - 1] < w) {
                top[j] = top[j - 1];
                --j;
            }
            top[j] = w;
        }
    };
    if (rep_cell(ri, q, c)) {
        rep_neighbourhood(base_grid, k, c, [&](uint32_t j) {
            offer(rep_weight(rp, ri, q, qn, base.pos + 3 * j, base.nrm + 3 * j));
        });
        if (extra_on != nullptr)
            rep_neighbourhood(extra_grid, k, c, [&](uint32_t j) {
                if (extra_on[j]) offer(rep_weight(rp, ri, q, qn, extra.pos + 3 * j, extra.nrm + 3 * j));
            });
    }
    counts[a] = n;
    const float s32 = (float)pairwise_sum(top, n, false);
    const double sq = pairwise_sum(top, n, true);
    sums[a] = s32;
    ess[a] = sq > 0.0 ? (float)(((double)s32 * (double)s32) / sq) : 0.0f;
}

// Candidate -> deficient audits it reaches (weight above epsilon).
template <bool kFill>
__global__ void k_rep_cover(RepairParams rp, RepairSet cand, RepairSet audits, RepairGrid audit_grid,
                            const int* deficit, const uint32_t* offsets, uint32_t* degree, uint32_t* list,
                            uint32_t* audit_degree) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cand.n) return;
    const uint32_t k = cand.inst[i];
    if (k >= rp.inst_count) {
        if (!kFill) degree[i] = 0;
        return;
    }
    const RepairInst ri = rp.inst[k];
    int c[3];
    uint32_t count = 0, out = kFill ? offsets[i] : 0u;
    if (rep_cell(ri, cand.pos + 3 * i, c)) {
        rep_neighbourhood(audit_grid, k, c, [&](uint32_t a) {
            if (deficit[a] <= 0) return;
            if (rep_weight(rp, ri, audits.pos + 3 * a, audits.nrm + 3 * a, cand.pos + 3 * i, cand.nrm + 3 * i) <=
                0.0f)
                return;
            if (kFill) {
                list[out++] = a;
            } else {
                ++count;
                atomicAdd(audit_degree + a, 1u);
            }
        });
    }
    if (!kFill) degree[i] = count;
}

__global__ void k_rep_transpose(uint32_t n, const uint32_t* offsets, const uint32_t* list,
                                const uint32_t* audit_offsets, uint32_t* audit_cursor, uint32_t* audit_list) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (uint32_t e = offsets[i]; e < offsets[i + 1]; ++e) {
        const uint32_t a = list[e];
        audit_list[audit_offsets[a] + atomicAdd(audit_cursor + a, 1u)] = i;
    }
}

__global__ void k_rep_score(uint32_t n, const uint32_t* offsets, const uint32_t* list, const int* deficit,
                            const uint8_t* chosen, long long* score, unsigned int* positive) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long s = 0;
    if (!chosen[i])
        for (uint32_t e = offsets[i]; e < offsets[i + 1]; ++e) {
            const int d = deficit[list[e]];
            if (d > 0) s += 2 * d - 1;
        }
    score[i] = s;
    if (s > 0) atomicAdd(positive, 1u);
}

__global__ void k_rep_mark(uint32_t n, const uint32_t* offsets, const uint32_t* list, const uint32_t* audit_offsets,
                           const uint32_t* audit_list, const long long* score, uint8_t* mark) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long si = score[i];
    bool top = si > 0;
    for (uint32_t e = offsets[i]; top && e < offsets[i + 1]; ++e) {
        const uint32_t a = list[e];
        for (uint32_t f = audit_offsets[a]; f < audit_offsets[a + 1]; ++f) {
            const uint32_t j = audit_list[f];
            if (j == i) continue;
            const long long sj = score[j];
            if (sj > 0 && !(si > sj || (si == sj && i < j))) {
                top = false;
                break;
            }
        }
    }
    mark[i] = top ? 1 : 0;
}

__global__ void k_rep_choose(uint32_t n, const uint32_t* offsets, const uint32_t* list, const long long* score,
                             const uint8_t* mark, int* deficit, uint8_t* chosen, long long* key) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !mark[i]) return;
    chosen[i] = 1;
    key[i] = score[i];
    // no two candidates chosen in one round share an audit
    for (uint32_t e = offsets[i]; e < offsets[i + 1]; ++e) {
        const uint32_t a = list[e];
        deficit[a] = max(deficit[a] - 1, 0);
    }
}

__global__ void k_rep_order_keys(uint32_t n, const uint8_t* chosen, const long long* key, unsigned long long* okey,
                                 uint32_t* idx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    okey[i] = chosen[i] ? (unsigned long long)(0x7fffffffffffffffLL - key[i]) : 0xffffffffffffffffull;
    idx[i] = i;
}

__global__ void k_rep_take(uint32_t take, const uint32_t* order, uint32_t* selected, uint8_t* on) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= take) return;
    selected[r] = order[r];
    on[order[r]] = 1;
}

__global__ void k_rep_count_chosen(uint32_t n, const uint8_t* chosen, unsigned int* total) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool c = i < n && chosen[i];
    const unsigned b = __ballot_sync(0xffffffffu, c);
    if ((threadIdx.x & 31u) == 0u && b) atomicAdd(total, (unsigned int)__popc(b));
}

// ---------------------------------------------------------------------------
// Support estimate (estimate_support_python, surface_probe_sampler.py:
// 1179-1260): per query site, support = sum over the reference points of its
// instance within R (normal past the hard gate) of kernel x area weight, the
// kernel as the gather's with values at or below epsilon set to 0; the sum in
// float64 over the points in ascending index order as numpy forms it for a
// float32 array summed in float64: the terms in buffers of 8192, each buffer
// summed by the pairwise scheme, the buffer sums added in order;
// f = clip(support / (pi R^2 / 3), 0, 1), m = min(M, 1 / max(f, 1/M)).
//
// The queries are grouped by (instance, grid cell). A cell's candidates --
// the reference points of its 3x3x3 neighbourhood, nine column ranges of
// the sorted grid -- are listed once and sorted by reference index, and one
// warp takes up to 32 of the cell's queries through that list in tiles of 32
// candidates staged in shared memory, so every lane tests the same candidate
// at the same step. A first pass counts each query's terms (the shape of the
// pairwise scheme depends on the count), a second feeds them to the sum.
// ---------------------------------------------------------------------------
constexpr uint32_t kSupportWarps = 4;    // warps per block of k_support_sum
constexpr unsigned long long kSupportBatch = 1ull << 26;  // list entries sorted at once

// numpy's float64 sum, fed one term at a time (nan_pairwise.h).
using PairwiseFeed = nan_pairwise::Feed;

// Reference points in index order as two float4: position and area weight,
// normal and 0.
__global__ void k_support_pack(RepairSet ref, const float* area, float4* packed) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ref.n) return;
    const float* p = ref.pos + 3 * (size_t)j;
    const float* n = ref.nrm + 3 * (size_t)j;
    packed[2 * (size_t)j] = make_float4(p[0], p[1], p[2], area[j]);
    packed[2 * (size_t)j + 1] = make_float4(n[0], n[1], n[2], 0.0f);
}

// Per query cell: the sorted-grid ranges of its nine neighbouring columns
// (three cells each), its candidate count and its number of 32-query warps.
// Keys are (instance 16 | x 16 | y 16 | z 16) bits, coordinates below 65535,
// so column + z + 2 is the first key past the column's cell z + 1.
__global__ void k_support_cells(uint32_t cells, const unsigned long long* cell_keys, const uint32_t* cell_queries,
                                RepairGrid g, uint32_t* range_b, uint32_t* range_e, unsigned long long* list_len,
                                uint32_t* warps) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= cells) return;
    const unsigned long long key = cell_keys[u];
    const int c0 = (int)((key >> 32) & 0xffffu), c1 = (int)((key >> 16) & 0xffffu), c2 = (int)(key & 0xffffu);
    const unsigned long long inst = (key >> 48) << 48;
    unsigned long long total = 0;
    int r = 0;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy, ++r) {
            uint32_t b = 0, e = 0;
            const int r0 = c0 + dx, r1 = c1 + dy;
            if (r0 >= 0 && r1 >= 0) {
                const unsigned long long column = inst + ((unsigned long long)r0 << 32) +
                                                  ((unsigned long long)r1 << 16);
                b = lower_bound_key(g.keys, g.n, column + (unsigned long long)max(c2 - 1, 0));
                e = lower_bound_key(g.keys, g.n, column + (unsigned long long)(c2 + 2));
            }
            range_b[9 * (size_t)u + r] = b;
            range_e[9 * (size_t)u + r] = e;
            total += e - b;
        }
    list_len[u] = total;
    warps[u] = (cell_queries[u] + 31u) / 32u;
}

// One block per cell of [u0, u1): its candidates as (cell - u0) << 32 |
// reference index, at its list offset; a key sort then orders each cell's
// list by reference index.
__global__ void k_support_fill(uint32_t u0, const uint32_t* range_b, const uint32_t* range_e,
                               const unsigned long long* list_off, const uint32_t* grid_idx,
                               unsigned long long* list_keys) {
    const uint32_t u = u0 + blockIdx.x;
    unsigned long long at = list_off[u] - list_off[u0];
    const unsigned long long tag = (unsigned long long)blockIdx.x << 32;
    for (int r = 0; r < 9; ++r) {
        const uint32_t b = range_b[9 * (size_t)u + r], e = range_e[9 * (size_t)u + r];
        for (uint32_t p = b + threadIdx.x; p < e; p += blockDim.x) list_keys[at + (p - b)] = tag | grid_idx[p];
        at += e - b;
    }
}

// The cell list's tile at t0 (m <= 32 entries) into this warp's shared tile.
__device__ __forceinline__ void support_tile(const unsigned long long* list, uint32_t t0, uint32_t m, uint32_t lane,
                                             const float4* packed, float4 (*tile)[2]) {
    __syncwarp();
    if (lane < m) {
        const size_t j = (uint32_t)list[t0 + lane];
        tile[lane][0] = packed[2 * j];
        tile[lane][1] = packed[2 * j + 1];
    }
    __syncwarp();
}

// One warp per (cell, 32 of its queries) of the cells [u0, u1); lane = query.
__global__ void __launch_bounds__(32 * kSupportWarps)
    k_support_sum(RepairParams rp, RepairSet query, const float4* packed, uint32_t u0, uint32_t u1,
                  const uint32_t* warp_off, const unsigned long long* cell_keys, const uint32_t* cell_first,
                  const uint32_t* cell_queries, const uint32_t* query_order, const unsigned long long* list_off,
                  const unsigned long long* list_keys, const double* flat_support, double max_density,
                  float* support_f, float* density_m) {
    __shared__ float4 tiles[kSupportWarps][32][2];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint32_t item = warp_off[u0] + blockIdx.x * kSupportWarps + w;
    if (item >= warp_off[u1]) return;  // the whole warp
    uint32_t lo = u0, hi = u1;         // warp_off[lo] <= item < warp_off[hi]
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (warp_off[mid] <= item) lo = mid;
        else hi = mid;
    }
    const uint32_t u = lo, chunk = item - warp_off[u];
    const bool active = lane < cell_queries[u] - 32u * chunk;
    const uint32_t qi = active ? query_order[cell_first[u] + 32u * chunk + lane] : 0u;
    const uint32_t k = (uint32_t)(cell_keys[u] >> 48);
    const RepairInst ri = rp.inst[k];
    const float q0 = query.pos[3 * (size_t)qi], q1 = query.pos[3 * (size_t)qi + 1], q2 = query.pos[3 * (size_t)qi + 2];
    const float n0 = query.nrm[3 * (size_t)qi], n1 = query.nrm[3 * (size_t)qi + 1], n2 = query.nrm[3 * (size_t)qi + 2];
    const unsigned long long* list = list_keys + (list_off[u] - list_off[u0]);
    const uint32_t len = (uint32_t)(list_off[u + 1] - list_off[u]);
    float4(*tile)[2] = tiles[w];

    uint32_t n = 0;
    for (uint32_t t0 = 0; t0 < len; t0 += 32u) {
        const uint32_t m = min(32u, len - t0);
        support_tile(list, t0, m, lane, packed, tile);
        if (active)
            for (uint32_t e = 0; e < m; ++e) {
                const float4 a = tile[e][0], b = tile[e][1];
                const float dx = a.x - q0, dy = a.y - q1, dz = a.z - q2;
                const float d2 = (dx * dx + dy * dy) + dz * dz;
                const float nc = (b.x * n0 + b.y * n1) + b.z * n2;
                n += (d2 <= ri.r2 && nc >= kRepairHardCos) ? 1u : 0u;
            }
    }
    PairwiseFeed sum;
    sum.begin(n);
    for (uint32_t t0 = 0; t0 < len; t0 += 32u) {
        const uint32_t m = min(32u, len - t0);
        support_tile(list, t0, m, lane, packed, tile);
        if (n)
            for (uint32_t e = 0; e < m; ++e) {
                const float4 a = tile[e][0], b = tile[e][1];
                const float dx = a.x - q0, dy = a.y - q1, dz = a.z - q2;
                const float d2 = (dx * dx + dy * dy) + dz * dz;
                const float nc = (b.x * n0 + b.y * n1) + b.z * n2;
                if (d2 <= ri.r2 && nc >= kRepairHardCos) {
                    const float t = ((dx * n0 + dy * n1) + dz * n2) / ri.plane_sigma;
                    const float pw = nbd::nan_exp(-0.5f * (t * t));
                    const float sp = fmaxf(1.0f - d2 / ri.r2, 0.0f);
                    const float g = fminf(fmaxf((nc - kRepairHardCos) / rp.ncos_span, 0.0f), 1.0f);
                    const float soft = ((g * g) * (3.0f - 2.0f * g)) * fmaxf(nc, 0.0f);
                    float kw = ((sp * sp) * pw) * soft;
                    kw = kw > rp.eps ? kw : 0.0f;
                    sum.push((double)(kw * a.w));
                }
            }
    }
    if (!active) return;
    const double flat = flat_support[k];
    const double v = fmin(fmax(sum.total / fmax(flat, 1e-30), 0.0), 1.0);
    support_f[qi] = (float)v;
    density_m[qi] = (float)fmin(max_density, 1.0 / fmax(v, 1.0 / max_density));
}

__global__ void k_rep_deficit(uint32_t n, const uint32_t* counts, uint32_t min_gather, int* deficit) {
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < n) deficit[a] = max((int)min_gather - (int)counts[a], 0);
}

}  // namespace

namespace nan_host {

int launch_wse_eliminate(NanContext* ctx, const float* positions, const float* normals, const float* densities,
                         const uint32_t* set_offsets, uint32_t set_count, const uint32_t* output_counts,
                         const float* surface_areas, const NanWseOptions* opt, uint8_t* keep, float* poisson_radii,
                         uint32_t* rounds_out, cudaStream_t st) {
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
            poisson_radii[k] = densities      ? (float)r
                               : count == out ? (float)std::sqrt(std::max((double)surface_areas[k], 1e-20) / out)
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
    unsigned int *removed = nullptr, *min_bits = nullptr;
    uint32_t *out_offsets = nullptr, *out_nbr = nullptr, *cursor = nullptr;
    long long* out_contrib = nullptr;
    void* tmp = nullptr;
    auto release = [&]() {
        for (void* p : {(void*)sets, (void*)set_of, (void*)idx, (void*)idx_sorted, (void*)degree, (void*)offsets,
                        (void*)nbr, (void*)set_begin, (void*)set_elim, (void*)set_sorted, (void*)keys,
                        (void*)keys_sorted, (void*)contrib, (void*)weight, (void*)rkey, (void*)active, (void*)mark,
                        (void*)status, (void*)removed, (void*)min_bits, (void*)out_offsets, (void*)out_nbr,
                        (void*)cursor, (void*)out_contrib, tmp})
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
    if (densities) {
        ok(alloc(&min_bits, set_count, st));
        ok(alloc(&out_offsets, n + 1, st));
        ok(alloc(&cursor, n, st));
    }
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "wse scratch");
    }
    ok(cudaMemcpyAsync(sets, host_sets.data(), set_count * sizeof(WseSet), cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(set_of, set_of_host.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(set_begin, begin_host.data(), set_count * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(set_elim, elim_host.data(), set_count * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    ok(cudaMemsetAsync(status, 0, sizeof(int), st));
    WseArgs a{positions, normals, set_of, sets, (double)opt->normal_cosine_threshold, n, densities,
              (double)opt->plane_distance_scale};
    const uint32_t g = blocks(n, 256);
    if (densities) {
        ok(cudaMemsetAsync(min_bits, 0xff, set_count * sizeof(unsigned int), st));
        k_wse_density_min<<<g, 256, 0, st>>>(a, min_bits, status);
        k_wse_set_cells<<<blocks(set_count, 128), 128, 0, st>>>(set_count, min_bits, sets);
        ctx->launches += 2;
    }
    k_wse_cells<<<g, 256, 0, st>>>(a, sets, status);
    k_wse_keys<<<g, 256, 0, st>>>(a, keys, idx, status);
    ctx->launches += 2;
    int host_status = 0;
    ok(cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    ok(cudaStreamSynchronize(st));
    if (e != cudaSuccess || host_status) {
        release();
        if (e != cudaSuccess) return cuda_fail(e, "wse cells");
        set_error(host_status & 32 ? "relative densities must be finite and positive"
                  : host_status & 2 ? "a candidate set spans more than 65535 cells of d_max on an axis"
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
    if (!ok(nan_host::scratch_alloc(&tmp, std::max<size_t>(tmp_bytes, 1), st))) {
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
    if (densities) {
        // transposed lists: who loses weight when a candidate goes
        ok(cudaMemsetAsync(degree, 0, (n + 1) * sizeof(uint32_t), st));
        ok(cudaMemsetAsync(cursor, 0, n * sizeof(uint32_t), st));
        k_wse_out_degree<<<g, 256, 0, st>>>(n, offsets, nbr, degree);
        cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, degree, out_offsets, (int)(n + 1), st);
        if (!ok(alloc(&out_nbr, edges, st)) || !ok(alloc(&out_contrib, edges, st))) {
            release();
            return cuda_fail(e, "wse transposed lists");
        }
        k_wse_out_fill<<<g, 256, 0, st>>>(n, offsets, nbr, contrib, out_offsets, cursor, out_nbr, out_contrib);
        ctx->launches += 2;
    }
    const uint32_t* lose_offsets = densities ? out_offsets : offsets;
    const uint32_t* lose_nbr = densities ? out_nbr : nbr;
    const long long* lose_contrib = densities ? out_contrib : contrib;
    // elimination rounds, until every candidate has its removal weight
    uint32_t rounds = 0, done = 0;
    ok(cudaMemsetAsync(removed, 0, sizeof(unsigned int), st));
    while (e == cudaSuccess && done < n) {
        for (int k = 0; k < 8; ++k) {
            k_wse_mark<<<g, 256, 0, st>>>(n, offsets, nbr, densities ? out_offsets : nullptr,
                                          densities ? out_nbr : nullptr, weight, active, mark);
            k_wse_remove<<<g, 256, 0, st>>>(n, lose_offsets, lose_nbr, lose_contrib, weight, active, mark, rkey,
                                            removed);
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

int launch_deficit_repair(NanContext* ctx, const float* const* base, const uint32_t* base_instances, uint32_t base_count,
                          const float* const* cand, const uint32_t* cand_instances, uint32_t cand_count,
                          const float* const* audit, const uint32_t* audit_instances, uint32_t audit_count,
                          const float* radii, uint32_t instance_count, const NanRepairOptions* opt, uint32_t* selected,
                          uint32_t* repair_count, uint32_t* counts_before, uint32_t* counts_after,
                          float* sums_before, float* sums_after, float* ess_before, float* ess_after,
                          uint32_t* rounds_out, cudaStream_t st) {
    std::vector<RepairInst> host_inst(instance_count);
    for (uint32_t k = 0; k < instance_count; ++k) {
        const double r = (double)radii[k];
        host_inst[k].inv_cell = 1.0 / std::max(r, 1e-8);
        host_inst[k].r2 = radii[k] * radii[k];
        host_inst[k].plane_sigma = (float)std::max(r * 0.25, 1e-6);
        host_inst[k].cmin[0] = host_inst[k].cmin[1] = host_inst[k].cmin[2] = 0x7fffffff;
    }
    const double hard = 0.17364817766693041;  // cos(80 degrees)
    const uint32_t limit = std::min(opt->max_repair_count, cand_count);
    RepairSet B{base[0], base[1], base_instances, base_count};
    RepairSet C{cand[0], cand[1], cand_instances, cand_count};
    RepairSet A{audit[0], audit[1], audit_instances, audit_count};
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
    RepairInst* inst = (RepairInst*)get(instance_count * sizeof(RepairInst));
    int* status = (int*)get(sizeof(int));
    unsigned long long* keys_in = (unsigned long long*)get(std::max({base_count, cand_count, audit_count}) * 8ull);
    uint32_t* idx_in = (uint32_t*)get(std::max({base_count, cand_count, audit_count}) * 4ull);
    unsigned long long* bkeys = (unsigned long long*)get(base_count * 8ull);
    uint32_t* bidx = (uint32_t*)get(base_count * 4ull);
    unsigned long long* ckeys = (unsigned long long*)get(cand_count * 8ull);
    uint32_t* cidx = (uint32_t*)get(cand_count * 4ull);
    unsigned long long* akeys = (unsigned long long*)get(audit_count * 8ull);
    uint32_t* aidx = (uint32_t*)get(audit_count * 4ull);
    int* deficit = (int*)get(audit_count * 4ull);
    uint32_t* cdeg = (uint32_t*)get((cand_count + 1) * 4ull);
    uint32_t* coff = (uint32_t*)get((cand_count + 1) * 4ull);
    uint32_t* adeg = (uint32_t*)get((audit_count + 1) * 4ull);
    uint32_t* aoff = (uint32_t*)get((audit_count + 1) * 4ull);
    uint32_t* acur = (uint32_t*)get(audit_count * 4ull);
    long long* score = (long long*)get(cand_count * 8ull);
    long long* key = (long long*)get(cand_count * 8ull);
    uint8_t* mark = (uint8_t*)get(cand_count);
    uint8_t* chosen = (uint8_t*)get(cand_count);
    uint8_t* on = (uint8_t*)get(cand_count);
    unsigned int* positive = (unsigned int*)get(64 * sizeof(unsigned int));
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "deficit repair scratch");
    }
    cudaMemcpyAsync(inst, host_inst.data(), instance_count * sizeof(RepairInst), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(status, 0, sizeof(int), st);
    for (const RepairSet* set : {&B, &C, &A})
        if (set->n) k_rep_cmin<<<blocks(set->n, 256), 256, 0, st>>>(*set, inst, instance_count, status);
    // sorted cell keys of each set
    size_t tmp_bytes = 0;
    const uint32_t nmax = std::max({base_count, cand_count, audit_count, 1u});
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys_in, bkeys, idx_in, bidx, (int)nmax, 0, 64, st);
    size_t need = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need, cdeg, coff, (int)(nmax + 1), st);
    tmp_bytes = std::max(tmp_bytes, need);
    void* tmp = get(tmp_bytes);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "deficit repair sort scratch");
    }
    const std::pair<const RepairSet*, std::pair<unsigned long long*, uint32_t*>> sets[3] = {
        {&B, {bkeys, bidx}}, {&C, {ckeys, cidx}}, {&A, {akeys, aidx}}};
    for (const auto& item : sets) {
        const RepairSet& set = *item.first;
        if (!set.n) continue;
        k_rep_keys<<<blocks(set.n, 256), 256, 0, st>>>(set, inst, instance_count, keys_in, idx_in, status);
        cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys_in, item.second.first, idx_in, item.second.second,
                                        (int)set.n, 0, 64, st);
    }
    int host_status = 0;
    cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess || host_status) {
        release();
        if (e != cudaSuccess) return cuda_fail(e, "deficit repair grids");
        set_error(host_status & 8 ? "an instance index is out of range"
                  : host_status & 2 ? "an instance spans more than 65535 kernel radii on an axis"
                                    : "positions must be finite");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    RepairParams rp{inst, instance_count,
                    (float)(std::max((double)opt->normal_cosine_threshold, hard + 1e-3) - hard), opt->weight_epsilon,
                    opt->min_gather_count};
    const RepairGrid BG{bkeys, bidx, base_count}, CG{ckeys, cidx, cand_count}, AG{akeys, aidx, audit_count};
    const uint32_t ga = blocks(audit_count, 128), gc = blocks(std::max(cand_count, 1u), 256);
    k_rep_gather<<<ga, 128, 0, st>>>(rp, A, B, BG, C, CG, nullptr, counts_before, sums_before, ess_before);
    k_rep_deficit<<<blocks(audit_count, 256), 256, 0, st>>>(audit_count, counts_before, opt->min_gather_count,
                                                             deficit);
    uint32_t rounds = 0, take = 0;
    if (cand_count && limit) {
        cudaMemsetAsync(adeg, 0, (audit_count + 1) * 4ull, st);
        cudaMemsetAsync(cdeg + cand_count, 0, 4, st);
        k_rep_cover<false><<<gc, 256, 0, st>>>(rp, C, A, AG, deficit, nullptr, cdeg, nullptr, adeg);
        cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cdeg, coff, (int)(cand_count + 1), st);
        cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, adeg, aoff, (int)(audit_count + 1), st);
        uint32_t pairs = 0;
        cudaMemcpyAsync(&pairs, coff + cand_count, 4, cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
        uint32_t* list = (uint32_t*)get(pairs * 4ull);
        uint32_t* alist = (uint32_t*)get(pairs * 4ull);
        if (e != cudaSuccess) {
            release();
            return cuda_fail(e, "deficit repair coverage");
        }
        k_rep_cover<true><<<gc, 256, 0, st>>>(rp, C, A, AG, deficit, coff, nullptr, list, nullptr);
        cudaMemsetAsync(acur, 0, audit_count * 4ull, st);
        k_rep_transpose<<<gc, 256, 0, st>>>(cand_count, coff, list, aoff, acur, alist);
        cudaMemsetAsync(chosen, 0, cand_count, st);
        cudaMemsetAsync(positive, 0, 64 * sizeof(unsigned int), st);
        // rounds, four at a time, until no candidate has a positive score
        for (;;) {
            for (int r = 0; r < 4; ++r) {
                k_rep_score<<<gc, 256, 0, st>>>(cand_count, coff, list, deficit, chosen, score,
                                                positive + ((rounds + r) & 63u));
                k_rep_mark<<<gc, 256, 0, st>>>(cand_count, coff, list, aoff, alist, score, mark);
                k_rep_choose<<<gc, 256, 0, st>>>(cand_count, coff, list, score, mark, deficit, chosen, key);
                ctx->launches += 3;
            }
            rounds += 4;
            unsigned int pos = 0;
            cudaMemcpyAsync(&pos, positive + ((rounds - 1) & 63u), sizeof(unsigned int), cudaMemcpyDeviceToHost, st);
            cudaMemsetAsync(positive + (rounds & 63u), 0, 4 * sizeof(unsigned int), st);
            e = cudaStreamSynchronize(st);
            if (e != cudaSuccess || pos == 0u) break;
            if (rounds > cand_count + 8u) {
                release();
                set_error("deficit repair did not finish");
                return NAN_ERR_LIMIT;
            }
        }
        if (e != cudaSuccess) {
            release();
            return cuda_fail(e, "deficit repair rounds");
        }
        // choices in sequential order: score at choice descending, index ascending
        unsigned long long* okey = keys_in;
        uint32_t* oidx = (uint32_t*)get(cand_count * 4ull);
        unsigned long long* okey_sorted = (unsigned long long*)get(cand_count * 8ull);
        uint32_t* oidx_sorted = (uint32_t*)get(cand_count * 4ull);
        if (e != cudaSuccess) {
            release();
            return cuda_fail(e, "deficit repair order");
        }
        k_rep_order_keys<<<gc, 256, 0, st>>>(cand_count, chosen, key, okey, oidx);
        cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, okey, okey_sorted, oidx, oidx_sorted, (int)cand_count, 0, 64,
                                        st);
        // how many were chosen
        unsigned int chosen_total = 0;
        {
            unsigned int* cnt = (unsigned int*)get(sizeof(unsigned int));
            cudaMemsetAsync(cnt, 0, sizeof(unsigned int), st);
            k_rep_count_chosen<<<gc, 256, 0, st>>>(cand_count, chosen, cnt);
            cudaMemcpyAsync(&chosen_total, cnt, sizeof(unsigned int), cudaMemcpyDeviceToHost, st);
            e = cudaStreamSynchronize(st);
        }
        take = std::min<uint32_t>(chosen_total, limit);
        cudaMemsetAsync(on, 0, cand_count, st);
        if (take) k_rep_take<<<blocks(take, 256), 256, 0, st>>>(take, oidx_sorted, selected, on);
    }
    k_rep_gather<<<ga, 128, 0, st>>>(rp, A, B, BG, C, CG, take ? on : nullptr, counts_after, sums_after, ess_after);
    ctx->launches += 12;
    e = cudaGetLastError();
    release();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    *repair_count = take;
    if (rounds_out) *rounds_out = rounds;
    return e == cudaSuccess ? NAN_OK : cuda_fail(e, "deficit repair");
}

int launch_estimate_support(NanContext* ctx, const float* ref_pos, const float* ref_nrm, const uint32_t* ref_inst,
                            const float* area_weights, uint32_t ref_count, const float* query_pos,
                            const float* query_nrm, const uint32_t* query_inst, uint32_t query_count,
                            const float* radii, uint32_t instance_count, const NanSupportOptions* opt,
                            float* support_f, float* density_m, cudaStream_t st) {
    std::vector<RepairInst> host_inst(instance_count);
    std::vector<double> flat(instance_count);
    for (uint32_t k = 0; k < instance_count; ++k) {
        const double r = (double)radii[k];
        host_inst[k].inv_cell = 1.0 / std::max(r, 1e-8);
        host_inst[k].r2 = radii[k] * radii[k];
        host_inst[k].plane_sigma = (float)std::max(r * 0.25, 1e-6);
        host_inst[k].cmin[0] = host_inst[k].cmin[1] = host_inst[k].cmin[2] = 0x7fffffff;
        flat[k] = 3.141592653589793 * r * r / 3.0;
    }
    const double hard = 0.17364817766693041;  // cos(80 degrees)
    RepairSet R{ref_pos, ref_nrm, ref_inst, ref_count};
    RepairSet Q{query_pos, query_nrm, query_inst, query_count};
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
    RepairInst* inst = (RepairInst*)get(instance_count * sizeof(RepairInst));
    double* flat_dev = (double*)get(instance_count * sizeof(double));
    // counters: [0] status, [1] query cells
    int* counters = (int*)get(2 * sizeof(int));
    const uint32_t nmax = std::max(ref_count, 1u), qmax = std::max(query_count, 1u);
    unsigned long long* keys_in = (unsigned long long*)get(std::max(nmax, qmax) * 8ull);
    uint32_t* idx_in = (uint32_t*)get(std::max(nmax, qmax) * 4ull);
    unsigned long long* rkeys = (unsigned long long*)get(nmax * 8ull);
    uint32_t* ridx = (uint32_t*)get(nmax * 4ull);
    float4* packed = (float4*)get(nmax * 32ull);
    unsigned long long* qkeys = (unsigned long long*)get(qmax * 8ull);
    uint32_t* qorder = (uint32_t*)get(qmax * 4ull);
    unsigned long long* cell_keys = (unsigned long long*)get(qmax * 8ull);
    uint32_t* cell_queries = (uint32_t*)get(qmax * 4ull);
    size_t tmp_bytes = 0, need = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, need, keys_in, rkeys, idx_in, ridx, (int)std::max(nmax, qmax), 0, 64,
                                    st);
    tmp_bytes = std::max(tmp_bytes, need);
    cub::DeviceRunLengthEncode::Encode(nullptr, need, qkeys, cell_keys, cell_queries, counters + 1, (int)qmax, st);
    tmp_bytes = std::max(tmp_bytes, need);
    void* tmp = get(tmp_bytes);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "support scratch");
    }
    cudaMemcpyAsync(inst, host_inst.data(), instance_count * sizeof(RepairInst), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(flat_dev, flat.data(), instance_count * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(counters, 0, 2 * sizeof(int), st);
    int* status = counters;
    for (const RepairSet* set : {&R, &Q})
        if (set->n) k_rep_cmin<<<blocks(set->n, 256), 256, 0, st>>>(*set, inst, instance_count, status);
    if (ref_count) {
        k_rep_keys<<<blocks(ref_count, 256), 256, 0, st>>>(R, inst, instance_count, keys_in, idx_in, status);
        cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys_in, rkeys, idx_in, ridx, (int)ref_count, 0, 64, st);
        k_support_pack<<<blocks(ref_count, 256), 256, 0, st>>>(R, area_weights, packed);
    }
    if (query_count) {
        k_rep_keys<<<blocks(query_count, 256), 256, 0, st>>>(Q, inst, instance_count, keys_in, idx_in, status);
        cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys_in, qkeys, idx_in, qorder, (int)query_count, 0, 64, st);
        cub::DeviceRunLengthEncode::Encode(tmp, tmp_bytes, qkeys, cell_keys, cell_queries, counters + 1,
                                           (int)query_count, st);
    }
    ctx->launches += 6;
    int host_counters[2] = {0, 0};
    cudaMemcpyAsync(host_counters, counters, sizeof(host_counters), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    const int host_status = host_counters[0];
    if (e != cudaSuccess || host_status) {
        release();
        if (e != cudaSuccess) return cuda_fail(e, "support grid");
        set_error(host_status & 8 ? "an instance index is out of range"
                  : host_status & 2 ? "an instance spans more than 65535 kernel radii on an axis"
                                    : "positions must be finite");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    const uint32_t cells = (uint32_t)host_counters[1];
    if (cells == 0) {
        release();
        return NAN_OK;
    }
    // per query cell: candidate ranges, list lengths and warps, and their
    // exclusive sums (cells + 1 entries: the last is the total)
    uint32_t* range_b = (uint32_t*)get(9ull * cells * 4);
    uint32_t* range_e = (uint32_t*)get(9ull * cells * 4);
    unsigned long long* list_len = (unsigned long long*)get((cells + 1ull) * 8);
    unsigned long long* list_off = (unsigned long long*)get((cells + 1ull) * 8);
    uint32_t* warps = (uint32_t*)get((cells + 1ull) * 4);
    uint32_t* warp_off = (uint32_t*)get((cells + 1ull) * 4);
    uint32_t* cell_first = (uint32_t*)get((cells + 1ull) * 4);
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need, list_len, list_off, (int)cells + 1, st);
    scan_bytes = std::max(scan_bytes, need);
    cub::DeviceScan::ExclusiveSum(nullptr, need, warps, warp_off, (int)cells + 1, st);
    scan_bytes = std::max(scan_bytes, need);
    void* scan_tmp = get(scan_bytes);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "support cell scratch");
    }
    const RepairGrid RG{rkeys, ridx, ref_count};
    cudaMemsetAsync(list_len + cells, 0, 8, st);
    cudaMemsetAsync(warps + cells, 0, 4, st);
    k_support_cells<<<blocks(cells, 128), 128, 0, st>>>(cells, cell_keys, cell_queries, RG, range_b, range_e,
                                                       list_len, warps);
    cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, list_len, list_off, (int)cells + 1, st);
    cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, warps, warp_off, (int)cells + 1, st);
    cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, cell_queries, cell_first, (int)cells, st);
    ctx->launches += 4;
    std::vector<unsigned long long> host_off(cells + 1ull);
    std::vector<uint32_t> host_warp_off(cells + 1ull);
    cudaMemcpyAsync(host_off.data(), list_off, (cells + 1ull) * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(host_warp_off.data(), warp_off, (cells + 1ull) * 4, cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "support cells");
    }
    // batches of whole cells of at most kSupportBatch list entries (a single
    // larger cell is a batch of its own)
    std::vector<uint32_t> cuts{0};
    while (cuts.back() < cells) {
        const uint32_t u0 = cuts.back();
        uint32_t u1 = u0 + 1;
        while (u1 < cells && host_off[u1 + 1] - host_off[u0] <= kSupportBatch) ++u1;
        if (host_off[u1] - host_off[u0] >= (1ull << 31)) {
            release();
            set_error("a query cell has 2^31 or more candidate reference points");
            return NAN_ERR_LIMIT;
        }
        cuts.push_back(u1);
    }
    unsigned long long widest = 0;
    for (size_t b = 0; b + 1 < cuts.size(); ++b) widest = std::max(widest, host_off[cuts[b + 1]] - host_off[cuts[b]]);
    unsigned long long* list_in = (unsigned long long*)get(std::max(widest, 1ull) * 8);
    unsigned long long* list_sorted = (unsigned long long*)get(std::max(widest, 1ull) * 8);
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, list_in, list_sorted, (int)std::max(widest, 1ull), 0, 64,
                                   st);
    void* sort_tmp = get(sort_bytes);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "support list scratch");
    }
    const RepairParams rp{inst, instance_count,
                          (float)(std::max((double)opt->normal_cosine_threshold, hard + 1e-3) - hard),
                          opt->weight_epsilon, 1u};
    const double max_density = std::max(1.0, (double)opt->max_density_multiplier);
    for (size_t b = 0; b + 1 < cuts.size(); ++b) {
        const uint32_t u0 = cuts[b], u1 = cuts[b + 1];
        const int count = (int)(host_off[u1] - host_off[u0]);
        const uint32_t batch_warps = host_warp_off[u1] - host_warp_off[u0];
        int end_bit = 32;
        for (uint32_t span = u1 - u0 - 1; span; span >>= 1) ++end_bit;
        if (count) {
            k_support_fill<<<u1 - u0, 128, 0, st>>>(u0, range_b, range_e, list_off, ridx, list_in);
            cub::DeviceRadixSort::SortKeys(sort_tmp, sort_bytes, list_in, list_sorted, count, 0, end_bit, st);
        }
        k_support_sum<<<blocks(batch_warps, kSupportWarps), 32 * kSupportWarps, 0, st>>>(
            rp, Q, packed, u0, u1, warp_off, cell_keys, cell_first, cell_queries, qorder, list_off, list_sorted,
            flat_dev, max_density, support_f, density_m);
        ctx->launches += count ? 3 : 1;
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    release();
    if (e != cudaSuccess) return cuda_fail(e, "support estimate");
    return NAN_OK;
}

}  // namespace nan_host
