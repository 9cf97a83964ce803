// nan_cache.cu -- learned radiance cache: a multiresolution hash encoding
// (16 levels x 2 FP16 features x 2^log2_table entries) feeding a ReLU MLP
// 48 -> 64 -> 64 -> 64 -> 64 -> 16 (3 outputs used: irradiance RGB), trained
// online with a relative L2 loss and Adam.
//
// The MLP runs on the 5th-generation tensor cores: BF16 operands in shared
// memory (interleaved core-matrix layout, nan_tcgen05.cuh), FP32
// accumulators in TMEM, one elected thread issuing tcgen05.mma and
// committing to an mbarrier that the CTA waits on (bounded). A tile is 128
// samples, one sample per thread; CTAs walk tiles persistently (inference
// CTAs hold two tiles that share one copy of the weights).
//
// Training (k_cache_train) runs forward and backward in one kernel. The
// activations of all five layers stay in shared memory. Weight gradients
// dW_i = delta_i^T a_i accumulate in TMEM across all the CTA's tiles, with
// the same shared tiles read as MN-major operands. Input gradients
// delta_i W_i use the weight images as MN-major operands, so no transposed
// copy exists. The hash-table gradient is scattered with float2 atomics.
//
// Method: Mueller et al., "Instant Neural Graphics Primitives with a
// Multiresolution Hash Encoding" (2022), sec. 3; Mueller et al., "Real-time
// Neural Radiance Caching for Path Tracing" (2021), sec. 4; Adam (Kingma and
// Ba 2015). The reference renderer has no learned cache.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "nan_internal.h"
#include "nan_tcgen05.cuh"

namespace {

using nan_host::cuda_fail;
using nan_host::set_error;
using namespace nbd;

constexpr int kLevels = 16;
constexpr int kInputs = 48;
constexpr int kHidden = 64;
constexpr int kTile = 128;
constexpr uint32_t kSpinLimit = 1u << 22;
constexpr uint32_t kStatusTensorWait = 8u;

// layer i: kRows[i] x kCols[i] weights (out x in), row-major in the master
// vector at kOff[i]; bf16 image at kImg[i] bytes (interleaved layout).
__host__ __device__ constexpr int rows_of(int i) { return i == 4 ? 16 : kHidden; }
__host__ __device__ constexpr int cols_of(int i) { return i == 0 ? kInputs : kHidden; }
__host__ __device__ constexpr int off_of(int i) { return i == 0 ? 0 : 3072 + (i - 1) * 4096; }
__host__ __device__ constexpr int img_of(int i) { return 2 * off_of(i); }
constexpr int kMlpParams = 16384;
constexpr int kImgBytes = 2 * kMlpParams;

struct CacheView {
    const __half2* table;  // [L][T] feature pairs
    float3 bmin;
    float3 inv_extent;
    uint32_t res[kLevels];
    uint32_t dense_mask;   // bit l: level l indexes densely
    uint32_t table_mask;   // T - 1
    uint32_t* status;
};

// Corner k of level l: table index and trilinear weight, in the oracle's
// float32 operation order.
struct LevelCell {
    uint32_t cx, cy, cz;
    float fx, fy, fz;
};

__device__ __forceinline__ float3 unit_position(const CacheView& c, float3 p) {
    float x = (p.x - c.bmin.x) * c.inv_extent.x;
    float y = (p.y - c.bmin.y) * c.inv_extent.y;
    float z = (p.z - c.bmin.z) * c.inv_extent.z;
    x = fminf(fmaxf(x, 0.0f), 1.0f);
    y = fminf(fmaxf(y, 0.0f), 1.0f);
    z = fminf(fmaxf(z, 0.0f), 1.0f);
    return make_float3(x, y, z);
}

__device__ __forceinline__ LevelCell level_cell(const CacheView& c, float3 u, int l) {
    const float r = (float)c.res[l];
    const float sx = __fmul_rn(u.x, r), sy = __fmul_rn(u.y, r), sz = __fmul_rn(u.z, r);
    const float cx = fminf(floorf(sx), r - 1.0f), cy = fminf(floorf(sy), r - 1.0f), cz = fminf(floorf(sz), r - 1.0f);
    LevelCell cell;
    cell.cx = (uint32_t)cx;
    cell.cy = (uint32_t)cy;
    cell.cz = (uint32_t)cz;
    cell.fx = __fsub_rn(sx, cx);
    cell.fy = __fsub_rn(sy, cy);
    cell.fz = __fsub_rn(sz, cz);
    return cell;
}

__device__ __forceinline__ uint32_t corner_index(const CacheView& c, const LevelCell& cell, int l, int k) {
    const uint32_t x = cell.cx + (k & 1), y = cell.cy + ((k >> 1) & 1), z = cell.cz + (k >> 2);
    uint32_t idx;
    if (c.dense_mask & (1u << l)) {
        const uint32_t s = c.res[l] + 1u;
        idx = x + y * s + z * s * s;
    } else {
        idx = x ^ (y * 2654435761u) ^ (z * 805459861u);
    }
    return idx & c.table_mask;
}

__device__ __forceinline__ float corner_weight(const LevelCell& cell, int k) {
    const float wx = (k & 1) ? cell.fx : __fsub_rn(1.0f, cell.fx);
    const float wy = (k & 2) ? cell.fy : __fsub_rn(1.0f, cell.fy);
    const float wz = (k & 4) ? cell.fz : __fsub_rn(1.0f, cell.fz);
    return __fmul_rn(__fmul_rn(wx, wy), wz);
}

// Network input row: 32 hash features, normal, 1, zeros (as float).
__device__ __forceinline__ void encode_row(const CacheView& c, float4 q0, float4 q1, float* x) {
    const float3 u = unit_position(c, make_float3(q0.x, q0.y, q0.z));
#pragma unroll 1
    for (int l = 0; l < kLevels; ++l) {
        const LevelCell cell = level_cell(c, u, l);
        const __half2* t = c.table + (size_t)l * (c.table_mask + 1u);
        float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float w = corner_weight(cell, k);
            const float2 f = __half22float2(__ldg(t + corner_index(c, cell, l, k)));
            a0 = __fadd_rn(a0, __fmul_rn(w, f.x));
            a1 = __fadd_rn(a1, __fmul_rn(w, f.y));
        }
        x[2 * l] = a0;
        x[2 * l + 1] = a1;
    }
    x[32] = q1.x;
    x[33] = q1.y;
    x[34] = q1.z;
    x[35] = 1.0f;
#pragma unroll
    for (int i = 36; i < kInputs; ++i) x[i] = 0.0f;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Store 8 consecutive values (columns c0..c0+7) of row r as bf16.
__device__ __forceinline__ void store8(unsigned char* tile, uint32_t r, uint32_t c0, uint32_t cols, const float* v) {
    uint4 w;
    w.x = pack_bf16(v[0], v[1]);
    w.y = pack_bf16(v[2], v[3]);
    w.z = pack_bf16(v[4], v[5]);
    w.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4*>(tile + tc::tile_offset(r, c0, cols)) = w;
}

__device__ __forceinline__ void load8(const unsigned char* tile, uint32_t r, uint32_t c0, uint32_t cols, float* v) {
    const uint4 w = *reinterpret_cast<const uint4*>(tile + tc::tile_offset(r, c0, cols));
    const uint32_t u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        v[2 * i] = __uint_as_float(u[i] << 16);
        v[2 * i + 1] = __uint_as_float(u[i] & 0xFFFF0000u);
    }
}

__device__ __forceinline__ void load_weights(unsigned char* s_w, const uint4* __restrict__ img) {
    uint4* d = reinterpret_cast<uint4*>(s_w);
    for (int i = threadIdx.x; i < kImgBytes / 16; i += blockDim.x) d[i] = __ldg(img + i);
}

// Issue the K/16 MMAs of one product D (+)= A B into TMEM.
__device__ __forceinline__ void issue_kmajor(uint32_t d, uint32_t a, uint32_t a_cols, uint32_t b, uint32_t b_cols,
                                             uint32_t k, uint32_t idesc, bool accumulate) {
    for (uint32_t kk = 0; kk < k / 16u; ++kk) {
        const uint64_t ad = tc::smem_desc(a + kk * 256u, 128u, a_cols * 16u);
        const uint64_t bd = tc::smem_desc(b + kk * 256u, 128u, b_cols * 16u);
        tc::mma_bf16(d, ad, bd, idesc, (accumulate || kk > 0) ? 1u : 0u);
    }
}

// ---------------------------------------------------------------------------
// Inference: out[q] = network(query q). With `image`, adds
// weight * max(out, 0) into image[pixel] instead (cached screen frames).
// ---------------------------------------------------------------------------
struct InferArgs {
    const float4* queries;  // 2 float4 per query: (position, pixel bits), (normal, 0)
    const float4* weights;  // optional: 1 float4 per query (rgb factor)
    uint32_t count;
    const uint32_t* count_dev;  // optional device-side count (overrides count when set)
    float4* out;            // [count] network output
    float4* image;          // optional accumulation target indexed by the query's pixel
};

// A CTA runs kSub tiles of 128 queries side by side (kSub x 128 threads):
// the tiles share one copy of the weight images, so more warps fit on an SM
// to wait on the hash gathers. Tile s accumulates in TMEM columns
// [64 s, 64 s + 64); its warps 4 s .. 4 s + 3 read lanes 32 (warp % 4) on.
template <int kSub>
constexpr int infer_smem() { return kImgBytes + kSub * kTile * kHidden * 2 + 64; }
// CTAs per SM that shared memory and the 512 TMEM columns allow.
template <int kSub>
constexpr int infer_ctas_per_sm() { return kSub == 1 ? 4 : kSub == 2 ? 3 : 2; }
// Measured render + inference time of a cached 1920x1080 frame on the
// 998k-triangle terrain: 1 tile 2.17 ms, 2 tiles 2.06 ms, 4 tiles 2.07 ms.
constexpr int kInferSub = 2;

template <int kSub>
__global__ void __launch_bounds__(kSub * kTile, infer_ctas_per_sm<kSub>())
    k_cache_infer(CacheView c, const uint4* __restrict__ img, InferArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr uint32_t kActTile = kTile * kHidden * 2;
    unsigned char* s_w = smem;
    const uint32_t warp = threadIdx.x >> 5, sub = warp >> 2, r = threadIdx.x & (kTile - 1);
    unsigned char* s_act = smem + kImgBytes + sub * kActTile;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kImgBytes + kSub * kActTile);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
    const uint32_t count = a.count_dev ? *a.count_dev : a.count;
    const uint32_t tiles = (count + kTile - 1) / kTile;
    const uint32_t groups = (tiles + kSub - 1) / kSub;
    if (blockIdx.x >= groups) return;

    load_weights(s_w, img);
    if (threadIdx.x == 0) tc::mbar_init(bar, 1);
    if (warp == 0) tc::tmem_alloc(tslot, 64 * kSub);
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t my_lane = tmem + (((warp & 3u) * 32u) << 16) + 64u * sub;
    const uint32_t w_addr = tc::smem_addr(s_w), act_addr = tc::smem_addr(smem + kImgBytes);
    uint32_t phase = 0;
    bool ok = true;

    for (uint32_t group = blockIdx.x; group < groups && ok; group += gridDim.x) {
        const uint32_t q = (group * kSub + sub) * kTile + r;
        const bool valid = q < count;
        {
            float x[kInputs];
            if (valid) {
                encode_row(c, a.queries[2 * q], a.queries[2 * q + 1], x);
            } else {
#pragma unroll
                for (int i = 0; i < kInputs; ++i) x[i] = 0.0f;
            }
#pragma unroll
            for (int c0 = 0; c0 < kInputs; c0 += 8) store8(s_act, r, c0, kInputs, x + c0);
        }
        for (int layer = 0; layer < 5 && ok; ++layer) {
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            __syncthreads();
            if (threadIdx.x == 0) {
                tc::fence_after_sync();
                const uint32_t n = rows_of(layer), k = cols_of(layer);
#pragma unroll
                for (int s = 0; s < kSub; ++s)
                    issue_kmajor(tmem + 64u * s, act_addr + s * kActTile, k, w_addr + img_of(layer), k, k,
                                 tc::idesc_bf16(128, n, 0, 0), false);
                tc::commit(bar);
            }
            ok = __syncthreads_and(tc::mbar_wait(bar, phase, kSpinLimit) ? 1 : 0) != 0;
            phase ^= 1u;
            tc::fence_after_sync();
            if (!ok) break;
            if (layer < 4) {
                // ReLU, bf16, written over the tile the finished MMA read
#pragma unroll
                for (int c0 = 0; c0 < kHidden; c0 += 16) {
                    float v[16];
                    tc::tmem_load16(my_lane + c0, v);
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i], 0.0f);
                    store8(s_act, r, c0, kHidden, v);
                    store8(s_act, r, c0 + 8, kHidden, v + 8);
                }
            } else {
                float v[16];
                tc::tmem_load16(my_lane, v);
                if (valid) {
                    if (a.image) {
                        const float4 w = a.weights[q];
                        const uint32_t pixel = __float_as_uint(a.queries[2 * q].w);
                        float4 o = a.image[pixel];
                        o.x = __fadd_rn(o.x, __fmul_rn(w.x, fmaxf(v[0], 0.0f)));
                        o.y = __fadd_rn(o.y, __fmul_rn(w.y, fmaxf(v[1], 0.0f)));
                        o.z = __fadd_rn(o.z, __fmul_rn(w.z, fmaxf(v[2], 0.0f)));
                        a.image[pixel] = o;
                    } else {
                        a.out[q] = make_float4(v[0], v[1], v[2], 0.0f);
                    }
                }
            }
        }
    }
    if (!ok && threadIdx.x == 0) atomicOr(c.status, kStatusTensorWait);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem, 64 * kSub);
}

// ---------------------------------------------------------------------------
// Training: forward + relative-L2 loss + backward for `count` samples.
// Gradients (of the loss averaged with `inv_batch`) are added into grad
// (MLP, float32 row-major) and table_grad (float2 per entry).
// ---------------------------------------------------------------------------
struct TrainArgs {
    const float4* queries;  // 2 float4 per sample
    const float4* targets;  // 1 float4 per sample (rgb, w < 0: no sample)
    uint32_t count;
    float batch;            // samples the loss is averaged over
    float inv_batch;        // 1 / batch
    float loss_eps;
    float* partials;        // [gridDim.x][16384] per-CTA weight gradients
    float2* table_grad;     // [L * T]
    float* loss;            // [1] sum of per-sample losses * inv_batch
};

// TMEM columns: forward accumulator, input-gradient accumulator, and the five
// weight-gradient accumulators (M = 64: rows live in lanes 0-15 of each warp
// quarter).
constexpr uint32_t kColFwd = 0, kColBwd = 64;
__host__ __device__ constexpr uint32_t dw_col(int i) { return 128u + 64u * (uint32_t)i; }
constexpr uint32_t kTrainTmemCols = 512;

constexpr int kActBytes0 = kTile * kInputs * 2;
constexpr int kActBytes = kTile * kHidden * 2;
constexpr int kTrainSmem = kImgBytes + kActBytes0 + 4 * kActBytes + kActBytes + 64;

__global__ void __launch_bounds__(kTile, 1) k_cache_train(CacheView c, const uint4* __restrict__ img, TrainArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* s_w = smem;
    unsigned char* s_act[5];
    s_act[0] = smem + kImgBytes;
    for (int i = 1; i < 5; ++i) s_act[i] = s_act[0] + kActBytes0 + (i - 1) * kActBytes;
    unsigned char* s_delta = s_act[4] + kActBytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(s_delta + kActBytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
    const uint32_t r = threadIdx.x, warp = r >> 5, lane = r & 31u;
    const uint32_t tiles = (a.count + kTile - 1) / kTile;
    if (blockIdx.x >= tiles) return;

    load_weights(s_w, img);
    if (r == 0) tc::mbar_init(bar, 1);
    if (warp == 0) tc::tmem_alloc(tslot, kTrainTmemCols);
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t my_lane = tmem + ((warp * 32u) << 16);
    const uint32_t w_addr = tc::smem_addr(s_w), delta_addr = tc::smem_addr(s_delta);
    uint32_t act_addr[5];
    for (int i = 0; i < 5; ++i) act_addr[i] = tc::smem_addr(s_act[i]);
    uint32_t phase = 0;
    bool ok = true, first = true;
    float loss = 0.0f;

    // one MMA group issued by thread 0, then the whole CTA waits for it
    auto sync_issue_wait = [&](auto issue) {
        tc::fence_smem_to_async();
        tc::fence_before_sync();
        __syncthreads();
        if (r == 0) {
            tc::fence_after_sync();
            issue();
            tc::commit(bar);
        }
        ok = __syncthreads_and(tc::mbar_wait(bar, phase, kSpinLimit) ? 1 : 0) != 0;
        phase ^= 1u;
        tc::fence_after_sync();
    };

    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const uint32_t q = tile * kTile + r;
        // a negative target .w marks a sample without a point; samples with
        // a non-finite target are skipped too
        bool valid = q < a.count;
        if (valid) {
            const float4 y = a.targets[q];
            valid = !(y.w < 0.0f) && isfinite(y.x) && isfinite(y.y) && isfinite(y.z);
        }
        float4 q0 = make_float4(0.f, 0.f, 0.f, 0.f), q1 = q0;
        {
            float x[kInputs];
            if (valid) {
                q0 = a.queries[2 * q];
                q1 = a.queries[2 * q + 1];
                encode_row(c, q0, q1, x);
            } else {
#pragma unroll
                for (int i = 0; i < kInputs; ++i) x[i] = 0.0f;
            }
#pragma unroll
            for (int c0 = 0; c0 < kInputs; c0 += 8) store8(s_act[0], r, c0, kInputs, x + c0);
        }
        // forward
        for (int layer = 0; layer < 5 && ok; ++layer) {
            sync_issue_wait([&] {
                const uint32_t n = rows_of(layer), k = cols_of(layer);
                issue_kmajor(tmem + kColFwd, act_addr[layer], k, w_addr + img_of(layer), k, k,
                             tc::idesc_bf16(128, n, 0, 0), false);
            });
            if (!ok) break;
            if (layer < 4) {
#pragma unroll
                for (int c0 = 0; c0 < kHidden; c0 += 16) {
                    float v[16];
                    tc::tmem_load16(my_lane + kColFwd + c0, v);
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i], 0.0f);
                    store8(s_act[layer + 1], r, c0, kHidden, v);
                    store8(s_act[layer + 1], r, c0 + 8, kHidden, v + 8);
                }
            } else {
                float v[16];
                tc::tmem_load16(my_lane + kColFwd, v);
                float d[64];
#pragma unroll
                for (int i = 0; i < 64; ++i) d[i] = 0.0f;
                if (valid) {
                    const float4 y = a.targets[q];
                    const float yy[3] = {y.x, y.y, y.z};
#pragma unroll
                    for (int ch = 0; ch < 3; ++ch) {
                        const float o = v[ch];
                        const float den = __fadd_rn(__fmul_rn(o, o), a.loss_eps);
                        const float e = __fsub_rn(o, yy[ch]);
                        loss = __fadd_rn(loss, __fmul_rn(__fdiv_rn(__fmul_rn(e, e), den), a.inv_batch));
                        d[ch] = __fdiv_rn(__fmul_rn(2.0f, e), __fmul_rn(den, a.batch));
                    }
                }
#pragma unroll
                for (int c0 = 0; c0 < 64; c0 += 8) store8(s_delta, r, c0, 64, d + c0);
            }
        }
        // backward
        for (int layer = 4; layer >= 0 && ok; --layer) {
            const uint32_t n_out = rows_of(layer), n_in = cols_of(layer);
            sync_issue_wait([&] {
                // dW += delta^T a: M = 64 (output rows, padded), N = n_in, K = 128 samples
                const uint32_t id_w = tc::idesc_bf16(64, n_in, 1, 1);
                for (uint32_t kk = 0; kk < kTile / 16u; ++kk) {
                    const uint64_t ad = tc::smem_desc(delta_addr + kk * 2u * 64u * 16u, 64u * 16u, 128u);
                    const uint64_t bd = tc::smem_desc(act_addr[layer] + kk * 2u * n_in * 16u, n_in * 16u, 128u);
                    tc::mma_bf16(tmem + dw_col(layer), ad, bd, id_w, (first && kk == 0) ? 0u : 1u);
                }
                // g = delta W: M = 128, N = n_in, K = n_out; W as an MN-major operand
                const uint32_t id_x = tc::idesc_bf16(128, n_in, 0, 1);
                for (uint32_t kk = 0; kk < n_out / 16u; ++kk) {
                    const uint64_t ad = tc::smem_desc(delta_addr + kk * 256u, 128u, 64u * 16u);
                    const uint64_t bd = tc::smem_desc(w_addr + img_of(layer) + kk * 2u * n_in * 16u, n_in * 16u, 128u);
                    tc::mma_bf16(tmem + kColBwd, ad, bd, id_x, kk > 0 ? 1u : 0u);
                }
            });
            if (!ok) break;
            if (layer > 0) {
                // delta of the layer below: g masked by its ReLU, as bf16
#pragma unroll
                for (int c0 = 0; c0 < kHidden; c0 += 16) {
                    float g[16], act[16];
                    tc::tmem_load16(my_lane + kColBwd + c0, g);
                    load8(s_act[layer], r, c0, kHidden, act);
                    load8(s_act[layer], r, c0 + 8, kHidden, act + 8);
#pragma unroll
                    for (int i = 0; i < 16; ++i) g[i] = act[i] > 0.0f ? g[i] : 0.0f;
                    store8(s_delta, r, c0, 64, g);
                    store8(s_delta, r, c0 + 8, 64, g + 8);
                }
            } else {
                float g[32];
                tc::tmem_load16(my_lane + kColBwd, g);
                tc::tmem_load16(my_lane + kColBwd + 16, g + 16);
                if (valid) {
                    const float3 u = unit_position(c, make_float3(q0.x, q0.y, q0.z));
                    const size_t T = (size_t)c.table_mask + 1u;
#pragma unroll 1
                    for (int l = 0; l < kLevels; ++l) {
                        const LevelCell cell = level_cell(c, u, l);
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            const float w = corner_weight(cell, k);
                            const uint32_t idx = corner_index(c, cell, l, k);
                            atomicAdd(a.table_grad + (size_t)l * T + idx,
                                      make_float2(__fmul_rn(w, g[2 * l]), __fmul_rn(w, g[2 * l + 1])));
                        }
                    }
                }
            }
        }
        first = false;
    }
    // flush the weight gradients accumulated over this CTA's tiles
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    // into this CTA's partial (summed by k_cache_reduce); zeros if it had no tile
    float* part = a.partials + (size_t)blockIdx.x * kMlpParams;
    for (int layer = 0; layer < 5; ++layer) {
        const int n_out = rows_of(layer), n_in = cols_of(layer);
        const int m = 16 * (int)warp + (int)lane;  // valid for lanes 0-15
        for (int c0 = 0; c0 < n_in; c0 += 16) {
            float v[16];
            tc::tmem_load16(my_lane + dw_col(layer) + c0, v);
            if (lane < 16 && m < n_out) {
                float4* gp = reinterpret_cast<float4*>(part + off_of(layer) + m * n_in + c0);
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    gp[i] = (ok && !first) ? make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3])
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
    }
    // loss: warp sums, one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0 && loss != 0.0f) atomicAdd(a.loss, loss);
    if (!ok && r == 0) atomicOr(c.status, kStatusTensorWait);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem, kTrainTmemCols);
}

// grad[i] += sum over CTAs of partials[c][i] (fixed order: deterministic).
__global__ void k_cache_reduce(const float* __restrict__ partials, int parts, float* __restrict__ grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    float acc = 0.0f;
    for (int c = 0; c < parts; ++c) acc += partials[(size_t)c * kMlpParams + i];
    grad[i] += acc;
}

// ---------------------------------------------------------------------------
// Adam over the MLP weights (also writing their bf16 images) and the hash
// table (also writing its fp16 copy); the gradient is cleared.
// ---------------------------------------------------------------------------
struct AdamArgs {
    float lr, beta1, beta2, eps, bc1, bc2;  // bc = 1 - beta^t
};

__device__ __forceinline__ float adam_one(float p, float& m, float& v, float g, const AdamArgs& h) {
    m = __fadd_rn(__fmul_rn(h.beta1, m), __fmul_rn(1.0f - h.beta1, g));
    v = __fadd_rn(__fmul_rn(h.beta2, v), __fmul_rn(1.0f - h.beta2, __fmul_rn(g, g)));
    const float mh = __fdiv_rn(m, h.bc1);
    const float vh = __fdiv_rn(v, h.bc2);
    return __fsub_rn(p, __fdiv_rn(__fmul_rn(h.lr, mh), __fadd_rn(__fsqrt_rn(vh), h.eps)));
}

__global__ void k_cache_adam_mlp(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                                 float* __restrict__ g, unsigned char* __restrict__ img, AdamArgs h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    float mi = m[i], vi = v[i];
    const float np = adam_one(p[i], mi, vi, g[i], h);
    p[i] = np;
    m[i] = mi;
    v[i] = vi;
    g[i] = 0.0f;
    int layer = 0;
    while (layer < 4 && i >= off_of(layer + 1)) ++layer;
    const int local = i - off_of(layer), cols = cols_of(layer);
    const int row = local / cols, col = local % cols;
    const __nv_bfloat16 b = __float2bfloat16_rn(np);
    *reinterpret_cast<__nv_bfloat16*>(img + img_of(layer) + tc::tile_offset(row, col, cols)) = b;
}

// kLazy: only the entries with a nonzero gradient pair in this step are
// updated (lazy Adam); the others keep their parameters and moments, and the
// pass reads just their gradient.
template <bool kLazy>
__global__ void k_cache_adam_table(float2* __restrict__ p, float2* __restrict__ m, float2* __restrict__ v,
                                   float2* __restrict__ g, __half2* __restrict__ t16, size_t n, AdamArgs h) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float2 gi = g[i];
        if (kLazy && gi.x == 0.0f && gi.y == 0.0f) continue;
        float2 pi = p[i], mi = m[i], vi = v[i];
        pi.x = adam_one(pi.x, mi.x, vi.x, gi.x, h);
        pi.y = adam_one(pi.y, mi.y, vi.y, gi.y, h);
        p[i] = pi;
        m[i] = mi;
        v[i] = vi;
        g[i] = make_float2(0.0f, 0.0f);
        t16[i] = __floats2half2_rn(pi.x, pi.y);
    }
}

// Images and fp16 copy from the master parameters (after a set).
__global__ void k_cache_publish(const float* __restrict__ p, unsigned char* __restrict__ img,
                                const float2* __restrict__ tp, __half2* __restrict__ t16, size_t n) {
    const size_t i0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i0 < (size_t)kMlpParams) {
        const int i = (int)i0;
        int layer = 0;
        while (layer < 4 && i >= off_of(layer + 1)) ++layer;
        const int local = i - off_of(layer), cols = cols_of(layer);
        *reinterpret_cast<__nv_bfloat16*>(img + img_of(layer) + tc::tile_offset(local / cols, local % cols, cols)) =
            __float2bfloat16_rn(p[i]);
    }
    for (size_t i = i0; i < n; i += (size_t)gridDim.x * blockDim.x) t16[i] = __floats2half2_rn(tp[i].x, tp[i].y);
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
namespace nan_host {

namespace {

CacheView cache_view(const NanCache* k) {
    CacheView c;
    c.table = reinterpret_cast<const __half2*>(k->table16);
    c.bmin = make_float3(k->cfg.bounds_min[0], k->cfg.bounds_min[1], k->cfg.bounds_min[2]);
    float inv[3];
    for (int i = 0; i < 3; ++i) {
        const float e = std::max(k->cfg.bounds_max[i] - k->cfg.bounds_min[i], 1e-20f);
        inv[i] = 1.0f / e;
    }
    c.inv_extent = make_float3(inv[0], inv[1], inv[2]);
    const uint64_t T = 1ull << k->cfg.log2_table;
    c.dense_mask = 0;
    for (int l = 0; l < kLevels; ++l) {
        c.res[l] = k->resolutions[l];
        const uint64_t s = (uint64_t)k->resolutions[l] + 1u;
        if (s * s * s <= T) c.dense_mask |= 1u << l;
    }
    c.table_mask = (uint32_t)(T - 1u);
    c.status = k->ctx->d_status;
    return c;
}

int sm_count(int device) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return sms;
}

}  // namespace

size_t cache_table_params(const NanCacheConfig* cfg) { return (size_t)kLevels * 2u * (1ull << cfg->log2_table); }
size_t cache_mlp_params() { return kMlpParams; }

int cache_create(NanContext* ctx, const NanCacheConfig* cfg, NanCache** out) {
    NanCache* k = new NanCache();
    k->ctx = ctx;
    k->cfg = *cfg;
    const double b = std::exp((std::log((double)cfg->max_resolution) - std::log((double)cfg->base_resolution)) /
                              (double)(kLevels - 1));
    for (int l = 0; l < kLevels; ++l)
        k->resolutions[l] = (uint32_t)std::floor((double)cfg->base_resolution * std::pow(b, (double)l));
    const size_t nt = cache_table_params(cfg);
    k->table_params = nt;
    cudaError_t err = cudaSuccess;
    auto grab = [&](void** p, size_t bytes) {
        if (err == cudaSuccess) err = cudaMalloc(p, bytes);
        if (err == cudaSuccess) err = cudaMemset(*p, 0, bytes);
    };
    grab(reinterpret_cast<void**>(&k->mlp), 4 * kMlpParams * sizeof(float));  // p, m, v, g
    grab(reinterpret_cast<void**>(&k->img), kImgBytes);
    grab(reinterpret_cast<void**>(&k->table), 4 * nt * sizeof(float));  // p, m, v, g
    grab(reinterpret_cast<void**>(&k->table16), nt * sizeof(__half));
    grab(reinterpret_cast<void**>(&k->loss), 16);
    grab(reinterpret_cast<void**>(&k->partials), (size_t)sm_count(ctx->device) * kMlpParams * sizeof(float));
    if (err == cudaSuccess) err = cudaFuncSetAttribute(k_cache_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       kTrainSmem);
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(k_cache_infer<kInferSub>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   infer_smem<kInferSub>());
    if (err != cudaSuccess) {
        cache_destroy(k);
        return cuda_fail(err, "cache allocation");
    }
    *out = k;
    return NAN_OK;
}

void cache_destroy(NanCache* k) {
    if (!k) return;
    cudaFree(k->mlp);
    cudaFree(k->img);
    cudaFree(k->table);
    cudaFree(k->table16);
    cudaFree(k->loss);
    cudaFree(k->partials);
    delete k;
}

int cache_set_params(NanCache* k, const float* mlp, const float* table, cudaStream_t st) {
    const size_t nt = k->table_params;
    cudaError_t err = cudaMemcpyAsync(k->mlp, mlp, kMlpParams * sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (err == cudaSuccess) err = cudaMemsetAsync(k->mlp + kMlpParams, 0, 3 * kMlpParams * sizeof(float), st);
    if (err == cudaSuccess) err = cudaMemcpyAsync(k->table, table, nt * sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (err == cudaSuccess) err = cudaMemsetAsync(k->table + nt, 0, 3 * nt * sizeof(float), st);
    if (err != cudaSuccess) return cuda_fail(err, "cache parameter upload");
    k->step = 0;
    const size_t pairs = nt / 2;
    const int blocks = (int)std::min<size_t>((pairs + 255) / 256, 148u * 16u);
    k_cache_publish<<<std::max(blocks, kMlpParams / 256), 256, 0, st>>>(
        k->mlp, k->img, reinterpret_cast<const float2*>(k->table), reinterpret_cast<__half2*>(k->table16), pairs);
    k->ctx->launches++;
    return cuda_fail(cudaGetLastError(), "cache publish");
}

int cache_get_params(NanCache* k, float* mlp, float* table, float* mlp_grad, float* table_grad, float* loss,
                     cudaStream_t st) {
    const size_t nt = k->table_params;
    cudaError_t err = cudaSuccess;
    if (mlp) err = cudaMemcpyAsync(mlp, k->mlp, kMlpParams * sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (err == cudaSuccess && table)
        err = cudaMemcpyAsync(table, k->table, nt * sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (err == cudaSuccess && mlp_grad)
        err = cudaMemcpyAsync(mlp_grad, k->mlp + 3 * kMlpParams, kMlpParams * sizeof(float), cudaMemcpyDeviceToDevice,
                              st);
    if (err == cudaSuccess && table_grad)
        err = cudaMemcpyAsync(table_grad, k->table + 3 * nt, nt * sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (err == cudaSuccess && loss) err = cudaMemcpyAsync(loss, k->loss, sizeof(float), cudaMemcpyDeviceToDevice, st);
    return cuda_fail(err, "cache parameter read");
}

int launch_cache_infer(NanCache* k, const float* queries, uint32_t count, const uint32_t* count_dev, float* out,
                       const float* weights, float* image, cudaStream_t st) {
    if (count == 0) return NAN_OK;
    InferArgs a;
    a.queries = reinterpret_cast<const float4*>(queries);
    a.weights = reinterpret_cast<const float4*>(weights);
    a.count = count;
    a.count_dev = count_dev;
    a.out = reinterpret_cast<float4*>(out);
    a.image = reinterpret_cast<float4*>(image);
    const uint32_t tiles = (count + kTile - 1) / kTile;
    const uint32_t groups = (tiles + kInferSub - 1) / kInferSub;
    const uint32_t grid =
        std::min<uint32_t>(groups, (uint32_t)sm_count(k->ctx->device) * infer_ctas_per_sm<kInferSub>());
    k_cache_infer<kInferSub><<<grid, kInferSub * kTile, infer_smem<kInferSub>(), st>>>(
        cache_view(k), reinterpret_cast<const uint4*>(k->img), a);
    k->ctx->launches++;
    return cuda_fail(cudaGetLastError(), "cache inference");
}

int launch_cache_backward(NanCache* k, const float* queries, const float* targets, uint32_t count, uint32_t batch,
                          cudaStream_t st) {
    if (count == 0) return NAN_OK;
    TrainArgs a;
    a.queries = reinterpret_cast<const float4*>(queries);
    a.targets = reinterpret_cast<const float4*>(targets);
    a.count = count;
    a.batch = (float)batch;
    a.inv_batch = (float)(1.0 / (double)batch);
    a.loss_eps = k->cfg.loss_epsilon;
    a.partials = k->partials;
    a.table_grad = reinterpret_cast<float2*>(k->table + 3 * k->table_params);
    a.loss = k->loss;
    const uint32_t tiles = (count + kTile - 1) / kTile;
    // one CTA per SM: 512 TMEM columns and 124 KB shared memory each
    const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)sm_count(k->ctx->device));
    k_cache_train<<<grid, kTile, kTrainSmem, st>>>(cache_view(k), reinterpret_cast<const uint4*>(k->img), a);
    k_cache_reduce<<<kMlpParams / 256, 256, 0, st>>>(k->partials, (int)grid, k->mlp + 3 * kMlpParams);
    k->ctx->launches += 2;
    return cuda_fail(cudaGetLastError(), "cache training");
}

int launch_cache_step(NanCache* k, cudaStream_t st) {
    k->step++;
    AdamArgs h;
    h.lr = k->cfg.learning_rate;
    h.beta1 = k->cfg.beta1;
    h.beta2 = k->cfg.beta2;
    h.eps = k->cfg.epsilon;
    h.bc1 = (float)(1.0 - std::pow((double)k->cfg.beta1, (double)k->step));
    h.bc2 = (float)(1.0 - std::pow((double)k->cfg.beta2, (double)k->step));
    float* m = k->mlp;
    k_cache_adam_mlp<<<kMlpParams / 256, 256, 0, st>>>(m, m + kMlpParams, m + 2 * kMlpParams, m + 3 * kMlpParams,
                                                       k->img, h);
    const size_t nt = k->table_params, pairs = nt / 2;
    float2* t = reinterpret_cast<float2*>(k->table);
    const int blocks = (int)std::min<size_t>((pairs + 255) / 256, (size_t)sm_count(k->ctx->device) * 16u);
    if (k->cfg.table_update == 1u)
        k_cache_adam_table<true><<<blocks, 256, 0, st>>>(t, t + pairs, t + 2 * pairs, t + 3 * pairs,
                                                         reinterpret_cast<__half2*>(k->table16), pairs, h);
    else
        k_cache_adam_table<false><<<blocks, 256, 0, st>>>(t, t + pairs, t + 2 * pairs, t + 3 * pairs,
                                                          reinterpret_cast<__half2*>(k->table16), pairs, h);
    k->ctx->launches += 2;
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaMemsetAsync(k->loss, 0, sizeof(float), st);
    return cuda_fail(err, "cache optimizer step");
}

}  // namespace nan_host
