// mlp.cuh — the surrogate's per-particle MLP (16 -> 64 -> 64 -> 3, SiLU) on
// the tcgen05 tensor cores: bf16 weights and activations, fp32 accumulation
// in TMEM. One CTA of 128 threads handles tiles of 128 particles; thread t
// owns row t of the tile (TMEM lane t).
//
// Model buffer (fp32, device), kMlpModelFloats floats:
//   [kW1, +16*64)  W1[in][out]   [kB1, +64) b1
//   [kW2, +64*64)  W2[in][out]   [kB2, +64) b2
//   [kW3, +64*3)   W3[in][out]   [kB3, +3)  b3
//   [kInMean, +16) feature means   [kInInvStd, +16) 1/std of the features
//   [kOutMean, +3) output means    [kOutStd, +3)    output stds
// The network sees (f - mean) * inv_std and its output y is de-normalised as
// y * out_std + out_mean. The fp32 weights are the training masters; each
// CTA rounds them to bf16 when it stages them in shared memory.
#pragma once

#include <cuda_bf16.h>

#include "umma.cuh"

namespace nsph {

constexpr int kMlpIn = 16;
constexpr int kMlpHid = 64;
constexpr int kMlpOut = 3;
constexpr int kMlpOutPad = 16;  // layer-3 MMA width (N >= 16)
constexpr int kMlpTile = 128;   // rows (particles) per tile = threads per CTA
constexpr int kW1 = 0;
constexpr int kB1 = kW1 + kMlpIn * kMlpHid;   // 1024
constexpr int kW2 = kB1 + kMlpHid;            // 1088
constexpr int kB2 = kW2 + kMlpHid * kMlpHid;  // 5184
constexpr int kW3 = kB2 + kMlpHid;            // 5248
constexpr int kB3 = kW3 + kMlpHid * kMlpOut;  // 5440
constexpr int kMlpParams = kB3 + kMlpOut;     // 5443 trainable
constexpr int kInMean = 5448;
constexpr int kInInvStd = kInMean + kMlpIn;
constexpr int kOutMean = kInInvStd + kMlpIn;
constexpr int kOutStd = kOutMean + 4;
constexpr int kMlpModelFloats = kOutStd + 4;  // 5488
constexpr int kMlpWaitLimit = 1 << 22;        // polls of an MMA-completion wait before giving up
constexpr uint32_t kMlpFwdCols = 64;          // inference TMEM: z1, z2 and the output in turn at column 0
constexpr int kTmemCols = 512;                // TMEM columns per SM

// shared memory of inference: one hidden tile serves both layers (layer 2's
// MMA has completed, so h1 is no longer read, before its epilogue writes
// silu(z2) over it), which keeps a CTA at about 34 KB
struct MlpFwdSmem {
    __nv_bfloat16 w1t[kMlpHid * kMlpIn];      // B of layer 1: [out][in], K = 16
    __nv_bfloat16 w2t[kMlpHid * kMlpHid];     // B of layer 2: [out][in], K = 64
    __nv_bfloat16 w3t[kMlpOutPad * kMlpHid];  // B of layer 3: [out (padded)][in], K = 64
    __nv_bfloat16 x[kMlpTile * kMlpIn];       // A of layer 1
    __nv_bfloat16 h1[kMlpTile * kMlpHid];     // A of layer 2 (silu(z1)), then of layer 3 (silu(z2))
    float b1[kMlpHid], b2[kMlpHid], b3[kMlpOutPad];
    float norm[kMlpModelFloats - kInMean];    // feature / output normalisation
    uint64_t bar;
    uint32_t tmem;
};

// the A tile of layer 3: its own buffer where the smem layout has one (the
// training kernel keeps silu(z2) for the weight gradients), else h1
template <class S>
__device__ __forceinline__ __nv_bfloat16* hidden2(S& s)
{
    return s.h2;
}
__device__ __forceinline__ __nv_bfloat16* hidden2(MlpFwdSmem& s) { return s.h1; }

__device__ __forceinline__ float tanh_approx(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// silu(z) = z * sigmoid(z), sigmoid(z) = (1 + tanh(z/2)) / 2
__device__ __forceinline__ float silu(float z)
{
    const float h = 0.5f * z;
    return fmaf(h, tanh_approx(h), h);
}

// d silu / dz = s (1 + z (1 - s)), s = sigmoid(z)
__device__ __forceinline__ float silu_grad(float z)
{
    const float s = fmaf(0.5f, tanh_approx(0.5f * z), 0.5f);
    return s * fmaf(z, 1.f - s, 1.f);
}

// all threads of the CTA: round the fp32 master weights to bf16 into the
// K-major core-matrix layouts, copy biases and normalisation constants
template <class S>
__device__ void mlp_stage_weights(const float* __restrict__ model, S& s)
{
    using umma::core_offset;
    for (int e = threadIdx.x; e < kMlpIn * kMlpHid; e += blockDim.x) {  // W1[i][o] -> w1t (o, i)
        const int i = e / kMlpHid, o = e % kMlpHid;
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(s.w1t) + core_offset(o, i, kMlpIn)) =
            __float2bfloat16_rn(model[kW1 + e]);
    }
    for (int e = threadIdx.x; e < kMlpHid * kMlpHid; e += blockDim.x) {  // W2[i][o] -> w2t (o, i)
        const int i = e / kMlpHid, o = e % kMlpHid;
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(s.w2t) + core_offset(o, i, kMlpHid)) =
            __float2bfloat16_rn(model[kW2 + e]);
    }
    for (int e = threadIdx.x; e < kMlpOutPad * kMlpHid; e += blockDim.x) {  // W3[i][o] -> w3t (o, i), o >= 3 zero
        const int o = e / kMlpHid, i = e % kMlpHid;
        const float w = o < kMlpOut ? model[kW3 + i * kMlpOut + o] : 0.f;
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(s.w3t) + core_offset(o, i, kMlpHid)) =
            __float2bfloat16_rn(w);
    }
    for (int e = threadIdx.x; e < kMlpHid; e += blockDim.x) {
        s.b1[e] = model[kB1 + e];
        s.b2[e] = model[kB2 + e];
    }
    for (int e = threadIdx.x; e < kMlpOutPad; e += blockDim.x) s.b3[e] = e < kMlpOut ? model[kB3 + e] : 0.f;
    for (int e = threadIdx.x; e < kMlpModelFloats - kInMean; e += blockDim.x) s.norm[e] = model[kInMean + e];
}

// store 8 consecutive bf16 values of row `row` (columns c0..c0+7, c0 % 8 == 0)
__device__ __forceinline__ void store_row8(__nv_bfloat16* tile, int row, int c0, int K, const float* v)
{
    __nv_bfloat162 p[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) p[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
    *reinterpret_cast<uint4*>(reinterpret_cast<char*>(tile) + umma::core_offset(row, c0, K)) =
        *reinterpret_cast<const uint4*>(p);
}

// CTA-wide barrier that also orders tcgen05 operations and makes this
// thread's shared-memory writes visible to the tensor core
__device__ __forceinline__ void mlp_sync()
{
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
}

// Layer epilogue: read this thread's 64 accumulator columns at `tcol`, add
// the bias, apply silu and store the row as bf16 into the next layer's A tile.
__device__ __forceinline__ void mlp_hidden_epilogue(uint32_t tmem_row, uint32_t tcol, const float* bias,
                                                    __nv_bfloat16* out_tile, int row)
{
#pragma unroll
    for (int c = 0; c < kMlpHid; c += 16) {
        float v[16];
        umma::tmem_ld16(tmem_row + tcol + c, v);
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = silu(v[j] + bias[c + j]);
        store_row8(out_tile, row, c, kMlpHid, v);
        store_row8(out_tile, row, c + 8, kMlpHid, v + 8);
    }
}

// Wait for the next completion of s.bar (all threads; the outcome is made
// uniform across the CTA). On success the phase advances; on failure it stays
// at the completion still outstanding, which the caller waits for (bounded)
// before it frees TMEM.
template <class S>
__device__ __forceinline__ bool mlp_wait(S& s, uint32_t& phase, int limit = kMlpWaitLimit)
{
    const bool ok = __syncthreads_and(umma::mbar_wait(&s.bar, phase, limit)) != 0;
    if (ok) phase ^= 1u;
    umma::fence_after_sync();
    return ok;
}

// Forward of one tile whose normalised bf16 inputs are already in s.x (and
// made visible with mlp_sync). Accumulators: z1 at TMEM column c1, z2 at c2,
// the output at c3 (each without bias); c2 may equal c1 and c3 may equal
// either, since each accumulator is read out before the next MMA is issued. Returns false if an MMA wait gave up
// (then no further MMA is issued). `phase` is the parity of the next
// completion of s.bar. `wait_limit` bounds each completion wait (polls).
template <class S>
__device__ bool mlp_forward_tile(S& s, uint32_t tmem, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t& phase,
                                 float (&y)[kMlpOut], int wait_limit = kMlpWaitLimit)
{
    using namespace umma;
    const int row = threadIdx.x;
    const uint32_t tmem_row = tmem + ((uint32_t)((threadIdx.x >> 5) * 32) << 16);
    const uint32_t xa = smem_addr(s.x), h1a = smem_addr(s.h1), h2a = smem_addr(hidden2(s));
    const uint32_t w1a = smem_addr(s.w1t), w2a = smem_addr(s.w2t), w3a = smem_addr(s.w3t);
    // layer 1: z1 = x W1 (K = 16, one MMA)
    if (threadIdx.x == 0) {
        mma_bf16(tmem + c1, smem_desc(xa, 128, 256), smem_desc(w1a, 128, 256), idesc_bf16_f32(128, kMlpHid), 0);
        mma_commit(&s.bar);
    }
    if (!mlp_wait(s, phase, wait_limit)) return false;
    mlp_hidden_epilogue(tmem_row, c1, s.b1, s.h1, row);
    mlp_sync();
    // layer 2: z2 = h1 W2 (K = 64, four MMAs)
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            mma_bf16(tmem + c2, smem_desc(h1a + 256 * k, 128, 1024), smem_desc(w2a + 256 * k, 128, 1024),
                     idesc_bf16_f32(128, kMlpHid), k > 0);
        mma_commit(&s.bar);
    }
    if (!mlp_wait(s, phase, wait_limit)) return false;
    mlp_hidden_epilogue(tmem_row, c2, s.b2, hidden2(s), row);
    mlp_sync();
    // layer 3: out = h2 W3 (K = 64, N = 16 of which 3 are used)
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            mma_bf16(tmem + c3, smem_desc(h2a + 256 * k, 128, 1024), smem_desc(w3a + 256 * k, 128, 1024),
                     idesc_bf16_f32(128, kMlpOutPad), k > 0);
        mma_commit(&s.bar);
    }
    if (!mlp_wait(s, phase, wait_limit)) return false;
    float v[16];
    tmem_ld16(tmem_row + c3, v);
#pragma unroll
    for (int o = 0; o < kMlpOut; ++o) y[o] = v[o] + s.b3[o];
    return true;
}

// Grid of an inference kernel: as many CTAs as can be resident at once, so
// every CTA runs in the first wave and strides over the tiles. Residency is
// computed from the kernel's registers (allocated per warp in units of 256),
// its shared memory (plus the per-CTA reservation) and the SM's TMEM columns;
// 0 on a CUDA error.
template <class K>
inline int mlp_resident_grid(K kernel, size_t smem, int device)
{
    cudaFuncAttributes fa;
    int sms = 0, smem_sm = 0, reserved = 0, regs_sm = 0;
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const int warp_regs = ((fa.numRegs * 32 + 255) / 256) * 256;
    const int by_regs = regs_sm / (warp_regs * (kMlpTile / 32));
    const int by_smem = smem_sm / (int)(smem + fa.sharedSizeBytes + reserved);
    int per_sm = by_regs < by_smem ? by_regs : by_smem;
    per_sm = per_sm > kTmemCols / (int)kMlpFwdCols ? kTmemCols / (int)kMlpFwdCols : per_sm;
    return (sms > 0 ? sms : 1) * (per_sm > 0 ? per_sm : 1);
}

// CTA start: stage the weights, initialise the barrier, allocate `ncols`
// TMEM columns (warp 0). Returns the TMEM base address.
template <class S>
__device__ uint32_t mlp_cta_begin(const float* __restrict__ model, S& s, uint32_t ncols)
{
    mlp_stage_weights(model, s);
    if (threadIdx.x == 0) umma::mbar_init(&s.bar, 1);
    if (threadIdx.x < 32) umma::tmem_alloc(&s.tmem, ncols);
    mlp_sync();
    return s.tmem;
}

// CTA end: if a completion is still outstanding (a wait gave up), wait for it
// once more (bounded), then free the TMEM columns (warp 0).
template <class S>
__device__ void mlp_cta_end(S& s, uint32_t tmem, uint32_t ncols, bool outstanding, uint32_t phase)
{
    if (outstanding) umma::mbar_wait(&s.bar, phase, kMlpWaitLimit);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (threadIdx.x < 32) umma::tmem_dealloc(tmem, ncols);
}

// stage one tile's inputs: feat (16 raw features of this thread's row) ->
// normalised bf16 row of s.x
template <class S>
__device__ __forceinline__ void mlp_stage_input(S& s, const float (&feat)[kMlpIn])
{
    float v[kMlpIn];
#pragma unroll
    for (int j = 0; j < kMlpIn; ++j) v[j] = (feat[j] - s.norm[j]) * s.norm[kMlpIn + j];
    store_row8(s.x, threadIdx.x, 0, kMlpIn, v);
    store_row8(s.x, threadIdx.x, 8, kMlpIn, v + 8);
}

// de-normalised output
template <class S>
__device__ __forceinline__ float mlp_denorm(const S& s, const float (&y)[kMlpOut], int o)
{
    return fmaf(y[o], s.norm[kOutStd - kInMean + o], s.norm[kOutMean - kInMean + o]);
}

// ---- inference with several tiles per CTA ------------------------------------
// kGroups groups of 128 threads share one copy of the weights; group g owns
// its input and hidden tiles, its completion barrier and TMEM columns
// [64 g, 64 g + 64). Groups synchronise on their own named barriers
// (ids 1 .. kGroups), so one group's MMA round trips overlap the other
// groups' work. TMEM lane quadrant q of a group is accessed by its warp
// q (warp index mod 4), as tcgen05.ld requires.
template <int kGroups>
struct MlpFwdGroupSmem {
    static_assert(kGroups == 2, "named barriers 1 and 2 serve two groups");
    __nv_bfloat16 w1t[kMlpHid * kMlpIn];
    __nv_bfloat16 w2t[kMlpHid * kMlpHid];
    __nv_bfloat16 w3t[kMlpOutPad * kMlpHid];
    __nv_bfloat16 x[kGroups][kMlpTile * kMlpIn];
    __nv_bfloat16 h1[kGroups][kMlpTile * kMlpHid];  // silu(z1), then silu(z2)
    float b1[kMlpHid], b2[kMlpHid], b3[kMlpOutPad];
    float norm[kMlpModelFloats - kInMean];
    uint64_t bar[kGroups];
    uint32_t tmem;
};

// named barrier of group g (id 1 + g, 128 threads), ordering this thread's
// shared-memory writes before the tensor core's reads and tcgen05 operations
// across the barrier
// (ids are immediates, so the kernel reserves only the barriers it names;
// groups 0 and 1)
__device__ __forceinline__ void mlp_group_sync(int g)
{
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    if (g == 0)
        asm volatile("barrier.cta.sync 1, 128;" ::: "memory");
    else
        asm volatile("barrier.cta.sync 2, 128;" ::: "memory");
    umma::fence_after_sync();
}

// AND of v over group g's 128 threads (named barrier 1 + g)
__device__ __forceinline__ bool mlp_group_and(bool v, int g)
{
    uint32_t r;
    if (g == 0)
        asm volatile(
            "{\n.reg .pred p, q;\nsetp.ne.u32 q, %1, 0;\nbarrier.cta.red.and.pred p, 1, 128, q;\n"
            "selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(r)
            : "r"((uint32_t)v)
            : "memory");
    else
        asm volatile(
            "{\n.reg .pred p, q;\nsetp.ne.u32 q, %1, 0;\nbarrier.cta.red.and.pred p, 2, 128, q;\n"
            "selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(r)
            : "r"((uint32_t)v)
            : "memory");
    return r != 0;
}

// wait for the next completion of group g's barrier (the outcome is uniform
// over the group); the phase advances on success
template <int kGroups>
__device__ __forceinline__ bool mlp_group_wait(MlpFwdGroupSmem<kGroups>& s, int g, uint32_t& phase, int limit)
{
    const bool ok = mlp_group_and(umma::mbar_wait(&s.bar[g], phase, limit), g);
    if (ok) phase ^= 1u;
    umma::fence_after_sync();
    return ok;
}

// stage group g's inputs: row `row` of its tile
template <int kGroups>
__device__ __forceinline__ void mlp_group_stage_input(MlpFwdGroupSmem<kGroups>& s, int g, int row,
                                                      const float (&feat)[kMlpIn])
{
    float v[kMlpIn];
#pragma unroll
    for (int j = 0; j < kMlpIn; ++j) v[j] = (feat[j] - s.norm[j]) * s.norm[kMlpIn + j];
    store_row8(s.x[g], row, 0, kMlpIn, v);
    store_row8(s.x[g], row, 8, kMlpIn, v + 8);
}

// forward of group g's tile (inputs staged and made visible with
// mlp_group_sync): z1, z2 and the output take the group's TMEM columns in
// turn; row 0 of the group issues the MMAs. Returns false if a wait gave up
// (then the group issues no further MMA).
template <int kGroups>
__device__ bool mlp_group_forward_tile(MlpFwdGroupSmem<kGroups>& s, int g, int row, uint32_t tmem, uint32_t& phase,
                                       float (&y)[kMlpOut], int wait_limit)
{
    using namespace umma;
    const uint32_t col = (uint32_t)(kMlpFwdCols * g);
    const uint32_t tmem_row = tmem + ((uint32_t)(((threadIdx.x >> 5) & 3) * 32) << 16);
    const uint32_t xa = smem_addr(s.x[g]), ha = smem_addr(s.h1[g]);
    const uint32_t w1a = smem_addr(s.w1t), w2a = smem_addr(s.w2t), w3a = smem_addr(s.w3t);
    if (row == 0) {
        mma_bf16(tmem + col, smem_desc(xa, 128, 256), smem_desc(w1a, 128, 256), idesc_bf16_f32(128, kMlpHid), 0);
        mma_commit(&s.bar[g]);
    }
    if (!mlp_group_wait(s, g, phase, wait_limit)) return false;
    mlp_hidden_epilogue(tmem_row, col, s.b1, s.h1[g], row);
    mlp_group_sync(g);
    if (row == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            mma_bf16(tmem + col, smem_desc(ha + 256 * k, 128, 1024), smem_desc(w2a + 256 * k, 128, 1024),
                     idesc_bf16_f32(128, kMlpHid), k > 0);
        mma_commit(&s.bar[g]);
    }
    if (!mlp_group_wait(s, g, phase, wait_limit)) return false;
    mlp_hidden_epilogue(tmem_row, col, s.b2, s.h1[g], row);
    mlp_group_sync(g);
    if (row == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            mma_bf16(tmem + col, smem_desc(ha + 256 * k, 128, 1024), smem_desc(w3a + 256 * k, 128, 1024),
                     idesc_bf16_f32(128, kMlpOutPad), k > 0);
        mma_commit(&s.bar[g]);
    }
    if (!mlp_group_wait(s, g, phase, wait_limit)) return false;
    float v[16];
    tmem_ld16(tmem_row + col, v);
#pragma unroll
    for (int o = 0; o < kMlpOut; ++o) y[o] = v[o] + s.b3[o];
    return true;
}

}  // namespace nsph
