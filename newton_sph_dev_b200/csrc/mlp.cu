// mlp.cu — batched inference, training gradient and Adam update of the
// surrogate MLP (mlp.cuh) on the tcgen05 tensor cores.
//
// Training of one batch (nsph_mlp_gradient): persistent CTAs of 128 threads
// stride over tiles of 128 samples. Per tile:
//   forward        three tcgen05 MMA chains (z1, z2, y stay in TMEM)
//   dY             2 (y - t) / (3 B) (mean squared error on normalised targets)
//   dZ2            (dY W3^T) * silu'(z2)            CUDA cores (K = 3)
//   dA1            dZ2 W2^T                          tcgen05, overlapped with:
//   dW2, dW3, db2, db3                               CUDA cores, fp32 accumulators
//   dZ1            dA1 * silu'(z1); dW1, db1         CUDA cores
// Each CTA keeps its gradient share in registers and writes it once; a
// second kernel sums the CTA partials in a fixed order (deterministic for a
// fixed launch shape). bf16 operands, fp32 accumulation throughout.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "mlp.cuh"
#include "nsph_internal.cuh"

namespace nsph {
namespace {

constexpr uint32_t kTrainCols = 256;  // training TMEM: z1 @0, z2 @64, y @128, dA1 @192
constexpr int kPartialStride = kMlpParams + 1;  // gradient + loss per CTA

struct MlpTrainSmem {
    __nv_bfloat16 w1t[kMlpHid * kMlpIn];
    __nv_bfloat16 w2t[kMlpHid * kMlpHid];
    __nv_bfloat16 w3t[kMlpOutPad * kMlpHid];
    __nv_bfloat16 x[kMlpTile * kMlpIn];
    __nv_bfloat16 h1[kMlpTile * kMlpHid];
    __nv_bfloat16 h2[kMlpTile * kMlpHid];
    __nv_bfloat16 w2b[kMlpHid * kMlpHid];  // B of dA1 = dZ2 W2^T: [in][out], K = 64 (out)
    __nv_bfloat16 g2[kMlpTile * kMlpHid];  // dZ2 (A of the dA1 MMA)
    __nv_bfloat16 g1[kMlpTile * kMlpHid];  // dZ1
    float w3f[kMlpHid * kMlpOut];          // W3 rounded to bf16, in fp32
    float dy[kMlpTile * 4];
    float b1[kMlpHid], b2[kMlpHid], b3[kMlpOutPad];
    float norm[kMlpModelFloats - kInMean];
    uint64_t bar;
    uint32_t tmem;
};

__device__ __forceinline__ float bf(const __nv_bfloat16* tile, int row, int col, int K)
{
    return __bfloat162float(
        *reinterpret_cast<const __nv_bfloat16*>(reinterpret_cast<const char*>(tile) + umma::core_offset(row, col, K)));
}

// 8 consecutive bf16 of a row (c0 % 8 == 0) as fp32
__device__ __forceinline__ void ld_row8(const __nv_bfloat16* tile, int row, int c0, int K, float* v)
{
    const uint4 u = *reinterpret_cast<const uint4*>(reinterpret_cast<const char*>(tile) + umma::core_offset(row, c0, K));
    const __nv_bfloat162* p = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float2 f = __bfloat1622float2(p[j]);
        v[2 * j] = f.x;
        v[2 * j + 1] = f.y;
    }
}

__global__ void __launch_bounds__(kMlpTile, 1) k_mlp_forward(const float* __restrict__ model,
                                                             const float* __restrict__ feat, int n,
                                                             float* __restrict__ out, unsigned* __restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    MlpFwdSmem& s = *reinterpret_cast<MlpFwdSmem*>(smem_raw);
    const uint32_t tmem = mlp_cta_begin(model, s, kMlpFwdCols);
    uint32_t phase = 0;
    bool ok = true;
    const int tiles = (n + kMlpTile - 1) / kMlpTile;
    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int r = t * kMlpTile + threadIdx.x;
        float f[kMlpIn];
#pragma unroll
        for (int j = 0; j < kMlpIn; ++j) f[j] = r < n ? feat[(size_t)r * kMlpIn + j] : 0.f;
        mlp_stage_input(s, f);
        mlp_sync();
        float y[kMlpOut];
        ok = mlp_forward_tile(s, tmem, 0, 0, 0, phase, y);
        if (ok && r < n)
            for (int o = 0; o < kMlpOut; ++o) out[(size_t)r * kMlpOut + o] = mlp_denorm(s, y, o);
        __syncthreads();
    }
    if (!ok && threadIdx.x == 0) atomicOr(err, 1u);
    mlp_cta_end(s, tmem, kMlpFwdCols, !ok, phase);
}

__global__ void __launch_bounds__(kMlpTile, 1) k_mlp_grad(const float* __restrict__ model,
                                                          const float* __restrict__ feat,
                                                          const float* __restrict__ target,
                                                          const int* __restrict__ idx, int batch,
                                                          float* __restrict__ partials, unsigned* __restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    MlpTrainSmem& s = *reinterpret_cast<MlpTrainSmem*>(smem_raw);
    using umma::core_offset;
    // extra operands of the backward pass
    for (int e = threadIdx.x; e < kMlpHid * kMlpHid; e += blockDim.x) {  // W2[i][o] -> w2b (i, o)
        const int i = e / kMlpHid, o = e % kMlpHid;
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(s.w2b) + core_offset(i, o, kMlpHid)) =
            __float2bfloat16_rn(model[kW2 + e]);
    }
    for (int e = threadIdx.x; e < kMlpHid * kMlpOut; e += blockDim.x)
        s.w3f[e] = __bfloat162float(__float2bfloat16_rn(model[kW3 + e]));
    const uint32_t tmem = mlp_cta_begin(model, s, kTrainCols);
    const int t = threadIdx.x;
    const uint32_t tmem_row = tmem + ((uint32_t)((t >> 5) * 32) << 16);
    const float inv3b = 1.f / (3.f * (float)batch);
    // this thread's gradient share
    const int o64 = t & 63, half = t >> 6;
    float gw2[32], gw1[8], gw3[3] = {0.f, 0.f, 0.f}, gb1 = 0.f, gb2 = 0.f, gb3 = 0.f, loss = 0.f;
#pragma unroll
    for (int j = 0; j < 32; ++j) gw2[j] = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) gw1[j] = 0.f;
    uint32_t phase = 0;
    bool ok = true;
    const int tiles = (batch + kMlpTile - 1) / kMlpTile;
    for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const int b = tile * kMlpTile + t;
        const bool valid = b < batch;
        const int row = valid ? idx[b] : 0;
        float f[kMlpIn], tg[kMlpOut];
#pragma unroll
        for (int j = 0; j < kMlpIn; ++j) f[j] = valid ? feat[(size_t)row * kMlpIn + j] : 0.f;
#pragma unroll
        for (int o = 0; o < kMlpOut; ++o)
            tg[o] = valid ? (target[(size_t)row * kMlpOut + o] - s.norm[kOutMean - kInMean + o]) /
                                s.norm[kOutStd - kInMean + o]
                          : 0.f;
        mlp_stage_input(s, f);
        mlp_sync();
        float y[kMlpOut];
        ok = mlp_forward_tile(s, tmem, 0, 64, 128, phase, y);
        if (!ok) break;
        // dY and the loss
        float dyv[kMlpOut];
#pragma unroll
        for (int o = 0; o < kMlpOut; ++o) {
            const float e = valid ? y[o] - tg[o] : 0.f;
            loss = fmaf(e, e, loss);
            dyv[o] = 2.f * e * inv3b;
            s.dy[t * 4 + o] = dyv[o];
        }
        // dZ2 = (dY W3^T) * silu'(z2), stored as bf16 (A of the dA1 MMA)
#pragma unroll
        for (int c = 0; c < kMlpHid; c += 16) {
            float z[16];
            umma::tmem_ld16(tmem_row + 64 + c, z);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const float* w = s.w3f + (c + j) * kMlpOut;
                const float da = fmaf(dyv[0], w[0], fmaf(dyv[1], w[1], dyv[2] * w[2]));
                z[j] = da * silu_grad(z[j] + s.b2[c + j]);
            }
            store_row8(s.g2, t, c, kMlpHid, z);
            store_row8(s.g2, t, c + 8, kMlpHid, z + 8);
        }
        mlp_sync();
        // dA1 = dZ2 W2^T on the tensor core ...
        if (t == 0) {
            const uint32_t ga = umma::smem_addr(s.g2), wa = umma::smem_addr(s.w2b);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                umma::mma_bf16(tmem + 192, umma::smem_desc(ga + 256 * k, 128, 1024),
                               umma::smem_desc(wa + 256 * k, 128, 1024), umma::idesc_bf16_f32(128, kMlpHid), k > 0);
            umma::mma_commit(&s.bar);
        }
        // ... while the CUDA cores accumulate dW2, dW3, db2, db3
        for (int r = 0; r < kMlpTile; ++r) {
            const float g = bf(s.g2, r, o64, kMlpHid);
#pragma unroll
            for (int c = 0; c < 32; c += 8) {
                float h[8];
                ld_row8(s.h1, r, half * 32 + c, kMlpHid, h);
#pragma unroll
                for (int j = 0; j < 8; ++j) gw2[c + j] = fmaf(h[j], g, gw2[c + j]);
            }
            if (half == 0) {
                gb2 += g;
                const float h2v = bf(s.h2, r, o64, kMlpHid);
#pragma unroll
                for (int o = 0; o < kMlpOut; ++o) gw3[o] = fmaf(h2v, s.dy[r * 4 + o], gw3[o]);
            } else if (o64 < kMlpOut) {
                gb3 += s.dy[r * 4 + o64];
            }
        }
        ok = mlp_wait(s, phase);
        if (!ok) break;
        // dZ1 = dA1 * silu'(z1)
#pragma unroll
        for (int c = 0; c < kMlpHid; c += 16) {
            float da[16], z[16];
            umma::tmem_ld16(tmem_row + 192 + c, da);
            umma::tmem_ld16(tmem_row + c, z);
#pragma unroll
            for (int j = 0; j < 16; ++j) da[j] *= silu_grad(z[j] + s.b1[c + j]);
            store_row8(s.g1, t, c, kMlpHid, da);
            store_row8(s.g1, t, c + 8, kMlpHid, da + 8);
        }
        __syncthreads();
        // dW1, db1
        for (int r = 0; r < kMlpTile; ++r) {
            const float g = bf(s.g1, r, o64, kMlpHid);
            float xv[8];
            ld_row8(s.x, r, half * 8, kMlpIn, xv);
#pragma unroll
            for (int j = 0; j < 8; ++j) gw1[j] = fmaf(xv[j], g, gw1[j]);
            if (half == 0) gb1 += g;
        }
        umma::fence_before_sync();
        __syncthreads();
        umma::fence_after_sync();
    }
    if (!ok && t == 0) atomicOr(err, 1u);
    // this CTA's share of the gradient (every entry is written by exactly one thread)
    float* P = partials + (size_t)blockIdx.x * kPartialStride;
#pragma unroll
    for (int j = 0; j < 32; ++j) P[kW2 + (half * 32 + j) * kMlpHid + o64] = gw2[j];
#pragma unroll
    for (int j = 0; j < 8; ++j) P[kW1 + (half * 8 + j) * kMlpHid + o64] = gw1[j];
    if (half == 0) {
        P[kB1 + o64] = gb1;
        P[kB2 + o64] = gb2;
#pragma unroll
        for (int o = 0; o < kMlpOut; ++o) P[kW3 + o64 * kMlpOut + o] = gw3[o];
    } else if (o64 < kMlpOut) {
        P[kB3 + o64] = gb3;
    }
    // loss: block sum in thread 0 (fixed order)
    __shared__ float lsum[kMlpTile];
    lsum[t] = loss;
    __syncthreads();
    if (t == 0) {
        float l = 0.f;
        for (int k = 0; k < kMlpTile; ++k) l += lsum[k];
        P[kMlpParams] = l / (3.f * (float)batch);
    }
    mlp_cta_end(s, tmem, kTrainCols, !ok, phase);
}

// grad[p] = sum over CTAs of partials[c][p] (p <= kMlpParams: the last entry is the loss)
__global__ void k_mlp_reduce(const float* __restrict__ partials, int ctas, float* __restrict__ grad)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kPartialStride) return;
    float g = 0.f;
    for (int c = 0; c < ctas; ++c) g += partials[(size_t)c * kPartialStride + p];
    grad[p] = g;
}

__global__ void k_mlp_adam(float* __restrict__ model, const float* __restrict__ grad, float* __restrict__ m,
                           float* __restrict__ v, float lr, float beta1, float beta2, float eps, float bc1, float bc2)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    const float g = grad[p];
    const float mp = fmaf(beta1, m[p], (1.f - beta1) * g);
    const float vp = fmaf(beta2, v[p], (1.f - beta2) * g * g);
    m[p] = mp;
    v[p] = vp;
    model[p] -= lr * (mp / bc1) / (sqrtf(vp / bc2) + eps);
}

std::mutex g_attr_mutex;
int g_attr_done[64];

// dynamic shared memory above 48 KB needs an opt-in per kernel (once per device)
cudaError_t mlp_kernel_attrs(int device)
{
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    if (g_attr_done[device]) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(MlpFwdSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpTrainSmem));
    if (e == cudaSuccess) g_attr_done[device] = 1;
    return e;
}

int sm_count(int device)
{
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return sms > 0 ? sms : 1;
}

}  // namespace
}  // namespace nsph

using namespace nsph;

extern "C" int nsph_mlp_model_floats(void) { return kMlpModelFloats; }

extern "C" int nsph_mlp_forward(int device, const float* model, const float* features, int n, float* out,
                                unsigned int* err, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_mlp_forward");
    if (n < 0) return fail(NSPH_ERR_INVALID_ARG, "negative count");
    if (n == 0) return NSPH_OK;
    if (!model || !features || !out || !err) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    DeviceGuard guard(device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    NSPH_CUDA_TRY(mlp_kernel_attrs(device));
    const int tiles = (n + kMlpTile - 1) / kMlpTile;
    const int resident = mlp_resident_grid(k_mlp_forward, sizeof(MlpFwdSmem), device);
    if (resident <= 0) return fail(NSPH_ERR_CUDA, "cannot size the k_mlp_forward grid");
    const int grid = std::min(tiles, resident);
    k_mlp_forward<<<grid, kMlpTile, sizeof(MlpFwdSmem), (cudaStream_t)stream>>>(model, features, n, out, err);
    NSPH_LAUNCH_CHECK("k_mlp_forward");
    return NSPH_OK;
}

extern "C" int nsph_mlp_gradient_ctas(int device, int batch)
{
    if (batch <= 0) return 0;
    const int tiles = (batch + kMlpTile - 1) / kMlpTile;
    return std::min(tiles, 2 * sm_count(device));
}

extern "C" int nsph_mlp_gradient(int device, const float* model, const float* features, const float* targets,
                                 const int* batch_idx, int batch, float* partials, int partial_rows, float* grad,
                                 unsigned int* err, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_mlp_gradient");
    if (batch <= 0) return fail(NSPH_ERR_INVALID_ARG, "batch must be positive");
    if (!model || !features || !targets || !batch_idx || !partials || !grad || !err)
        return fail(NSPH_ERR_INVALID_ARG, "null argument");
    const int ctas = nsph_mlp_gradient_ctas(device, batch);
    if (partial_rows < ctas)
        return fail(NSPH_ERR_CAPACITY, "partials needs nsph_mlp_gradient_ctas(device, batch) rows");
    DeviceGuard guard(device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    NSPH_CUDA_TRY(mlp_kernel_attrs(device));
    cudaStream_t cs = (cudaStream_t)stream;
    k_mlp_grad<<<ctas, kMlpTile, sizeof(MlpTrainSmem), cs>>>(model, features, targets, batch_idx, batch, partials,
                                                                  err);
    NSPH_LAUNCH_CHECK("k_mlp_grad");
    k_mlp_reduce<<<(kPartialStride + 255) / 256, 256, 0, cs>>>(partials, ctas, grad);
    NSPH_LAUNCH_CHECK("k_mlp_reduce");
    return NSPH_OK;
}

extern "C" int nsph_mlp_adam(int device, float* model, const float* grad, float* m, float* v, float lr, float beta1,
                             float beta2, float eps, int step, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_mlp_adam");
    if (!model || !grad || !m || !v) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    if (step < 1) return fail(NSPH_ERR_INVALID_ARG, "step counts from 1");
    DeviceGuard guard(device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    const float bc1 = 1.f - powf(beta1, (float)step), bc2 = 1.f - powf(beta2, (float)step);
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(model, grad, m, v, lr, beta1, beta2, eps,
                                                                            bc1, bc2);
    NSPH_LAUNCH_CHECK("k_mlp_adam");
    return NSPH_OK;
}
