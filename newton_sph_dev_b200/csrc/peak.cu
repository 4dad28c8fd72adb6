// peak.cu — measured FP32 / instruction-issue peak of the device (no
// counterpart in the reference: the denominator of the issue roofline that
// bounds the neighbour passes).
//
// Every SM runs 64 resident warps; each thread keeps 8 independent FMA
// chains, so the FMA pipes never wait on a dependency. One FFMA is one warp
// instruction issued per warp, so the rate measured here is both the FP32
// peak (2 flops per lane per FFMA) and the sustained warp-instruction issue
// rate the neighbour passes compete for.
#include "nsph_internal.cuh"

namespace nsph {
namespace {

constexpr int kPeakThreads = 256;
constexpr int kPeakBlocksPerSm = 8;
constexpr int kPeakChains = 8;
constexpr int kPeakUnroll = 16;

__global__ void __launch_bounds__(kPeakThreads) k_ffma_peak(float* __restrict__ out, int iters, float a, float b)
{
    float x[kPeakChains];
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) x[c] = (float)(threadIdx.x + c) * 1.0e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < kPeakUnroll; ++u) {
#pragma unroll
            for (int c = 0; c < kPeakChains; ++c) x[c] = __fmaf_rn(x[c], a, b);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) s += x[c];
    if (s == 12345.678f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains alive
}

}  // namespace
}  // namespace nsph

using namespace nsph;

extern "C" int nsph_fp32_peak(int device, int iters, float* tflops, float* warp_inst_per_s, float* ms, void* stream)
{
    clear_error();
    if (iters <= 0 || !tflops || !warp_inst_per_s || !ms) return fail(NSPH_ERR_INVALID_ARG, "bad argument");
    DeviceGuard guard(device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    int sms = 0;
    NSPH_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int blocks = sms * kPeakBlocksPerSm;
    float* sink = nullptr;
    NSPH_CUDA_TRY(cudaMalloc(&sink, sizeof(float) * (size_t)blocks * kPeakThreads));
    cudaStream_t cs = (cudaStream_t)stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) {
        k_ffma_peak<<<blocks, kPeakThreads, 0, cs>>>(sink, std::max(1, iters / 8), 0.9999f, 1.0e-4f);  // warm-up
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e0, cs);
    if (e == cudaSuccess) {
        k_ffma_peak<<<blocks, kPeakThreads, 0, cs>>>(sink, iters, 0.9999f, 1.0e-4f);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, cs);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_fail(e, "fp32 peak");
    const double ffma = (double)blocks * kPeakThreads * iters * kPeakUnroll * kPeakChains;
    *ms = t;
    *tflops = (float)(2.0 * ffma / (t * 1e-3) / 1e12);
    *warp_inst_per_s = (float)(ffma / 32.0 / (t * 1e-3));
    return NSPH_OK;
}
