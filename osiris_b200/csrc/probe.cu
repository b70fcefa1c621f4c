// FP64 pipe peak probe: the denominator of the flash kernel's roofline.
//
// Each thread runs kChains independent dependent-FMA chains for kIters
// rounds, enough independent work per warp to keep the FP64 pipe saturated;
// the grid fills every SM.  Result = 2 * FMAs / elapsed seconds.
#include <cuda_runtime.h>
#include "osiris_b200.h"
#include "eos_device.cuh"

namespace {

// The branch-free quotient and reciprocal of the flash kernels on arrays of
// operands, with the range predicate their callers gather.
__global__ void __launch_bounds__(256) quotient_probe_kernel(const double *a, const double *b, long n, double *q,
                                                             double *r, signed char *ok) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        q[i] = osr::qdiv(a[i], b[i]);
        r[i] = osr::qrcp(b[i]);
        ok[i] = osr::qdiv_ok(a[i], b[i]) ? 1 : 0;
    }
}

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) dfma_probe_kernel(double seed, double *sink) {
    double a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) a[c] = seed + threadIdx.x * 1e-9 + c * 1e-7;
    const double m = 0.999999999, q = 1e-12;
#pragma unroll 4
    for (int it = 0; it < kIters; it++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) a[c] = fma(a[c], m, q);
    }
    double s = 0;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += a[c];
    if (s == 1234.5678) sink[0] = s;  // keeps the chains live; never true
}

}  // namespace

extern "C" osr_status osr_probe_quotients(const double *d_a, const double *d_b, long n, double *d_q, double *d_r,
                                          signed char *d_ok, void *stream) {
    if (n < 0 || (n > 0 && (!d_a || !d_b || !d_q || !d_r || !d_ok))) return OSR_ERR_ARG;
    if (n == 0) return OSR_OK;
    long blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    quotient_probe_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(d_a, d_b, n, d_q, d_r, d_ok);
    return cudaGetLastError() == cudaSuccess ? OSR_OK : OSR_ERR_CUDA;
}

extern "C" osr_status osr_probe_fp64_peak(double *tflops, void *stream) {
    if (!tflops) return OSR_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return OSR_ERR_NODEVICE;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return OSR_ERR_CUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dfma_probe_kernel, 256, 0) != cudaSuccess)
        return OSR_ERR_CUDA;
    const int blocks = sms * (per_sm > 0 ? per_sm : 1) * 4;
    double *sink = nullptr;
    cudaEvent_t e0, e1;
    if (cudaMallocAsync((void **)&sink, sizeof(double), s) != cudaSuccess) return OSR_ERR_CUDA;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    dfma_probe_kernel<<<blocks, 256, 0, s>>>(1.0, sink);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
        cudaEventRecord(e0, s);
        dfma_probe_kernel<<<blocks, 256, 0, s>>>(1.0 + r, sink);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaFreeAsync(sink, s);
    cudaStreamSynchronize(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) return OSR_ERR_CUDA;
    double flops = 2.0 * kChains * (double)kIters * 256.0 * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return OSR_OK;
}
