// fgpe_peak.cu -- FP64 FMA throughput of the device, the compute-roofline
// denominator of the step kernels (their pointwise exponentials, spin-2
// matrix products and FFT butterflies run on the FP64 pipe).
//
// Every thread runs 8 independent FMA chains (enough to cover the FP64 pipe
// latency at full occupancy) for `iters` rounds; the chains fold into one
// store so the compiler keeps every FMA.  Timed with CUDA events on a
// private stream after one warm-up launch.
#include <cuda_runtime.h>

#include "../../include/fgpe.h"

namespace {

__global__ void __launch_bounds__(256) k_fp64_fma(double* sink, int iters, double a, double b) {
    double v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = (double)(threadIdx.x + j) * 1e-9;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = fma(v[j], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += v[j];
    if (s == 12345.678) sink[0] = s;   // never true for these inputs; keeps the chains live
}

}  // namespace

extern "C" int fgpe_fp64_fma_rate(int iters, double* tflops) {
    if (!tflops || iters < 1) return FGPE_E_ARG;
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return FGPE_E_CUDA;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return FGPE_E_CUDA;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double* sink = nullptr;
    int rc = FGPE_E_CUDA;
    const int blocks = nsm * 8, threads = 256;
    float ms = 0.f;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) goto done;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) goto done;
    if (cudaMallocAsync((void**)&sink, sizeof(double), st) != cudaSuccess) goto done;
    k_fp64_fma<<<blocks, threads, 0, st>>>(sink, iters, 0.999999, 1e-12);
    cudaEventRecord(e0, st);
    k_fp64_fma<<<blocks, threads, 0, st>>>(sink, iters, 0.999999, 1e-12);
    cudaEventRecord(e1, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) goto done;
    if (cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0.f) goto done;
    *tflops = 2.0 * 8.0 * (double)iters * blocks * threads / (ms * 1e-3) / 1e12;
    rc = FGPE_OK;
done:
    if (sink) cudaFreeAsync(sink, st);
    if (st) cudaStreamSynchronize(st);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    cudaGetLastError();
    return rc;
}
