// fma_peak.cu -- attainable FP64 / FP32 FMA throughput of the current device.
//
// Measurement only: built into libws_peaks.so, which bench.py loads for the
// roofline denominator of the fused RHS kernels (the FP64 pipe bounds them,
// and no FP64 peak is measured elsewhere).  It is not part of
// libwindstencil_b200.so or of its C ABI.
//
// Independent FMA chains (8 per thread, CTAs of 512 threads, 4 per SM); one
// short warm-up launch, then three timed launches between CUDA events.
#include <cuda_runtime.h>

namespace {
template <typename T>
__global__ void fma_peak_kernel(T* out, int iters, T a, T b) {
    T x0 = T(threadIdx.x) * T(1e-3), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
    T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == T(-1.2345)) out[0] = s;    // keeps the chains live
}

// 0 on success, else the CUDA error code
template <typename T>
int peak(double* tflops, cudaStream_t st) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    T* out = nullptr;
    if (e == cudaSuccess) e = cudaMallocAsync(&out, sizeof(T), st);
    if (e != cudaSuccess) return (int)e;
    const int threads = 512, blocks = sms * 4, iters = 2048;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_peak_kernel<T><<<blocks, threads, 0, st>>>(out, iters / 4, T(0.999999), T(1e-7));
    cudaEventRecord(e0, st);
    for (int r = 0; r < 3; ++r)
        fma_peak_kernel<T><<<blocks, threads, 0, st>>>(out, iters, T(0.999999), T(1e-7));
    cudaEventRecord(e1, st);
    e = cudaEventSynchronize(e1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(out, st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    const double flop = 3.0 * 2.0 * 8.0 * 16.0 * iters * (double)threads * blocks;
    *tflops = flop / (ms * 1e-3) / 1e12;
    return 0;
}
}  // namespace

extern "C" {
__attribute__((visibility("default"))) int wsp_fp64_fma_peak(double* tflops, void* stream) {
    return tflops ? peak<double>(tflops, (cudaStream_t)stream) : -1;
}
__attribute__((visibility("default"))) int wsp_fp32_fma_peak(double* tflops, void* stream) {
    return tflops ? peak<float>(tflops, (cudaStream_t)stream) : -1;
}
}
