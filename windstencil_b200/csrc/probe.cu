// probe.cu -- attainable FP64 / FP32 FMA throughput of the current device.
//
// The fused RHS is bound by the FP64 pipe; its roofline denominator is the
// FMA rate this device sustains, measured here with independent FMA chains
// (8 per thread, one CTA of 512 threads per SM slot, 4 per SM).
#include "ws_internal.h"

namespace ws {
namespace {
template <typename T>
__global__ void fma_probe_kernel(T* out, int iters, T a, T b) {
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

template <typename T>
int probe(double* tflops, cudaStream_t st) {
    int dev = 0, sms = 0;
    WS_CUDA(cudaGetDevice(&dev));
    WS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    T* out = nullptr;
    WS_CUDA(cudaMallocAsync(&out, sizeof(T), st));
    const int threads = 512, blocks = sms * 4, iters = 2048;
    cudaEvent_t e0, e1;
    WS_CUDA(cudaEventCreate(&e0));
    WS_CUDA(cudaEventCreate(&e1));
    fma_probe_kernel<T><<<blocks, threads, 0, st>>>(out, iters / 4, T(0.999999), T(1e-7));
    WS_CUDA(cudaEventRecord(e0, st));
    for (int r = 0; r < 3; ++r)
        fma_probe_kernel<T><<<blocks, threads, 0, st>>>(out, iters, T(0.999999), T(1e-7));
    WS_CUDA(cudaEventRecord(e1, st));
    WS_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(out, st);
    WS_CUDA(cudaGetLastError());
    const double flop = 3.0 * 2.0 * 8.0 * 16.0 * iters * (double)threads * blocks;
    *tflops = flop / (ms * 1e-3) / 1e12;
    return WS_OK;
}
}  // namespace
}  // namespace ws

extern "C" {
int ws_probe_fp64_peak(double* tflops, ws_stream_t stream) {
    if (!tflops) return ws::fail(WS_ERR_INVALID, "tflops is NULL");
    return ws::probe<double>(tflops, (cudaStream_t)stream);
}
int ws_probe_fp32_peak(double* tflops, ws_stream_t stream) {
    if (!tflops) return ws::fail(WS_ERR_INVALID, "tflops is NULL");
    return ws::probe<float>(tflops, (cudaStream_t)stream);
}
}
