// Non-tensor FP64 / FP32 FMA throughput of the current device, measured with
// an FMA-only kernel: the roofline denominators of the cell kernels, which do
// no dense contraction and so never use the tensor cores.
#include "../../include/sdot_gpu.h"
#include "common.cuh"

namespace {

template <class T>
__global__ void k_fma(T *out, int iters, T a, T b) {
    // 8 independent chains per thread keep the FMA pipe full
    T x0 = T(threadIdx.x), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
    T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
            x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
        }
    }
    const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == T(-1.2345)) out[0] = s;  // keeps the chains live
}

template <class T>
double measure(int sms) {
    T *out = nullptr;
    SDOT_CUDA(cudaMalloc(&out, sizeof(T)));
    const int threads = 256, blocks = sms * 8, iters = 4096;
    cudaEvent_t e0, e1;
    SDOT_CUDA(cudaEventCreate(&e0));
    SDOT_CUDA(cudaEventCreate(&e1));
    k_fma<T><<<blocks, threads>>>(out, 16, T(0.999), T(0.001));  // warm-up
    SDOT_CUDA(cudaGetLastError());
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        SDOT_CUDA(cudaEventRecord(e0));
        k_fma<T><<<blocks, threads>>>(out, iters, T(0.999), T(0.001));
        SDOT_CUDA(cudaEventRecord(e1));
        SDOT_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        SDOT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double flops = 2.0 * 64.0 * iters * double(threads) * blocks;
    return flops / (best * 1e-3) / 1e12;
}

}  // namespace

extern "C" int sdot_measure_fma_peaks(double *tflops2) {
    if (!tflops2) return SDOT_BAD_ARG;
    try {
        int dev = 0, sms = 0;
        SDOT_CUDA(cudaGetDevice(&dev));
        SDOT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        tflops2[0] = measure<double>(sms);
        tflops2[1] = measure<float>(sms);
    } catch (const sdot::CudaError &) {
        return SDOT_CUDA_ERROR;
    }
    return SDOT_OK;
}
