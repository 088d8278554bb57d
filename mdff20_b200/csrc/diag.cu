// Diagnostics: the FMA-pipe roofline of this GPU, measured with a kernel of
// independent fused multiply-add chains (the pair and k-space kernels are bound by the
// FP64 or FP32 pipe, not by HBM or the tensor cores).
#include "engine.cuh"

namespace mdffgpu {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(T *out, int iters, T a, T b) {
    grid_dep();
    T x0 = (T)threadIdx.x, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
    T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
            x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
        }
    }
    T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)-12345.0) out[blockIdx.x] = s;  // keeps the chains alive
}

template <typename T>
static double run_peak(int iters) {
    int nsm = 148;
    int dev = 0;
    MDFF_CK(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int blocks = nsm * 8;
    T *out = nullptr;
    MDFF_CK(cudaMalloc(&out, sizeof(T) * blocks));
    cudaEvent_t e0, e1;
    MDFF_CK(cudaEventCreate(&e0));
    MDFF_CK(cudaEventCreate(&e1));
    k_fma_peak<T><<<blocks, 256>>>(out, 8, (T)0.999999, (T)1e-7);  // warm-up
    MDFF_CK(cudaEventRecord(e0));
    k_fma_peak<T><<<blocks, 256>>>(out, iters, (T)0.999999, (T)1e-7);
    MDFF_CK(cudaEventRecord(e1));
    MDFF_CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    MDFF_CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    double flops = 2.0 * 8 * 16 * (double)iters * blocks * 256;
    return flops / (ms * 1e-3) / 1e12;
}

}  // namespace mdffgpu

extern "C" int mdffgpu_fma_peak(int device, int precision, double *tflops) {
    if (!tflops) return MDFFGPU_ERR_ARG;
    try {
        if (device >= 0) MDFF_CK(cudaSetDevice(device));
        *tflops = precision == MDFFGPU_FP64 ? mdffgpu::run_peak<double>(2048) : mdffgpu::run_peak<float>(4096);
        return MDFFGPU_OK;
    } catch (const mdffgpu::Error &x) {
        return x.code;
    }
}
