// peak.cu — measures this device's FP32 / FP64 / packed-FP32x2 CUDA-core FMA throughput with
// a dependent-chain-free FMA loop, so the field kernels' roofline fraction is
// taken against a number measured on the same GPU (the FP32/FP64 vector pipes
// are the bound of this path, not HBM or the tensor cores).
#include "../../include/bielcc_gpu.h"
#include "internal.h"

namespace bielcc_gpu {

template <typename T>
__global__ void fma_loop_kernel(T* out, int iters, T seed) {
    T a[8];
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = seed + (T)(threadIdx.x + i);
    const T b = (T)0.9999999, c = (T)1e-7;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] = a[i] * b + c;
    }
    T s = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) s += a[i];
    if (s == (T)-1.2345) out[0] = s;  // never true; keeps the loop live
}

// Packed FP32 pairs: one fma.rn.f32x2 per element pair (sm_100).
__global__ void fma2_loop_kernel(float* out, int iters, float seed) {
    float2 a[8];
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = make_float2(seed + (float)(threadIdx.x + i), seed - (float)i);
    const float2 b = make_float2(0.9999999f, 0.9999998f), c = make_float2(1e-7f, 2e-7f);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] = __ffma2_rn(a[i], b, c);
    }
    float s = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) s += a[i].x + a[i].y;
    if (s == -1.2345f) out[0] = s;  // never true; keeps the loop live
}

}  // namespace bielcc_gpu

extern "C" int bielcc_measure_fma_peak(int kind, double* tflops) {
    const int fp64 = kind == 1;
    using namespace bielcc_gpu;
    if (!tflops || kind < 0 || kind > 2) return BIELCC_ERR_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return BIELCC_ERR_CUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    void* out = nullptr;
    if (cudaMalloc(&out, 64) != cudaSuccess) return BIELCC_ERR_OOM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int threads = 256, blocks = sms * 8, iters = fp64 ? 4096 : 8192;
    double best = 0.;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        if (kind == 1) fma_loop_kernel<double><<<blocks, threads>>>((double*)out, iters, 1.0);
        else if (kind == 2) fma2_loop_kernel<<<blocks, threads>>>((float*)out, iters, 1.0f);
        else fma_loop_kernel<float><<<blocks, threads>>>((float*)out, iters, 1.0f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        double flops = 2.0 * 8.0 * iters * (double)threads * blocks * (kind == 2 ? 2.0 : 1.0);
        if (rep > 0 && ms > 0) best = best > flops / (ms * 1e-3) ? best : flops / (ms * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return BIELCC_ERR_CUDA;
    *tflops = best / 1e12;
    return BIELCC_OK;
}
