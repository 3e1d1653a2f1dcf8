// fma_probe.cu -- FP32 throughput probe for the roofline denominator (not
// part of the engine): independent FFMA chains on every SM, best of three
// timed launches after a warm-up.  bench.py loads it from tests/_build.
#include <cuda_runtime.h>

namespace {

// 8 independent FFMA chains per thread; the values converge to a fixed point
// (x = 0.999 x + 0.001), so nothing overflows or goes subnormal.
__global__ void __launch_bounds__(256) fma_rate_kernel(float* out, int iters)
{
    float a0 = threadIdx.x * 1e-3f, a1 = a0 + 0.1f, a2 = a0 + 0.2f, a3 = a0 + 0.3f;
    float a4 = a0 + 0.4f, a5 = a0 + 0.5f, a6 = a0 + 0.6f, a7 = a0 + 0.7f;
    const float m = 0.999f, c = 0.001f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = __fmaf_rn(a0, m, c); a1 = __fmaf_rn(a1, m, c); a2 = __fmaf_rn(a2, m, c); a3 = __fmaf_rn(a3, m, c);
            a4 = __fmaf_rn(a4, m, c); a5 = __fmaf_rn(a5, m, c); a6 = __fmaf_rn(a6, m, c); a7 = __fmaf_rn(a7, m, c);
        }
    }
    const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.0f) out[blockIdx.x] = s;   // keeps the chains alive
}

}  // namespace

// Measured FFMA throughput of `device` in TFLOP/s (2 flops per FFMA).
// Returns 0, or the CUDA error code.
extern "C" int pfd_probe_fp32_fma_rate(int device, double* tflops)
{
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return (int)e;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, threads = 256, iters = 512;
    float* out = nullptr;
    e = cudaMalloc((void**)&out, sizeof(float) * blocks);
    if (e != cudaSuccess) return (int)e;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    fma_rate_kernel<<<blocks, threads>>>(out, iters);    // warm-up
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(a);
        fma_rate_kernel<<<blocks, threads>>>(out, iters);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float t = 0.0f;
        cudaEventElapsedTime(&t, a, b);
        if (t < best) best = t;
    }
    e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    const double flops = 2.0 * 8.0 * 16.0 * (double)iters * (double)blocks * (double)threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return (int)e;
}
