/* FP32 FMA throughput of the device: the denominator of the roofline of
 * the kernels that run on the CUDA cores (the measured peaks of the pool
 * cover HBM copies and BF16 tensor-core GEMMs only). */
#include "tcoh_internal.h"

#define TC_API extern "C" __attribute__((visibility("default")))

__global__ void __launch_bounds__(256) tc_fma_kernel(float *out, int iters, float a, float b)
{
    float x[16];

#pragma unroll
    for (int i = 0; i < 16; i++)
        x[i] = threadIdx.x * 1e-7f + i;
    for (int it = 0; it < iters; it++)
#pragma unroll
        for (int i = 0; i < 16; i++)
            x[i] = fmaf(x[i], a, b);
    float s = 0.f;

#pragma unroll
    for (int i = 0; i < 16; i++)
        s += x[i];
    if (s == 1234.5f)
        out[blockIdx.x] = s;
}

TC_API int tc_fp32_peak(int device, double *tflops)
{
    cudaDeviceProp p;
    float *out = nullptr, best = 1e30f;
    cudaEvent_t e0, e1;
    const int iters = 1 << 14;

    if (cudaSetDevice(device < 0 ? 0 : device) != cudaSuccess ||
        cudaGetDeviceProperties(&p, device < 0 ? 0 : device) != cudaSuccess)
        return TC_ERR_DEVICE;
    const int blocks = p.multiProcessorCount * 8;

    if (cudaMalloc(&out, sizeof(float) * blocks) != cudaSuccess)
        return TC_ERR_MEMORY;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int rep = 0; rep < 4; rep++) {
        float ms = 0.f;

        cudaEventRecord(e0);
        tc_fma_kernel<<<blocks, 256>>>(out, iters, 0.9999f, 1e-6f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best)
            best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess)
        return TC_ERR_CUDA;
    *tflops = 2.0 * 16.0 * iters * (double)blocks * 256 / (best * 1e-3) / 1e12;
    return TC_OK;
}
