/* FP32 and FP64 FMA throughput of the device: the denominators of the
 * roofline of the kernels that run on the CUDA cores (the measured peaks of
 * the pool cover HBM copies and BF16 tensor-core GEMMs only). */
#include "tcoh_internal.h"

#define TC_API extern "C" __attribute__((visibility("default")))

template <typename R>
__global__ void __launch_bounds__(256) tc_fma_kernel(R *out, int iters, R a, R b)
{
    R x[16];

#pragma unroll
    for (int i = 0; i < 16; i++)
        x[i] = (R)threadIdx.x * (R)1e-7 + (R)i;
    for (int it = 0; it < iters; it++)
#pragma unroll
        for (int i = 0; i < 16; i++)
            x[i] = fma(x[i], a, b);
    R s = 0;

#pragma unroll
    for (int i = 0; i < 16; i++)
        s += x[i];
    if (s == (R)1234.5)
        out[blockIdx.x] = s;
}

template <typename R>
static int fma_peak(int device, int iters, double *tflops)
{
    cudaDeviceProp p;
    R *out = nullptr;
    float best = 1e30f;
    cudaEvent_t e0, e1;

    if (cudaSetDevice(device < 0 ? 0 : device) != cudaSuccess ||
        cudaGetDeviceProperties(&p, device < 0 ? 0 : device) != cudaSuccess)
        return TC_ERR_DEVICE;
    const int blocks = p.multiProcessorCount * 8;

    if (cudaMalloc(&out, sizeof(R) * blocks) != cudaSuccess)
        return TC_ERR_MEMORY;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int rep = 0; rep < 4; rep++) {
        float ms = 0.f;

        cudaEventRecord(e0);
        tc_fma_kernel<R><<<blocks, 256>>>(out, iters, (R)0.9999, (R)1e-6);
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

TC_API int tc_fp32_peak(int device, double *tflops)
{
    return fma_peak<float>(device, 1 << 14, tflops);
}

TC_API int tc_fp64_peak(int device, double *tflops)
{
    return fma_peak<double>(device, 1 << 12, tflops);
}
