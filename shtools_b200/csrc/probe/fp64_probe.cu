// FP64 throughput probe (libshtc_probe.so), used by bench.py to measure the
// FP64-pipe peak that the Legendre kernels are compared with: the measured
// peak file of this machine pool lists only HBM and bf16 tensor rates.
//
// Each thread runs 8 independent FMA chains; the caller times a launch with
// CUDA events and counts 2 flops per FMA.
#include <cuda_runtime.h>

__global__ void __launch_bounds__(256) k_dfma(double* out, int iters, double a,
                                              double b) {
    double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
    double x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b);
            x3 = fma(x3, a, b); x4 = fma(x4, a, b); x5 = fma(x5, a, b);
            x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const double s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 1234.5) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// flops of one launch = blocks * 256 * iters * 16 * 8 * 2
extern "C" __attribute__((visibility("default"))) int shtc_probe_dfma(
    double* out, int blocks, int iters, void* stream) {
    k_dfma<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters, 0.999999, 1e-7);
    return cudaGetLastError() == cudaSuccess ? 0 : 6;
}
