// FMA-throughput microbenchmark: the FP64 and FP32 peaks that the ring pass and the NUFFT
// are measured against (the driver-measured peaks cover only HBM and bf16 GEMM).
// Each thread runs 8 independent FMA chains; the grid fills every SM several times over.
#include <cuda_runtime.h>

#include <string>

#include "../../include/pfsht_b200.h"
#include "internal.cuh"

namespace pf {

template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T* out, int iters, T a, T b) {
    T x0 = (T)threadIdx.x, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
    T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)-1.2345) out[threadIdx.x] = s;  // keeps the chains live
}

template <typename T>
static int run_peak(int iters, double* flops_per_s, double* ms_out) {
    int dev = 0, nsm = 0;
    PF_CUDA(cudaGetDevice(&dev));
    PF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    DevBuf out;
    PF_TRY(out.alloc(256 * sizeof(T)));
    const int blocks = nsm * 8;
    cudaEvent_t e0, e1;
    PF_CUDA(cudaEventCreate(&e0));
    PF_CUDA(cudaEventCreate(&e1));
    fma_peak_kernel<T><<<blocks, 256>>>(out.as<T>(), iters / 10 + 1, (T)0.999999, (T)1e-7);
    PF_CUDA(cudaEventRecord(e0));
    fma_peak_kernel<T><<<blocks, 256>>>(out.as<T>(), iters, (T)0.999999, (T)1e-7);
    PF_CUDA(cudaEventRecord(e1));
    PF_CUDA(cudaEventSynchronize(e1));
    PF_TRY(check_launch("fma_peak_kernel"));
    float ms = 0;
    PF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double fmas = (double)blocks * 256.0 * iters * 16.0 * 8.0;
    *flops_per_s = 2.0 * fmas / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    return 0;
}

}  // namespace pf

extern "C" pfsht_status pfsht_fma_peak(int32_t fp64, int32_t iters, double* flops_per_s,
                                       double* ms) {
    if (!flops_per_s || iters < 1) {
        pf::set_error("bad arguments");
        return PFSHT_ERR_ARGUMENT;
    }
    return (pfsht_status)(fp64 ? pf::run_peak<double>(iters, flops_per_s, ms)
                               : pf::run_peak<float>(iters, flops_per_s, ms));
}
