// FP64 FMA-pipe throughput probe: the measured denominator of the sum
// kernels' roofline (the driver's peak file holds HBM and bf16 figures only).
// Every thread runs 8 independent FMA chains; 2 flops per FMA.
#include "few_internal.h"

namespace few {
namespace {
__global__ void __launch_bounds__(256) k_fp64_fma_probe(double *out, int iters, double a, double b)
{
    double x[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = threadIdx.x * 1e-3 + q;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = fma(x[q], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += x[q];
    out[(long long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace
}  // namespace few

extern "C" int few_probe_fp64_fma(double *out, int blocks, int iters, void *stream)
{
    few::clear_error();
    if (!out) return few::fail(FEW_ERR_ARG, "few_probe_fp64_fma: null pointer");
    if (blocks < 1 || iters < 1) return few::fail(FEW_ERR_SIZE, "few_probe_fp64_fma: bad sizes");
    few::k_fp64_fma_probe<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters, 0.999999999, 1e-9);
    FEW_LAUNCH_CHECK("k_fp64_fma_probe");
    return FEW_OK;
}
