// Direct mode sum on dense inputs: amplitudes and phases given at every output
// sample, no splines.
//
// Reference: DirectModeSum.sum (src/few/summation/directmodesum.py:30-131):
//     h_i = sum_j Y_j A_ij exp(-i phi_ij)
//         + sum_{j: m_j > 0} (-1)^{l_j} Y_{K+j} conj(A_ij) exp(+i phi_ij),
//     phi_ij = (m_j Phi_phi,i + k_j Phi_theta,i) + n_j Phi_r,i,
// the phase rounded in numpy's order (explicitly rounded operations here).
// One warp per sample: lanes take modes j = lane, lane + 32, ... (the lanes
// of a warp read consecutive amplitudes of the sample's row), then a warp
// reduction; the two sums are reduced separately and added, as the reference
// adds its two arrays.  The large phases are reduced mod 2 pi (Cody & Waite,
// three-part 2 pi) before sincos.  FP64 throughout.
#include <cuda_runtime.h>

#include <cmath>

#include "few_internal.h"

namespace few {
namespace direct {

__device__ __forceinline__ void sincos_big(double ph, double *s, double *c) {
    const double kInv2Pi = 0.15915494309189535;
    const double kC1 = 0x1.921fb54400000p+2, kC2 = 0x1.0b4611a600000p-32, kC3 = 0x1.3198a2e037073p-67;
    double r = ph;
    double kq = rint(ph * kInv2Pi);
    if (fabs(kq) < 2097152.0) {
        r = __fma_rn(-kq, kC1, ph);
        r = __fma_rn(-kq, kC2, r);
        r = __fma_rn(-kq, kC3, r);
    }
    sincos(r, s, c);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

__global__ void __launch_bounds__(256) k_direct_sum(const double2 *__restrict__ teuk, const double2 *__restrict__ ylms,
                                                    const double *__restrict__ Pphi, const double *__restrict__ Pth,
                                                    const double *__restrict__ Pr, const int *__restrict__ l,
                                                    const int *__restrict__ m, const int *__restrict__ k,
                                                    const int *__restrict__ n, int N, int K,
                                                    double2 *__restrict__ out) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long i = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < N; i += warps) {
        const double pp = Pphi[i], pt = Pth[i], pr = Pr[i];
        double2 w1 = make_double2(0.0, 0.0), w2 = make_double2(0.0, 0.0);
        for (int j = lane; j < K; j += 32) {
            const int mj = m[j];
            const double phase =
                __dadd_rn(__dadd_rn(__dmul_rn((double)mj, pp), __dmul_rn((double)k[j], pt)), __dmul_rn((double)n[j], pr));
            double s, c;
            sincos_big(phase, &s, &c);
            const double2 a = teuk[i * K + j];
            const double2 e1 = make_double2(c, -s);  // exp(-i phase)
            const double2 t1 = cmul(cmul(ylms[j], a), e1);
            w1.x = __dadd_rn(w1.x, t1.x);
            w1.y = __dadd_rn(w1.y, t1.y);
            if (mj > 0) {
                const double sg = (l[j] & 1) ? -1.0 : 1.0;
                const double2 y2 = make_double2(sg * ylms[K + j].x, sg * ylms[K + j].y);
                const double2 t2 = cmul(cmul(y2, make_double2(a.x, -a.y)), make_double2(c, s));  // exp(+i phase)
                w2.x = __dadd_rn(w2.x, t2.x);
                w2.y = __dadd_rn(w2.y, t2.y);
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            w1.x += __shfl_down_sync(0xffffffffu, w1.x, off);
            w1.y += __shfl_down_sync(0xffffffffu, w1.y, off);
            w2.x += __shfl_down_sync(0xffffffffu, w2.x, off);
            w2.y += __shfl_down_sync(0xffffffffu, w2.y, off);
        }
        if (lane == 0) out[i] = make_double2(w1.x + w2.x, w1.y + w2.y);
    }
}

}  // namespace direct
}  // namespace few

// DirectModeSum.sum's kernel: teuk [device] (N, K) complex, ylms [device] (2K)
// complex (+m, then -m), phases [device] (3, N) = (Phi_phi, Phi_theta, Phi_r),
// l, m, k, n [device] (K,) int; out [device] (N,) complex.
extern "C" FEW_API int few_direct_sum(const void *teuk, const void *ylms, const double *phases, const int *l,
                                      const int *m, const int *k, const int *n, int N, int K, void *out,
                                      void *stream) {
    few::clear_error();
    if (N < 0 || K < 0) return few::fail(FEW_ERR_SIZE, "few_direct_sum: N=%d K=%d", N, K);
    if (N == 0) return FEW_OK;
    if (!out || (K > 0 && (!teuk || !ylms || !phases || !l || !m || !k || !n)))
        return few::fail(FEW_ERR_ARG, "few_direct_sum: null pointer");
    if (K == 0) {
        FEW_CUDA_TRY(cudaMemsetAsync(out, 0, (size_t)N * 16, static_cast<cudaStream_t>(stream)));
        return FEW_OK;
    }
    long long blocks = ((long long)N + 7) / 8;
    if (blocks > 148 * 64) blocks = 148 * 64;
    few::direct::k_direct_sum<<<(int)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const double2 *>(teuk), static_cast<const double2 *>(ylms), phases, phases + N, phases + 2LL * N, l,
        m, k, n, N, K, static_cast<double2 *>(out));
    FEW_LAUNCH_CHECK("k_direct_sum");
    return FEW_OK;
}
