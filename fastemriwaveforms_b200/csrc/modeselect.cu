// Mode selection by estimated power (the threshold branch of
// ModeSelector.__call__, src/few/utils/modeselector.py:393-486).
//
// k_mode_snr2: one thread per mode j (consecutive threads read consecutive
// modes of a knot row of the (N, K) amplitude array, so the loads coalesce):
//   p_n = |A_nj Y_j|^2 (+ |conj(A_nj) Y_j^-|^2 for m != 0),
//   snr2_j = sum_{n < N-1} (p_n / psd_nj) (t_{n+1} - t_n),
// accumulated in knot order, as numpy's reduction over the leading axis does
// (|z|^2 as hypot(re, im)^2, numpy's abs followed by its square).
// k_mode_keep: the cumulative sum of the descending-sorted estimates in
// sorted order (one thread: numpy's cumsum is sequential) and the keep rule
// keep_0 = true, keep_i = cumsum_{i-1} < cumsum_{K-1} (1 - threshold)^2.
#include <cuda_runtime.h>

#include <cmath>

#include "few_internal.h"

namespace few {
namespace msel {

__global__ void k_mode_snr2(const double2 *__restrict__ teuk, int N, int K, const double2 *__restrict__ ylms,
                            const int *__restrict__ minus_index, const double *__restrict__ psd,
                            const double *__restrict__ t, double *__restrict__ snr2) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= K) return;
    const double2 yp = ylms[j];
    const int mi = minus_index[j];
    const double2 ym = mi >= 0 ? ylms[mi] : make_double2(0.0, 0.0);
    double acc = 0.0;
    for (int n = 0; n < N - 1; ++n) {
        const double2 a = teuk[(long long)n * K + j];
        double re = __dsub_rn(__dmul_rn(a.x, yp.x), __dmul_rn(a.y, yp.y));
        double im = __dadd_rn(__dmul_rn(a.x, yp.y), __dmul_rn(a.y, yp.x));
        double h = hypot(re, im);
        double p = __dmul_rn(h, h);
        if (mi >= 0) {  // conj(A) Y^-
            double re2 = __dsub_rn(__dmul_rn(a.x, ym.x), __dmul_rn(-a.y, ym.y));
            double im2 = __dadd_rn(__dmul_rn(a.x, ym.y), __dmul_rn(-a.y, ym.x));
            double h2 = hypot(re2, im2);
            p = __dadd_rn(p, __dmul_rn(h2, h2));
        }
        if (psd) p = __ddiv_rn(p, psd[(long long)n * K + j]);
        acc = __dadd_rn(acc, __dmul_rn(p, __dsub_rn(t[n + 1], t[n])));
    }
    snr2[j] = acc;
}

__global__ void k_mode_keep(const double *__restrict__ sorted_desc, int K, double threshold, int *__restrict__ keep) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double total = 0.0;
    for (int i = 0; i < K; ++i) total = __dadd_rn(total, sorted_desc[i]);
    const double one_m = __dsub_rn(1.0, threshold);
    const double lim = __dmul_rn(total, __dmul_rn(one_m, one_m));
    double run = 0.0;
    for (int i = 0; i < K; ++i) {
        keep[i] = (i == 0) ? 1 : (run < lim ? 1 : 0);
        run = __dadd_rn(run, sorted_desc[i]);
    }
}

}  // namespace msel
}  // namespace few

extern "C" FEW_API int few_mode_snr2(const void *teuk, int N, int K, const void *ylms, const int *minus_index,
                                     const double *psd, const double *t, double *snr2, void *stream) {
    few::clear_error();
    if (N < 1 || K < 0) return few::fail(FEW_ERR_SIZE, "few_mode_snr2: N=%d K=%d", N, K);
    if (K == 0) return FEW_OK;
    if (!teuk || !ylms || !minus_index || !t || !snr2) return few::fail(FEW_ERR_ARG, "few_mode_snr2: null pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    few::msel::k_mode_snr2<<<(K + 127) / 128, 128, 0, st>>>(static_cast<const double2 *>(teuk), N, K,
                                                             static_cast<const double2 *>(ylms), minus_index, psd,
                                                             t, snr2);
    FEW_LAUNCH_CHECK("k_mode_snr2");
    return FEW_OK;
}

extern "C" FEW_API int few_mode_keep(const double *sorted_desc, int K, double threshold, int *keep, void *stream) {
    few::clear_error();
    if (K < 0) return few::fail(FEW_ERR_SIZE, "few_mode_keep: K=%d", K);
    if (K == 0) return FEW_OK;
    if (!sorted_desc || !keep) return few::fail(FEW_ERR_ARG, "few_mode_keep: null pointer");
    few::msel::k_mode_keep<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(sorted_desc, K, threshold, keep);
    FEW_LAUNCH_CHECK("k_mode_keep");
    return FEW_OK;
}
