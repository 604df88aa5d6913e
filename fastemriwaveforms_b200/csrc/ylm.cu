// Spin-weighted spherical harmonics of spin weight -2, the Y_lm of the mode sum.
//
// Drop-in for GetYlms (src/few/utils/ylm.py:278-365), whose kernel
// (ylm.py:17-276) spells out each (l, m) with l <= 10 in closed form.  Here
// every (l, m) comes from one sum (Goldberg et al., J. Math. Phys. 8 (1967)
// 2155, with s = -2):
//   sY_lm(theta, phi) = (-1)^m sqrt((l+m)! (l-m)! (2l+1) / (4 pi (l+s)! (l-s)!))
//                       e^{i m phi} sum_r C(l-s, r) C(l+s, r+s-m) (-1)^{l-r-s}
//                       cos(theta/2)^{2r+s-m} sin(theta/2)^{2l-2r-s+m},
// which is the reference's convention (checked term by term on its (2, +-2),
// (2, 1) and (3, -1) entries, and against its values for every l <= 10).
// Powers of cos and sin replace the cotangent of the textbook form, so the
// poles need no special case.
#include <cuda_runtime.h>

#include <cmath>

#include "few_internal.h"

namespace few {
namespace ylm {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr int kS = -2;
constexpr int kMaxL = 64;

__device__ __forceinline__ double binom(int n, int k) {
    if (k < 0 || k > n) return 0.0;
    if (k > n - k) k = n - k;
    double b = 1.0;
    for (int j = 1; j <= k; ++j) b = b * (n - k + j) / j;
    return b;
}

__device__ __forceinline__ double ipow(double x, int e) {
    double r = 1.0;
    for (int j = 0; j < e; ++j) r *= x;
    return r;
}

// sqrt((l+m)! (l-m)! / ((l+s)! (l-s)!)) as a product of ratios (no overflow)
__device__ __forceinline__ double fact_ratio(int l, int m) {
    // (l+m)!/(l+s)! * (l-m)!/(l-s)!
    double r = 1.0;
    int a = l + m, b = l + kS;
    if (a >= b) for (int j = b + 1; j <= a; ++j) r *= j;
    else for (int j = a + 1; j <= b; ++j) r /= j;
    a = l - m; b = l - kS;
    if (a >= b) for (int j = b + 1; j <= a; ++j) r *= j;
    else for (int j = a + 1; j <= b; ++j) r /= j;
    return sqrt(r);
}

__global__ void k_ylm(const int *__restrict__ l_arr, const int *__restrict__ m_arr, int n, int flip_second_half,
                      double theta, double phi, double2 *__restrict__ out, int *status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int src = i, sgn = 1;
    if (flip_second_half) {  // output i >= n/2 is (l, -m) of input i - n/2
        int half = n / 2;
        if (i >= half) { src = i - half; sgn = -1; }
    }
    const int l = l_arr[src], m = sgn * m_arr[src];
    if (l < 2 || l > kMaxL || m < -l || m > l) {
        out[i] = make_double2(nan(""), nan(""));
        if (status) atomicOr(status, 1);
        return;
    }
    const double c = cos(theta / 2.0), s = sin(theta / 2.0);
    double sum = 0.0;
    const int r0 = (m - kS) > 0 ? (m - kS) : 0, r1 = (l - kS) < (l + m) ? (l - kS) : (l + m);
    for (int r = r0; r <= r1; ++r) {
        const int ec = 2 * r + kS - m, es = 2 * l - ec;
        const double term = binom(l - kS, r) * binom(l + kS, r + kS - m) * ipow(c, ec) * ipow(s, es);
        sum += ((l - r - kS) & 1) ? -term : term;
    }
    const double pref = ((m & 1) ? -1.0 : 1.0) * fact_ratio(l, m) * sqrt((2 * l + 1) / (4.0 * kPi));
    double sp, cp;
    sincos(m * phi, &sp, &cp);
    out[i] = make_double2(pref * sum * cp, pref * sum * sp);
}

}  // namespace ylm
}  // namespace few

extern "C" FEW_API int few_ylm(const int *l, const int *m, int n, int include_minus_m, double theta, double phi,
                               void *out, int *status, void *stream) {
    few::clear_error();
    if (n < 0) return few::fail(FEW_ERR_SIZE, "few_ylm: n=%d < 0", n);
    if (n == 0) return FEW_OK;
    if (!l || !m || !out) return few::fail(FEW_ERR_ARG, "few_ylm: null pointer");
    const int nout = include_minus_m ? 2 * n : n;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    few::ylm::k_ylm<<<(nout + 127) / 128, 128, 0, st>>>(l, m, nout, include_minus_m ? 1 : 0, theta, phi,
                                                         static_cast<double2 *>(out), status);
    FEW_LAUNCH_CHECK("k_ylm");
    return FEW_OK;
}
