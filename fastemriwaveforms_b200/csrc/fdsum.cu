// Frequency-domain interpolated mode sum (stationary-phase approximation).
//
// Reference: FDInterpolatedModeSum.sum (src/few/summation/fdinterp.py:138-542)
// and its kernel make_generic_kerr_waveform_fd / get_waveform_generic_fd
// (src/few/cutils/interpolate.cu:1141-1563, helpers cube_roots :1113-1133 and
// SPAFunc :1041-1097).
//
// For every mode (l, m, k, n) and trajectory segment [t_j, t_j+1), the mode
// frequency f_mode(t) = m f_phi(t) + k f_theta(t) + n f_r(t) is a cubic in
// x = t - t_j (from the frequency splines).  Every frequency bin f_i in the
// segment's range gets, for each real root x of f_mode(t_j + x) = f_i inside
// the segment, the stationary-phase term
//     A(t) Y_lm SPA(fdot, fddot) exp(i (2 pi f_i t - Phi_mode(t)))
// and, for m != 0, its conjugate image at -f_i with Y_l,-m.
//
// Work layout (B200): the per-(mode, segment) bin ranges are planned on the
// device (k_fd_extrema, k_fd_bins); a prefix over their bin counts turns the
// ragged work into one flat bin index space, which k_fd_sum splits into equal
// contiguous slices, one per warp (lanes take consecutive bins, so the
// waveform atomics of a warp hit consecutive addresses).  FP64 throughout.
//
// Numerics follow the reference operation by operation (Cardano roots with the
// principal complex branches, the same complex arithmetic, the SPA series) so
// that results agree to the rounding of the transcendental functions; the
// planning arithmetic that decides integer bin ranges uses explicitly rounded
// operations (no contraction) so that it matches numpy's bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "few_internal.h"

namespace few {
namespace fd {

constexpr double kPi = 3.141592653589793238462643383279502884;

// ---- complex arithmetic (C99 Annex G definitions, principal branches) --------
struct cx {
    double re, im;
};

__device__ __forceinline__ cx mk(double r, double i) { return cx{r, i}; }
__device__ __forceinline__ cx cadd(cx a, cx b) { return mk(a.re + b.re, a.im + b.im); }
__device__ __forceinline__ cx csub(cx a, cx b) { return mk(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ cx cscale(cx a, double s) { return mk(a.re * s, a.im * s); }
__device__ __forceinline__ cx cdivr(cx a, double s) { return mk(a.re / s, a.im / s); }
__device__ __forceinline__ cx cmul(cx a, cx b) { return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
__device__ __forceinline__ cx cconj(cx a) { return mk(a.re, -a.im); }

// Quotient with the denominator scaled by a power of two first (the Annex G
// example algorithm), which avoids spurious overflow and underflow.
__device__ __forceinline__ cx cdiv(cx z, cx w) {
    double a = z.re, b = z.im, c = w.re, d = w.im;
    // Scaling by a power of two is exact, so when every intermediate stays a
    // normal number the unscaled quotient has the same bits.
    double mw = fmax(fabs(c), fabs(d)), mz = fmax(fabs(a), fabs(b));
    if (mw > 0x1p-250 && mw < 0x1p250 && mz < 0x1p250 && (mz > 0x1p-250 || mz == 0.0)) {
        double den = c * c + d * d;
        return mk((a * c + b * d) / den, (b * c - a * d) / den);
    }
    int sc = 0;
    double lg = logb(fmax(fabs(c), fabs(d)));
    if (isfinite(lg)) {
        sc = static_cast<int>(lg);
        c = scalbn(c, -sc);
        d = scalbn(d, -sc);
    }
    double den = c * c + d * d;
    return mk(scalbn((a * c + b * d) / den, -sc), scalbn((b * c - a * d) / den, -sc));
}

__device__ __forceinline__ double cabs_(cx z) { return hypot(z.re, z.im); }
__device__ __forceinline__ double carg(cx z) { return atan2(z.im, z.re); }

__device__ __forceinline__ cx cpolar(double rho, double th) {
    if (isnan(rho) || signbit(rho)) return mk(nan(""), nan(""));
    double s, c;
    sincos(th, &s, &c);
    double x = rho * c, y = rho * s;
    if (isnan(x)) x = 0.0;
    if (isnan(y)) y = 0.0;
    return mk(x, y);
}

__device__ __forceinline__ cx cexp_(cx z) {
    double e = exp(z.re), s, c;
    sincos(z.im, &s, &c);
    return mk(e * c, e * s);
}

__device__ __forceinline__ cx clog_(cx z) { return mk(log(cabs_(z)), carg(z)); }

__device__ __forceinline__ cx csqrt_(cx z) {
    if (isinf(z.im)) return mk(INFINITY, z.im);
    return cpolar(sqrt(cabs_(z)), carg(z) / 2.0);
}

// e^{i ph} for the large phases of the sum (|ph| up to ~1e7 rad): the angle is
// first reduced mod 2 pi by Cody & Waite's method with 2 pi split in three
// parts (the first two of 32 significant bits, so k*C1 and k*C2 are exact for
// |k| < 2^21); the reduced angle is within a few units in the last place of
// the exact remainder, and sincos then runs on |r| <= pi.  Larger angles go to
// sincos directly.
__device__ __forceinline__ cx cexp_i(double ph) {
    const double kInv2Pi = 0.15915494309189535;
    const double kC1 = 0x1.921fb54400000p+2, kC2 = 0x1.0b4611a600000p-32, kC3 = 0x1.3198a2e037073p-67;
    double r = ph;
    double kq = rint(ph * kInv2Pi);
    if (fabs(kq) < 2097152.0) {
        r = __fma_rn(-kq, kC1, ph);
        r = __fma_rn(-kq, kC2, r);
        r = __fma_rn(-kq, kC3, r);
    }
    double s, c;
    sincos(r, &s, &c);
    return mk(c, s);
}

// z^p for real p, as exp(p log z) with p promoted to complex.
__device__ __forceinline__ cx cpowr(cx z, double p) { return cexp_(cmul(mk(p, 0.0), clog_(z))); }

// ---- SPA function ----------------------------------------------------------------
// SPA(x) stands for i sqrt(x) e^{-ix} K_{1/3}(-ix) in the reference's sign and
// branch convention (interpolate.cu:1041-1097).  |x| <= 7: the power series of
// K_{1/3} = pi/sqrt(3) (I_{-1/3} - I_{1/3}),
//     SPA = e^{-ix} (P1 x^{5/6} S1(x^2) + P2 x^{1/6} S2(x^2)),
//     S1 = 1/2 sum_j (-x^2/4)^j Gamma(4/3) / (j! Gamma(j + 4/3)),
//     S2 =     sum_j (-x^2/4)^j Gamma(2/3) / (j! Gamma(j + 2/3)),
// P1 = e^{-2 pi i/3} Gamma(-1/3) / 2^{1/3}, P2 = e^{-pi i/3} Gamma(1/3) / 2^{2/3},
// fourteen terms each.  |x| > 7: the asymptotic expansion of K_nu (nu = 1/3),
//     SPA = e^{-3 pi i/4} sqrt(pi/2) sum_j a_j i^{j+1} x^{-j},
//     a_0 = 1, a_{j+1} = a_j (4 nu^2 - (2j + 1)^2) / (8 (j + 1)),
// nine terms.  The coefficients are generated here from those recurrences.
struct SpaTable {
    double s1[14], s2[14];  // S1, S2 coefficients of (x^2)^j
    double ar[9], ai[9];    // a_j i^{j+1} (real, imaginary parts)
};

constexpr SpaTable make_spa_table() {
    SpaTable t{};
    double c1 = 0.5, c2 = 1.0;
    for (int j = 0; j < 14; ++j) {
        t.s1[j] = c1;
        t.s2[j] = c2;
        c1 = c1 * (-0.25) / ((j + 1) * (j + 4.0 / 3.0));
        c2 = c2 * (-0.25) / ((j + 1) * (j + 2.0 / 3.0));
    }
    double a = 1.0;
    const double nu2x4 = 4.0 / 9.0;
    for (int j = 0; j < 9; ++j) {
        // i^{j+1}: j=0 -> i, 1 -> -1, 2 -> -i, 3 -> 1
        int q = (j + 1) & 3;
        t.ar[j] = (q == 0) ? a : (q == 2 ? -a : 0.0);
        t.ai[j] = (q == 1) ? a : (q == 3 ? -a : 0.0);
        a = a * (nu2x4 - (2.0 * j + 1.0) * (2.0 * j + 1.0)) / (8.0 * (j + 1));
    }
    return t;
}

__constant__ SpaTable c_spa = make_spa_table();

constexpr double kGammaP13 = 2.678938534707747633;   // Gamma(1/3)
constexpr double kGammaM13 = -4.062353818279201250;  // Gamma(-1/3)
constexpr double kCbrt2 = 1.259921049894873165;      // 2^{1/3}
constexpr double kCbrt4 = 1.587401051968199475;      // 2^{2/3}

// Phase factors computed at run time with the same complex exponential as
// the reference (their roundings are part of its values).
struct SpaConsts {
    cx e23, e13, e34;  // e^{-2 pi i/3}, e^{-pi i/3}, e^{-3 pi i/4}
    double sqrt_half_pi;
    // For a real argument r + 0i, the general csqrt_ and cpowr take the angle
    // atan2(+0, r): +0 for r > 0 (sincos gives exactly (0, 1)) and pi for
    // r < 0.  The sincos of the angles that follow from pi (pi/2 for the square
    // root, p*pi for z^p) are computed once here with the same functions, so
    // the real-argument paths below return the general functions' bits.
    double half_s, half_c;    // sincos(pi / 2)
    double third_s, third_c;  // sincos((1/3) pi)
    double sixth_s, sixth_c;  // sincos((1/6) pi)
};

__device__ __forceinline__ SpaConsts spa_consts() {
    SpaConsts k;
    k.e23 = cexp_(cdivr(cscale(mk(0.0, 1.0), -2.0 * kPi), 3.0));
    k.e13 = cexp_(cdivr(cscale(mk(0.0, 1.0), -kPi), 3.0));
    k.e34 = cexp_(cscale(cscale(mk(-0.0, -1.0), 0.75), kPi));
    k.sqrt_half_pi = sqrt(0.5 * kPi);
    const double pi_arg = atan2(0.0, -1.0);
    sincos(pi_arg / 2.0, &k.half_s, &k.half_c);
    sincos(__dmul_rn(1.0 / 3.0, pi_arg), &k.third_s, &k.third_c);
    sincos(__dmul_rn(1.0 / 6.0, pi_arg), &k.sixth_s, &k.sixth_c);
    return k;
}

// csqrt_(r + 0i): the same bits without atan2 and sincos.
__device__ __forceinline__ cx csqrt_real(double r, const SpaConsts &K) {
    if (!isfinite(r)) return csqrt_(mk(r, 0.0));
    const double rho = sqrt(fabs(r));  // hypot(r, +-0) is fabs(r) (CUDA's documented special case)
    if (r > 0.0 || (r == 0.0 && !signbit(r))) return mk(rho * 1.0, rho * 0.0);
    return mk(rho * K.half_c, rho * K.half_s);
}

// cpowr(r + 0i, p) for p = 1/3 (third = true) or 1/6: exp(p log|r|) times the
// phase factor of the angle 0 (r > 0) or p*pi (r < 0).
__device__ __forceinline__ cx cpowr_real(double r, double p, bool third, const SpaConsts &K) {
    if (!isfinite(r) || r == 0.0) return cpowr(mk(r, 0.0), p);
    const double e = exp(p * log(fabs(r)));  // hypot(r, +-0) is fabs(r)
    if (r > 0.0) return mk(e * 1.0, e * 0.0);
    return third ? mk(e * K.third_c, e * K.third_s) : mk(e * K.sixth_c, e * K.sixth_s);
}

__device__ cx spa(double x, const SpaConsts &K) {
    if (fabs(x) <= 7.0) {
        cx p6 = cpowr_real(x, 1.0 / 6.0, false, K);
        cx pref1 = cdivr(cscale(cmul(cmul(cmul(cmul(cmul(K.e23, p6), p6), p6), p6), p6), kGammaM13), kCbrt2);
        cx pref2 = cdivr(cscale(cmul(K.e13, p6), kGammaP13), kCbrt4);
        double x2 = x * x;
        double s1 = c_spa.s1[13], s2 = c_spa.s2[13];
#pragma unroll
        for (int j = 12; j >= 0; --j) {
            s1 = c_spa.s1[j] + x2 * s1;
            s2 = c_spa.s2[j] + x2 * s2;
        }
        // cexp_(-0 x - i x): exp(+-0) is exactly 1, so the factor is (cos x, -sin x)
        double sx, cxv;
        sincos(-x, &sx, &cxv);
        cx ph = mk(cxv, sx);
        return cmul(ph, cadd(cscale(pref1, s1), cscale(pref2, s2)));
    }
    cx y = mk(1.0 / x, 0.0);
    cx pref = cscale(K.e34, K.sqrt_half_pi);
    cx ser = mk(c_spa.ar[8], c_spa.ai[8]);
#pragma unroll
    for (int j = 7; j >= 0; --j) ser = cadd(mk(c_spa.ar[j], c_spa.ai[j]), cmul(y, ser));
    return cmul(pref, ser);
}

// Roots of a x^3 + b x^2 + c x + d by Cardano's formula with principal complex
// branches (interpolate.cu:1113-1133); the real parts are returned.
__device__ __forceinline__ void cube_roots(double a, double b, double c, double d, cx xi, double r[3],
                                           const SpaConsts &K) {
    double b2 = b * b, b3 = b2 * b, a2 = a * a;
    double D0 = b2 - 3 * a * c;
    double D1 = 2 * b3 - 9 * a * b * c + 27 * a2 * d;
    cx S = csqrt_real(D1 * D1 - 4 * (D0 * D0 * D0), K);
    cx z = cdivr(mk(S.re + D1, S.im), 2.0);
    cx C = (z.im == 0.0 && !signbit(z.im)) ? cpowr_real(z.re, 1.0 / 3.0, true, K) : cpowr(z, 1.0 / 3.0);
    double s = -(1.0 / (3 * a));
    cx D0c = mk(D0, 0.0);
    cx xC = cmul(xi, C);
    cx xxC = cmul(cmul(xi, xi), C);
    r[0] = cscale(cadd(mk(b + C.re, C.im), cdiv(D0c, C)), s).re;
    r[1] = cscale(cadd(mk(b + xC.re, xC.im), cdiv(D0c, xC)), s).re;
    r[2] = cscale(cadd(mk(b + xxC.re, xxC.im), cdiv(D0c, xxC)), s).re;
}

// ---- planning (fdinterp.py:262-430) ----------------------------------------------
// Explicitly rounded helpers: the planning must reproduce numpy's roundings.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// m*f0 + k*f1 + n*f2 in numpy's order for integer mode numbers.
__device__ __forceinline__ double mode_comb(int m, int k, int n, double f0, double f1, double f2) {
    return add(add(mul((double)m, f0), mul((double)k, f1)), mul((double)n, f2));
}

// x^3 rounded once (numpy's x**3 is libm pow): exact x^2 by a two-product, then
// the exact product with x split in two, summed with a single final rounding
// up to a last-place tie.
__device__ __forceinline__ double cube_rn(double x) {
    double p = __dmul_rn(x, x);
    double pe = __fma_rn(x, x, -p);
    double q = __dmul_rn(p, x);
    double qe = __fma_rn(p, x, -q);
    return __dadd_rn(q, __fma_rn(pe, x, qe));
}

// numpy argmax/argmin: the first maximum (minimum); a NaN wins, the first one.
// i == kEmpty marks a thread that saw no element.
constexpr int kEmpty = 0x7fffffff;

struct Arg {
    double v;
    int i;
};

__device__ __forceinline__ bool better_max(const Arg &a, const Arg &b) {  // a before b?
    if (a.i == kEmpty) return false;
    if (b.i == kEmpty) return true;
    bool an = isnan(a.v), bn = isnan(b.v);
    if (an || bn) return an && (!bn || a.i < b.i);
    return a.v > b.v || (a.v == b.v && a.i < b.i);
}

__device__ __forceinline__ bool better_min(const Arg &a, const Arg &b) {
    if (a.i == kEmpty) return false;
    if (b.i == kEmpty) return true;
    bool an = isnan(a.v), bn = isnan(b.v);
    if (an || bn) return an && (!bn || a.i < b.i);
    return a.v < b.v || (a.v == b.v && a.i < b.i);
}

// np.sort of two or three values (NaN sorts last).
__device__ __forceinline__ bool lt_nan_last(double a, double b) { return !isnan(a) && (isnan(b) || a < b); }

// Output of k_fd_extrema per mode and list (0: the frequency maximum, 1: the
// minimum): flag (turnover inside (0, t[-1])), target segment, the turnover
// frequency, and the root keep bits.
struct Turn {
    double fext;
    int valid, seg;  // seg: the segment whose range is widened (Python's -1 -> N-2)
    int keep;        // bit 0: root 1 kept, bit 1: root 2 kept
    int pad;
};

// flags[0] bits (few_fd_plan_extrema / few_fd_plan_bins); flags[1] counts the
// interior turnovers over all modes and both lists.
constexpr int kFlagAnyKeep = 1;    // some turnover root lies inside its segment
constexpr int kFlagBothKeep = 2;   // a segment holds both roots (the reference stops there)
constexpr int kFlagDiscBad = 4;    // a discriminant below -1e10 (the reference stops there)
constexpr int kFlagNan = 8;        // a NaN among the dense frequencies

__device__ __forceinline__ int search_left(const double *t, int N, double v) {
    int lo = 0, hi = N;  // first index with t[i] >= v
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (t[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ double t_dense(int d, int D, double start, double step, double stop) {
    return d == D - 1 ? stop : add(mul((double)d, step), start);
}

// One block per mode.  fd: (3, D) frequencies on the dense grid; fc: the
// frequency spline coefficients (4, N, 3) (knot-major).
__global__ void k_fd_extrema(const double *__restrict__ fdense, int D, double tn_start, double tn_step,
                             double tn_stop, const double *__restrict__ t, int N, const double *__restrict__ fc,
                             const int *__restrict__ m_arr, const int *__restrict__ k_arr,
                             const int *__restrict__ n_arr, int K, Turn *__restrict__ turns, int *flags) {
    int mode = blockIdx.x;
    if (mode >= K) return;
    int m = m_arr[mode], k = k_arr[mode], n = n_arr[mode];
    Arg mx{0.0, kEmpty}, mn{0.0, kEmpty};
    for (int d = threadIdx.x; d < D; d += blockDim.x) {
        Arg v{mode_comb(m, k, n, fdense[d], fdense[D + d], fdense[2 * D + d]), d};
        if (better_max(v, mx)) mx = v;
        if (better_min(v, mn)) mn = v;
    }
    __shared__ Arg s_mx[32], s_mn[32];
    for (int off = 16; off > 0; off >>= 1) {
        Arg o{__shfl_down_sync(0xffffffffu, mx.v, off), __shfl_down_sync(0xffffffffu, mx.i, off)};
        if (better_max(o, mx)) mx = o;
        Arg p{__shfl_down_sync(0xffffffffu, mn.v, off), __shfl_down_sync(0xffffffffu, mn.i, off)};
        if (better_min(p, mn)) mn = p;
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) { s_mx[w] = mx; s_mn[w] = mn; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int i = 1; i < nw; ++i) {
        if (better_max(s_mx[i], mx)) mx = s_mx[i];
        if (better_min(s_mn[i], mn)) mn = s_mn[i];
    }
    if (isnan(mx.v) || isnan(mn.v)) atomicOr(flags, kFlagNan);
    const double tlast = t[N - 1];
    for (int which = 0; which < 2; ++which) {
        Turn o{0.0, 0, 0, 0, 0};
        double tof = t_dense(which == 0 ? mx.i : mn.i, D, tn_start, tn_step, tn_stop);
        if (tof > 0.0 && tof < tlast) {
            o.valid = 1;
            atomicAdd(flags + 1, 1);
            int seg = search_left(t, N, tof) - 1;          // may be -1 (Python wraps it)
            int sc = seg < 0 ? seg + N : seg;              // coefficient column
            double t0 = t[sc], t1 = t[seg + 1 < N ? seg + 1 : seg + 1 - N];
            o.seg = seg < 0 ? seg + (N - 1) : seg;         // target segment of the widening
            // cubic a x^3 + b x^2 + c x + d of this mode's frequency on the segment
            double cf[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double *row = fc + (size_t)q * N * 3 + (size_t)sc * 3;
                cf[q] = mode_comb(m, k, n, row[0], row[1], row[2]);
            }
            double a = cf[3], b = cf[2], c = cf[1], d = cf[0];
            double inner = sub(mul(mul(2.0, b), mul(2.0, b)), mul(mul(4.0, mul(3.0, a)), c));
            if (inner < -1e10) atomicOr(flags, kFlagDiscBad);
            if (inner < 0.0) inner = 0.0;
            double sq = sqrt(inner);
            double den = mul(2.0, mul(3.0, a));
            double r1 = __ddiv_rn(add(-mul(2.0, b), sq), den);
            double r2 = __ddiv_rn(sub(-mul(2.0, b), sq), den);
            double tr1 = add(t0, r1), tr2 = add(t0, r2);
            int k1 = (t0 < tr1) && (t1 > tr1), k2 = (t0 < tr2) && (t1 > tr2);
            o.keep = k1 | (k2 << 1);
            if (k1 && k2) atomicOr(flags, kFlagBothKeep);
            if (k1 || k2) atomicOr(flags, kFlagAnyKeep);
            double tfix = add(mul(tr1, (double)k1), mul(tr2, (double)k2));
            double x = sub(tfix, t0);
            o.fext = add(add(add(mul(a, cube_rn(x)), mul(b, mul(x, x))), mul(c, x)), d);
        }
        turns[2 * mode + which] = o;
    }
}

// numpy float64 -> int64 (astype(int), x86 semantics): NaN and values out of
// range give INT64_MIN.
__device__ __forceinline__ long long to_i64(double x) {
    if (!(x > -9223372036854775808.0 && x < 9223372036854775808.0)) return (long long)0x8000000000000000ULL;
    return (long long)x;  // truncation toward zero
}

__device__ __forceinline__ long long bin_index(double v, double f0, double df, int has_farr, double fpos1,
                                               int zero_index) {
    long long i = to_i64(fabs(__ddiv_rn(sub(v, f0), df)));
    if (has_farr && v > 0.0)  // int64 arithmetic wraps, as numpy's does
        i = (long long)((unsigned long long)to_i64(fabs(__ddiv_rn(sub(v, fpos1), df))) + zero_index + 1);
    return i;
}

// One thread per (mode, segment) entry e = mode*(N-1) + seg.  fk: frequencies
// at the knots (3, N).  Writes the reference's int32 start/end (before the
// kernel's range check) and the clamped range [lo, lo + count).
__global__ void k_fd_bins(const double *__restrict__ fk, const int *__restrict__ m_arr,
                          const int *__restrict__ k_arr, const int *__restrict__ n_arr, int K, int N,
                          const Turn *__restrict__ turns, const int *__restrict__ flags, double f0, double df,
                          int has_farr, double fpos1, int zero_index, int L, int *__restrict__ start32,
                          int *__restrict__ end32, int *__restrict__ lo_out, long long *__restrict__ count) {
    long long E = (long long)K * (N - 1);
    // fdinterp.py:367-376 joins the (n, 2) segment bounds with the (1, n) row of
    // turnover frequencies; for n != 1 that raises the ValueError its handler
    // swallows, so the widening happens only for a single interior turnover.
    bool apply = (flags[0] & kFlagAnyKeep) != 0 && flags[1] == 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < E;
         e += (long long)gridDim.x * blockDim.x) {
        int mode = (int)(e / (N - 1)), seg = (int)(e % (N - 1));
        int m = m_arr[mode], k = k_arr[mode], n = n_arr[mode];
        double v0 = mode_comb(m, k, n, fk[seg], fk[N + seg], fk[2 * N + seg]);
        double v1 = mode_comb(m, k, n, fk[seg + 1], fk[N + seg + 1], fk[2 * N + seg + 1]);
        double lo = lt_nan_last(v1, v0) ? v1 : v0, hi = lt_nan_last(v1, v0) ? v0 : v1;
        if (apply) {
            const double blo = lo, bhi = hi;
            for (int which = 0; which < 2; ++which) {  // the minimum's widening is assigned last
                Turn tr = turns[2 * mode + which];
                if (!tr.valid || tr.seg != seg) continue;
                double w3[3] = {blo, bhi, tr.fext};
                // sort three, NaN last
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2 - a; ++b)
                        if (lt_nan_last(w3[b + 1], w3[b])) { double s = w3[b]; w3[b] = w3[b + 1]; w3[b + 1] = s; }
                lo = w3[0];
                hi = w3[2];
            }
        }
        long long s64 = (long long)((unsigned long long)bin_index(lo, f0, df, has_farr, fpos1, zero_index) + 1);
        long long e64 = bin_index(hi, f0, df, has_farr, fpos1, zero_index);
        int s = (int)(uint32_t)(unsigned long long)s64, en = (int)(uint32_t)(unsigned long long)e64;
        start32[e] = s;
        end32[e] = en;
        int a = s < 0 ? 0 : s, b = en > L - 1 ? L - 1 : en;
        lo_out[e] = a;
        count[e] = b >= a ? (long long)(b - a + 1) : 0;
    }
}

// ---- the sum ----------------------------------------------------------------------
struct SumArgs {
    double2 *wf;
    int L, zero_index, include_minus_m, N, K;
    const double *freq;
    const double *amp;  // amplitude spline: coefficient q of series p at knot j: amp[q*aq + p*ap + j*aj]
    long long aq, ap, aj;
    const double *fco;  // frequency spline, same indexing with fq, fp, fj (series 0..2)
    long long fq, fp, fj;
    const double *pc;   // phase coefficients: pc[c*pcc + field*pcf + seg*pcs], c = 0..7
    long long pcc, pcf, pcs;
    const double *phase_t, *t;
    const int *m, *k, *n;
    const double2 *ylms;  // (2K): +m then -m (already times (-1)^l)
    const int *lo;
    const long long *prefix;  // (E + 1) exclusive prefix of the bin counts
    long long E;
};

// Last e in [lo, hi] with prefix[e] <= b (prefix[lo] <= b assumed).
__device__ __forceinline__ long long find_entry(const long long *prefix, long long lo, long long hi, long long b) {
    while (lo < hi) {
        long long mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Advance a lane's entry e (prefix[e] <= b) to the entry holding bin b: a
// look at the next boundary, then an exponential search, then bisection.
__device__ __forceinline__ long long advance_entry(const long long *prefix, long long E, long long e, long long b) {
    if (prefix[e + 1] > b) return e;
    long long step = 1, lo = e + 1;
    while (lo + step < E && prefix[lo + step] <= b) {
        lo += step;
        step <<= 1;
    }
    long long hi = lo + step < E ? lo + step : E - 1;
    return find_entry(prefix, lo, hi, b);
}

__device__ __forceinline__ void red_add(double2 *p, cx v) {
    atomicAdd(&p->x, v.re);
    atomicAdd(&p->y, v.im);
}

template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_fd_sum(SumArgs A) {
    const long long B = A.prefix[A.E];
    const long long W = (long long)gridDim.x * (blockDim.x >> 5);
    const long long w = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const long long b0 = B * w / W, b1 = B * (w + 1) / W;
    // run-time constants of the SPA function and of Cardano's formula, once per
    // CTA in shared memory (they would hold 18 registers for the whole kernel)
    __shared__ SpaConsts s_sk;
    __shared__ cx s_xi;
    if (threadIdx.x == 0) {
        s_sk = spa_consts();
        s_xi = cdivr(cadd(mk(-1.0, 0.0), csqrt_(mk(-3.0, 0.0))), 2.0);
    }
    __syncthreads();
    if (b0 >= b1) return;
    const SpaConsts &SK = s_sk;
    const cx &xi = s_xi;
    const int nseg = A.N - 1;
    long long e = find_entry(A.prefix, 0, A.E - 1, b0 + lane < b1 ? b0 + lane : b1 - 1);
    for (long long base = b0; base < b1; base += 32) {
        long long b = base + lane;
        if (b >= b1) break;
        e = advance_entry(A.prefix, A.E, e, b);
        int i = A.lo[e] + (int)(b - A.prefix[e]);
        int mode = (int)(e / nseg), seg = (int)(e % nseg);
        int m = A.m[mode], k = A.k[mode], n = A.n[mode];
        double f = A.freq[i];
        // mode-frequency cubic on this segment
        const double *fy = A.fco + (long long)seg * A.fj;
        double fyv = m * fy[0] + k * fy[A.fp] + n * fy[2 * A.fp];
        double fc1 = m * fy[A.fq] + k * fy[A.fq + A.fp] + n * fy[A.fq + 2 * A.fp];
        double fc2 = m * fy[2 * A.fq] + k * fy[2 * A.fq + A.fp] + n * fy[2 * A.fq + 2 * A.fp];
        double fc3 = m * fy[3 * A.fq] + k * fy[3 * A.fq + A.fp] + n * fy[3 * A.fq + 2 * A.fp];
        double roots[3];
        cube_roots(fc3, fc2, fc1, fyv - f, xi, roots, SK);
        const double ts = A.t[seg], te = A.t[seg + 1];
        for (int r = 0; r < 3; ++r) {
            double x = roots[r];
            double tt = ts + x;
            if (!(tt < te && tt >= ts)) continue;
            double x2 = x * x, x3 = x * x2;
            const double *ar = A.amp + (long long)mode * A.ap + (long long)seg * A.aj;
            const double *ai = ar + (long long)A.K * A.ap;
            double Rre = ar[0] + ar[A.aq] * x + ar[2 * A.aq] * x2 + ar[3 * A.aq] * x3;
            double Rim = ai[0] + ai[A.aq] * x + ai[2 * A.aq] * x2 + ai[3 * A.aq] * x3;
            double h = A.phase_t[seg + 1] - A.phase_t[seg];
            double s = (tt - A.phase_t[seg]) / h;
            double s1 = 1.0 - s, s2 = s * s, s3 = s * s2, s4 = s * s3, s5 = s * s4;
            double h2 = h * h, h3 = h * h2;
            double phase = 0.0, fdot = 0.0, fddot = 0.0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int mult = q == 0 ? m : (q == 1 ? k : n);
                const double *c = A.pc + (long long)q * A.pcf + (long long)seg * A.pcs;
                double c0 = c[0], c1 = c[A.pcc], c2 = c[2 * A.pcc], c3 = c[3 * A.pcc];
                double c4 = c[4 * A.pcc], c5 = c[5 * A.pcc], c6 = c[6 * A.pcc], c7 = c[7 * A.pcc];
                double P = c0 + s * (c1 + s1 * (c2 + s * (c3 + s1 * (c4 + s * (c5 + s1 * (c6 + s * c7))))));
                double d2 = (-2. * c2 + c3 * (2. - 6. * s) + c4 * (2. - 12. * s + 12. * s2) +
                             c5 * (6. * s - 24. * s2 + 20. * s3) + c6 * (6. * s - 36. * s2 + 60. * s3 - 30. * s4) +
                             c7 * (12. * s2 - 60. * s3 + 90. * s4 - 42. * s5)) /
                            (2. * kPi * h2);
                double d3 = (-6. * c3 + c4 * (-12. + 24. * s) + c5 * (6. - 48. * s + 60. * s2) +
                             c6 * (6. - 72. * s + 180. * s2 - 120. * s3) +
                             c7 * (24. * s - 180. * s2 + 360. * s3 - 210. * s4)) /
                            (2. * kPi * h3);
                if (q == 0) { phase = mult * P; fdot = mult * d2; fddot = mult * d3; }
                else { phase += mult * P; fdot += mult * d2; fddot += mult * d3; }
            }
            double arg = 2. * kPi * fdot * fdot * fdot / (3. * fddot * fddot);
            double pre = -1.0 * fdot / fabs(fddot) * 2. / sqrt(3.);
            cx amp2 = cdiv(cscale(spa(arg, SK), pre), csqrt_real(arg, SK));
            double ph = 2. * kPi * f * tt - phase;
            cx te_ = cmul(cmul(mk(Rre, Rim), amp2), cexp_i(ph));
            double2 yp = A.ylms[mode];
            red_add(A.wf + i, cmul(mk(yp.x, yp.y), te_));
            if (m != 0 && A.include_minus_m) {
                int im = 2 * A.zero_index - i;
                if (im >= 0 && im < A.L) {
                    double2 ym = A.ylms[A.K + mode];
                    red_add(A.wf + im, cmul(mk(ym.x, ym.y), cconj(te_)));
                }
            }
        }
    }
}

// (h+, hx) from the two-sided spectrum (fdinterp.py:518-536):
//   s = -flip(w);  p = Re(s + flip s)/2 + i Im(s - flip s)/2,
//   c = -Im(s + flip s)/2 + i Re(s - flip s)/2,  j = first .. first+count-1.
__global__ void k_fd_finalize(const double2 *__restrict__ w, int L, int first, int count,
                              double2 *__restrict__ out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) {
        int jj = first + j;
        double2 a = w[L - 1 - jj], b = w[jj];  // s[jj] = -a, flip(s)[jj] = -b
        double pre = add(-a.x, -b.x), pim = add(-a.y, -b.y);
        double mre = sub(-a.x, -b.x), mim = sub(-a.y, -b.y);
        out[j] = make_double2(pre / 2.0, mim / 2.0);
        out[count + j] = make_double2(-pim / 2.0, mre / 2.0);
    }
}

// Default two-sided frequency grid (fdinterp.py:398-403): f_j = (j - L/2) / (L dt),
// the integer numerator exact, one rounding in the quotient (as numpy's).
__global__ void k_fd_grid(double *f, int L, double Ldt) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < L; j += gridDim.x * blockDim.x)
        f[j] = __ddiv_rn((double)(j - L / 2), Ldt);
}

// The kernel's range rule on given int32 start/end indices: bins
// [max(start, 0), min(end, L-1)].
__global__ void k_fd_range(const int *__restrict__ start32, const int *__restrict__ end32, long long E, int L,
                           int *__restrict__ lo, long long *__restrict__ count) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < E;
         e += (long long)gridDim.x * blockDim.x) {
        int s = start32[e], en = end32[e];
        int a = s < 0 ? 0 : s, b = en > L - 1 ? L - 1 : en;
        lo[e] = a;
        count[e] = b >= a ? (long long)(b - a + 1) : 0;
    }
}

// Exclusive prefix of count (E,) into prefix (E + 1,) in three launches over
// G contiguous chunks: the chunk totals, their scan (one CTA), then each
// chunk's own scan offset by its chunk's prefix, in tiles of 256 x 4 counts.
constexpr int kScanThreads = 256, kScanPer = 4, kScanMaxChunks = 1024;

__device__ __forceinline__ long long block_exclusive_scan(long long v, long long *s_warp, long long *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    long long x = v;
    for (int off = 1; off < 32; off <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        long long t = lane < nw ? s_warp[lane] : 0;
        for (int off = 1; off < 32; off <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, t, off);
            if (lane >= off) t += y;
        }
        if (lane < nw) s_warp[lane] = t;  // inclusive warp totals
    }
    __syncthreads();
    long long before = (w > 0 ? s_warp[w - 1] : 0) + x - v;
    *total = s_warp[nw - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(kScanThreads) k_fd_scan_totals(const long long *__restrict__ count, long long E,
                                                                 long long chunk, long long *__restrict__ totals) {
    __shared__ long long s_warp[32];
    const long long c0 = blockIdx.x * chunk, c1 = c0 + chunk < E ? c0 + chunk : E;
    long long sum = 0;
    for (long long e = c0 + threadIdx.x; e < c1; e += blockDim.x) sum += count[e];
    long long tot;
    block_exclusive_scan(sum, s_warp, &tot);
    if (threadIdx.x == 0) totals[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanMaxChunks) k_fd_scan_chunks(long long *__restrict__ totals, int G,
                                                                  long long *__restrict__ prefix, long long E) {
    __shared__ long long s_warp[32];
    long long v = threadIdx.x < G ? totals[threadIdx.x] : 0, tot;
    long long before = block_exclusive_scan(v, s_warp, &tot);
    if (threadIdx.x < G) totals[threadIdx.x] = before;
    if (threadIdx.x == 0) prefix[E] = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_fd_scan_write(const long long *__restrict__ count, long long E,
                                                                long long chunk, const long long *__restrict__ offs,
                                                                long long *__restrict__ prefix) {
    __shared__ long long s_warp[32];
    const long long c0 = blockIdx.x * chunk, c1 = c0 + chunk < E ? c0 + chunk : E;
    long long run = offs[blockIdx.x];
    for (long long base = c0; base < c1; base += (long long)kScanThreads * kScanPer) {
        const long long e0 = base + (long long)threadIdx.x * kScanPer;
        long long v[kScanPer], sum = 0;
#pragma unroll
        for (int j = 0; j < kScanPer; ++j) {
            v[j] = e0 + j < c1 ? count[e0 + j] : 0;
            sum += v[j];
        }
        long long tot;
        long long p = run + block_exclusive_scan(sum, s_warp, &tot);
#pragma unroll
        for (int j = 0; j < kScanPer; ++j) {
            if (e0 + j < c1) prefix[e0 + j] = p;
            p += v[j];
        }
        run += tot;
    }
}

}  // namespace fd
}  // namespace few

using few::fd::Turn;

extern "C" FEW_API int few_fd_turn_bytes(void) { return (int)sizeof(Turn); }

extern "C" FEW_API int few_fd_plan_extrema(const double *fdense, int D, double tn_start, double tn_step,
                                           double tn_stop, const double *t, int N, const double *fcoef,
                                           const int *m, const int *k, const int *n, int K, void *turns, int *flags,
                                           void *stream) {
    few::clear_error();
    if (K < 0 || N < 4 || D < 2) return few::fail(FEW_ERR_SIZE, "few_fd_plan_extrema: K=%d N=%d D=%d", K, N, D);
    if (K == 0) return FEW_OK;
    if (!fdense || !t || !fcoef || !m || !k || !n || !turns || !flags)
        return few::fail(FEW_ERR_ARG, "few_fd_plan_extrema: null pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    few::fd::k_fd_extrema<<<K, 256, 0, st>>>(fdense, D, tn_start, tn_step, tn_stop, t, N, fcoef, m, k, n, K,
                                              static_cast<Turn *>(turns), flags);
    FEW_LAUNCH_CHECK("k_fd_extrema");
    return FEW_OK;
}

extern "C" FEW_API int few_fd_plan_bins(const double *fknots, const int *m, const int *k, const int *n, int K, int N,
                                        const void *turns, const int *flags, double f0, double df, int has_farr,
                                        double fpos1, int zero_index, int L, int *start32, int *end32, int *lo,
                                        long long *count, void *stream) {
    few::clear_error();
    if (K < 0 || N < 2 || L < 1) return few::fail(FEW_ERR_SIZE, "few_fd_plan_bins: K=%d N=%d L=%d", K, N, L);
    if (K == 0) return FEW_OK;
    if (!fknots || !m || !k || !n || !turns || !flags || !start32 || !end32 || !lo || !count)
        return few::fail(FEW_ERR_ARG, "few_fd_plan_bins: null pointer");
    if (!(df != 0.0)) return few::fail(FEW_ERR_ARG, "few_fd_plan_bins: zero frequency spacing");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    long long E = (long long)K * (N - 1);
    int blocks = (int)((E + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    few::fd::k_fd_bins<<<blocks, 256, 0, st>>>(fknots, m, k, n, K, N, static_cast<const Turn *>(turns), flags, f0,
                                               df, has_farr, fpos1, zero_index, L, start32, end32, lo, count);
    FEW_LAUNCH_CHECK("k_fd_bins");
    return FEW_OK;
}

extern "C" FEW_API int few_fd_sum(void *wf, int L, const double *freq, int zero_index, int include_minus_m,
                                  const double *amp, long long aq, long long ap, long long aj, const double *fco,
                                  long long fq, long long fp, long long fj, const double *pc, long long pcc,
                                  long long pcf, long long pcs, const double *phase_t, const double *t, int N,
                                  const int *m, const int *k, const int *n, int K, const void *ylms, const int *lo,
                                  const long long *prefix, int blocks, int ctas_per_sm, void *stream) {
    few::clear_error();
    if (K < 0 || N < 2 || L < 1) return few::fail(FEW_ERR_SIZE, "few_fd_sum: K=%d N=%d L=%d", K, N, L);
    if (K == 0) return FEW_OK;
    if (!wf || !freq || !amp || !fco || !pc || !phase_t || !t || !m || !k || !n || !ylms || !lo || !prefix)
        return few::fail(FEW_ERR_ARG, "few_fd_sum: null pointer");
    if (zero_index < 0 || zero_index >= L) return few::fail(FEW_ERR_ARG, "few_fd_sum: zero_index=%d", zero_index);
    few::fd::SumArgs A;
    A.wf = static_cast<double2 *>(wf);
    A.L = L;
    A.zero_index = zero_index;
    A.include_minus_m = include_minus_m;
    A.N = N;
    A.K = K;
    A.freq = freq;
    A.amp = amp; A.aq = aq; A.ap = ap; A.aj = aj;
    A.fco = fco; A.fq = fq; A.fp = fp; A.fj = fj;
    A.pc = pc; A.pcc = pcc; A.pcf = pcf; A.pcs = pcs;
    A.phase_t = phase_t;
    A.t = t;
    A.m = m; A.k = k; A.n = n;
    A.ylms = static_cast<const double2 *>(ylms);
    A.lo = lo;
    A.prefix = prefix;
    A.E = (long long)K * (N - 1);
    // ctas_per_sm selects the register budget of the kernel (1: 255, 2: 128,
    // 3: 80 registers a thread); blocks is the grid (0: 32 CTAs per SM: the
    // static slices of the bin space are short enough that the last warps to
    // finish trail by little; measured 83.9 ms against 85.6 ms at 8 per SM on
    // the one-year, 3843-mode case).
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (blocks <= 0) blocks = 148 * 32;
    if (ctas_per_sm <= 0) ctas_per_sm = 2;
    if (ctas_per_sm == 1) few::fd::k_fd_sum<1><<<blocks, 256, 0, st>>>(A);
    else if (ctas_per_sm == 3) few::fd::k_fd_sum<3><<<blocks, 256, 0, st>>>(A);
    else few::fd::k_fd_sum<2><<<blocks, 256, 0, st>>>(A);
    FEW_LAUNCH_CHECK("k_fd_sum");
    return FEW_OK;
}

extern "C" FEW_API int few_fd_finalize(const void *wf, int L, int first, int count, void *out, void *stream) {
    few::clear_error();
    if (L < 1 || first < 0 || count < 0 || first + count > L)
        return few::fail(FEW_ERR_SIZE, "few_fd_finalize: L=%d first=%d count=%d", L, first, count);
    if (count == 0) return FEW_OK;
    if (!wf || !out) return few::fail(FEW_ERR_ARG, "few_fd_finalize: null pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int blocks = (count + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    few::fd::k_fd_finalize<<<blocks, 256, 0, st>>>(static_cast<const double2 *>(wf), L, first, count,
                                                   static_cast<double2 *>(out));
    FEW_LAUNCH_CHECK("k_fd_finalize");
    return FEW_OK;
}

extern "C" FEW_API int few_fd_frequency_grid(double *f, int L, double Ldt, void *stream) {
    few::clear_error();
    if (L < 1) return few::fail(FEW_ERR_SIZE, "few_fd_frequency_grid: L=%d", L);
    if (!f) return few::fail(FEW_ERR_ARG, "few_fd_frequency_grid: null pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int blocks = (L + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    few::fd::k_fd_grid<<<blocks, 256, 0, st>>>(f, L, Ldt);
    FEW_LAUNCH_CHECK("k_fd_grid");
    return FEW_OK;
}

namespace few {
namespace fd {

// prefix (E + 1) of count (E); scratch holds kScanMaxChunks long longs.
static int launch_scan(const long long *count, long long E, long long *prefix, long long *scratch, cudaStream_t st) {
    long long G = (E + 4095) / 4096;  // at least 4096 counts a chunk
    if (G < 1) G = 1;
    if (G > kScanMaxChunks) G = kScanMaxChunks;
    const long long chunk = (E + G - 1) / G > 0 ? (E + G - 1) / G : 1;
    k_fd_scan_totals<<<(int)G, kScanThreads, 0, st>>>(count, E, chunk, scratch);
    k_fd_scan_chunks<<<1, kScanMaxChunks, 0, st>>>(scratch, (int)G, prefix, E);
    k_fd_scan_write<<<(int)G, kScanThreads, 0, st>>>(count, E, chunk, scratch, prefix);
    FEW_LAUNCH_CHECK("k_fd_scan");
    return FEW_OK;
}

}  // namespace fd
}  // namespace few

extern "C" FEW_API int few_fd_scan(const long long *count, long long E, long long *prefix, long long *scratch,
                                   void *stream) {
    few::clear_error();
    if (E < 0) return few::fail(FEW_ERR_SIZE, "few_fd_scan: E=%lld", E);
    if (!count || !prefix || !scratch) return few::fail(FEW_ERR_ARG, "few_fd_scan: null pointer");
    return few::fd::launch_scan(count, E, prefix, scratch, static_cast<cudaStream_t>(stream));
}

// Drop-in for get_waveform_generic_fd (interpolate.hh:33-38, interpolate.cu:1525-1563)
// with the reference's argument list and layouts: interp_array (4, 2K+3, N)
// (amplitude series then f_phi, f_theta, f_r), phase_interp_coeffs (8, 3, N-1),
// seg_start/end_inds (K, N-1) int32, Ylm_all (2K) with the -m half already
// multiplied by (-1)^l.  Plus the stream.  Accumulates into waveform (L).
extern "C" FEW_API int few_get_waveform_fd(void *waveform, const double *interp_array, const double *phase_interp_t,
                                           const double *phase_interp_coeffs, const int *m, const int *k,
                                           const int *n, int num_teuk_modes, double delta_t,
                                           const double *old_time_arr, int init_length, int data_length,
                                           const double *frequencies, const int *seg_start_inds,
                                           const int *seg_end_inds, int num_segments, const void *Ylm_all,
                                           int zero_index, int include_minus_m, int separate_modes, void *stream) {
    (void)delta_t;
    few::clear_error();
    const int K = num_teuk_modes, N = init_length, L = data_length;
    if (separate_modes)
        return few::fail(FEW_ERR_ARG, "few_get_waveform_fd: separate_modes is not supported (the reference kernel "
                                      "writes mode_i * data_length + i into a data_length buffer)");
    if (K < 0 || N < 2 || L < 1 || num_segments != N - 1)
        return few::fail(FEW_ERR_SIZE, "few_get_waveform_fd: K=%d init_length=%d data_length=%d num_segments=%d", K, N,
                         L, num_segments);
    if (K == 0) return FEW_OK;
    if (!waveform || !interp_array || !phase_interp_t || !phase_interp_coeffs || !m || !k || !n || !old_time_arr ||
        !frequencies || !seg_start_inds || !seg_end_inds || !Ylm_all)
        return few::fail(FEW_ERR_ARG, "few_get_waveform_fd: null pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long E = (long long)K * (N - 1);
    void *buf = nullptr;
    size_t bytes = (size_t)E * sizeof(int) + (size_t)(2 * E + 1 + few::fd::kScanMaxChunks) * sizeof(long long) + 64;
    FEW_CUDA_TRY(cudaMallocAsync(&buf, bytes, st));
    long long *count = static_cast<long long *>(buf);
    long long *prefix = count + E;
    long long *scratch = prefix + E + 1;
    int *lo = reinterpret_cast<int *>(scratch + few::fd::kScanMaxChunks);
    int blocks = (int)((E + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    few::fd::k_fd_range<<<blocks, 256, 0, st>>>(seg_start_inds, seg_end_inds, E, L, lo, count);
    cudaError_t e1 = cudaGetLastError();
    int status = FEW_OK;
    if (e1 != cudaSuccess) {
        status = few::fail(FEW_ERR_CUDA, "few_get_waveform_fd: launch failed: %s", cudaGetErrorString(e1));
    } else if ((status = few::fd::launch_scan(count, E, prefix, scratch, st)) != FEW_OK) {
    } else {
        const long long ns = 2LL * K + 3;
        status = few_fd_sum(waveform, L, frequencies, zero_index, include_minus_m, interp_array, ns * N, N, 1,
                            interp_array + 2LL * K * N, ns * N, N, 1, phase_interp_coeffs, 3LL * (N - 1), N - 1, 1,
                            phase_interp_t, old_time_arr, N, m, k, n, K, Ylm_all, lo, prefix, 0, 0, stream);
    }
    cudaError_t e2 = cudaFreeAsync(buf, st);
    if (status != FEW_OK) return status;
    if (e2 != cudaSuccess) return few::fail(FEW_ERR_CUDA, "few_get_waveform_fd: free failed: %s", cudaGetErrorString(e2));
    return FEW_OK;
}
