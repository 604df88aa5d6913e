// Batched not-a-knot cubic splines: build (tridiagonal solve) and evaluation.
//
// Build.  The reference fills the not-a-knot rows (src/few/cutils/interpolate.cu:48-145),
// solves every system with a pivoting tridiagonal solver (cuSPARSE gtsv2StridedBatch
// on the GPU, LAPACK dgtsv on the CPU, interpolate.cu:201-239) and then derives
// the cubic coefficients (interpolate.cu:29-43, 149-198, 241-280) in three more
// launches with host synchronisations between them.
//
// Here one thread owns one interpolant and does all of it in one launch:
//   * The first and last not-a-knot rows are not diagonally dominant, so they
//     are eliminated up front.  Row 0 reads h1*s0 + (x2-x0)*s1 = b0 and row 1
//     has h1 as its s0 coefficient, so row1 - row0 removes s0 with an exact
//     factor of 1 (the same elimination a pivoting solver makes at that step);
//     the last row is removed from row N-2 the same way.  Rows 1..N-2 are then
//     strictly diagonally dominant and a Thomas sweep without pivoting is
//     stable.
//   * The forward sweep writes its two running values (c'_i, r'_i) into the
//     c2/c3 output rows of knot i; the backward sweep reads them back, forms the
//     slope s_i and immediately overwrites knot i with the final coefficients,
//     so no scratch memory is used.
//   * The coefficient formulas are those of fill_coefficients and
//     fill_final_derivs (the last knot carries the derivative-extrapolated
//     c1, c2, c3 of the last segment).
// y is read through a strided view, so the (N, K) complex Teukolsky amplitudes
// are splined in place (real parts as interpolants 0..K-1, imaginary parts as
// K..2K-1) with no (2K, N) copy.  Output layout (4, N, ninterps) makes every
// store of a warp one contiguous run.
//
// Evaluation restates CubicSplineInterpolant.__call__
// (src/few/summation/interpolatedmodesum.py:118-257): interval by
// searchsorted(side="right") - 1 with the last knot mapped to the last interval,
// y + c1 x + c2 x^2 + c3 x^3 (or a derivative), edge values outside the range.
#include "few_common.cuh"
#include "few_internal.h"

namespace few {

namespace {

struct SplineArgs {
    const double *t;
    long long t_rs;
    const double *y;
    long long sk, sp, off2;
    int split;
    int ni, N;
    double *out;
    long long os_i, os_p;  // output stride per knot / per interpolant inside one plane
};

__device__ __forceinline__ void write_segment(double *o1, double *o2, double *o3, long long off, double s_i,
                                              double s_ip1, double y_i, double y_ip1, double dx)
{
    // fill_coefficients (interpolate.cu:29-43)
    double slope = (y_ip1 - y_i) / dx;
    double tt = (s_i + s_ip1 - 2 * slope) / dx;
    o1[off] = s_i;
    o2[off] = (slope - s_i) / dx - tt;
    o3[off] = tt / dx;
}

__global__ void __launch_bounds__(128) k_spline_build(SplineArgs a)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.ni) return;
    const int N = a.N;
    const double *x = a.t + (long long)p * a.t_rs;
    const double *yb = (p < a.split) ? a.y + (long long)p * a.sp : a.y + a.off2 + (long long)(p - a.split) * a.sp;
    const long long sk = a.sk;
    const long long plane = (long long)N * a.ni, oi = a.os_i;
    double *o0 = a.out + (long long)p * a.os_p;
    double *o1 = o0 + plane;
    double *o2 = o1 + plane;
    double *o3 = o2 + plane;

    // First not-a-knot row (interpolate.cu:71-86).
    const double x0 = x[0], x1 = x[1], x2 = x[2];
    const double y0 = yb[0], y1 = yb[sk], y2 = yb[2 * sk];
    const double h0 = x1 - x0, h1 = x2 - x1, d0 = x2 - x0;
    const double b0 = ((h0 + 2 * d0) * h1 * ((y1 - y0) / h0) + h0 * h0 * ((y2 - y1) / h1)) / d0;
    // Last not-a-knot row (interpolate.cu:56-69).
    const double xa = x[N - 3], xb = x[N - 2], xc = x[N - 1];
    const double ya = yb[(long long)(N - 3) * sk], yv = yb[(long long)(N - 2) * sk], yc = yb[(long long)(N - 1) * sk];
    const double hA = xb - xa, hB = xc - xb, dE = xc - xa;
    const double bE = (hB * hB * ((yv - ya) / hA) + (2 * dE + hB) * hA * ((yc - yv) / hB)) / dE;

    // Forward sweep over rows 1..N-2 (interior rows of interpolate.cu:88-101).
    double cprev = 0.0, rprev = 0.0;
    double xm = x0, xi = x1, ym = y0, yi = y1;
    for (int i = 1; i <= N - 2; ++i) {
        const double xn = x[i + 1];
        const double yn = yb[(long long)(i + 1) * sk];
        const double hl = xi - xm, hr = xn - xi;
        double lo = hr, dg = 2 * (hl + hr), up = hl;
        double rhs = 3.0 * (hr * ((yi - ym) / hl) + hl * ((yn - yi) / hr));
        if (i == 1) {  // row 1 - row 0
            dg -= d0;
            rhs -= b0;
            lo = 0.0;
        }
        if (i == N - 2) {  // row N-2 - row N-1
            dg -= dE;
            rhs -= bE;
            up = 0.0;
        }
        const double den = dg - lo * cprev;
        const double cp = up / den;
        const double rp = (rhs - lo * rprev) / den;
        o2[i * oi] = cp;
        o3[i * oi] = rp;
        cprev = cp;
        rprev = rp;
        xm = xi;
        xi = xn;
        ym = yi;
        yi = yn;
    }

    // Backward sweep.  s_{N-2} = r'_{N-2}; s_{N-1} from the last row.
    double s_ip1 = rprev;
    const double s_last = (bE - dE * s_ip1) / hA;
    {
        const long long off = (long long)(N - 2) * oi;
        write_segment(o1, o2, o3, off, s_ip1, s_last, yv, yc, hB);
        o0[off] = yv;
        // fill_final_derivs (interpolate.cu:241-280)
        const double c1 = o1[off], c2 = o2[off], c3 = o3[off];
        const double xx = hB, x2v = xx * xx;
        const long long offe = (long long)(N - 1) * oi;
        o0[offe] = yc;
        o1[offe] = c1 + 2 * c2 * xx + 3 * c3 * x2v;
        o2[offe] = (2. * c2 + 6. * c3 * xx) / 2.;
        o3[offe] = c3;
    }
    double xr = xb, yr = yv;  // knot i+1
    for (int i = N - 3; i >= 1; --i) {
        const long long off = (long long)i * oi;
        const double cp = o2[off], rp = o3[off];
        const double s_i = rp - cp * s_ip1;
        const double xl = x[i];
        const double yl = yb[(long long)i * sk];
        write_segment(o1, o2, o3, off, s_i, s_ip1, yl, yr, xr - xl);
        o0[off] = yl;
        s_ip1 = s_i;
        xr = xl;
        yr = yl;
    }
    // s_0 from the first row.
    const double s0 = (b0 - d0 * s_ip1) / h1;
    write_segment(o1, o2, o3, 0, s0, s_ip1, y0, y1, h0);
    o0[0] = y0;
}

// Shared-knot build from a host factorization (few_spline_factor), in scan form.
// The sweeps are linear recurrences whose factors depend on the knots only:
//     r'_i = A_i r'_{i-1} + (alpha_i delta_{i-1} + beta_i delta_i) / den_i,  A_i = -lo_i / den_i
//     s_i  = C_i s_{i+1} + r'_i,                                            C_i = -c'_i
// so the interior rows are cut into kScanChunks chunks (one warp each; lane =
// series, 32 series per CTA, every access coalesced across the series): each
// warp runs its chunk's forward sweep from a zero carry, the chunk carries are
// chained through shared memory (r'_end = rho_end + (prod A) r'_in), the
// warp corrects its rows (r' = rho + prod_{chunk start..i} A x carry) and runs
// the backward sweep from a zero carry the same way, and finally writes the
// coefficients of its segments from the corrected slopes.  The products come
// from the factor table; the sweep temporaries are parked in the c3 output
// row, which the last pass overwrites.  Loads are issued kSweepBatch steps
// ahead of the arithmetic that uses them.
constexpr int kSweepBatch = 8;

__global__ void __launch_bounds__(32 * kScanChunks) k_spline_build_factored(
    const double *__restrict__ fac, const double *__restrict__ y, long long sk, long long sp, int split,
    long long off2, int ni, int N, double *__restrict__ out, long long os_i, long long os_p)
{
    constexpr int W = kFacWidth;
    constexpr int P = kScanChunks;
    __shared__ double s_end[P][32];
    __shared__ double s_carry[P + 1][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int p0 = blockIdx.x * 32 + lane;
    const bool live = p0 < ni;
    const int p = live ? p0 : ni - 1;  // idle lanes compute on a valid series and store nothing
    const double *yb = (p < split) ? y + (long long)p * sp : y + off2 + (long long)(p - split) * sp;
    const long long plane = (long long)N * ni;
    double *o0 = out + (long long)p * os_p;
    double *o1 = o0 + plane;
    double *o2 = o1 + plane;
    double *o3 = o2 + plane;
    const int L = (N - 2 + P - 1) / P;
    const int a = 1 + w * L, e = min(a + L, N - 1);  // this warp's rows [a, e); empty if a >= e

    // pass 1: forward sweep from a zero carry
    double rho = 0.0;
    if (a < e) {
        double ym = yb[(long long)a * sk];
        double dprev = (ym - yb[(long long)(a - 1) * sk]) * __ldg(fac + W * (a - 1) + 6);
        for (int i0 = a; i0 < e; i0 += kSweepBatch) {
            double yv[kSweepBatch], fl[kSweepBatch], fi[kSweepBatch], fa[kSweepBatch], fb[kSweepBatch], fh[kSweepBatch];
#pragma unroll
            for (int q = 0; q < kSweepBatch; ++q) {
                const int i = min(i0 + q, e - 1);
                yv[q] = yb[(long long)(i + 1) * sk];
                const double *f = fac + (long long)W * i;
                fl[q] = __ldg(f + 0);
                fi[q] = __ldg(f + 1);
                fa[q] = __ldg(f + 3);
                fb[q] = __ldg(f + 4);
                fh[q] = __ldg(f + 6);
            }
#pragma unroll
            for (int q = 0; q < kSweepBatch; ++q) {
                const int i = i0 + q;
                if (i < e) {
                    const double del = (yv[q] - ym) * fh[q];
                    rho = (fa[q] * dprev + fb[q] * del - fl[q] * rho) * fi[q];
                    if (live) o3[(long long)i * os_i] = rho;
                    dprev = del;
                    ym = yv[q];
                }
            }
        }
    }
    s_end[w][lane] = rho;
    __syncthreads();
    if (w == 0) {  // chain the forward carries: r' entering chunk q
        double c = 0.0;
        for (int q = 0; q < P; ++q) {
            s_carry[q][lane] = c;
            const int aq = 1 + q * L, eq = min(aq + L, N - 1);
            if (aq < eq) c = s_end[q][lane] + __ldg(fac + (long long)W * (eq - 1) + 10) * c;
        }
    }
    __syncthreads();
    const double cf = s_carry[w][lane];

    // pass 2: r' = rho + prod(A) cf, then the backward sweep from a zero carry
    double sig = 0.0;
    if (a < e) {
        for (int i0 = e - 1; i0 >= a; i0 -= kSweepBatch) {
            double rv[kSweepBatch], fp[kSweepBatch], fc[kSweepBatch];
#pragma unroll
            for (int q = 0; q < kSweepBatch; ++q) {
                const int i = max(i0 - q, a);
                rv[q] = o3[(long long)i * os_i];
                fp[q] = __ldg(fac + (long long)W * i + 10);
                fc[q] = __ldg(fac + (long long)W * i + 2);
            }
#pragma unroll
            for (int q = 0; q < kSweepBatch; ++q) {
                const int i = i0 - q;
                if (i >= a) {
                    const double r = fma(fp[q], cf, rv[q]);
                    sig = r - fc[q] * sig;
                    if (live) o3[(long long)i * os_i] = sig;
                }
            }
        }
    }
    __syncthreads();
    s_end[w][lane] = sig;
    __syncthreads();
    if (w == 0) {  // chain the backward carries: s at the row after chunk q; s_1 last
        double c = 0.0;
        for (int q = P - 1; q >= 0; --q) {
            s_carry[q][lane] = c;
            const int aq = 1 + q * L, eq = min(aq + L, N - 1);
            if (aq < eq) c = s_end[q][lane] + __ldg(fac + (long long)W * aq + 11) * c;
        }
        s_carry[P][lane] = c;
    }
    __syncthreads();
    if (a >= e || !live) return;
    const double cb = s_carry[w][lane];

    // pass 3: slopes s_i = sig_i + prod(C) cb and the coefficients of segments
    // [a, e) (fill_coefficients, interpolate.cu:29-43); the last chunk also the
    // extrapolated last knot (fill_final_derivs, interpolate.cu:241-280), the
    // first chunk segment 0 from the first not-a-knot row
    double s_ip1, yr;
    int top = e - 1;
    if (e == N - 1) {
        const double *bnd = fac + (long long)W * N;
        const double e0 = __ldg(bnd + 4), e1 = __ldg(bnd + 5), dE = __ldg(bnd + 6), hA = __ldg(bnd + 7);
        const long long i = N - 2;
        const double ya = yb[(i - 1) * sk], yl = yb[i * sk], yc = yb[(i + 1) * sk];
        const double sN2 = fma(__ldg(fac + W * i + 11), cb, o3[i * os_i]);
        const double dA = (yl - ya) * __ldg(fac + W * (i - 1) + 6);
        const double ih = __ldg(fac + W * i + 6), xx = __ldg(fac + W * i + 5);
        const double dl = (yc - yl) * ih;
        const double bE = e0 * dA + e1 * dl;
        const double s_last = (bE - dE * sN2) / hA;
        const double tt = (sN2 + s_last - 2 * dl) * ih;
        const double c1 = sN2, c2 = (dl - sN2) * ih - tt, c3 = tt * ih;
        const long long off = i * os_i, offe = (long long)(N - 1) * os_i;
        __stcs(o0 + off, yl);
        __stcs(o1 + off, c1);
        __stcs(o2 + off, c2);
        __stcs(o3 + off, c3);
        __stcs(o0 + offe, yc);
        __stcs(o1 + offe, c1 + 2 * c2 * xx + 3 * c3 * xx * xx);
        __stcs(o2 + offe, (2. * c2 + 6. * c3 * xx) / 2.);
        __stcs(o3 + offe, c3);
        s_ip1 = sN2;
        yr = yl;
        top = N - 3;
    } else {
        s_ip1 = cb;
        yr = yb[(long long)e * sk];
    }
    for (int i0 = top; i0 >= a; i0 -= kSweepBatch) {
        double yv[kSweepBatch], rv[kSweepBatch], fq[kSweepBatch], fh[kSweepBatch];
#pragma unroll
        for (int q = 0; q < kSweepBatch; ++q) {
            const int i = max(i0 - q, a);
            yv[q] = yb[(long long)i * sk];
            rv[q] = o3[(long long)i * os_i];
            fq[q] = __ldg(fac + (long long)W * i + 11);
            fh[q] = __ldg(fac + (long long)W * i + 6);
        }
#pragma unroll
        for (int q = 0; q < kSweepBatch; ++q) {
            const int i = i0 - q;
            if (i >= a) {
                const long long off = (long long)i * os_i;
                const double s_i = fma(fq[q], cb, rv[q]);
                const double dl = (yr - yv[q]) * fh[q];
                const double tt = (s_i + s_ip1 - 2 * dl) * fh[q];
                // final coefficients: streaming stores (evict first), so that they do
                // not push the sweep temporaries and y out of L2
                __stcs(o0 + off, yv[q]);
                __stcs(o1 + off, s_i);
                __stcs(o2 + off, (dl - s_i) * fh[q] - tt);
                __stcs(o3 + off, tt * fh[q]);
                s_ip1 = s_i;
                yr = yv[q];
            }
        }
    }
    if (w == 0) {
        // s_0 from the first row: b0 = gamma0 delta_0 + gamma1 delta_1
        const double *bnd = fac + (long long)W * N;
        const double g0 = __ldg(bnd + 0), g1 = __ldg(bnd + 1), d0 = __ldg(bnd + 2), h1 = __ldg(bnd + 3);
        const double y0 = yb[0], y1 = yr, y2 = yb[2 * sk];
        const double ih0 = __ldg(fac + 6);
        const double del0 = (y1 - y0) * ih0, del1 = (y2 - y1) * __ldg(fac + W + 6);
        const double s0 = (g0 * del0 + g1 * del1 - d0 * s_ip1) / h1;
        const double tt = (s0 + s_ip1 - 2 * del0) * ih0;
        o0[0] = y0;
        o1[0] = s0;
        o2[0] = (del0 - s0) * ih0 - tt;
        o3[0] = tt * ih0;
    }
}

__global__ void k_spline_eval(const double *__restrict__ t, long long t_rs, const double *__restrict__ coeffs,
                              int ni, int N, const double *__restrict__ tnew, long long tn_rs, int M, int deriv,
                              double *__restrict__ out, int *__restrict__ flags)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)ni * M) return;
    const int p = (int)(idx / M);
    const int j = (int)(idx - (long long)p * M);
    const double *x = t + (long long)p * t_rs;
    const double tv = tnew[(long long)p * tn_rs + j];
    // searchsorted(x, tv, side="right") - 1
    int lo = 0, hi = N;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (x[mid] <= tv) lo = mid + 1;
        else hi = mid;
    }
    int ind = lo - 1;
    if (tv == x[N - 1]) ind = N - 2;
    const bool left = tv < x[0];
    const bool right = tv > x[N - 1];
    if (left) atomicOr(&flags[0], 1);
    if (right) atomicOr(&flags[1], 1);
    if (ind < 0) ind = 0;  // only reached when left; value replaced below
    const long long plane = (long long)N * ni;
    const long long o = (long long)ind * ni + p;
    const double xx = tv - x[ind];
    const double y = coeffs[o], c1 = coeffs[plane + o], c2 = coeffs[2 * plane + o], c3 = coeffs[3 * plane + o];
    double v;
    if (deriv == 0) {
        const double x2 = xx * xx, x3 = x2 * xx;
        v = y + c1 * xx + c2 * x2 + c3 * x3;
        if (left) v = coeffs[p];
        if (right) v = coeffs[(long long)(N - 1) * ni + p];
    } else if (deriv == 1) {
        v = c1 + 2 * c2 * xx + 3 * c3 * (xx * xx);
    } else if (deriv == 2) {
        v = 2 * c2 + 6 * c3 * xx;
    } else {
        v = 6 * c3;
    }
    out[idx] = v;
}

}  // namespace

int launch_spline_build(const double *t, long long t_rs, const double *y, long long sk, long long sp, int split,
                        long long off2, int ni, int N, double *out, int layout, cudaStream_t st)
{
    SplineArgs a;
    a.t = t;
    a.t_rs = t_rs;
    a.y = y;
    a.sk = sk;
    a.sp = sp;
    a.off2 = off2;
    a.split = split;
    a.ni = ni;
    a.N = N;
    a.out = out;
    if (layout == FEW_LAYOUT_KNOT_MAJOR) {
        a.os_i = ni;
        a.os_p = 1;
    } else {
        a.os_i = 1;
        a.os_p = N;
    }
    const int threads = 128;
    const int blocks = (ni + threads - 1) / threads;
    k_spline_build<<<blocks, threads, 0, st>>>(a);
    FEW_LAUNCH_CHECK("k_spline_build");
    return FEW_OK;
}

}  // namespace few

extern "C" int few_spline_build_factored(const double *fac, const double *y, long long y_knot_stride,
                                         long long y_interp_stride, int y_split, long long y_split_offset, int ninterps,
                                         int length, double *coeffs, int layout, void *stream)
{
    few::clear_error();
    if (!fac || !y || !coeffs) return few::fail(FEW_ERR_ARG, "few_spline_build_factored: null pointer");
    if (ninterps < 1) return few::fail(FEW_ERR_SIZE, "few_spline_build_factored: ninterps=%d < 1", ninterps);
    if (length < 4) return few::fail(FEW_ERR_SIZE, "few_spline_build_factored: length=%d < 4", length);
    if (layout != FEW_LAYOUT_KNOT_MAJOR && layout != FEW_LAYOUT_INTERP_MAJOR)
        return few::fail(FEW_ERR_ARG, "few_spline_build_factored: unknown layout %d", layout);
    if (y_split < 0 || y_split > ninterps) return few::fail(FEW_ERR_ARG, "few_spline_build_factored: bad y_split");
    const long long os_i = layout == FEW_LAYOUT_KNOT_MAJOR ? ninterps : 1;
    const long long os_p = layout == FEW_LAYOUT_KNOT_MAJOR ? 1 : length;
    few::k_spline_build_factored<<<(ninterps + 31) / 32, 32 * few::kScanChunks, 0, (cudaStream_t)stream>>>(
        fac, y, y_knot_stride, y_interp_stride, y_split, y_split_offset, ninterps, length, coeffs, os_i, os_p);
    FEW_LAUNCH_CHECK("k_spline_build_factored");
    return FEW_OK;
}

extern "C" int few_spline_build(const double *t, long long t_row_stride, const double *y, long long y_knot_stride,
                                long long y_interp_stride, int y_split, long long y_split_offset, int ninterps,
                                int length, double *coeffs, int layout, void *stream)
{
    few::clear_error();
    if (!t || !y || !coeffs) return few::fail(FEW_ERR_ARG, "few_spline_build: null pointer");
    if (ninterps < 1) return few::fail(FEW_ERR_SIZE, "few_spline_build: ninterps=%d < 1", ninterps);
    if (length < 4)
        return few::fail(FEW_ERR_SIZE, "few_spline_build: length=%d; not-a-knot splines need at least 4 knots",
                         length);
    if (layout != FEW_LAYOUT_KNOT_MAJOR && layout != FEW_LAYOUT_INTERP_MAJOR)
        return few::fail(FEW_ERR_ARG, "few_spline_build: unknown layout %d", layout);
    if (y_split < 0 || y_split > ninterps) return few::fail(FEW_ERR_ARG, "few_spline_build: bad y_split");
    if ((long long)ninterps * length * 4 > (1LL << 40)) return few::fail(FEW_ERR_SIZE, "few_spline_build: too large");
    return few::launch_spline_build(t, t_row_stride, y, y_knot_stride, y_interp_stride, y_split, y_split_offset,
                                    ninterps, length, coeffs, layout, (cudaStream_t)stream);
}

extern "C" int few_spline_eval(const double *t, long long t_row_stride, const double *coeffs, int ninterps,
                               int length, const double *tnew, long long tnew_row_stride, int M, int deriv_order,
                               double *out, int *flags, void *stream)
{
    few::clear_error();
    if (!t || !coeffs || !tnew || !out || !flags) return few::fail(FEW_ERR_ARG, "few_spline_eval: null pointer");
    if (ninterps < 1 || length < 2 || M < 0) return few::fail(FEW_ERR_SIZE, "few_spline_eval: bad sizes");
    if (deriv_order < 0 || deriv_order > 3)
        return few::fail(FEW_ERR_ARG, "deriv_order must be within 0 <= deriv_order <= 3.");
    if (M == 0) return FEW_OK;
    const long long total = (long long)ninterps * M;
    const int threads = 256;
    const long long blocks = (total + threads - 1) / threads;
    if (blocks > 0x7fffffffLL) return few::fail(FEW_ERR_SIZE, "few_spline_eval: too many points");
    few::k_spline_eval<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(
        t, t_row_stride, coeffs, ninterps, length, tnew, tnew_row_stride, M, deriv_order, out, flags);
    FEW_LAUNCH_CHECK("k_spline_eval");
    return FEW_OK;
}
