/*
 * few_oracle.c -- CPU restatement of the FastEMRIWaveforms time-domain
 * interpolated mode sum, the amplitude grid evaluation and the
 * frequency-domain (stationary-phase) sum.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA path is checked
 * against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it; the product path (fastemriwaveforms_b200) never does.
 *
 * Parity pin: the restatement is checked against the reference itself, built
 * from its own sources by oracle/Makefile into oracle/_ref, and against the
 * golden vectors under tests/golden (made by tests/golden/make_golden.py from
 * that build) plus scipy.interpolate.CubicSpline for the spline build.
 *
 * Reference functions restated (paths inside the FastEMRIWaveforms project):
 *   src/few/cutils/interpolate.cu:29-43    fill_coefficients
 *   src/few/cutils/interpolate.cu:48-102   prep_splines (not-a-knot rows)
 *   src/few/cutils/interpolate.cu:201-239  fit_wrap (CPU branch: LAPACK dgtsv)
 *   src/few/cutils/interpolate.cu:241-280  fill_final_derivs
 *   src/few/cutils/interpolate.cu:284-325  interpolate_arrays
 *   src/few/cutils/interpolate.cu:444-689  make_waveform (CPU branch)
 *   src/few/cutils/interpolate.cu:694-723  find_start_inds
 *   src/few/cutils/interpolate.cu:726-797  get_waveform
 *   src/few/cutils/interpolate.cu:1041-1520 SPAFunc, cube_roots, make_generic_kerr_waveform_fd
 *
 * Build with -ffp-contract=off: every a*b+c in the reference source is two
 * rounded operations here, in the order the source writes them.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Spline build                                                              */
/* ------------------------------------------------------------------------- */

/* Not-a-knot row i of the slope system for one interpolant
 * (interpolate.cu:48-102).  Row i reads lower*s[i-1] + diag*s[i] + upper*s[i+1]. */
static void oracle_row(int i, int n, const double *x, const double *y,
                       double *b, double *ud, double *dg, double *ld)
{
    double dx1, dx2, d, slope1, slope2;
    if (i == n - 1) {
        dx1 = x[n - 2] - x[n - 3];
        dx2 = x[n - 1] - x[n - 2];
        d = x[n - 1] - x[n - 3];
        slope1 = (y[n - 2] - y[n - 3]) / dx1;
        slope2 = (y[n - 1] - y[n - 2]) / dx2;
        b[i] = ((dx2 * dx2 * slope1 + (2 * d + dx2) * dx1 * slope2) / d);
        dg[i] = dx1;
        ld[i] = d;
        ud[i] = 0.0;
    } else if (i == 0) {
        dx1 = x[1] - x[0];
        dx2 = x[2] - x[1];
        d = x[2] - x[0];
        slope1 = (y[1] - y[0]) / dx1;
        slope2 = (y[2] - y[1]) / dx2;
        b[0] = ((dx1 + 2 * d) * dx2 * slope1 + dx1 * dx1 * slope2) / d;
        dg[0] = dx2;
        ud[0] = d;
        ld[0] = 0.0;
    } else {
        dx1 = x[i] - x[i - 1];
        dx2 = x[i + 1] - x[i];
        slope1 = (y[i] - y[i - 1]) / dx1;
        slope2 = (y[i + 1] - y[i]) / dx2;
        b[i] = 3.0 * (dx2 * slope1 + dx1 * slope2);
        dg[i] = 2 * (dx1 + dx2);
        ud[i] = dx1;
        ld[i] = dx2;
    }
}

/* Tridiagonal solve by Gaussian elimination with partial (row) pivoting, the
 * published algorithm of LAPACK xGTSV that fit_wrap calls on the CPU
 * (interpolate.cu:231-236).  sub[i] = A[i+1][i] (n-1 entries), dg[i] = A[i][i],
 * sup[i] = A[i][i+1] (n-1 entries).  A row swap moves a second superdiagonal
 * entry into sup2.  b is overwritten with the solution.  Returns 0, or i+1 when
 * pivot i is exactly zero. */
static int oracle_gtsv(int n, double *sub, double *dg, double *sup, double *b, double *sup2)
{
    for (int i = 0; i < n - 1; ++i) {
        if (fabs(dg[i]) >= fabs(sub[i])) {
            if (dg[i] == 0.0) return i + 1;
            double f = sub[i] / dg[i];
            dg[i + 1] = dg[i + 1] - f * sup[i];
            b[i + 1] = b[i + 1] - f * b[i];
            sup2[i] = 0.0;
        } else {
            /* the next row becomes the pivot row */
            double f = dg[i] / sub[i];
            double old_d1 = dg[i + 1];
            double old_u1 = (i < n - 2) ? sup[i + 1] : 0.0;
            dg[i] = sub[i];
            dg[i + 1] = sup[i] - f * old_d1;
            sup[i] = old_d1;
            sup2[i] = old_u1;
            if (i < n - 2) sup[i + 1] = -f * old_u1;
            double bi = b[i];
            b[i] = b[i + 1];
            b[i + 1] = bi - f * b[i];
        }
    }
    if (dg[n - 1] == 0.0) return n;
    b[n - 1] = b[n - 1] / dg[n - 1];
    if (n > 1) b[n - 2] = (b[n - 2] - sup[n - 2] * b[n - 1]) / dg[n - 2];
    for (int i = n - 3; i >= 0; --i)
        b[i] = (b[i] - sup[i] * b[i + 1] - sup2[i] * b[i + 2]) / dg[i];
    return 0;
}

/* interpolate_arrays (interpolate.cu:284-325), CPU branch.
 * t_arr: (ninterps, length) knots, one row per interpolant.
 * interp_array: (4, ninterps, length); row 0 holds y on entry, rows 1..3
 * receive c1, c2, c3.  B/upper/diag/lower: (ninterps*length) scratch, as in
 * the reference.  Returns 0, or a negative code on bad sizes, or the first
 * failing pivot of the first singular system. */
int oracle_interpolate_arrays(const double *t_arr, double *interp_array, int ninterps, int length,
                              double *B, double *upper_diag, double *diag, double *lower_diag)
{
    if (ninterps < 1 || length < 3) return -1;
    double *sup2 = (double *)malloc(sizeof(double) * (size_t)length);
    if (!sup2) return -2;
    const size_t plane = (size_t)ninterps * (size_t)length;
    int status = 0;
    for (int p = 0; p < ninterps; ++p) {
        const size_t lead = (size_t)p * (size_t)length;
        const double *x = t_arr + lead;
        double *y = interp_array + lead;
        for (int i = 0; i < length; ++i)
            oracle_row(i, length, x, y, B + lead, upper_diag + lead, diag + lead, lower_diag + lead);
        /* fit_wrap passes dl = &lower[j*m+1]: sub-diagonal entry i is row i+1's lower coefficient */
        int info = oracle_gtsv(length, lower_diag + lead + 1, diag + lead, upper_diag + lead, B + lead, sup2);
        if (info != 0 && status == 0) status = info;
        double *c1 = interp_array + plane + lead;
        double *c2 = interp_array + 2 * plane + lead;
        double *c3 = interp_array + 3 * plane + lead;
        const double *dydx = B + lead;
        /* fill_coefficients (interpolate.cu:29-43) */
        for (int i = 0; i < length - 1; ++i) {
            double dx = x[i + 1] - x[i];
            double slope = (y[i + 1] - y[i]) / dx;
            double dydx_i = dydx[i];
            double tt = (dydx_i + dydx[i + 1] - 2 * slope) / dx;
            c1[i] = dydx_i;
            c2[i] = (slope - dydx_i) / dx - tt;
            c3[i] = tt / dx;
        }
        /* fill_final_derivs (interpolate.cu:241-280) */
        {
            double a1 = c1[length - 2], a2 = c2[length - 2], a3 = c3[length - 2];
            double xx = x[length - 1] - x[length - 2];
            double x2 = xx * xx;
            c1[length - 1] = a1 + 2 * a2 * xx + 3 * a3 * x2;
            c2[length - 1] = (2. * a2 + 6. * a3 * xx) / 2.;
            c3[length - 1] = a3;
        }
    }
    free(sup2);
    return status;
}

/* ------------------------------------------------------------------------- */
/* Mode sum                                                                  */
/* ------------------------------------------------------------------------- */

/* find_start_inds (interpolate.cu:694-723).  Segment j owns output samples
 * [start[j], start[j+1]).  Returns the number of usable segments, or -1 when
 * no knot reaches the end of the output (a case the reference leaves
 * undefined; this restatement refuses it). */
int oracle_find_start_inds(int *start, const double *h_t, double dt, int length, int out_len)
{
    double T = (out_len - 1) * dt;
    start[0] = 0;
    for (int i = 1; i < length; ++i) {
        double t = h_t[i];
        if (t < T) {
            start[i] = (int)ceil(t / dt);
        } else {
            start[i] = out_len;
            return i; /* segments 0..i-1 */
        }
    }
    return -1;
}

/* The sum body of make_waveform (interpolate.cu:618-686) for the samples
 * [i_lo, i_hi) of segment `seg`, double precision, operation order as written
 * in the reference.  wf: interleaved complex, absolute sample index. */
static void oracle_segment_f64(double *wf, const double *interp, const double *pc,
                               const int *m_arr, const int *k_arr, const int *n_arr, int K,
                               const double *ylm, double dt, double start_t, int seg,
                               int i_lo, int i_hi, int init_len, double pt0, double pwidth)
{
    const size_t num_base = (size_t)init_len * (size_t)(2 * K);
    const size_t nps = (size_t)(init_len - 1) * 3;
    double pp[8], pt[8], pr[8];
    for (int c = 0; c < 8; ++c) {
        pp[c] = pc[c * nps + (size_t)seg * 3 + 0];
        pt[c] = pc[c * nps + (size_t)seg * 3 + 1];
        pr[c] = pc[c * nps + (size_t)seg * 3 + 2];
    }
    const double *cr[4], *ci[4];
    for (int c = 0; c < 4; ++c) {
        cr[c] = interp + c * num_base + (size_t)seg * (2 * K);
        ci[c] = cr[c] + K;
    }
    for (int i = i_lo; i < i_hi; ++i) {
        double t = dt * i;
        double x = t - start_t;
        double x2 = x * x;
        double x3 = x * x2;
        double s = (t - pt0) / pwidth;
        double s1 = 1.0 - s;
        double Pp = pp[0] + s * (pp[1] + s1 * (pp[2] + s * (pp[3] + s1 * (pp[4] + s * (pp[5] + s1 * (pp[6] + s * pp[7]))))));
        double Pt = pt[0] + s * (pt[1] + s1 * (pt[2] + s * (pt[3] + s1 * (pt[4] + s * (pt[5] + s1 * (pt[6] + s * pt[7]))))));
        double Pr = pr[0] + s * (pr[1] + s1 * (pr[2] + s * (pr[3] + s1 * (pr[4] + s * (pr[5] + s1 * (pr[6] + s * pr[7]))))));
        double tr = 0.0, ti = 0.0;
        for (int j = 0; j < K; ++j) {
            int m = m_arr[j], k = k_arr[j], n = n_arr[j];
            double phase = m * Pp + k * Pt + n * Pr;
            double ang = -phase;                 /* imag part of -i*phase */
            double er = cos(ang), ei = sin(ang); /* exp(0 + i*ang) */
            double re = cr[0][j] + cr[1][j] * x + cr[2][j] * x2 + cr[3][j] * x3;
            double im = ci[0][j] + ci[1][j] * x + ci[2][j] * x2 + ci[3][j] * x3;
            double qr = er * re - ei * im;       /* exp * amplitude */
            double qi = er * im + ei * re;
            double ypr = ylm[2 * j], ypi = ylm[2 * j + 1];
            double tpr = qr * ypr - qi * ypi;
            double tpi = qr * ypi + qi * ypr;
            double tmr = 0.0, tmi = 0.0;
            if (m != 0) {
                double ymr = ylm[2 * (K + j)], ymi = ylm[2 * (K + j) + 1];
                double nqi = -qi;                /* conj(partial_mode) */
                tmr = qr * ymr - nqi * ymi;
                tmi = qr * ymi + nqi * ymr;
            }
            tr = tr + tmr + tpr;
            ti = ti + tmi + tpi;
        }
        wf[2 * (size_t)i] += tr;
        wf[2 * (size_t)i + 1] += ti;
    }
}

/* The same sum in 80-bit extended arithmetic after the phase polynomials:
 * Phi is evaluated exactly as the reference does (double), then the mode phase
 * m*Phi_phi + k*Phi_theta + n*Phi_r, its sine/cosine, the amplitude and the
 * products are formed in long double.  This is the accuracy reference for the
 * recurrence form, which does not round the combined mode phase. */
/* The 8-term basis in long double (the nested form of interpolate.cu:642-644). */
static long double basis_ld(const double *c, long double s)
{
    long double s1 = 1.0L - s;
    return c[0] + s * (c[1] + s1 * (c[2] + s * (c[3] + s1 * (c[4] + s * (c[5] + s1 * (c[6] + s * (long double)c[7]))))));
}

/* dpc (same layout as pc) and delta: when dpc is given, the phases are
 * Phi + delta * dPhi evaluated in long double (a finite-difference probe whose
 * step is not rounded into the large phase coefficients); otherwise Phi is
 * evaluated in double exactly as the reference does. */
static void oracle_segment_ext(double *wf, const double *interp, const double *pc,
                               const int *m_arr, const int *k_arr, const int *n_arr, int K,
                               const double *ylm, double dt, double start_t, int seg,
                               int i_lo, int i_hi, int init_len, double pt0, double pwidth,
                               const double *dpc, long double delta)
{
    const size_t num_base = (size_t)init_len * (size_t)(2 * K);
    const size_t nps = (size_t)(init_len - 1) * 3;
    double pp[8], pt[8], pr[8], dp[8], dt8[8], dr[8];
    for (int c = 0; c < 8; ++c) {
        pp[c] = pc[c * nps + (size_t)seg * 3 + 0];
        pt[c] = pc[c * nps + (size_t)seg * 3 + 1];
        pr[c] = pc[c * nps + (size_t)seg * 3 + 2];
        if (dpc) {
            dp[c] = dpc[c * nps + (size_t)seg * 3 + 0];
            dt8[c] = dpc[c * nps + (size_t)seg * 3 + 1];
            dr[c] = dpc[c * nps + (size_t)seg * 3 + 2];
        }
    }
    const double *cr[4], *ci[4];
    for (int c = 0; c < 4; ++c) {
        cr[c] = interp + c * num_base + (size_t)seg * (2 * K);
        ci[c] = cr[c] + K;
    }
    for (int i = i_lo; i < i_hi; ++i) {
        double t = dt * i;
        double x = t - start_t;
        double s = (t - pt0) / pwidth;
        double s1 = 1.0 - s;
        long double Pp, Pt, Pr;
        if (dpc) {
            long double sl = ((long double)t - pt0) / pwidth;
            Pp = basis_ld(pp, sl) + delta * basis_ld(dp, sl);
            Pt = basis_ld(pt, sl) + delta * basis_ld(dt8, sl);
            Pr = basis_ld(pr, sl) + delta * basis_ld(dr, sl);
        } else {
            Pp = pp[0] + s * (pp[1] + s1 * (pp[2] + s * (pp[3] + s1 * (pp[4] + s * (pp[5] + s1 * (pp[6] + s * pp[7]))))));
            Pt = pt[0] + s * (pt[1] + s1 * (pt[2] + s * (pt[3] + s1 * (pt[4] + s * (pt[5] + s1 * (pt[6] + s * pt[7]))))));
            Pr = pr[0] + s * (pr[1] + s1 * (pr[2] + s * (pr[3] + s1 * (pr[4] + s * (pr[5] + s1 * (pr[6] + s * pr[7]))))));
        }
        long double X = x;
        long double tr = 0.0L, ti = 0.0L;
        for (int j = 0; j < K; ++j) {
            int m = m_arr[j], k = k_arr[j], n = n_arr[j];
            long double phase = (long double)m * Pp + (long double)k * Pt + (long double)n * Pr;
            long double er = cosl(phase), ei = -sinl(phase);
            long double re = ((cr[3][j] * X + cr[2][j]) * X + cr[1][j]) * X + cr[0][j];
            long double im = ((ci[3][j] * X + ci[2][j]) * X + ci[1][j]) * X + ci[0][j];
            long double qr = er * re - ei * im;
            long double qi = er * im + ei * re;
            long double ypr = ylm[2 * j], ypi = ylm[2 * j + 1];
            tr += qr * ypr - qi * ypi;
            ti += qr * ypi + qi * ypr;
            if (m != 0) {
                long double ymr = ylm[2 * (K + j)], ymi = ylm[2 * (K + j) + 1];
                tr += qr * ymr + qi * ymi;
                ti += qr * ymi - qi * ymr;
            }
        }
        wf[2 * (size_t)i] += (double)tr;
        wf[2 * (size_t)i + 1] += (double)ti;
    }
}

/* get_waveform (interpolate.cu:726-797), CPU branch, restricted to the output
 * samples [s_lo, s_hi) (pass 0 and out_len for the whole waveform).
 * wf: (out_len,) complex128 as interleaved doubles, accumulated with +=.
 * interp_array: (4, init_len, 2K); phase_coeffs: (8, init_len-1, 3);
 * ylm: (2K,) complex with the -m half already multiplied by (-1)^l.
 * extended = 0: double precision in the reference's operation order;
 * extended = 1: the long double restatement above.
 * Returns 0, or a negative code when the knots do not reach the output end. */
static int get_waveform_impl(double *wf, const double *interp_array, const double *phase_interp_t,
                             const double *phase_interp_coeffs, const int *m_arr, const int *k_arr,
                             const int *n_arr, int init_len, int out_len, int K, const double *ylm,
                             double dt, const double *h_t, int s_lo, int s_hi, int extended,
                             const double *dpc, long double delta);

int oracle_get_waveform(double *wf, const double *interp_array, const double *phase_interp_t,
                        const double *phase_interp_coeffs, const int *m_arr, const int *k_arr,
                        const int *n_arr, int init_len, int out_len, int K, const double *ylm,
                        double dt, const double *h_t, int s_lo, int s_hi, int extended)
{
    return get_waveform_impl(wf, interp_array, phase_interp_t, phase_interp_coeffs, m_arr, k_arr, n_arr, init_len,
                             out_len, K, ylm, dt, h_t, s_lo, s_hi, extended, 0, 0.0L);
}

/* The long double sum with the phases Phi + delta * dPhi (dpc: the basis of a
 * phase perturbation, laid out as phase_interp_coeffs), for finite
 * differences of the phase inputs. */
int oracle_get_waveform_dphase(double *wf, const double *interp_array, const double *phase_interp_t,
                               const double *phase_interp_coeffs, const double *dpc, double delta,
                               const int *m_arr, const int *k_arr, const int *n_arr, int init_len, int out_len,
                               int K, const double *ylm, double dt, const double *h_t, int s_lo, int s_hi)
{
    return get_waveform_impl(wf, interp_array, phase_interp_t, phase_interp_coeffs, m_arr, k_arr, n_arr, init_len,
                             out_len, K, ylm, dt, h_t, s_lo, s_hi, 1, dpc, (long double)delta);
}

static int get_waveform_impl(double *wf, const double *interp_array, const double *phase_interp_t,
                             const double *phase_interp_coeffs, const int *m_arr, const int *k_arr,
                             const int *n_arr, int init_len, int out_len, int K, const double *ylm,
                             double dt, const double *h_t, int s_lo, int s_hi, int extended,
                             const double *dpc, long double delta)
{
    if (init_len < 2 || out_len < 1 || K < 1) return -1;
    int *start = (int *)malloc(sizeof(int) * (size_t)init_len);
    if (!start) return -2;
    int nseg = oracle_find_start_inds(start, h_t, dt, init_len, out_len);
    if (nseg < 0) { free(start); return -3; }
    for (int j = 0; j < nseg; ++j) {
        int a = start[j] > s_lo ? start[j] : s_lo;
        int b = start[j + 1] < s_hi ? start[j + 1] : s_hi;
        if (a >= b) continue;
        double pt0 = phase_interp_t[j], pw = phase_interp_t[j + 1] - phase_interp_t[j];
        if (extended)
            oracle_segment_ext(wf, interp_array, phase_interp_coeffs, m_arr, k_arr, n_arr, K, ylm,
                               dt, h_t[j], j, a, b, init_len, pt0, pw, dpc, delta);
        else
            oracle_segment_f64(wf, interp_array, phase_interp_coeffs, m_arr, k_arr, n_arr, K, ylm,
                               dt, h_t[j], j, a, b, init_len, pt0, pw);
    }
    free(start);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Amplitude grids: tensor-product B-spline evaluation                       */
/* ------------------------------------------------------------------------- */

/* The k+1 non-zero B-splines of degree k at x, for t[l-1] <= x < t[l]: the
 * de Boor-Cox recurrence as FITPACK's fpbspl states it (Dierckx), the form
 * AmpInterp2D.cu:20-44 restates; each operation rounded separately. */
static void oracle_bspl(const double *t, int k, double x, int l, double *h)
{
    double hh[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    h[0] = 1.0;
    for (int j = 1; j <= k; ++j) {
        for (int i = 0; i < k; ++i) hh[i] = h[i];
        h[0] = 0.0;
        for (int i = 0; i < j; ++i) {
            const int li = l + i, lj = li - j;
            const double f = hh[i] / (t[li] - t[lj]);
            h[i] = h[i] + f * (t[li] - x);
            h[i + 1] = f * (x - t[lj]);
        }
    }
}

/* Interval of x (clamped to [t[k], t[n-k-1]]): the first l >= k+1 with
 * x < t[l], at most n-k-1 (FITPACK fpbisp's search, AmpInterp2D.cu:68-79);
 * fills the basis and returns l - (k+1). */
static int oracle_basis(const double *t, int n, int k, double x, double *h)
{
    const int k1 = k + 1, nk1 = n - k1;
    double arg = x;
    if (arg < t[k1 - 1]) arg = t[k1 - 1];
    if (arg > t[nk1]) arg = t[nk1];
    int l = k1;
    while (!(arg < t[l] || l == nk1)) ++l;
    oracle_bspl(t, k, arg, l, h);
    return l - k1;
}

/* interp2D (AmpInterp2D.cu:86-176), CPU branch: z[g * m + i] = grid g at
 * (x[i], y[i]), summed over the (kx+1)(ky+1) coefficients in FITPACK's order. */
void oracle_interp2d(double *z, const double *tx, int nx, const double *ty, int ny, const double *c, int kx, int ky,
                     const double *x, const double *y, int m, int ngrid, int len_indiv_c)
{
    const int nky1 = ny - ky - 1;
    for (int i = 0; i < m; ++i) {
        double wx[6], wy[6];
        const int lx = oracle_basis(tx, nx, kx, x[i], wx);
        const int ly = oracle_basis(ty, ny, ky, y[i], wy);
        for (int g = 0; g < ngrid; ++g) {
            const double *cg = c + (size_t)g * len_indiv_c;
            double sp = 0.0;
            int l1 = lx * nky1 + ly;
            for (int a = 0; a <= kx; ++a) {
                for (int b = 0; b <= ky; ++b) sp += cg[l1 + b] * wx[a] * wy[b];
                l1 += nky1;
            }
            z[(size_t)g * m + i] = sp;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Frequency-domain sum (stationary phase)                                   */
/* ------------------------------------------------------------------------- */
/* Restates make_generic_kerr_waveform_fd (src/few/cutils/interpolate.cu:
 * 1141-1520) with its helpers cube_roots (:1113-1133) and SPAFunc
 * (:1041-1097), and the complex arithmetic of cuda_complex.hpp (C99 Annex G
 * forms: products without contraction, the quotient with a power-of-two
 * scaled divisor, principal branches through atan2/hypot).  Inputs in the
 * reference kernel's layouts: interp (4, 2K+3, N), pc (8, 3, N-1), start/end
 * (K, N-1), ylms (2K) interleaved with the -m half already times (-1)^l;
 * wf (L) interleaved, accumulated, visited in the reference's order
 * (mode, segment, bin, root).  The SPA series coefficients are generated
 * from their recurrences (the same numbers the reference writes out). */

typedef struct { double re, im; } ocx;

static ocx ocx_mk(double r, double i) { ocx z; z.re = r; z.im = i; return z; }
static ocx ocx_add(ocx a, ocx b) { return ocx_mk(a.re + b.re, a.im + b.im); }
static ocx ocx_scale(ocx a, double s) { return ocx_mk(a.re * s, a.im * s); }
static ocx ocx_divr(ocx a, double s) { return ocx_mk(a.re / s, a.im / s); }
static ocx ocx_mul(ocx a, ocx b)
{
    double ac = a.re * b.re, bd = a.im * b.im, ad = a.re * b.im, bc = a.im * b.re;
    return ocx_mk(ac - bd, ad + bc);
}
static ocx ocx_div(ocx z, ocx w)
{
    double a = z.re, b = z.im, c = w.re, d = w.im, lg = logb(fmax(fabs(c), fabs(d)));
    int sc = 0;
    if (isfinite(lg)) { sc = (int)lg; c = scalbn(c, -sc); d = scalbn(d, -sc); }
    double den = c * c + d * d;
    return ocx_mk(scalbn((a * c + b * d) / den, -sc), scalbn((b * c - a * d) / den, -sc));
}
static ocx ocx_polar(double rho, double th)
{
    if (isnan(rho) || signbit(rho)) return ocx_mk(NAN, NAN);
    double x = rho * cos(th), y = rho * sin(th);
    if (isnan(x)) x = 0.0;
    if (isnan(y)) y = 0.0;
    return ocx_mk(x, y);
}
static ocx ocx_exp(ocx z) { double e = exp(z.re); return ocx_mk(e * cos(z.im), e * sin(z.im)); }
static ocx ocx_log(ocx z) { return ocx_mk(log(hypot(z.re, z.im)), atan2(z.im, z.re)); }
static ocx ocx_sqrt(ocx z)
{
    if (isinf(z.im)) return ocx_mk(INFINITY, z.im);
    return ocx_polar(sqrt(hypot(z.re, z.im)), atan2(z.im, z.re) / 2.0);
}
static ocx ocx_powr(ocx z, double p) { return ocx_exp(ocx_mul(ocx_mk(p, 0.0), ocx_log(z))); }

static double spa_s1[14], spa_s2[14], spa_ar[9], spa_ai[9];
static int spa_ready = 0;

static void spa_init(void)
{
    double c1 = 0.5, c2 = 1.0, a = 1.0;
    for (int j = 0; j < 14; ++j) {
        spa_s1[j] = c1;
        spa_s2[j] = c2;
        c1 = c1 * (-0.25) / ((j + 1) * (j + 4.0 / 3.0));
        c2 = c2 * (-0.25) / ((j + 1) * (j + 2.0 / 3.0));
    }
    for (int j = 0; j < 9; ++j) {
        int q = (j + 1) & 3;
        spa_ar[j] = (q == 0) ? a : (q == 2 ? -a : 0.0);
        spa_ai[j] = (q == 1) ? a : (q == 3 ? -a : 0.0);
        a = a * (4.0 / 9.0 - (2.0 * j + 1.0) * (2.0 * j + 1.0)) / (8.0 * (j + 1));
    }
    spa_ready = 1;
}

static ocx oracle_spa(double x)
{
    const double pi = 3.141592653589793238462643383279502884;
    if (fabs(x) <= 7.0) {
        ocx e23 = ocx_exp(ocx_divr(ocx_scale(ocx_mk(0.0, 1.0), -2.0 * pi), 3.0));
        ocx e13 = ocx_exp(ocx_divr(ocx_scale(ocx_mk(0.0, 1.0), -pi), 3.0));
        ocx p6 = ocx_powr(ocx_mk(x, 0.0), 1.0 / 6.0);
        ocx q = e23;
        for (int i = 0; i < 5; ++i) q = ocx_mul(q, p6);
        ocx pref1 = ocx_divr(ocx_scale(q, -4.062353818279201250), 1.259921049894873165);
        ocx pref2 = ocx_divr(ocx_scale(ocx_mul(e13, p6), 2.678938534707747633), 1.587401051968199475);
        double x2 = x * x, s1 = spa_s1[13], s2 = spa_s2[13];
        for (int j = 12; j >= 0; --j) { s1 = spa_s1[j] + x2 * s1; s2 = spa_s2[j] + x2 * s2; }
        ocx ph = ocx_exp(ocx_scale(ocx_mk(-0.0, -1.0), x));
        return ocx_mul(ph, ocx_add(ocx_scale(pref1, s1), ocx_scale(pref2, s2)));
    }
    ocx y = ocx_mk(1.0 / x, 0.0);
    ocx pref = ocx_scale(ocx_exp(ocx_scale(ocx_scale(ocx_mk(-0.0, -1.0), 0.75), pi)), sqrt(0.5 * pi));
    ocx ser = ocx_mk(spa_ar[8], spa_ai[8]);
    for (int j = 7; j >= 0; --j) ser = ocx_add(ocx_mk(spa_ar[j], spa_ai[j]), ocx_mul(y, ser));
    return ocx_mul(pref, ser);
}

static void oracle_cube_roots(double a, double b, double c, double d, ocx xi, double r[3])
{
    double b2 = b * b, b3 = b2 * b, a2 = a * a;
    double D0 = b2 - 3 * a * c;
    double D1 = 2 * b3 - 9 * a * b * c + 27 * a2 * d;
    ocx S = ocx_sqrt(ocx_mk(D1 * D1 - 4 * (D0 * D0 * D0), 0.0));
    ocx C = ocx_powr(ocx_divr(ocx_mk(S.re + D1, S.im), 2.0), 1.0 / 3.0);
    double s = -(1.0 / (3 * a));
    ocx D0c = ocx_mk(D0, 0.0), xC = ocx_mul(xi, C), xxC = ocx_mul(ocx_mul(xi, xi), C);
    r[0] = ocx_scale(ocx_add(ocx_mk(b + C.re, C.im), ocx_div(D0c, C)), s).re;
    r[1] = ocx_scale(ocx_add(ocx_mk(b + xC.re, xC.im), ocx_div(D0c, xC)), s).re;
    r[2] = ocx_scale(ocx_add(ocx_mk(b + xxC.re, xxC.im), ocx_div(D0c, xxC)), s).re;
}

void oracle_fd_sum(double *wf, const double *interp, const double *phase_t, const double *pc, const int *m_arr,
                   const int *k_arr, const int *n_arr, int K, const double *t, int N, int L, const double *freq,
                   const int *start, const int *end, const double *ylms, int zero_index, int include_minus_m)
{
    const double pi = 3.141592653589793238462643383279502884;
    if (!spa_ready) spa_init();
    const long nb = (long)(2 * K + 3) * N, nps = (long)(N - 1) * 3;
    ocx S3 = ocx_sqrt(ocx_mk(-3.0, 0.0));
    ocx xi = ocx_divr(ocx_mk(S3.re + -1.0, S3.im), 2.0);
    for (int mode = 0; mode < K; ++mode) {
        const int m = m_arr[mode], k = k_arr[mode], n = n_arr[mode];
        ocx yp = ocx_mk(ylms[2 * mode], ylms[2 * mode + 1]);
        ocx ym = ocx_mk(ylms[2 * (K + mode)], ylms[2 * (K + mode) + 1]);
        for (int seg = 0; seg < N - 1; ++seg) {
            const double ts = t[seg], te = t[seg + 1];
            const double *re = interp + (long)mode * N + seg, *im = interp + (long)(K + mode) * N + seg;
            const double *fp = interp + (long)(2 * K) * N + seg, *ft = fp + N, *fr = fp + 2 * N;
            double fy = m * fp[0] + k * ft[0] + n * fr[0];
            double fc1 = m * fp[nb] + k * ft[nb] + n * fr[nb];
            double fc2 = m * fp[2 * nb] + k * ft[2 * nb] + n * fr[2 * nb];
            double fc3 = m * fp[3 * nb] + k * ft[3 * nb] + n * fr[3 * nb];
            double h = phase_t[seg + 1] - phase_t[seg], h2 = h * h, h3 = h * h2;
            int s0 = start[mode * (N - 1) + seg], s1e = end[mode * (N - 1) + seg];
            for (int i = s0 < 0 ? 0 : s0; i <= s1e && i <= L - 1; ++i) {
                double f = freq[i], roots[3];
                oracle_cube_roots(fc3, fc2, fc1, fy - f, xi, roots);
                for (int r = 0; r < 3; ++r) {
                    double x = roots[r], tt = ts + x;
                    if (!(tt < te && tt >= ts)) continue;
                    double x2 = x * x, x3 = x * x2;
                    double Rre = re[0] + re[nb] * x + re[2 * nb] * x2 + re[3 * nb] * x3;
                    double Rim = im[0] + im[nb] * x + im[2 * nb] * x2 + im[3 * nb] * x3;
                    double s = (tt - phase_t[seg]) / h, sm = 1.0 - s;
                    double q2 = s * s, q3 = s * q2, q4 = s * q3, q5 = s * q4;
                    double phase = 0.0, fdot = 0.0, fddot = 0.0;
                    for (int q = 0; q < 3; ++q) {
                        const int mult = q == 0 ? m : (q == 1 ? k : n);
                        const double *c = pc + (long)q * (N - 1) + seg;
                        double c0 = c[0], c1 = c[nps], c2 = c[2 * nps], c3 = c[3 * nps], c4 = c[4 * nps],
                               c5 = c[5 * nps], c6 = c[6 * nps], c7 = c[7 * nps];
                        double P = c0 + s * (c1 + sm * (c2 + s * (c3 + sm * (c4 + s * (c5 + sm * (c6 + s * c7))))));
                        double d2 = (-2. * c2 + c3 * (2. - 6. * s) + c4 * (2. - 12. * s + 12. * q2) +
                                     c5 * (6. * s - 24. * q2 + 20. * q3) + c6 * (6. * s - 36. * q2 + 60. * q3 - 30. * q4) +
                                     c7 * (12. * q2 - 60. * q3 + 90. * q4 - 42. * q5)) / (2. * pi * h2);
                        double d3 = (-6. * c3 + c4 * (-12. + 24. * s) + c5 * (6. - 48. * s + 60. * q2) +
                                     c6 * (6. - 72. * s + 180. * q2 - 120. * q3) +
                                     c7 * (24. * s - 180. * q2 + 360. * q3 - 210. * q4)) / (2. * pi * h3);
                        if (q == 0) { phase = mult * P; fdot = mult * d2; fddot = mult * d3; }
                        else { phase += mult * P; fdot += mult * d2; fddot += mult * d3; }
                    }
                    double arg = 2. * pi * fdot * fdot * fdot / (3. * fddot * fddot);
                    double pre = -1.0 * fdot / fabs(fddot) * 2. / sqrt(3.);
                    ocx amp2 = ocx_div(ocx_scale(oracle_spa(arg), pre), ocx_sqrt(ocx_mk(arg, 0.0)));
                    double ph = 2. * pi * f * tt - phase;
                    ocx tex = ocx_mul(ocx_mul(ocx_mk(Rre, Rim), amp2), ocx_exp(ocx_mk(0.0 * ph, ph)));
                    ocx rt = ocx_mul(yp, tex);
                    wf[2 * i] += rt.re;
                    wf[2 * i + 1] += rt.im;
                    if (m != 0 && include_minus_m) {
                        int imn = 2 * zero_index - i;
                        if (imn >= 0 && imn < L) {
                            ocx lt = ocx_mul(ym, ocx_mk(tex.re, -tex.im));
                            wf[2 * imn] += lt.re;
                            wf[2 * imn + 1] += lt.im;
                        }
                    }
                }
            }
        }
    }
}
