// Dense output of the Dormand-Prince 8(5,3) integrator on the GPU: the map
// from the stages a step stored to the 8-term interpolation basis of that step
// (the phase coefficients the mode sum consumes), and the evaluation of that
// basis and of its time derivatives.
//
// Restates DOPR853.prep_evaluate / eval / eval_derivative
// (src/few/trajectory/dopr853.py:621-875), batched over steps: every step's
// basis depends only on its own end points, stored stages and four right-hand
// side evaluations (the derivative at the step's end and three extra stages),
// so a batch of steps is one index space of (component, step).  The
// right-hand side belongs to the trajectory's ODE and is evaluated by the
// caller between the launches, for all steps at once:
//   phase 0: rcont1..4, the stored-stage part of rcont5..8, argument of stage 14
//   phase 1: argument of stage 15 (needs stage 14's derivative)
//   phase 2: argument of stage 16 (needs stages 14 and 15)
//   phase 3: rcont5..8 completed with the new derivative and stages 14..16
// The coefficients are the published dense-output coefficients of DOP853
// (Hairer, Norsett & Wanner, Solving ODEs I, 2nd ed., section II.6, and the
// authors' dop853 code), which the reference tabulates at dopr853.py:10-181;
// they define the method, so the same values appear here.  Every sum is
// formed in the reference's order with explicitly rounded operations (no
// contraction), so the basis equals the reference's numpy result bit for bit
// when the right-hand side values do.
//
// Layouts (the reference's batch layout, systems = steps):
//   x0, h0, x1        (nsys,)
//   y0, y1, dydx1     (node, nsys)         dydx1 = f(x1, y1)
//   stages            (10, node, nsys)     k1..k10 as take_step leaves them:
//                                          slots 2 and 3 hold stages 11 and 12
//   k14, k15, k16     (node, nsys)         f at the extra stages
//   arg               (node, nsys)         out: the next extra stage's argument
//   xarg              (nsys,)              out: its time
//   rcont             (nsys, node, 8)      out
#include "few_common.cuh"
#include "few_internal.h"

namespace few {

namespace {

// extra stages: nodes and couplings
constexpr double c14 = 0.1, c15 = 0.2, c16 = 0.777777777777777777777777777778;
constexpr double a141 = 5.61675022830479523392909219681e-2, a147 = 2.53500210216624811088794765333e-1,
                 a148 = -2.46239037470802489917441475441e-1, a149 = -1.24191423263816360469010140626e-1,
                 a1410 = 1.5329179827876569731206322685e-1, a1411 = 8.20105229563468988491666602057e-3,
                 a1412 = 7.56789766054569976138603589584e-3, a1413 = -8.298e-3;
constexpr double a151 = 3.18346481635021405060768473261e-2, a156 = 2.83009096723667755288322961402e-2,
                 a157 = 5.35419883074385676223797384372e-2, a158 = -5.49237485713909884646569340306e-2,
                 a1511 = -1.08347328697249322858509316994e-4, a1512 = 3.82571090835658412954920192323e-4,
                 a1513 = -3.40465008687404560802977114492e-4, a1514 = 1.41312443674632500278074618366e-1;
constexpr double a161 = -4.28896301583791923408573538692e-1, a166 = -4.69762141536116384314449447206e0,
                 a167 = 7.68342119606259904184240953878e0, a168 = 4.06898981839711007970213554331e0,
                 a169 = 3.56727187455281109270669543021e-1, a1613 = -1.39902416515901462129418009734e-3,
                 a1614 = 2.9475147891527723389556272149e0, a1615 = -9.15095847217987001081870187138e0;

// dense-output weights: row q of D (q = 4..7 for rcont5..8), columns in the
// order the reference sums them: k1, k6, k7, k8, k9, k10, k11 (slot 2),
// k12 (slot 3), then f(x1), k14, k15, k16
__constant__ double c_D[4][12] = {
    {-0.84289382761090128651353491142e01, 0.56671495351937776962531783590e00, -0.30689499459498916912797304727e01,
     0.23846676565120698287728149680e01, 0.21170345824450282767155149946e01, -0.87139158377797299206789907490e00,
     0.22404374302607882758541771650e01, 0.63157877876946881815570249290e00, -0.88990336451333310820698117400e-01,
     0.18148505520854727256656404962e02, -0.91946323924783554000451984436e01, -0.44360363875948939664310572000e01},
    {0.10427508642579134603413151009e02, 0.24228349177525818288430175319e03, 0.16520045171727028198505394887e03,
     -0.37454675472269020279518312152e03, -0.22113666853125306036270938578e02, 0.77334326684722638389603898808e01,
     -0.30674084731089398182061213626e02, -0.93321305264302278729567221706e01, 0.15697238121770843886131091075e02,
     -0.31139403219565177677282850411e02, -0.93529243588444783865713862664e01, 0.35816841486394083752465898540e02},
    {0.19985053242002433820987653617e02, -0.38703730874935176555105901742e03, -0.18917813819516756882830838328e03,
     0.52780815920542364900561016686e03, -0.11573902539959630126141871134e02, 0.68812326946963000169666922661e01,
     -0.10006050966910838403183860980e01, 0.77771377980534432092869265740e00, -0.27782057523535084065932004339e01,
     -0.60196695231264120758267380846e02, 0.84320405506677161018159903784e02, 0.11992291136182789328035130030e02},
    {-0.25693933462703749003312586129e02, -0.15418974869023643374053993627e03, -0.23152937917604549567536039109e03,
     0.35763911791061412378285349910e03, 0.93405324183624310003907691704e02, -0.37458323136451633156875139351e02,
     0.10409964950896230045147246184e03, 0.29840293426660503123344363579e02, -0.43533456590011143754432175058e02,
     0.96324553959188282948394950600e02, -0.39177261675615439165231486172e02, -0.14972683625798562581422125276e03}};

struct DenseArgs {
    const double *x0, *h0, *x1, *y0, *y1, *dydx1, *stages, *k14, *k15, *k16;
    double *arg, *xarg, *rcont;
    int node, nsys, phase;
};

// a * b + c with both operations rounded (numpy's order, no FMA)
__device__ __forceinline__ double mad_rn(double a, double b, double c) { return radd(rmul(a, b), c); }

__global__ void __launch_bounds__(256) k_dense_output(DenseArgs a)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)a.node * a.nsys;
    if (idx >= n) return;
    const int j = (int)(idx % a.nsys);  // step (system)
    const int e = (int)(idx / a.nsys);  // component
    auto K = [&](int s) { return a.stages[((long long)s * a.node + e) * a.nsys + j]; };  // s = 0 for k1
    const double h = a.h0[j], y0 = a.y0[idx];
    double *out = a.rcont + ((long long)j * a.node + e) * 8;

    if (a.phase == 0) {
        const double y1 = a.y1[idx], f1 = a.dydx1[idx];
        const double k1 = K(0), k2 = K(1), k3 = K(2), k6 = K(5), k7 = K(6), k8 = K(7), k9 = K(8), k10 = K(9);
        const double diff = rsub(y1, y0);
        const double bspl = rsub(rmul(h, k1), diff);
        out[0] = y0;
        out[1] = diff;
        out[2] = bspl;
        out[3] = rsub(rsub(diff, rmul(h, f1)), bspl);
        // stored-stage part of rcont5..8: d1 k1 + d6 k6 + ... + d12 k12, left to right
        const double ks[8] = {k1, k6, k7, k8, k9, k10, k2, k3};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double s = rmul(c_D[q][0], ks[0]);
#pragma unroll
            for (int c = 1; c < 8; ++c) s = mad_rn(c_D[q][c], ks[c], s);
            out[4 + q] = s;
        }
        double s = rmul(a141, k1);
        s = mad_rn(a147, k7, s);
        s = mad_rn(a148, k8, s);
        s = mad_rn(a149, k9, s);
        s = mad_rn(a1410, k10, s);
        s = mad_rn(a1411, k2, s);
        s = mad_rn(a1412, k3, s);
        s = mad_rn(a1413, f1, s);
        a.arg[idx] = radd(y0, rmul(h, s));
        if (e == 0) a.xarg[j] = radd(a.x0[j], rmul(c14, h));
    } else if (a.phase == 1) {
        const double f1 = a.dydx1[idx], k14 = a.k14[idx];
        double s = rmul(a151, K(0));
        s = mad_rn(a156, K(5), s);
        s = mad_rn(a157, K(6), s);
        s = mad_rn(a158, K(7), s);
        s = mad_rn(a1511, K(1), s);
        s = mad_rn(a1512, K(2), s);
        s = mad_rn(a1513, f1, s);
        s = mad_rn(a1514, k14, s);
        a.arg[idx] = radd(y0, rmul(h, s));
        if (e == 0) a.xarg[j] = radd(a.x0[j], rmul(c15, h));
    } else if (a.phase == 2) {
        const double f1 = a.dydx1[idx], k14 = a.k14[idx], k15 = a.k15[idx];
        double s = rmul(a161, K(0));
        s = mad_rn(a166, K(5), s);
        s = mad_rn(a167, K(6), s);
        s = mad_rn(a168, K(7), s);
        s = mad_rn(a169, K(8), s);
        s = mad_rn(a1613, f1, s);
        s = mad_rn(a1614, k14, s);
        s = mad_rn(a1615, k15, s);
        a.arg[idx] = radd(y0, rmul(h, s));
        if (e == 0) a.xarg[j] = radd(a.x0[j], rmul(c16, h));
    } else {
        const double f1 = a.dydx1[idx], k14 = a.k14[idx], k15 = a.k15[idx], k16 = a.k16[idx];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double s = out[4 + q];
            s = mad_rn(c_D[q][8], f1, s);
            s = mad_rn(c_D[q][9], k14, s);
            s = mad_rn(c_D[q][10], k15, s);
            s = mad_rn(c_D[q][11], k16, s);
            out[4 + q] = rmul(h, s);
        }
    }
}

// Correctly rounded x^p for small integer p >= 3 (numpy's ** calls the C
// library's pow for these exponents, which rounds the exact power once):
// the power is carried as an unevaluated sum hi + lo (error-free products),
// then rounded once.
__device__ __forceinline__ double powi_rn(double x, int p)
{
    double hi = x, lo = 0.0;
    for (int i = 1; i < p; ++i) {
        const double ph = hi * x;
        const double pl = fma(hi, x, -ph);
        lo = fma(lo, x, pl);
        hi = ph;
    }
    return hi + lo;
}

struct EvalArgs {
    const double *t_new, *t_old, *coeffs;
    double *out;
    int npts, nold, node, order;
};

// One thread per (point, component): the step by binary search (numpy's
// searchsorted(side="right") - 1, the last knot mapped to the last step),
// s = (t - t_j) / (t_{j+1} - t_j), the basis or its order-th derivative in s
// in the reference's expression order, divided by the step's length^order.
__global__ void __launch_bounds__(256) k_dense_eval(EvalArgs a)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)a.npts * a.node) return;
    const int i = (int)(idx / a.node), e = (int)(idx % a.node);
    const double t = a.t_new[i];
    const double tmax = a.t_old[a.nold - 1];
    int lo = 0, hi = a.nold;  // first index with t_old > t
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a.t_old[mid] <= t) lo = mid + 1;
        else hi = mid;
    }
    int seg = lo - 1;
    if (t == tmax) seg = a.nold - 2;
    const double *c = a.coeffs + ((long long)seg * a.node + e) * 8;
    const double diff = rsub(a.t_old[seg + 1], a.t_old[seg]);
    const double s = rdiv(rsub(t, a.t_old[seg]), diff);
    const double s1 = rsub(1.0, s);
    double r;
    if (a.order == 0) {
        r = phase_poly(c, s, s1);
    } else {
        const double s2 = rmul(s, s), s3 = powi_rn(s, 3), s4 = powi_rn(s, 4), s5 = powi_rn(s, 5),
                     s6 = powi_rn(s, 6);
        auto lin = [](double a0, double b0, double x) { return radd(a0, rmul(b0, x)); };
        if (a.order == 1) {
            // rcont2 + rcont3 (1 - 2 s) + rcont4 (2 s - 3 s^2) + ...
            r = c[1];
            r = mad_rn(c[2], rsub(1.0, rmul(2.0, s)), r);
            r = mad_rn(c[3], rsub(rmul(2.0, s), rmul(3.0, s2)), r);
            r = mad_rn(c[4], radd(rsub(rmul(2.0, s), rmul(6.0, s2)), rmul(4.0, s3)), r);
            r = mad_rn(c[5], radd(rsub(rmul(3.0, s2), rmul(8.0, s3)), rmul(5.0, s4)), r);
            r = mad_rn(c[6], rsub(radd(rsub(rmul(3.0, s2), rmul(12.0, s3)), rmul(15.0, s4)), rmul(6.0, s5)), r);
            r = mad_rn(c[7], rsub(radd(rsub(rmul(4.0, s3), rmul(15.0, s4)), rmul(18.0, s5)), rmul(7.0, s6)), r);
        } else if (a.order == 2) {
            r = rmul(-2.0, c[2]);
            r = mad_rn(c[3], rsub(2.0, rmul(6.0, s)), r);
            r = mad_rn(c[4], radd(rsub(2.0, rmul(12.0, s)), rmul(12.0, s2)), r);
            r = mad_rn(c[5], radd(rsub(rmul(6.0, s), rmul(24.0, s2)), rmul(20.0, s3)), r);
            r = mad_rn(c[6], rsub(radd(rsub(rmul(6.0, s), rmul(36.0, s2)), rmul(60.0, s3)), rmul(30.0, s4)), r);
            r = mad_rn(c[7], rsub(radd(rsub(rmul(12.0, s2), rmul(60.0, s3)), rmul(90.0, s4)), rmul(42.0, s5)), r);
        } else {
            r = rmul(-6.0, c[3]);
            r = mad_rn(c[4], lin(-12.0, 24.0, s), r);
            r = mad_rn(c[5], radd(rsub(6.0, rmul(48.0, s)), rmul(60.0, s2)), r);
            r = mad_rn(c[6], rsub(radd(rsub(6.0, rmul(72.0, s)), rmul(180.0, s2)), rmul(120.0, s3)), r);
            r = mad_rn(c[7], rsub(radd(rsub(rmul(24.0, s), rmul(180.0, s2)), rmul(360.0, s3)), rmul(210.0, s4)), r);
        }
        const double dp = a.order == 1 ? diff : (a.order == 2 ? rmul(diff, diff) : powi_rn(diff, 3));
        r = rdiv(r, dp);
    }
    a.out[idx] = r;
}

}  // namespace

}  // namespace few

extern "C" int few_dopr853_dense(const double *x0, const double *h0, const double *x1, const double *y0,
                                 const double *y1, const double *dydx1, const double *stages, const double *k14,
                                 const double *k15, const double *k16, double *arg, double *xarg, double *rcont,
                                 int node, int nsys, int phase, void *stream)
{
    few::clear_error();
    if (phase < 0 || phase > 3) return few::fail(FEW_ERR_ARG, "few_dopr853_dense: phase %d is not 0..3", phase);
    if (!x0 || !h0 || !y0 || !dydx1 || !stages || !rcont)
        return few::fail(FEW_ERR_ARG, "few_dopr853_dense: null pointer");
    if ((phase == 0 && (!y1 || !arg || !xarg)) || (phase == 1 && (!k14 || !arg || !xarg)) ||
        (phase == 2 && (!k14 || !k15 || !arg || !xarg)) || (phase == 3 && (!k14 || !k15 || !k16)))
        return few::fail(FEW_ERR_ARG, "few_dopr853_dense: null pointer for phase %d", phase);
    if (node < 1 || nsys < 0 || (long long)node * nsys > (1LL << 40))
        return few::fail(FEW_ERR_SIZE, "few_dopr853_dense: bad sizes");
    if (nsys == 0) return FEW_OK;
    (void)x1;
    few::DenseArgs a{x0, h0, x1, y0, y1, dydx1, stages, k14, k15, k16, arg, xarg, rcont, node, nsys, phase};
    const long long n = (long long)node * nsys;
    few::k_dense_output<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a);
    FEW_LAUNCH_CHECK("k_dense_output");
    return FEW_OK;
}

extern "C" int few_dopr853_eval(const double *t_new, int npts, const double *t_old, int nold, const double *coeffs,
                                int node, int order, double *out, void *stream)
{
    few::clear_error();
    if (!t_new || !t_old || !coeffs || !out) return few::fail(FEW_ERR_ARG, "few_dopr853_eval: null pointer");
    if (order < 0 || order > 3) return few::fail(FEW_ERR_ARG, "few_dopr853_eval: order %d is not 0..3", order);
    if (npts < 0 || nold < 2 || node < 1) return few::fail(FEW_ERR_SIZE, "few_dopr853_eval: bad sizes");
    if (npts == 0) return FEW_OK;
    few::EvalArgs a{t_new, t_old, coeffs, out, npts, nold, node, order};
    const long long n = (long long)npts * node;
    few::k_dense_eval<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a);
    FEW_LAUNCH_CHECK("k_dense_eval");
    return FEW_OK;
}
