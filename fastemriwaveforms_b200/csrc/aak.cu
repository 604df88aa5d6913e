// Augmented analytic kludge (AAK) waveform: the harmonic sum of the AAK model
// over a sparse trajectory.
//
// Reference: AAKSummation.sum (src/few/summation/aakwave.py:35-196) and its
// kernel make_waveform / get_waveform (src/few/cutils/gpuAAK.cu:181-578,
// geometry d_RotCoeff :141-177).  Per output sample t = i dt, on the
// trajectory segment holding it: e, Y = cos(iota), Phi_phi, Phi_theta, Phi_r
// and the three frequencies from the 8-term dense-output basis; the orbit
// orientation (L), the spin (S) and the line of sight give the polarisation
// rotation and the precession angle gamma; the optional long-wavelength LISA
// response (mich); then the sum over harmonics n = 1..nmodes of the Peters &
// Mathews amplitudes with J_{n-2..n+2}(n e), rotated and projected.  The
// sample is (hI, -hII).
//
// B200 layout: one launch over all samples (the reference launches one kernel
// per trajectory segment); a thread finds its segment by bisection over the
// segments' first samples.  The five Bessel values of a harmonic come from
// one backward (Miller) recurrence normalised by J_0 + 2 sum J_2k = 1, instead
// of five separate evaluations; the harmonic phase n Phi (+ Doppler) is formed
// as the reference forms it (its rounding is part of the result) and reduced
// mod 2 pi before sincos (phases reach ~1e7 rad).  FP64 throughout.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "few_internal.h"

namespace few {
namespace aak {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kMTSUN = 4.9254909491978065e-06;      // solar mass in s (global.h:24)
constexpr double kGPCINSEC = 1.02927125054339e+17;     // Gpc in s (global.h:26)
constexpr double kAUsec = 499.00478383615643;          // AU in s (global.h:27)
constexpr double kYRSID = 31558149.763545595;          // sidereal year in s (global.h:23)

// e^{i ph} for large ph: Cody & Waite reduction mod 2 pi (three-part split,
// k*C1 and k*C2 exact for |k| < 2^21), then sincos on |r| <= pi.
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

// J_{n-2}(x) .. J_{n+2}(x) into J[0..4] for n >= 1, x >= 0 (J_{-1} = -J_1), by
// Miller's backward recurrence b_{k-1} = (2k/x) b_k - b_{k+1} from a start
// index M = top + 16 + sqrt(30 top) above top = max(n + 2, x), normalised by
// b_0 + 2 (b_2 + b_4 + ...).  The start's relative error is of order
// (x/2)^{2M} / (M! (M-1)!): below 1e-38 for every x <= top <= 64.
__device__ void bessel_band(int n, double x, double J[5]) {
    if (x == 0.0) {
#pragma unroll
        for (int q = 0; q < 5; ++q) J[q] = (n - 2 + q == 0) ? 1.0 : 0.0;
        return;
    }
    const int top = n + 2 > (int)x ? n + 2 : (int)x;
    int M = top + 16 + (int)sqrt(30.0 * top);
    M += M & 1;  // even start
    const double tox = 2.0 / x;
    double bp = 0.0, b = 1.0, sum = 0.0;
    double Jm1 = 0.0;  // b_1, for J_{-1} = -J_1
    double got[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int k = M; k >= 1; --k) {
        // b holds b_k, bp holds b_{k+1}; constant indices keep got[] in registers
#pragma unroll
        for (int q = 0; q < 5; ++q)
            if (k == n - 2 + q) got[q] = b;
        if ((k & 1) == 0) sum += b;
        double bm = k * tox * b - bp;  // b_{k-1}
        bp = b;
        b = bm;
        if (fabs(b) > 1e250) {  // rescale everything carried
            b *= 1e-250;
            bp *= 1e-250;
            sum *= 1e-250;
#pragma unroll
            for (int q = 0; q < 5; ++q) got[q] *= 1e-250;
        }
    }
    // b = b_0, bp = b_1
    Jm1 = bp;
#pragma unroll
    for (int q = 0; q < 5; ++q)
        if (n - 2 + q == 0) got[q] = b;  // k = 0 lies in the band when n <= 2
    const double norm = b + 2.0 * sum;
#pragma unroll
    for (int q = 0; q < 5; ++q) J[q] = got[q] / norm;
    if (n == 1) J[0] = -Jm1 / norm;  // J_{-1} = -J_1
}

// bessel_band for two harmonics at once (n and n + 1 at x1 = n e and x2 =
// (n + 1) e): one recurrence loop from a common start index (the larger one,
// which only adds accuracy to the other), two independent chains for the
// scheduler to interleave.  The loop runs in three phases so that only the six
// steps inside the bands capture values (with constant indices, so the bands
// stay in registers).
// One recurrence step of both chains at index k.  EVEN: k is even (b_k joins
// the normalisation sum); CHECK: test for overflow after the step (every
// other step suffices: two steps grow the values by less than 1e58 for any
// argument the kernel sees).
template <bool EVEN, bool CHECK>
__device__ __forceinline__ void miller_step(double kf, double t1, double t2, double &b1, double &bp1, double &s1,
                                            double &b2, double &bp2, double &s2, double g1[5], double g2[5]) {
    if (EVEN) {
        s1 += b1;
        s2 += b2;
    }
    const double m1 = kf * t1 * b1 - bp1, m2 = kf * t2 * b2 - bp2;
    bp1 = b1; b1 = m1;
    bp2 = b2; b2 = m2;
    if (CHECK) {
        if (fabs(b1) > 1e250) {
            b1 *= 1e-250; bp1 *= 1e-250; s1 *= 1e-250;
#pragma unroll
            for (int q = 0; q < 5; ++q) g1[q] *= 1e-250;
        }
        if (fabs(b2) > 1e250) {
            b2 *= 1e-250; bp2 *= 1e-250; s2 *= 1e-250;
#pragma unroll
            for (int q = 0; q < 5; ++q) g2[q] *= 1e-250;
        }
    }
}

__device__ void bessel_band2(int n, double x1, double x2, double J1[5], double J2[5]) {
    if (x1 == 0.0 || x2 == 0.0) {
        bessel_band(n, x1, J1);
        bessel_band(n + 1, x2, J2);
        return;
    }
    const int top = n + 3 > (int)x2 ? n + 3 : (int)x2;
    int M = top + 16 + (int)sqrt(30.0 * top);
    M += M & 1;
    const double t1 = 2.0 / x1, t2 = 2.0 / x2;
    double bp1 = 0.0, b1 = 1.0, s1 = 0.0, bp2 = 0.0, b2 = 1.0, s2 = 0.0;
    double g1[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, g2[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    // n is odd and M even: the steps pair up as (even k, odd k) in every phase
    for (int k = M; k > n + 3; k -= 2) {
        miller_step<true, false>((double)k, t1, t2, b1, bp1, s1, b2, bp2, s2, g1, g2);
        miller_step<false, true>((double)(k - 1), t1, t2, b1, bp1, s1, b2, bp2, s2, g1, g2);
    }
    // k = n+3 .. n-2: band 1 holds k = n-2+q (q = 0..4), band 2 holds k = n-1+q;
    // k = n-2+q is even exactly when q is odd
#pragma unroll
    for (int q = 5; q >= 0; --q) {
        const int k = n - 2 + q;
        if (k >= 1) {
            if (q <= 4) g1[q] = b1;
            if (q >= 1) g2[q - 1] = b2;
            if (q & 1) miller_step<true, false>((double)k, t1, t2, b1, bp1, s1, b2, bp2, s2, g1, g2);
            else miller_step<false, true>((double)k, t1, t2, b1, bp1, s1, b2, bp2, s2, g1, g2);
        }
    }
    for (int k = n - 3; k >= 1; k -= 2) {
        miller_step<true, false>((double)k, t1, t2, b1, bp1, s1, b2, bp2, s2, g1, g2);
        miller_step<false, true>((double)(k - 1), t1, t2, b1, bp1, s1, b2, bp2, s2, g1, g2);
    }
    // k = 0 (b = b_0, bp = b_1) lies in band 1 when n <= 2 and in band 2 when n == 1
    if (n == 1) { g1[1] = b1; g2[0] = b2; }
    if (n == 2) g1[0] = b1;
    const double nm1 = b1 + 2.0 * s1, nm2 = b2 + 2.0 * s2;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        J1[q] = g1[q] / nm1;
        J2[q] = g2[q] / nm2;
    }
    if (n == 1) J1[0] = -bp1 / nm1;  // J_{-1} = -J_1
}

struct AakArgs {
    double2 *wf;
    const double *coef;  // (8, cstride, 6): coefficient c of parameter q on segment j at (c*cstride + j)*6 + q
    const double *t;     // knots
    const int *first;    // (nseg + 1,): segment j writes samples [first[j], first[j+1])
    int nseg, cstride, nmodes, mich;
    double M, S, mu, qS, phiS, qK, phiK, dist, dt;
};

__device__ __forceinline__ double nested(const double *c, double s, double s1) {
    return c[0] + s * (c[1] + s1 * (c[2] + s * (c[3] + s1 * (c[4] + s * (c[5] + s1 * (c[6] + s * c[7]))))));
}

__device__ __forceinline__ double nested_ds(const double *c, double s, double h) {
    const double s2 = s * s, s3 = s * s2, s4 = s * s3, s5 = s * s4, s6 = s * s5;
    return (c[1] + c[2] * (1. - 2. * s) + c[3] * (2. * s - 3. * s2) + c[4] * (2. * s - 6. * s2 + 4. * s3) +
            c[5] * (3. * s2 - 8. * s3 + 5. * s4) + c[6] * (3. * s2 - 12. * s3 + 15 * s4 - 6. * s5) +
            c[7] * (4. * s3 - 15. * s4 + 18. * s5 - 7. * s6)) /
           h;
}

__device__ __forceinline__ void cross3(const double *u, const double *v, double *w) {
    w[0] = u[1] * v[2] - u[2] * v[1];
    w[1] = u[2] * v[0] - u[0] * v[2];
    w[2] = u[0] * v[1] - u[1] * v[0];
}

__global__ void __launch_bounds__(128) k_aak(AakArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int i0 = A.first[0], i1 = A.first[A.nseg];
    if (i < i0 || i >= i1) return;
    // segment j with first[j] <= i < first[j+1]
    int lo = 0, hi = A.nseg - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (A.first[mid] <= i) lo = mid; else hi = mid - 1;
    }
    const int j = lo;
    double c[5][8];
#pragma unroll
    for (int q = 0; q < 5; ++q)
#pragma unroll
        for (int k = 0; k < 8; ++k) c[q][k] = A.coef[((long long)k * A.cstride + j) * 6 + (q + 1)];

    double qS = A.qS, qK = A.qK;
    const double fill = 1e-6;
    if (qS < fill) qS = fill;
    if (qK < fill) qK = fill;
    if (qS > kPi - fill) qS = kPi - fill;
    if (qK > kPi - fill) qK = kPi - fill;
    double sinqS, cosqS, sinqK, cosqK, sinphiK, cosphiK;
    sincos(qS, &sinqS, &cosqS);
    sincos(qK, &sinqK, &cosqK);
    sincos(A.phiK, &sinphiK, &cosphiK);
    const double halfsqrt3 = sqrt(3.) / 2.;
    const double zeta = A.mu * kMTSUN / A.dist / kGPCINSEC;

    const double t = A.dt * i;
    const double h = A.t[j + 1] - A.t[j];
    const double s = (t - A.t[j]) / h, s1 = 1.0 - s;
    const double e = nested(c[0], s, s1), Y = nested(c[1], s, s1);
    const double Phi_phi = nested(c[2], s, s1), Phi_theta = nested(c[3], s, s1), Phi_r = nested(c[4], s, s1);
    const double Om_phi = nested_ds(c[2], s, h), Om_theta = nested_ds(c[3], s, h), Om_r = nested_ds(c[4], s, h);

    const double Phi = Phi_r, gim = Phi_theta - Phi_r, alp = Phi_phi - Phi_theta;
    const double nu = Om_r / (2. * kPi), gimdot = Om_theta - Om_r;
    const double lam = acos(Y);
    double sinlam, coslam, sinalp, cosalp;
    sincos(lam, &sinlam, &coslam);
    sincos_big(alp, &sinalp, &cosalp);
    const double cosqL = cosqK * coslam + sinqK * sinlam * cosalp;
    const double sinqL = sqrt(1. - cosqL * cosqL);
    const double phiLup = sinqK * sinphiK * coslam - cosphiK * sinlam * sinalp - cosqK * sinphiK * sinlam * cosalp;
    const double phiLdown = sinqK * cosphiK * coslam + sinphiK * sinlam * sinalp - cosqK * cosphiK * sinlam * cosalp;
    const double phiL = atan2(phiLup, phiLdown);
    const double Ldotn = cosqL * cosqS + sinqL * sinqS * cos(phiL - A.phiS);
    const double Ldotn2 = Ldotn * Ldotn;
    const double Sdotn = cosqK * cosqS + sinqK * sinqS * cos(A.phiK - A.phiS);
    double beta = 0.0;
    if (!(A.S == 0.0 || lam < 1e-10 || lam > (kPi - 1e-10))) {
        const double up = -Sdotn + coslam * Ldotn;
        const double down = sinqS * sin(A.phiK - A.phiS) * sinlam * cosalp + (cosqK * Sdotn - cosqS) / sinqK * sinlam * sinalp;
        beta = atan2(up, down);
    }
    double sin2gam, cos2gam;
    sincos_big(2. * (gim + beta), &sin2gam, &cos2gam);

    double FpI = 1.0, FcI = 0.0, FpII = 0.0, FcII = 1.0, cosorb = 0.0;
    if (A.mich) {
        const double orb = 2. * kPi * t / kYRSID;
        double sinorb;
        sincos(orb - A.phiS, &sinorb, &cosorb);
        const double cosq = .5 * cosqS - halfsqrt3 * sinqS * cosorb;
        const double phiw = orb + atan2(halfsqrt3 * cosqS + .5 * sinqS * cosorb, sinqS * sinorb);
        const double psiup = .5 * cosqK - halfsqrt3 * sinqK * cos(orb - A.phiK) -
                             cosq * (cosqK * cosqS + sinqK * sinqS * cos(A.phiK - A.phiS));
        const double psidown = .5 * sinqK * sinqS * sin(A.phiK - A.phiS) -
                               halfsqrt3 * cos(orb) * (cosqK * sinqS * sin(A.phiS) - cosqS * sinqK * sin(A.phiK)) -
                               halfsqrt3 * sin(orb) * (cosqS * sinqK * cos(A.phiK) - cosqK * sinqS * cos(A.phiS));
        const double psi = atan2(psiup, psidown);
        const double cosq1 = .5 * (1. + cosq * cosq);
        double s2phi, c2phi, s2psi, c2psi;
        sincos(2. * phiw, &s2phi, &c2phi);
        sincos(2. * psi, &s2psi, &c2psi);
        FpI = cosq1 * c2phi * c2psi - cosq * s2phi * s2psi;
        FcI = cosq1 * c2phi * s2psi + cosq * s2phi * c2psi;
        FpII = cosq1 * s2phi * c2psi + cosq * c2phi * s2psi;
        FcII = cosq1 * s2phi * s2psi - cosq * c2phi * c2psi;
    }
    const double Amp = pow(fabs(Om_phi) * A.M * kMTSUN, 2. / 3.) * zeta;

    // polarisation rotation (gpuAAK.cu:141-177)
    double rot0, rot1;
    {
        double sinS, cosS, sinPS, cosPS, sinK, cosK, sinPK, cosPK, sini, cosi;
        sincos(qS, &sinS, &cosS);
        sincos(A.phiS, &sinPS, &cosPS);
        sincos(qK, &sinK, &cosK);
        sincos(A.phiK, &sinPK, &cosPK);
        sincos(lam, &sini, &cosi);
        const double nv[3] = {sinS * cosPS, sinS * sinPS, cosS};
        const double Sv[3] = {sinK * cosPK, sinK * sinPK, cosK};
        const double Lv[3] = {cosi * sinK * cosPK + sini * (sinalp * sinPK - cosalp * cosK * cosPK),
                              cosi * sinK * sinPK - sini * (sinalp * cosPK + cosalp * cosK * sinPK),
                              cosi * cosK + sini * cosalp * sinK};
        double nxL[3], nxS[3];
        cross3(nv, Lv, nxL);
        cross3(nv, Sv, nxS);
        double norm = sqrt(nxL[0] * nxL[0] + nxL[1] * nxL[1] + nxL[2] * nxL[2]) *
                      sqrt(nxS[0] * nxS[0] + nxS[1] * nxS[1] + nxS[2] * nxS[2]);
        if (norm < 1e-6) norm = 1e-6;
        const double cosrot = (nxL[0] * nxS[0] + nxL[1] * nxS[1] + nxL[2] * nxS[2]) / norm;
        double sinrot = Lv[0] * nxS[0] + Lv[1] * nxS[1] + Lv[2] * nxS[2];
        sinrot -= Sv[0] * nxL[0] + Sv[1] * nxL[1] + Sv[2] * nxL[2];
        sinrot /= norm;
        rot0 = 2. * cosrot * cosrot - 1.;
        rot1 = cosrot * sinrot;
    }
    const double rot2 = -rot1, rot3 = rot0;
    const double sqrt1me2 = sqrt(1 - e * e);

    double hI = 0.0, hII = 0.0;
    double Ja[5], Jb[5];  // Bessel bands of the odd harmonic n and of n + 1
    for (int n = 1; n <= A.nmodes; ++n) {
        double nPhi;
        if (A.mich) {
            const double fn = n * nu + gimdot / kPi;
            const double Doppler = 2. * kPi * fn * kAUsec * sinqS * cosorb;
            nPhi = n * Phi + Doppler;
        } else {
            nPhi = n * Phi;
        }
        // Bessel values two harmonics at a time (odd n computes n and n + 1)
        const bool odd = (n & 1) != 0;
        if (odd) bessel_band2(n, n * e, (n + 1) * e, Ja, Jb);  // the last n + 1 may go unused
        double J[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) J[q] = odd ? Ja[q] : Jb[q];
        double sn, cn;
        sincos_big(nPhi, &sn, &cn);
        const double a = -n * Amp * (J[0] - 2. * e * J[1] + 2. / n * J[2] + 2. * e * J[3] - J[4]) * cn;
        const double b = -n * Amp * sqrt1me2 * (J[0] - 2. * J[2] + J[4]) * sn;
        const double cc = 2. * Amp * J[2] * cn;
        const double Ap0 = -(1. + Ldotn2) * (a * cos2gam - b * sin2gam) + cc * (1 - Ldotn2);
        const double Ac0 = 2. * Ldotn * (b * cos2gam + a * sin2gam);
        const double Ap = Ap0 * rot0 + Ac0 * rot1;
        const double Ac = Ap0 * rot2 + Ac0 * rot3;
        if (A.mich) {
            hI += halfsqrt3 * (FpI * Ap + FcI * Ac);
            hII += halfsqrt3 * (FpII * Ap + FcII * Ac);
        } else {
            hI += FpI * Ap + FcI * Ac;
            hII += FpII * Ap + FcII * Ac;
        }
    }
    A.wf[i] = make_double2(hI, -hII);
}

}  // namespace aak
}  // namespace few

// Segment ownership of the reference (gpuAAK.cu:495-519): first[0] = 0, then
// ceil(t_j / dt) for knots before T = (out_len - 1) dt; the first knot at or
// after T closes the list with out_len.  Returns the number of segments.
static int aak_segments(const double *h_t, int init_len, int out_len, double dt, std::vector<int> &first) {
    const double T = (out_len - 1) * dt;
    first.assign(init_len, 0);
    int i = 1;
    for (; i < init_len; ++i) {
        const double tt = h_t[i];
        if (tt < T) {
            first[i] = (int)std::ceil(tt / dt);
        } else {
            first[i] = out_len;
            break;
        }
    }
    const int npts = (i + 1 < init_len ? i + 1 : init_len);
    first.resize(npts);
    return npts - 1;
}

// The kernel on device tables, without allocation or synchronisation (what
// AAKSummation calls): t_knots [device] (>= nseg + 1), first [device]
// (nseg + 1) from the segment rule below, coef [device] (8, cstride, 6).
extern "C" FEW_API int few_aak_sum(void *waveform, const double *coef, int cstride, const double *t_knots,
                                   const int *first, int nseg, int total, double M_phys, double S_phys, double mu,
                                   double qS, double phiS, double qK, double phiK, double dist, int nmodes, int mich,
                                   double delta_t, void *stream) {
    few::clear_error();
    if (nseg < 0 || cstride < nseg || total < 0 || nmodes < 0 || nmodes > 4096)
        return few::fail(FEW_ERR_SIZE, "few_aak_sum: nseg=%d cstride=%d total=%d nmodes=%d", nseg, cstride, total,
                         nmodes);
    if (nseg == 0 || total == 0) return FEW_OK;
    if (!waveform || !coef || !t_knots || !first) return few::fail(FEW_ERR_ARG, "few_aak_sum: null pointer");
    few::aak::AakArgs A;
    A.wf = static_cast<double2 *>(waveform);
    A.coef = coef;
    A.t = t_knots;
    A.first = first;
    A.nseg = nseg;
    A.cstride = cstride;
    A.nmodes = nmodes;
    A.mich = mich;
    A.M = M_phys; A.S = S_phys; A.mu = mu; A.qS = qS; A.phiS = phiS; A.qK = qK; A.phiK = phiK; A.dist = dist;
    A.dt = delta_t;
    few::aak::k_aak<<<(total + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(A);
    FEW_LAUNCH_CHECK("k_aak");
    return FEW_OK;
}

// Drop-in for get_waveform of gpuAAK.hh:6-10 (AAKSummation's kernel call,
// aakwave.py:175-192): interp_array [device] (8, init_len-1, 6) =
// the trajectory's dense-output coefficients of (p, e, Y, Phi_phi, Phi_theta,
// Phi_r); h_t [host] (init_len,) knots; waveform [device] (out_len,) complex,
// samples of covered segments overwritten.  Plus the stream.
extern "C" FEW_API int few_aak_waveform(void *waveform, const double *interp_array, double M_phys, double S_phys,
                                        double mu, double qS, double phiS, double qK, double phiK, double dist,
                                        int nmodes, int mich, int init_len, int out_len, double delta_t,
                                        const double *h_t, void *stream) {
    few::clear_error();
    if (init_len < 2 || out_len < 1 || nmodes < 0 || nmodes > 4096)
        return few::fail(FEW_ERR_SIZE, "few_aak_waveform: init_len=%d out_len=%d nmodes=%d", init_len, out_len,
                         nmodes);
    if (!waveform || !interp_array || !h_t) return few::fail(FEW_ERR_ARG, "few_aak_waveform: null pointer");
    if (!(delta_t > 0.0)) return few::fail(FEW_ERR_ARG, "few_aak_waveform: delta_t must be positive");
    std::vector<int> first;
    const int nseg = aak_segments(h_t, init_len, out_len, delta_t, first);
    if (nseg < 1) return FEW_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    void *buf = nullptr;
    const size_t tbytes = (size_t)init_len * sizeof(double), fbytes = first.size() * sizeof(int);
    FEW_CUDA_TRY(cudaMallocAsync(&buf, tbytes + fbytes, st));
    double *t_d = static_cast<double *>(buf);
    int *first_d = reinterpret_cast<int *>(t_d + init_len);
    cudaError_t e1 = cudaMemcpyAsync(t_d, h_t, tbytes, cudaMemcpyHostToDevice, st);
    if (e1 == cudaSuccess) e1 = cudaMemcpyAsync(first_d, first.data(), fbytes, cudaMemcpyHostToDevice, st);
    int status = FEW_OK;
    if (e1 != cudaSuccess) {
        status = few::fail(FEW_ERR_CUDA, "few_aak_waveform: upload failed: %s", cudaGetErrorString(e1));
    } else {
        few::aak::AakArgs A;
        A.wf = static_cast<double2 *>(waveform);
        A.coef = interp_array;
        A.t = t_d;
        A.first = first_d;
        A.nseg = nseg;
        A.cstride = init_len - 1;
        A.nmodes = nmodes;
        A.mich = mich;
        A.M = M_phys; A.S = S_phys; A.mu = mu; A.qS = qS; A.phiS = phiS; A.qK = qK; A.phiK = phiK; A.dist = dist;
        A.dt = delta_t;
        const int total = first.back();
        few::aak::k_aak<<<(total + 127) / 128, 128, 0, st>>>(A);
        cudaError_t e2 = cudaGetLastError();
        if (e2 != cudaSuccess) status = few::fail(FEW_ERR_CUDA, "launch of k_aak failed: %s", cudaGetErrorString(e2));
    }
    // the host vector must outlive the copy
    cudaError_t e3 = cudaStreamSynchronize(st);
    cudaError_t e4 = cudaFreeAsync(buf, st);
    if (status != FEW_OK) return status;
    if (e3 != cudaSuccess) return few::fail(FEW_ERR_CUDA, "few_aak_waveform: %s", cudaGetErrorString(e3));
    if (e4 != cudaSuccess) return few::fail(FEW_ERR_CUDA, "few_aak_waveform: free failed: %s", cudaGetErrorString(e4));
    return FEW_OK;
}
