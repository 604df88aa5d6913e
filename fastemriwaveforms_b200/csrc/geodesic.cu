// Fundamental frequencies of Kerr geodesics, (a, p, e, x) -> (Omega_phi,
// Omega_theta, Omega_r) in units of 1/M, for the frequency-domain sum.
//
// Restates get_fundamental_frequencies (src/few/utils/geodesic.py:470-535) and
// the kernels it dispatches to (geodesic.py:157-451):
//   a == 0                  Schwarzschild closed form   (geodesic.py:285-347)
//   e == 0 and |x| == 1     circular equatorial Kerr    (geodesic.py:261-282)
//   |x| == 1                eccentric equatorial Kerr   (geodesic.py:350-426)
//   otherwise               generic Kerr                (geodesic.py:169-258)
// The generic and equatorial forms are the Mino-time frequencies of Fujita &
// Hikida (arXiv:0906.1420, eqs. 13, 15, 21) divided by Gamma; the constants of
// motion follow Schmidt (gr-qc/0202090) with the spherical-orbit formulas of
// arXiv:2102.02713 (A13-A17) below e = 1e-10 (geodesic.py:950-1050).
//
// The complete elliptic integrals are Carlson's symmetric forms by the
// duplication theorem (B. C. Carlson, Numer. Algorithms 10 (1995) 13-26), with
// the reference's stopping rule (largest relative deviation below 5e-4, then
// the fifth-order series; src/few/utils/elliptic.py:13-300) and its closed form
// for R_C (elliptic.py:61-85), and the Abramowitz & Stegun 17.3.34 / 17.3.36
// polynomials for K and E when k > 1 - 1e-10 (elliptic.py:220-265): these
// choices define the reference's values, so they are kept.
#include <cuda_runtime.h>

#include <cmath>

#include "few_internal.h"

namespace few {
namespace geo {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kTol = 5e-4;

// Error bits written to the status word.
constexpr int kErrModulus = 1;  // elliptic modulus outside [0, 1]

__device__ __forceinline__ double max3(double a, double b, double c) { return fmax(fmax(a, b), c); }

// R_F(x, y, z) = 1/2 int_0^inf dt / sqrt((t+x)(t+y)(t+z)).
__device__ double carlson_rf(double x, double y, double z) {
    double mu, dx, dy, dz;
    for (;;) {
        double sx = sqrt(x), sy = sqrt(y), sz = sqrt(z);
        double lam = sx * (sy + sz) + sy * sz;
        x = (x + lam) * 0.25;
        y = (y + lam) * 0.25;
        z = (z + lam) * 0.25;
        mu = (x + y + z) / 3.0;
        dx = 2.0 - (mu + x) / mu;
        dy = 2.0 - (mu + y) / mu;
        dz = 2.0 - (mu + z) / mu;
        if (!(max3(fabs(dx), fabs(dy), fabs(dz)) > kTol)) break;
    }
    double e2 = dx * dy - dz * dz;
    double e3 = dx * dy * dz;
    // 1 - E2/10 + E3/14 + E2^2/24 - 3 E2 E3/44
    double s = 1.0 + (e2 / 24.0 - 0.1 - 3.0 / 44.0 * e3) * e2 + e3 / 14.0;
    return s / sqrt(mu);
}

// R_C(x, y) = R_F(x, y, y), closed form.
__device__ double carlson_rc(double x, double y) {
    double d = x - y;
    if (d < -1e-8) return acos(sqrt(x / y)) / sqrt(-d);
    if (d > 1e-8) return acosh(sqrt(x / y)) / sqrt(d);
    return 1.0 / sqrt(y);
}

// R_D(x, y, z) = R_J(x, y, z, z).
__device__ double carlson_rd(double x, double y, double z) {
    double sum = 0.0, fac = 1.0, mu, dx, dy, dz;
    for (;;) {
        double sx = sqrt(x), sy = sqrt(y), sz = sqrt(z);
        double lam = sx * (sy + sz) + sy * sz;
        sum += fac / (sz * (z + lam));
        fac *= 0.25;
        x = (x + lam) * 0.25;
        y = (y + lam) * 0.25;
        z = (z + lam) * 0.25;
        mu = (x + y + 3.0 * z) * 0.2;
        dx = (mu - x) / mu;
        dy = (mu - y) / mu;
        dz = (mu - z) / mu;
        if (!(max3(fabs(dx), fabs(dy), fabs(dz)) > kTol)) break;
    }
    double ea = dx * dy, eb = dz * dz;
    double ec = ea - eb, ed = ea - 6.0 * eb;
    double ef = ed + 2.0 * ec;
    double s1 = ed * (-3.0 / 14.0 + 0.25 * (9.0 / 22.0) * ed - 1.5 * (3.0 / 26.0) * dz * ef);
    double s2 = dz * (ef / 6.0 + dz * (-(9.0 / 22.0) * ec + dz * (3.0 / 26.0) * ea));
    return 3.0 * sum + fac * (1.0 + s1 + s2) / (mu * sqrt(mu));
}

// R_J(x, y, z, p) = 3/2 int_0^inf dt / ((t+p) sqrt((t+x)(t+y)(t+z))).
__device__ double carlson_rj(double x, double y, double z, double p) {
    double sum = 0.0, fac = 1.0, mu, dx, dy, dz, dp;
    for (;;) {
        double sx = sqrt(x), sy = sqrt(y), sz = sqrt(z);
        double lam = sx * (sy + sz) + sy * sz;
        double al = p * (sx + sy + sz) + sx * sy * sz;
        al = al * al;
        double pl = p + lam;
        double be = p * (pl * pl);
        sum += fac * carlson_rc(al, be);
        fac *= 0.25;
        x = (x + lam) * 0.25;
        y = (y + lam) * 0.25;
        z = (z + lam) * 0.25;
        p = (p + lam) * 0.25;
        mu = (x + y + z + 2.0 * p) * 0.2;
        dx = (mu - x) / mu;
        dy = (mu - y) / mu;
        dz = (mu - z) / mu;
        dp = (mu - p) / mu;
        if (!(fmax(max3(fabs(dx), fabs(dy), fabs(dz)), fabs(dp)) > kTol)) break;
    }
    double ea = dx * (dy + dz) + dy * dz;
    double eb = dx * dy * dz;
    double ec = dp * dp;
    double e2 = ea - 3.0 * ec;
    double e3 = eb + 2.0 * dp * (ea - ec);
    const double c1 = 3.0 / 14.0, c2 = 1.0 / 3.0, c3 = 3.0 / 22.0, c4 = 3.0 / 26.0;
    double s1 = 1.0 + e2 * (-c1 + 0.75 * c3 * e2 - 1.5 * c4 * e3);
    double s2 = eb * (0.5 * c2 + dp * (-c3 - c3 + dp * c4));
    double s3 = dp * ea * (c2 - dp * c3) - c2 * dp * ec;
    return 3.0 * sum + fac * (s1 + s2 + s3) / (mu * sqrt(mu));
}

// Complete elliptic integrals with modulus k (not the parameter m = k^2).
__device__ double ellip_k(double k, int *err) {
    if (k < 0.0 || k > 1.0) { *err |= kErrModulus; return nan(""); }
    double y = 1.0 - k * k;
    if (k > 1.0 - 1e-10)
        return 1.38629436112 + y * (0.09666344259 + y * 0.03590092383) -
               log(y) * (0.5 + y * (0.12498593597 + y * 0.06880248576));
    return carlson_rf(0.0, y, 1.0);
}

__device__ double ellip_e(double k, int *err) {
    if (k < 0.0 || k > 1.0) { *err |= kErrModulus; return nan(""); }
    double y = 1.0 - k * k;
    if (k > 1.0 - 1e-10)
        return 1.0 + y * (0.44325141463 + y * (0.06260601220 + y * 0.04757383546)) -
               y * log(y) * (0.24998368310 + y * (0.09200180037 + y * 0.04069697526));
    return carlson_rf(0.0, y, 1.0) - (1.0 / 3.0) * (k * k) * carlson_rd(0.0, y, 1.0);
}

// Pi(n, k) = int_0^{pi/2} dtheta / ((1 - n sin^2) sqrt(1 - k^2 sin^2)).
__device__ double ellip_pi(double n, double k, int *err) {
    if (k < 0.0 || k > 1.0) { *err |= kErrModulus; return nan(""); }
    double y = 1.0 - k * k;
    return carlson_rf(0.0, y, 1.0) + (1.0 / 3.0) * n * carlson_rj(0.0, y, 1.0, 1.0 - n);
}

// ---- constants of motion (geodesic.py:899-1050) --------------------------------
// Potentials of Schmidt's energy equation with z_- = zm (here sqrt(1 - x^2)).
struct Pot {
    double f, g, h, d;
};

__device__ __forceinline__ double delta_r(double r, double a) { return r * r - 2.0 * r + a * a; }

__device__ Pot potentials(double r, double a, double zm) {
    double zm2 = zm * zm, D = delta_r(r, a);
    Pot o;
    o.f = r * r * r * r + a * a * (r * (r + 2.0) + zm2 * D);
    o.g = 2.0 * a * r;
    o.h = r * (r - 2.0) + zm2 / (1.0 - zm2) * D;
    o.d = (r * r + a * a * zm2) * D;
    return o;
}

// d/dr of the potentials (spherical orbits).
__device__ Pot potentials_dr(double r, double a, double zm) {
    double zm2 = zm * zm, a2 = a * a;
    Pot o;
    o.f = 4.0 * r * r * r + a2 * (2.0 * r * (1.0 + zm2) + 2.0 * (1.0 - zm2));
    o.g = 2.0 * a;
    o.h = 2.0 * (r - 1.0) * (1.0 + zm2 / (1.0 - zm2));
    o.d = 4.0 * r * r * r - 6.0 * r * r + 2.0 * a2 * r * (1.0 + zm2) - 2.0 * a2 * zm2;
    return o;
}

__device__ double kerr_energy(double a, double p, double e, double x) {
    double zm = sqrt(1.0 - x * x);
    double sgnax = (a * x > 0.0) ? 1.0 : -1.0;
    Pot P, Q;  // the two rows of the 2x2 system: (r1, r2), or (r, d/dr) for spherical orbits
    if (e < 1e-10) {
        P = potentials(p, a, zm);
        Q = potentials_dr(p, a, zm);
    } else if (fabs(x) == 1.0) {
        double e2 = e * e, a2 = a * a, em1 = -1.0 + e2;
        double t3 = 3.0 + e2 - p;
        double denom = -4.0 * a2 * (em1 * em1) + (t3 * t3) * p;
        double rad = (a2 * a2 * a2 * (em1 * em1) + a2 * (-4.0 * e2 + (p - 2.0) * (p - 2.0)) * (p * p) +
                      2.0 * (a2 * a2) * p * (-2.0 + p + e2 * (2.0 + p))) /
                     (p * p * p);
        double numer = em1 * (a2 * (1.0 + 3.0 * e2 + p) + p * (-3.0 - e2 + p - sgnax * 2.0 * sqrt(rad)));
        double ratio = (fabs(denom) < 1e-14 || fabs(numer) < 1e-14) ? 0.0 : numer / denom;
        return sqrt(1.0 - ((1.0 - e2) * (1.0 + ratio)) / p);
    } else {
        P = potentials(p / (1.0 - e), a, zm);
        Q = potentials(p / (1.0 + e), a, zm);
    }
    double kap = P.d * Q.h - P.h * Q.d;
    double eps = P.d * Q.g - P.g * Q.d;
    double rho = P.f * Q.h - P.h * Q.f;
    double eta = P.f * Q.g - P.g * Q.f;
    double sig = P.g * Q.h - P.h * Q.g;
    double disc = sig * (sig * eps * eps + rho * eps * kap - eta * kap * kap);
    return sqrt((kap * rho + 2.0 * eps * sig - sgnax * 2.0 * sqrt(disc)) / (rho * rho + 4.0 * eta * sig));
}

__device__ double kerr_angular_momentum(double a, double p, double e, double x, double En) {
    double zm = sqrt(1.0 - x * x);
    double sgnx = x > 0.0 ? 1.0 : -1.0;
    Pot P = potentials(p / (1.0 - e), a, zm);
    return (-En * P.g + sgnx * sqrt(-P.d * P.h + En * En * (P.g * P.g + P.f * P.h))) / P.h;
}

__device__ double kerr_carter(double a, double x, double En, double L) {
    double zm = sqrt(1.0 - x * x);
    double zm2 = zm * zm;
    return zm2 * (a * a * (1.0 - En * En) + L * L / (1.0 - zm2));
}

struct Roots {
    double r1, r2, r3, r4;
};

__device__ Roots radial_roots(double a, double p, double e, double En, double Q) {
    Roots o;
    o.r1 = p / (1.0 - e);
    o.r2 = p / (1.0 + e);
    double one_m_E2 = 1.0 - En * En;
    double s = 2.0 / one_m_E2 - (o.r1 + o.r2);
    double prod = (a * a * Q) / (one_m_E2 * o.r1 * o.r2);
    o.r3 = (s + sqrt(s * s - 4.0 * prod)) / 2.0;
    o.r4 = prod / o.r3;
    return o;
}

struct Mino {
    double gam, ups_phi, ups_theta, ups_r;
};

// Terms shared by the generic and equatorial Mino frequencies: the radial
// parts of Upsilon_phi and Gamma (Fujita & Hikida eq. 21).
struct RadialPart {
    double phi;  // coefficient bracket of Upsilon_phi's radial term
    double gam;  // Gamma minus 4 E (the radial bracket)
};

__device__ RadialPart radial_part(double a, double En, double L, const Roots &R, double ups_r, double K, double E,
                                  bool equatorial, int *err) {
    const double M = 1.0;
    double rp = M + sqrt(1.0 - a * a), rm = M - sqrt(1.0 - a * a);
    double kr = sqrt((R.r1 - R.r2) / (R.r1 - R.r3) * (R.r3 - R.r4) / (R.r2 - R.r4));
    double hr = (R.r1 - R.r2) / (R.r1 - R.r3);
    double hp = ((R.r1 - R.r2) * (R.r3 - rp)) / ((R.r1 - R.r3) * (R.r2 - rp));
    double hm = ((R.r1 - R.r2) * (R.r3 - rm)) / ((R.r1 - R.r3) * (R.r2 - rm));
    double Pi_r = ellip_pi(hr, kr, err), Pi_p = ellip_pi(hp, kr, err), Pi_m = ellip_pi(hm, kr, err);
    double root = sqrt((1.0 - En * En) * (R.r1 - R.r3) * (R.r2 - R.r4));
    double Kp = K - (R.r2 - R.r3) / (R.r2 - rp) * Pi_p;
    double Km = K - (R.r2 - R.r3) / (R.r2 - rm) * Pi_m;
    double tp = (2.0 * M * En * rp - a * L) * (equatorial ? Kp : 1.0);
    double tp2 = ((4.0 * En - a * L) * rp - 2.0 * M * (a * a) * En) * (equatorial ? Kp : 1.0);
    if (equatorial) {
        // geodesic.py:395-397 and 407-412: the + horizon term vanishes when r3 == r+
        if (fabs(tp) != 0.0) tp = tp / (R.r3 - rp);
        if (fabs(tp2) != 0.0) tp2 = tp2 / (R.r3 - rp);
    } else {
        tp = tp / (R.r3 - rp) * Kp;
        tp2 = tp2 / (R.r3 - rp) * Kp;
    }
    RadialPart o;
    o.phi = (2.0 * a * ups_r) / (kPi * (rp - rm) * root) *
            (tp - (2.0 * M * En * rm - a * L) / (R.r3 - rm) * Km);
    o.gam = (2.0 * ups_r) / (kPi * root) *
            (En / 2.0 *
                 ((R.r3 * (R.r1 + R.r2 + R.r3) - R.r1 * R.r2) * K +
                  (R.r2 - R.r3) * (R.r1 + R.r2 + R.r3 + R.r4) * Pi_r + (R.r1 - R.r3) * (R.r2 - R.r4) * E) +
             2.0 * M * En * (R.r3 * K + (R.r2 - R.r3) * Pi_r) +
             (2.0 * M) / (rp - rm) * (tp2 - ((4.0 * En - a * L) * rm - 2.0 * M * (a * a) * En) / (R.r3 - rm) * Km));
    return o;
}

__device__ Mino mino_generic(double a, double p, double e, double x, int *err) {
    double En = kerr_energy(a, p, e, x);
    double L = kerr_angular_momentum(a, p, e, x, En);
    double Q = kerr_carter(a, x, En, L);
    Roots R = radial_roots(a, p, e, En, Q);
    double zm = 1.0 - x * x;
    double E2m1 = -1.0 + En * En;
    double num = L * L + a * a * E2m1 * (-1.0 + zm);
    double a2zp = num / (E2m1 * (-1.0 + zm));
    double eps0zp = -(num / (L * L * (-1.0 + zm)));
    double zm_over_zp = zm / (num / (a * a * E2m1 * (-1.0 + zm)));
    double kr = sqrt((R.r1 - R.r2) / (R.r1 - R.r3) * (R.r3 - R.r4) / (R.r2 - R.r4));
    double kth = sqrt(zm_over_zp);
    double K_r = ellip_k(kr, err), K_th = ellip_k(kth, err);
    double ups_th = (kPi * L * sqrt(eps0zp)) / (2.0 * K_th);
    double ups_r = (kPi * sqrt((1.0 - En * En) * (R.r1 - R.r3) * (R.r2 - R.r4))) / (2.0 * K_r);
    RadialPart rad = radial_part(a, En, L, R, ups_r, K_r, ellip_e(kr, err), false, err);
    Mino o;
    o.ups_phi = (2.0 * ups_th) / (kPi * sqrt(eps0zp)) * ellip_pi(zm, kth, err) + rad.phi;
    o.gam = 4.0 * En + (2.0 * a2zp * En * ups_th) / (kPi * L * sqrt(eps0zp)) * (K_th - ellip_e(kth, err)) + rad.gam;
    o.ups_theta = fabs(ups_th);
    o.ups_r = ups_r;
    return o;
}

__device__ Mino mino_equatorial(double a, double p, double e, double x, int *err) {
    double En = kerr_energy(a, p, e, x);
    double L = kerr_angular_momentum(a, p, e, x, En);
    Roots R = radial_roots(a, p, e, En, 0.0);
    double eps0zp = -((L * L + a * a * (-1.0 + En * En) * (-1.0)) / (L * L * (-1.0)));
    double zp = a * a * (1.0 - En * En) + L * L;
    double kr = sqrt((R.r1 - R.r2) / (R.r1 - R.r3) * (R.r3 - R.r4) / (R.r2 - R.r4));
    double K = ellip_k(kr, err);
    double ups_r = (kPi * sqrt((1.0 - En * En) * (R.r1 - R.r3) * (R.r2))) / (2.0 * K);
    double ups_th = x * pow(zp, 0.5);
    RadialPart rad = radial_part(a, En, L, R, ups_r, K, ellip_e(kr, err), true, err);
    Mino o;
    o.ups_phi = ups_th / sqrt(eps0zp) + rad.phi;
    o.gam = 4.0 * En + rad.gam;
    o.ups_theta = fabs(ups_th);
    o.ups_r = ups_r;
    return o;
}

__device__ Mino mino_circular(double a, double p) {
    double sp = sqrt(p), a2 = a * a;
    double q = a2 - 4.0 * a * sp - (-4.0 + p) * p;
    double am = a - sp;
    double ups_r = sqrt((p * (-2.0 * a2 + 6.0 * a * sp + (-5.0 + p) * p + (am * am * q) / fabs(q))) /
                        (2.0 * a * sp + (-3.0 + p) * p));
    double den = sqrt(2.0 * a + (-3.0 + p) * sp);
    Mino o;
    o.ups_theta = fabs((pow(p, 0.25) * sqrt(3.0 * a2 - 4.0 * a * sp + p * p)) / den);
    o.ups_phi = pow(p, 1.25) / den;
    o.gam = (pow(p, 1.25) * (a + pow(p, 1.5))) / den;
    o.ups_r = ups_r;
    return o;
}

// Schwarzschild (a = 0): Omega_phi and Omega_r in closed form.
__device__ void schwarzschild(double p, double e, double *Ophi, double *Or, int *err) {
    double k = sqrt(4.0 * e / (p - 6.0 + 2.0 * e));
    double E = ellip_e(k, err), K = ellip_k(k, err);
    double Pi1 = ellip_pi(16.0 * e / (12.0 + 8.0 * e - 4.0 * e * e - 8.0 * p + p * p), k, err);
    double Pi2 = ellip_pi(2.0 * e * (p - 4.0) / ((1.0 + e) * (p - 6.0 + 2.0 * e)), k, err);
    double p2 = p * p, pm4 = p - 4.0, pm4sq = pm4 * pm4;
    double br = (-2.0 * Pi2 * (6.0 + 2.0 * e - p) * (3.0 + e * e - p) * p2) / ((-1.0 + e) * ((1.0 + e) * (1.0 + e))) -
                (E * pm4 * p2 * (-6.0 + 2.0 * e + p)) / (-1.0 + e * e) +
                (K * p2 * (28.0 + 4.0 * e * e - 12.0 * p + p2)) / (-1.0 + e * e) +
                (4.0 * pm4 * p * (2.0 * (1.0 + e) * K + Pi2 * (-6.0 - 2.0 * e + p))) / (1.0 + e) +
                2.0 * pm4sq * (K * pm4 + (Pi1 * p * (-6.0 - 2.0 * e + p)) / (2.0 + 2.0 * e - p));
    double q = -4.0 * e * e + (p - 2.0) * (p - 2.0);
    *Ophi = (2.0 * pow(p, 1.5)) / (sqrt(q) * (8.0 + br / (K * pm4sq)));
    *Or = (p * sqrt((-6.0 + 2.0 * e + p) / q) * kPi) / (8.0 * K + br / pm4sq);
}

__device__ void coordinate_frequencies(double a, double p, double e, double x, double *Ophi, double *Oth, double *Or,
                                       int *err) {
    if (a != 0.0) {
        Mino m;
        if (e > 0.0 || fabs(x) < 1.0) {
            m = fabs(x) < 1.0 ? mino_generic(a, p, e, x, err) : mino_equatorial(a, p, e, x, err);
        } else {
            m = mino_circular(a * x, p);
            m.ups_phi = x * m.ups_phi;
        }
        *Ophi = m.ups_phi / m.gam;
        *Oth = m.ups_theta / m.gam;
        *Or = m.ups_r / m.gam;
    } else {
        double ophi, orr;
        schwarzschild(p, e, &ophi, &orr, err);
        *Ophi = (x > 0.0 ? 1.0 : -1.0) * ophi;
        *Oth = ophi;
        *Or = orr;
    }
}

// One thread per trajectory point.  Outputs are divided by `denom` (1 for the
// dimensionless frequencies; 2 pi M MTSUN_SI for Hz); abs_phi takes |f_phi|
// (the frequency-domain sum's convention, fdinterp.py:232-236).
__global__ void k_fundamental_frequencies(const double *a, int a_stride, const double *p, const double *e,
                                          const double *x, int n, double denom, int abs_phi, double *o_phi,
                                          double *o_theta, double *o_r, int *status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int err = 0;
    double ophi, oth, orr;
    coordinate_frequencies(a[(long long)i * a_stride], p[i], e[i], x[i], &ophi, &oth, &orr, &err);
    ophi = ophi / denom;
    o_phi[i] = abs_phi ? fabs(ophi) : ophi;
    o_theta[i] = oth / denom;
    o_r[i] = orr / denom;
    if (err && status) atomicOr(status, err);
}

}  // namespace geo
}  // namespace few

extern "C" FEW_API int few_fundamental_frequencies(const double *a, int a_stride, const double *p, const double *e,
                                                   const double *x, int n, double denom, int abs_phi, double *o_phi,
                                                   double *o_theta, double *o_r, int *status, void *stream) {
    few::clear_error();
    if (n < 0) return few::fail(FEW_ERR_SIZE, "few_fundamental_frequencies: n=%d < 0", n);
    if (n == 0) return FEW_OK;
    if (!a || !p || !e || !x || !o_phi || !o_theta || !o_r)
        return few::fail(FEW_ERR_ARG, "few_fundamental_frequencies: null pointer");
    if (a_stride != 0 && a_stride != 1)
        return few::fail(FEW_ERR_ARG, "few_fundamental_frequencies: a_stride=%d (0 or 1)", a_stride);
    if (!(denom != 0.0)) return few::fail(FEW_ERR_ARG, "few_fundamental_frequencies: denom must be non-zero");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    few::geo::k_fundamental_frequencies<<<(n + 127) / 128, 128, 0, st>>>(a, a_stride, p, e, x, n, denom, abs_phi,
                                                                          o_phi, o_theta, o_r, status);
    FEW_LAUNCH_CHECK("k_fundamental_frequencies");
    return FEW_OK;
}
