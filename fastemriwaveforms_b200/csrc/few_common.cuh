// Shared device helpers for the B200 interpolated mode sum.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "few_b200.h"

namespace few {

// Nanoseconds of the GPU's global timer.
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// Complex FP64 helpers (double2: x = real, y = imaginary).  These are ordinary
// FP64 expressions; nvcc may contract them into FMAs, which is intended.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// a * (1 + i e) for a tiny angle e (first order of exp(i e); |e| < 1e-8 keeps
// the dropped e^2/2 term below 1e-16).
__device__ __forceinline__ double2 crot_small(double2 a, double e)
{
    return make_double2(fma(-a.y, e, a.x), fma(a.x, e, a.y));
}

// z^p for an integer p by binary powering (conjugate base for p < 0).
__device__ __forceinline__ double2 cpow_int(double2 z, int p)
{
    if (p < 0) {
        z = cconj(z);
        p = -p;
    }
    double2 r = make_double2(1.0, 0.0);
    while (p) {
        if (p & 1) r = cmul(r, z);
        p >>= 1;
        if (p) z = cmul(z, z);
    }
    return r;
}

// ---------------------------------------------------------------------------
// Exactly rounded operations used where the reference's rounding is replayed.
// The intrinsics stop nvcc from contracting a*b+c into one FMA.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }

// Error of the rounded sum s = fl(a + b): a + b = s + err exactly (Knuth's TwoSum).
__device__ __forceinline__ double two_sum_err(double a, double b, double s)
{
    double bb = __dsub_rn(s, a);
    return __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}

// sin and cos of a large angle: Cody & Waite reduction mod 2 pi (2 pi split in
// three parts, k*C1 and k*C2 exact for |k| < 2^21), then sincos on |r| <= pi,
// which stays on the function's short path (large arguments take its slow,
// table-driven reduction).
__device__ __forceinline__ void sincos_reduced(double ph, double *s, double *c)
{
    const double kInv2Pi = 0.15915494309189535;
    const double kC1 = 0x1.921fb54400000p+2, kC2 = 0x1.0b4611a600000p-32, kC3 = 0x1.3198a2e037073p-67;
    double r = ph;
    const double kq = rint(ph * kInv2Pi);
    if (fabs(kq) < 2097152.0) {
        r = __fma_rn(-kq, kC1, ph);
        r = __fma_rn(-kq, kC2, r);
        r = __fma_rn(-kq, kC3, r);
    }
    sincos(r, s, c);
}

// The 8-term dense-output phase polynomial in s, s1 = 1 - s, in the
// operation order of src/few/cutils/interpolate.cu:642-644, every product and
// sum rounded separately.
__device__ __forceinline__ double phase_poly(const double *c, double s, double s1)
{
    double a = rmul(s, c[7]);
    a = rmul(s1, radd(c[6], a));
    a = rmul(s, radd(c[5], a));
    a = rmul(s1, radd(c[4], a));
    a = rmul(s, radd(c[3], a));
    a = rmul(s1, radd(c[2], a));
    a = rmul(s, radd(c[1], a));
    return radd(c[0], a);
}

}  // namespace few
