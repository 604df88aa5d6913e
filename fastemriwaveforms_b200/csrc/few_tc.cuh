// tcgen05 building blocks shared by the tensor-core kernels: shared-memory and
// instruction descriptors, MMA issue and commit, bounded mbarrier waits, TMEM
// loads, bf16 hi/lo splitting, FP32 complex helpers and the FP64-reduced phase
// anchor.  sm_100a only.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "few_common.cuh"

namespace few {

constexpr unsigned long long kWaitLimitNs = 1000000000ull;  // 1 s of global time per wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Arrival that also announces `bytes` of asynchronous copies completing on the barrier.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bulk (untiled, no multicast) copy of `bytes` from global into this CTA's shared
// memory, completing on `bar`; both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void *smem_dst, const void *gmem_src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem_dst)),
                 "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Bounded wait; false if the phase did not complete within kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (global_ns() - t0 < kWaitLimitNs)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100; base offset 0; no swizzle
    return d;
}

// kind::f16 instruction descriptor: D f32, A and B bf16, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate)
{
    uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

// kind::i8 instruction descriptor: D s32, A and B signed 8-bit, both MN-major
// (bit 15 / 16), M x N.
__host__ __device__ constexpr uint32_t idesc_s8_mn(int M, int N)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

// One kind::i8 MMA (K = 32): D[s32] (+)= A[s8] B[s8], exact integer arithmetic.
__device__ __forceinline__ void mma_s8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate)
{
    uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

// Signed base-256 digits.  An operand value x is scaled to an integer
// |Y| <= 127 2^24 and written as Y = d0 2^24 + d1 2^16 + d2 2^8 + d3 with
// |d0| <= 127 and d1..d3 in [-128, 127] (each an int8).  Products of two such
// expansions, summed by the integer tensor core level by level (level = digit
// index sum), are exact; levels >= 4 weigh below 2^-31 of the scales.
//
// The digits come straight out of the bytes of Y + kDigitBias (kDigitBias =
// 128 (1 + 2^8 + 2^16)): its bytes 0..2 are d3..d1 + 128, its byte 3 is d0.
// scaled_biased gives Y + kDigitBias as the low 32 bits of the FMA
// x * scale + 1.5 * 2^52 + kDigitBias (rounded once: rint(x * scale)), so no
// conversion instruction is needed.
constexpr int kDigitBias = 128 + (128 << 8) + (128 << 16);
constexpr double kDigitScale = 127.0 * 16777216.0;  // |x| <= 1 -> |Y| <= 127 2^24

__device__ __forceinline__ uint32_t scaled_biased(double x, double scale)
{
    return (uint32_t)__double2loint(__fma_rn(x, scale, 6755399441055744.0 + (double)kDigitBias));
}

// The biased integer of -x from that of x: -Y + B = 2B - (Y + B).
__device__ __forceinline__ uint32_t negated_biased(uint32_t y) { return 2u * (uint32_t)kDigitBias - y; }

// Four biased values -> one word per digit plane (byte e = value e), plane 0
// the most significant.
__device__ __forceinline__ void digit_words8(uint32_t y0, uint32_t y1, uint32_t y2, uint32_t y3, uint32_t *w)
{
    w[0] = __byte_perm(__byte_perm(y0, y1, 0x0073), __byte_perm(y2, y3, 0x0073), 0x5410);
    w[1] = __byte_perm(__byte_perm(y0, y1, 0x0062), __byte_perm(y2, y3, 0x0062), 0x5410) ^ 0x80808080u;
    w[2] = __byte_perm(__byte_perm(y0, y1, 0x0051), __byte_perm(y2, y3, 0x0051), 0x5410) ^ 0x80808080u;
    w[3] = __byte_perm(__byte_perm(y0, y1, 0x0040), __byte_perm(y2, y3, 0x0040), 0x5410) ^ 0x80808080u;
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Byte offset of element (row, k) of a K-major, no-swizzle tile whose K-steps
// of 16 hold `groups` 8-row groups: K-step stride groups*256, 8-row group
// stride (SBO) 256, K-half stride (LBO) 128, row 16, element 2.
__host__ __device__ __forceinline__ uint32_t tile_off(int row, int k, int groups)
{
    return (uint32_t)((k >> 4) * groups * 256 + (row >> 3) * 256 + ((k >> 3) & 1) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// x = hi + lo with hi, lo bf16, packed two complex numbers (re, im, re, im) at a time.
__device__ __forceinline__ void split2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    float2 hf = __bfloat1622float2(h);
    __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
    hi = *reinterpret_cast<uint32_t *>(&h);
    lo = *reinterpret_cast<uint32_t *>(&l);
}

__device__ __forceinline__ float2 fcmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 fcpow(float2 z, int p)
{
    if (p < 0) {
        z.y = -z.y;
        p = -p;
    }
    float2 r = make_float2(1.f, 0.f);
    while (p) {
        if (p & 1) r = fcmul(r, z);
        p >>= 1;
        if (p) z = fcmul(z, z);
    }
    return r;
}

// exp(-i phi): the argument is reduced mod 2 pi in FP64 (phi reaches ~1e7 rad,
// where FP32 would keep no fraction of a turn), then sine and cosine are taken
// in FP32 on the reduced value in [-pi, pi].
__device__ __forceinline__ float2 anchor(double phi)
{
    const double two_pi = 6.283185307179586476925286766559;
    const double k = rint(phi * 0.15915494309189533576888376337251);
    const float red = (float)fma(-k, two_pi, phi);
    float s, c;
    sincosf(red, &s, &c);
    return make_float2(c, -s);
}

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }


// Tensor-core state a CTA carries across units: TMEM accumulator, one
// mbarrier per A/B buffer, their phases and whether a commit is outstanding
// (scalars, so that nothing is indexed at run time and all stays in registers).
struct MixedPipe {
    uint32_t tmem;
    uint64_t *bar;  // [2]
    uint32_t ph0, ph1;
    int pend0, pend1;
};

// Bounded wait for buffer b's outstanding MMAs.  On a timeout the commit
// stays pending, so a later drain (the teardown's) waits for it again.
__device__ __forceinline__ bool pipe_drain(MixedPipe &p, int b)
{
    if (b == 0) {
        if (!p.pend0) return true;
        const bool ok = mbar_wait_bounded(&p.bar[0], p.ph0);
        if (ok) {
            p.ph0 ^= 1u;
            p.pend0 = 0;
        }
        return ok;
    }
    if (!p.pend1) return true;
    const bool ok = mbar_wait_bounded(&p.bar[1], p.ph1);
    if (ok) {
        p.ph1 ^= 1u;
        p.pend1 = 0;
    }
    return ok;
}

__device__ __forceinline__ void mixed_setup(uint32_t *s_tmem, uint64_t *bars, int tmem_cols, MixedPipe &pp)
{
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                     "r"((uint32_t)tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    pp.tmem = *s_tmem;
    pp.bar = bars;
    pp.ph0 = pp.ph1 = 0;
    pp.pend0 = pp.pend1 = 0;
}

// End of a CTA: wait (bounded) for any MMA still in flight, then free TMEM.
// When that wait itself times out, an MMA may still be writing the
// accumulator, so the columns are left allocated rather than handed to the
// next CTA, and the error word stays set.
__device__ __forceinline__ void mixed_teardown(bool failed, MixedPipe &pp, int tmem_cols, int *err)
{
    const bool ok0 = pipe_drain(pp, 0);
    const bool ok1 = pipe_drain(pp, 1);
    tc_fence_before();
    const bool drained = __syncthreads_and(ok0 && ok1) != 0;
    if ((failed || !drained) && threadIdx.x == 0) atomicExch(err, 1);
    if (!drained) return;
    if ((threadIdx.x >> 5) == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(pp.tmem),
                     "r"((uint32_t)tmem_cols)
                     : "memory");
    }
}

}  // namespace few
