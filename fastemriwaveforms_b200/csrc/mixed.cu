// Mixed-precision mode sum on the 5th-generation tensor cores (tcgen05).
//
// Per knot segment s the folded sum is
//     h_i = sum_r u_r(t_i) Y_r(t_i),   Y_r = sum_c tau_i^c Z_{c,r}(t_i),
//     Z_{c,r}(t_i) = sum_{n'} v_{n'}(t_i) W'[c][n'][r]
// with tau = (t - t_s)/h_s in [0, 1), W'[c] = W[c] h_s^c (the folded
// coefficients rescaled so that every power of tau is <= 1),
// v_{n'} = exp(-i n' Phi_r), u_r = exp(-i (m' Phi_phi + k' Phi_theta)).  The
// contraction over n' runs on the tensor cores as a real GEMM
//     [Re v | Im v interleaved] (128 samples x 2 NNp)  x  B (2 NNp x 8R)
// whose 8 columns per (m', k') row hold (Re Z_{c,r}, Im Z_{c,r}) for c = 0..3;
// the epilogue applies tau^c (Horner) and u_r in FP32.  (The adjoints run in
// exact integer arithmetic on the tensor cores: mixed_adjoint.cu, mixed_phase.cu.)
//
// Precision plan:
//   * FP64: the phase polynomials, the per-sample anchors exp(-i Phi) and the
//     anchors of the n' recurrence (every 16 steps), each reduced mod 2 pi;
//   * FP32: the phasor recurrence between anchors, the row phasors u_r, the
//     powers of tau and the epilogue sums;
//   * tensor cores: split BF16 (x = hi + lo, three products hi*hi + hi*lo +
//     lo*hi) with FP32 accumulation in TMEM.
//
// Layout: A and B tiles are K-major, no swizzle: 8x8 bf16 core matrices of
// 128 contiguous bytes; stride 128 B between the two K halves of a K=16 step
// (LBO) and 256 B between 8-row groups (SBO).  A CTA of 8 producer warps and one
// MMA warp owns a work unit (<= 1024 samples of one segment) at a time, in
// 128-sample tiles; two producer threads share a sample row.  K runs in chunks
// of 32 (16 n' x {Re, Im}) through a two-stage ring: the producer half h writes
// the A chunks k = h, h + 2, ... into stage h while the MMA warp brings each
// chunk's B into its stage with one bulk copy and issues its MMAs (2 K-steps x
// 3 split products per group of <= 256 columns); mbarriers gate every hand-off
// (details at the kernels).  Every wait is bounded and a timeout sets an error
// word and ends the kernel, freeing TMEM only once the MMAs have drained.
#include <cuda_bf16.h>

#include "few_common.cuh"
#include "few_internal.h"
#include "few_tc.cuh"

namespace few {

namespace {

constexpr int kMT = 128;   // samples per tile (MMA M)
constexpr int kKC = 32;    // real K per chunk: 16 n' x {Re, Im}
constexpr int kAStage = 2 * kMT * kKC * 2;  // A hi + lo planes of one stage (16 KB)

// ---------------------------------------------------------------------------
// B operand: per segment and K chunk, hi and lo bf16 tiles in the smem layout.
// ---------------------------------------------------------------------------
// Columns: 8 per (m', k') row r, slot = j % 8 = 2 c + re/im.  K chunk ch
// covers the 16 n' of block ch, element kk = 2 (n' - 16 ch) + part.  One
// thread per 16-byte row of a core matrix (column j, K elements 8 kg ..
// 8 kg + 7 = 4 n' x 2 parts); writes the hi and the lo chunk.
__global__ void __launch_bounds__(256) k_fold_mixed(const double2 *__restrict__ W, const double *__restrict__ t_knots,
                                                    int nseg, int R, int NN, int NB, int nchunks,
                                                    __nv_bfloat16 *__restrict__ Bpk)
{
    const long long per_chunk = (long long)NB * kKC;  // elements of one plane of one chunk
    const long long total = (long long)nseg * nchunks * (kKC / 8) * NB;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int j = (int)(idx % NB);
    long long rest = idx / NB;
    const int kg = (int)(rest % (kKC / 8));
    rest /= (kKC / 8);
    const int ch = (int)(rest % nchunks);
    const int s = (int)(rest / nchunks);
    const int r = j >> 3, slot = j & 7;
    const bool im_col = slot & 1;
    const int nblk = ch, c = slot >> 1;
    const double h = t_knots[s + 1] - t_knots[s];
    const double hc = (c == 0) ? 1.0 : (c == 1 ? h : (c == 2 ? h * h : h * h * h));
    float f[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int nidx = 16 * nblk + 4 * kg + q;
        double v0 = 0.0, v1 = 0.0;
        if (r < R && nidx < NN) {
            const double2 w = W[(((long long)s * R + r) * NN + nidx) * 4 + c];
            const double wr = w.x * hc, wi = w.y * hc;
            v0 = im_col ? wi : wr;   // part 0: Re Z += Re v Re W ; Im Z += Re v Im W
            v1 = im_col ? wr : -wi;  // part 1: Re Z -= Im v Im W ; Im Z += Im v Re W
        }
        f[2 * q] = (float)v0;
        f[2 * q + 1] = (float)v1;
    }
    uint32_t h4[4], l4[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) split2(f[2 * e], f[2 * e + 1], h4[e], l4[e]);
    const uint32_t off = tile_off(j, 8 * kg, NB / 8);  // bytes; 16-byte aligned
    unsigned char *base = reinterpret_cast<unsigned char *>(Bpk + (((long long)s * nchunks + ch) * 2) * per_chunk);
    *reinterpret_cast<uint4 *>(base + off) = make_uint4(h4[0], h4[1], h4[2], h4[3]);
    *reinterpret_cast<uint4 *>(base + per_chunk * 2 + off) = make_uint4(l4[0], l4[1], l4[2], l4[3]);
}

struct MixedArgs {
    double2 *wf;
    const __nv_bfloat16 *Bpk;
    const double *pc;
    const double *seg_info;
    const double *t_knots;
    const int *units;
    const int *row_m;
    const int *row_k;
    int *err;
    int N, R, nlo, NN, NNp, NB, nchunks, use_theta, tmem_cols;
    double dt;
};

__host__ __device__ __forceinline__ void mixed_dims_core(int R, int NN, int &NNp, int &NB, int &nchunks)
{
    NNp = (NN + 15) / 16 * 16;
    NB = (8 * R + 15) / 16 * 16;
    nchunks = NNp / 16;
}

// ---------------------------------------------------------------------------
// Warp-specialized sum: 8 producer warps and one MMA warp per CTA.
// ---------------------------------------------------------------------------
// Producer warp w owns TMEM lane quarter w & 3 (samples 32 (w & 3) .. +31 of a
// 128-sample tile) and half h = w >> 2: half h writes the A chunks k = h, h + 2,
// ... of every tile into its nas (1 or 2) A stages in turn (with two, it writes
// the next chunk while the tensor cores still read the previous one) and reads
// accumulator column groups [h G/2, ...) in the epilogue; two threads share a
// sample.  The B chunks go through their own ring of nbs (2..4) slots: lane 0 of
// the MMA warp brings each chunk in with one bulk copy nbs - 1 chunks ahead of
// its MMAs, waits for the chunk's A stage, issues the MMAs and commits them to
// the A stage's and the B slot's "empty" barriers, and after a tile's last chunk
// to "accumulator full".  Barriers: full[b] (4 producer arrivals) and empty[b]
// (MMA commit) per A stage, bfull[s] (the bulk copy's bytes),
// bempty[s] (MMA commit), accf (MMA commit), acce (8 producer arrivals once the
// accumulator has been read).  Every wait is bounded; a timeout sets the CTA's
// fail word, after which no role waits again, every producer still reaches
// every named barrier and arrival, and the MMA warp stops issuing.
constexpr int kSumProd = 8;                        // producer warps: two per TMEM lane quarter
constexpr int kSumProdThreads = 32 * kSumProd;     // 256
constexpr int kSumThreads = kSumProdThreads + 32;  // + the MMA warp
constexpr int kMaxBSlots = kMaxBStages;
constexpr int kMaxAStages = 4;     // two per producer half
constexpr int kMixedMaxRows = 64;  // (m', k') rows the accumulator holds

struct SumShared {
    uint64_t full[kMaxAStages], empty[kMaxAStages], bfull[kMaxBSlots], bempty[kMaxBSlots], accf, acce, done;
    uint32_t tmem;
    int fail;
    int rm[kMixedMaxRows], rk[kMixedMaxRows];
    double pc[24];
    float2 part[2][kMT];  // half 1's epilogue sums, by tile parity
};

// Ring layout of the dynamic shared memory: 2 nas A stages, then nbs B slots.
struct SumRing {
    int nas;       // A stages per producer half (1 or 2)
    int nbs;       // B slots
    int bslot;     // bytes per B slot (>= every unit's chunk)
};

// A stage of chunk k of a tile: half k & 1, its stages taken in turn.
__device__ __forceinline__ int sum_stage(int k, int nas) { return nas == 2 ? 2 * (k & 1) + ((k >> 1) & 1) : (k & 1); }

// Phases a role has consumed so far (registers; the same sequence in every role).
struct SumRole {
    uint32_t par, used; // A stage b: bit b = parity of its fills so far / filled at least once
    uint32_t tiles;     // accumulator uses
    uint32_t gi, gc;    // MMA warp: B chunks issued / consumed (all units)
    bool dead;
};

__device__ __forceinline__ void sum_prod_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kSumProdThreads) : "memory"); }

__device__ __forceinline__ void sum_setup(SumShared &s, int tmem_cols, SumRole &ro)
{
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                     "r"((uint32_t)tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int b = 0; b < kMaxAStages; ++b) {
            mbar_init(&s.full[b], kSumProd / 2);
            mbar_init(&s.empty[b], 1);
        }
        for (int q = 0; q < kMaxBSlots; ++q) {
            mbar_init(&s.bfull[q], 1);
            mbar_init(&s.bempty[q], 1);
        }
        mbar_init(&s.accf, 1);
        mbar_init(&s.acce, kSumProd);
        mbar_init(&s.done, 1);
        s.fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    ro.par = ro.used = ro.tiles = ro.gi = ro.gc = 0;
    ro.dead = false;
}

// End of a CTA: the MMA warp waits (bounded) for every MMA and bulk copy it
// issued; TMEM is freed only if that drain completed (otherwise an MMA may
// still be writing the accumulator and the columns stay allocated), and the
// error word is set on any timeout.
__device__ __forceinline__ void sum_teardown(SumShared &s, SumRole &ro, const SumRing &rg, int tmem_cols, int *err)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    bool drained = true;
    if (warp == kSumProd && lane == 0) {
        mma_commit(&s.done);
        drained = mbar_wait_bounded(&s.done, 0);
        for (uint32_t g = ro.gc; g < ro.gi; ++g)  // copies issued but not yet observed
            drained = mbar_wait_bounded(&s.bfull[g % rg.nbs], (g / rg.nbs) & 1u) && drained;
    }
    tc_fence_before();
    drained = __syncthreads_and(drained) != 0;
    if ((s.fail || !drained) && threadIdx.x == 0) atomicExch(err, 1);
    if (drained && warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem), "r"((uint32_t)tmem_cols)
                     : "memory");
    }
}

// MMA warp: bulk copy of B chunk k of the unit's segment into the next slot,
// once the MMAs of that slot's previous chunk are done.
__device__ __forceinline__ bool sum_issue_b(const unsigned char *Bseg, int k, uint32_t bchunk,
                                            unsigned char *smem_raw, const SumRing &rg, SumShared &s, SumRole &ro)
{
    const uint32_t g = ro.gi, slot = g % rg.nbs, use = g / rg.nbs;
    if (use >= 1 && !mbar_wait_bounded(&s.bempty[slot], (use - 1) & 1u)) return false;
    mbar_arrive_expect_tx(&s.bfull[slot], bchunk);
    bulk_copy_g2s(smem_raw + 2 * rg.nas * kAStage + slot * rg.bslot, Bseg + (size_t)k * bchunk, bchunk,
                  &s.bfull[slot]);
    ro.gi = g + 1;
    return true;
}

// MMA warp, lane 0: the B chunks and the MMAs of every tile of one unit.
__device__ void sum_mma_unit(const MixedArgs &a, int seg, int lo, int hi, unsigned char *smem_raw, const SumRing &rg,
                             SumShared &s, SumRole &ro)
{
    const int NB = a.NB, nch = a.nchunks;
    const uint32_t bchunk = (uint32_t)(2 * NB * kKC * 2);  // hi then lo planes
    const unsigned char *Bseg = reinterpret_cast<const unsigned char *>(a.Bpk) + (size_t)seg * nch * bchunk;
    const int nfill = (hi - lo + kMT - 1) / kMT * nch;     // (tile, chunk) pairs of the unit
    const int ahead = rg.nbs - 1;
    bool ok = !*(volatile int *)&s.fail;
    for (int f = 0; f < min(ahead, nfill) && ok; ++f) ok = sum_issue_b(Bseg, f % nch, bchunk, smem_raw, rg, s, ro);
    for (int f = 0; f < nfill && ok; ++f) {
        const int k = f % nch, b = sum_stage(k, rg.nas);
        const uint32_t pb = (ro.par >> b) & 1u;
        ok = !*(volatile int *)&s.fail;
        // the accumulator is free once every producer has read the previous tile
        if (ok && k == 0 && ro.tiles >= 1) ok = mbar_wait_bounded(&s.acce, (ro.tiles - 1) & 1u);
        const uint32_t g = ro.gc, slot = g % rg.nbs;
        if (ok) ok = mbar_wait_bounded(&s.bfull[slot], (g / rg.nbs) & 1u);
        if (!ok) break;
        ro.gc = g + 1;
        ok = mbar_wait_bounded(&s.full[b], pb);
        if (!ok) break;
        ro.par ^= 1u << b;
        tc_fence_after();
        const uint32_t a_h = smem_u32(smem_raw + b * kAStage), a_l = a_h + kMT * kKC * 2;
        const uint32_t b_h = smem_u32(smem_raw + 2 * rg.nas * kAStage + slot * rg.bslot), b_l = b_h + NB * kKC * 2;
#pragma unroll
        for (int st = 0; st < kKC / 16; ++st) {
            const uint64_t da_h = smem_desc(a_h + st * (kMT / 8) * 256, 128, 256);
            const uint64_t da_l = smem_desc(a_l + st * (kMT / 8) * 256, 128, 256);
            for (int n0 = 0; n0 < NB; n0 += 256) {  // column groups of <= 256 (one MMA each)
                const int nq = min(256, NB - n0);
                const uint32_t idesc = idesc_bf16(kMT, nq);
                const uint32_t boff = st * (NB / 8) * 256 + (n0 / 8) * 256;
                const uint64_t db_h = smem_desc(b_h + boff, 128, 256);
                const uint64_t db_l = smem_desc(b_l + boff, 128, 256);
                const uint32_t d = s.tmem + (uint32_t)n0;
                mma_bf16(d, da_h, db_h, idesc, (k | st) != 0);
                mma_bf16(d, da_h, db_l, idesc, 1u);
                mma_bf16(d, da_l, db_h, idesc, 1u);
            }
        }
        mma_commit(&s.empty[b]);
        mma_commit(&s.bempty[slot]);
        if (k == nch - 1) {
            mma_commit(&s.accf);
            ro.tiles++;
        }
        // next copy: into the slot of chunk f - 1, whose MMAs were issued one step ago
        if (f + ahead < nfill) ok = sum_issue_b(Bseg, (f + ahead) % nch, bchunk, smem_raw, rg, s, ro);
    }
    if (!ok) {
        ro.dead = true;
        atomicExch(&s.fail, 1);
    }
}

// Producer warps: one unit's A chunks and epilogues.  Every producer runs every
// tile of the unit and reaches every named barrier and arrival; after a failed
// wait it only skips the work.
__device__ void sum_prod_unit(const MixedArgs &a, int seg, int lo, int hi, unsigned char *smem_raw, const SumRing &rg,
                              SumShared &s, SumRole &ro)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int h = warp >> 2, row = 32 * (warp & 3) + lane;  // half; sample row = TMEM lane
    const int NB = a.NB, R = a.R, nlo = a.nlo, nch = a.nchunks;
    const long long nps = (long long)(a.N - 1) * 3;
    sum_prod_sync();  // the previous unit's readers of the row tables are done
    for (int r = tid; r < R; r += kSumProdThreads) {
        s.rm[r] = a.row_m[r];
        s.rk[r] = a.row_k[r];
    }
    if (tid < 24) {
        const int q = tid >> 3, c = tid & 7;
        s.pc[tid] = a.pc[c * nps + (long long)seg * 3 + q];
    }
    sum_prod_sync();
    const double t0 = a.seg_info[3 * seg], pt0 = a.seg_info[3 * seg + 1];
    // reciprocals once per unit: s and tau by multiplication (within an ulp of the
    // quotients, far below this form's FP32 phasor error)
    const double ipw = 1.0 / a.seg_info[3 * seg + 2];
    const double ihs = 1.0 / (a.t_knots[seg + 1] - a.t_knots[seg]);
    const int ng = NB / 16, gs = (ng + 1) / 2;  // 16-column groups; half 0 takes [0, gs)
    const int g_lo = h ? gs : 0, g_hi = h ? ng : gs;

    for (int base = lo; base < hi; base += kMT) {
        const int i = base + row;
        const bool valid = i < hi;
        // the output sample, read early (half 0 adds both halves' sums into it)
        double2 o = make_double2(0.0, 0.0);
        if (!h && valid) o = a.wf[i];
        // FP64 prelude: phases (interpolate.cu:626-644) and anchors.  Rows past the
        // unit (and n' past NN, whose B rows are zero) hold finite phasors whose
        // products are discarded or vanish, so nothing is masked.
        const double t = (double)i * a.dt;
        const float tau = (float)((t - t0) * ihs);
        const double sp = (t - pt0) * ipw;
        const double sp1 = 1.0 - sp;
        const double Pr = phase_poly(s.pc + 16, sp, sp1);
        const float2 Er = anchor(Pr);
        const float2 Er2 = fcmul(Er, Er);
        // the epilogue's phasors, ahead of the chunk loop so that their latency is hidden
        const float2 Ep = anchor(phase_poly(s.pc, sp, sp1));
        const float2 Et = a.use_theta ? anchor(phase_poly(s.pc + 8, sp, sp1)) : make_float2(1.f, 0.f);
        for (int k = h; k < nch; k += 2) {
            const int b = sum_stage(k, rg.nas);
            const uint32_t pb = (ro.par >> b) & 1u;
            bool dead = ro.dead || *(volatile int *)&s.fail;
            // the stage is free once the MMAs of its previous fill are done
            if (!dead && ((ro.used >> b) & 1u) && !mbar_wait_bounded(&s.empty[b], pb ^ 1u)) {
                atomicExch(&s.fail, 1);
                dead = true;
            }
            ro.dead = __any_sync(0xffffffffu, dead);
            unsigned char *const aH = smem_raw + b * kAStage, *const aL = aH + kMT * kKC * 2;
            if (!ro.dead) {
                // two interleaved chains (even and odd n') stepping by Er^2: half the
                // dependent depth of one chain, and 8 FP32 steps from the anchor at most
                float2 v[16];
                v[0] = anchor((double)(nlo + 16 * k) * Pr);
                v[1] = fcmul(v[0], Er);
#pragma unroll
                for (int q = 2; q < 16; ++q) v[q] = fcmul(v[q - 2], Er2);
#pragma unroll
                for (int g = 0; g < 4; ++g) {  // 4 groups of 4 complex = 8 bf16 = 16 bytes
                    uint32_t h4[4], l4[4];
#pragma unroll
                    for (int e2 = 0; e2 < 4; ++e2) split2(v[4 * g + e2].x, v[4 * g + e2].y, h4[e2], l4[e2]);
                    const uint32_t off = tile_off(row, 8 * g, kMT / 8);
                    *reinterpret_cast<uint4 *>(aH + off) = make_uint4(h4[0], h4[1], h4[2], h4[3]);
                    *reinterpret_cast<uint4 *>(aL + off) = make_uint4(l4[0], l4[1], l4[2], l4[3]);
                }
            }
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&s.full[b]);
            ro.par ^= 1u << b;
            ro.used |= 1u << b;
        }
        // accumulator of this tile: this thread's row (TMEM lane), half h's column
        // groups; two (m', k') rows of 8 columns per 16-column load, two loads in
        // flight; u_r by one multiplication when m' steps by one
        bool dead = ro.dead || *(volatile int *)&s.fail;
        if (!dead && !mbar_wait_bounded(&s.accf, ro.tiles & 1u)) {
            atomicExch(&s.fail, 1);
            dead = true;
        }
        ro.dead = __any_sync(0xffffffffu, dead);
        tc_fence_after();
        float2 Sp = make_float2(0.f, 0.f), Sq = Sp;  // even and odd rows: two accumulation chains
        if (!ro.dead && g_lo < g_hi) {
            const uint32_t trow = s.tmem + ((uint32_t)(32 * (warp & 3)) << 16);
            float2 uu = make_float2(1.f, 0.f);
            int pm = 0x7fffffff, pk = 0x7fffffff;
            for (int g0 = g_lo; g0 < g_hi; g0 += 2) {
                float D[32];
                tmem_ld16(trow + 16 * g0, D);
                if (g0 + 1 < g_hi) tmem_ld16(trow + 16 * (g0 + 1), D + 16);
                tmem_wait_ld();
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int r = 2 * g0 + q;
                    if (r < R && (q < 2 || g0 + 1 < g_hi)) {
                        const int mm = s.rm[r], kk = s.rk[r];
                        if (kk == pk && mm == pm + 1) {
                            uu = fcmul(uu, Ep);
                        } else {
                            uu = fcpow(Ep, mm);
                            if (kk) uu = fcmul(uu, fcpow(Et, kk));
                        }
                        pm = mm;
                        pk = kk;
                        const float *d8 = D + 8 * q;
                        // Y = sum_c tau^c Z_c (Horner)
                        const float yr = fmaf(fmaf(fmaf(d8[6], tau, d8[4]), tau, d8[2]), tau, d8[0]);
                        const float yi = fmaf(fmaf(fmaf(d8[7], tau, d8[5]), tau, d8[3]), tau, d8[1]);
                        float2 &S = (q & 1) ? Sq : Sp;
                        S.x = fmaf(uu.x, yr, fmaf(-uu.y, yi, S.x));
                        S.y = fmaf(uu.x, yi, fmaf(uu.y, yr, S.y));
                    }
                }
            }
            Sp.x += Sq.x;
            Sp.y += Sq.y;
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&s.acce);
        if (h) s.part[ro.tiles & 1u][row] = Sp;
        sum_prod_sync();
        if (!h && valid && !ro.dead) {
            const float2 o2 = s.part[ro.tiles & 1u][row];
            o.x += (double)(Sp.x + o2.x);
            o.y += (double)(Sp.y + o2.y);
            a.wf[i] = o;
        }
        ro.tiles++;
    }
}

__global__ void __launch_bounds__(kSumThreads, 2) k_sum_mixed(MixedArgs a, SumRing rg)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ SumShared s;
    SumRole ro;
    sum_setup(s, a.tmem_cols, ro);
    const int u = blockIdx.x;
    const int seg = a.units[3 * u], lo = a.units[3 * u + 1], hi = a.units[3 * u + 2];
    if ((int)(threadIdx.x >> 5) == kSumProd) {
        if ((threadIdx.x & 31) == 0) sum_mma_unit(a, seg, lo, hi, smem_raw, rg, s, ro);
        __syncwarp();
    } else {
        sum_prod_unit(a, seg, lo, hi, smem_raw, rg, s, ro);
    }
    sum_teardown(s, ro, rg, a.tmem_cols, a.err);
}

// Persistent form over many waveforms: TMEM and the mbarriers are set up once
// per CTA; units {waveform, segment, first, end} are taken in stride.  The B
// slots keep the size of the largest chunk (max_NB) for every unit, so that a
// unit with a wider B never writes where the previous unit's MMAs may still
// read.
__global__ void __launch_bounds__(kSumThreads, 2) k_sum_mixed_batched(const few_wave_desc *__restrict__ descs,
                                                                      const int *__restrict__ units4, int nunits,
                                                                      SumRing rg, int tmem_cols, int *err,
                                                                      unsigned long long *__restrict__ done)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ SumShared s;
    SumRole ro;
    sum_setup(s, tmem_cols, ro);
    const bool mma = (int)(threadIdx.x >> 5) == kSumProd;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const few_wave_desc d = descs[units4[4 * u]];
        MixedArgs a;
        a.wf = (double2 *)d.wf;
        a.Bpk = (const __nv_bfloat16 *)d.Bpk;
        a.pc = d.phase_coeffs;
        a.seg_info = d.seg_info;
        a.t_knots = d.t_knots;
        a.units = nullptr;
        a.row_m = d.row_m;
        a.row_k = d.row_k;
        a.err = err;
        a.N = d.N;
        a.R = d.R;
        a.nlo = d.nlo;
        a.NN = d.NN;
        a.use_theta = d.use_theta;
        a.dt = d.dt;
        a.tmem_cols = tmem_cols;
        mixed_dims_core(d.R, d.NN, a.NNp, a.NB, a.nchunks);
        const int seg = units4[4 * u + 1], lo = units4[4 * u + 2], hi = units4[4 * u + 3];
        if (mma) {
            if ((threadIdx.x & 31) == 0 && !ro.dead) sum_mma_unit(a, seg, lo, hi, smem_raw, rg, s, ro);
        } else {
            sum_prod_unit(a, seg, lo, hi, smem_raw, rg, s, ro);
            if (done) {
                sum_prod_sync();  // every output row of the unit written
                if (threadIdx.x == 0 && !ro.dead) atomicMax(done + units4[4 * u], global_ns());  // unit complete
            }
        }
    }
    if (mma) __syncwarp();
    sum_teardown(s, ro, rg, tmem_cols, err);
}

}  // namespace

// Tensor-core shapes of an R x NN fold grid.
int mixed_dims(int R, int NN, int *NNp, int *NB, int *nchunks, int *tmem_cols)
{
    if (R > 64) return fail(FEW_ERR_SIZE, "mixed form: %d (m, k) rows exceed the 64 the accumulator holds", R);
    mixed_dims_core(R, NN, *NNp, *NB, *nchunks);
    int cols = 32;
    while (cols < *NB) cols <<= 1;
    *tmem_cols = cols;
    return FEW_OK;
}

// Ring shape of the sum for chunks of NB columns.  By default one A stage per
// producer half and as many B slots (2..4) as keep two CTAs per SM (<=
// kTwoCtaBytes of dynamic shared memory): at the one-year 3843-mode workload this
// measured 0.75 ms against 0.77 ms for two A stages per half with two B slots,
// and the autotuner's search over both agrees.  nas, nbs > 0 ask for a shape.
constexpr int kTwoCtaBytes = 112 * 1024;
size_t mixed_smem_bytes(const SumRing &rg) { return (size_t)2 * rg.nas * kAStage + (size_t)rg.nbs * rg.bslot; }
SumRing mixed_ring(int NB, int nbs = 0, int nas = 0)
{
    SumRing rg;
    rg.bslot = 2 * NB * kKC * 2;
    rg.nas = nas > 0 ? nas : 1;
    rg.nbs = nbs > 0 ? nbs
                     : std::max(2, std::min(kMaxBSlots, (kTwoCtaBytes - 2 * rg.nas * kAStage) / rg.bslot));
    return rg;
}

size_t mixed_bpk_bytes(int nseg, int R, int NN)
{
    int NNp, NB, nch, cols;
    if (mixed_dims(R, NN, &NNp, &NB, &nch, &cols)) return 0;
    return (size_t)nseg * nch * 2 * NB * kKC * sizeof(__nv_bfloat16);
}

int launch_fold_mixed(const double2 *W, const double *t_knots, int nseg, int R, int NN, void *Bpk,
                      cudaStream_t st)
{
    int NNp, NB, nch, cols;
    int rc = mixed_dims(R, NN, &NNp, &NB, &nch, &cols);
    if (rc) return rc;
    const long long total = (long long)nseg * nch * (kKC / 8) * NB;
    if (total == 0) return FEW_OK;
    const int threads = 256;
    k_fold_mixed<<<(unsigned)((total + threads - 1) / threads), threads, 0, st>>>(W, t_knots, nseg, R, NN, NB, nch,
                                                                                 (__nv_bfloat16 *)Bpk);
    FEW_LAUNCH_CHECK("k_fold_mixed");
    return FEW_OK;
}

int launch_sum_mixed(double2 *wf, const void *Bpk, const double *pc, int N, const double *seg_info,
                     const double *t_knots, const int *units, int nunits, const int *row_m, const int *row_k, int R,
                     int nlo, int NN, double dt, int use_theta, int *err, cudaStream_t st)
{
    if (nunits == 0) return FEW_OK;
    MixedArgs a;
    int rc = mixed_dims(R, NN, &a.NNp, &a.NB, &a.nchunks, &a.tmem_cols);
    if (rc) return rc;
    a.wf = wf;
    a.Bpk = (const __nv_bfloat16 *)Bpk;
    a.pc = pc;
    a.seg_info = seg_info;
    a.t_knots = t_knots;
    a.units = units;
    a.row_m = row_m;
    a.row_k = row_k;
    a.err = err;
    a.N = N;
    a.R = R;
    a.nlo = nlo;
    a.NN = NN;
    a.use_theta = use_theta;
    a.dt = dt;
    const SumRing rg = mixed_ring(a.NB);
    const size_t smem = mixed_smem_bytes(rg);
    FEW_CUDA_TRY(ensure_smem_attr((const void *)k_sum_mixed, (int)smem));
    k_sum_mixed<<<nunits, kSumThreads, smem, st>>>(a, rg);
    FEW_LAUNCH_CHECK("k_sum_mixed");
    return FEW_OK;
}

int launch_sum_mixed_batched(const few_wave_desc *descs, const int *units4, int nunits, int max_R, int ctas,
                             int astages, int bstages, int *err, unsigned long long *done, cudaStream_t st)
{
    if (nunits == 0) return FEW_OK;
    int NNp, NB, nch, cols;
    int rc = mixed_dims(max_R, 32, &NNp, &NB, &nch, &cols);
    if (rc) return rc;
    if (ctas <= 0) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        ctas = 2 * sms;
    }
    ctas = std::min(ctas, nunits);
    const SumRing rg = mixed_ring(NB, bstages, astages);
    const size_t smem = mixed_smem_bytes(rg);
    if (smem > 220 * 1024)
        return fail(FEW_ERR_SIZE, "few_sum_mixed_batched: %d A stages per half and %d B stages of %d bytes exceed "
                    "shared memory", rg.nas, rg.nbs, rg.bslot);
    FEW_CUDA_TRY(ensure_smem_attr((const void *)k_sum_mixed_batched, (int)smem));
    k_sum_mixed_batched<<<ctas, kSumThreads, smem, st>>>(descs, units4, nunits, rg, cols, err, done);
    FEW_LAUNCH_CHECK("k_sum_mixed_batched");
    return FEW_OK;
}

}  // namespace few

extern "C" int few_sum_mixed_batched(const few_wave_desc *descs, int nwave, const int *units4, int nunits, int max_R,
                                     int ctas, int astages, int bstages, int *err, unsigned long long *done,
                                     void *stream)
{
    few::clear_error();
    if (!descs || !units4 || !err) return few::fail(FEW_ERR_ARG, "few_sum_mixed_batched: null pointer");
    if (nwave < 1 || nunits < 0 || max_R < 1 || max_R > 64)
        return few::fail(FEW_ERR_SIZE, "few_sum_mixed_batched: bad sizes (max_R <= 64)");
    if (bstages != 0 && (bstages < 2 || bstages > few::kMaxBStages))
        return few::fail(FEW_ERR_ARG, "few_sum_mixed_batched: bstages=%d not in 2..%d", bstages, few::kMaxBStages);
    if (astages != 0 && astages != 1 && astages != 2)
        return few::fail(FEW_ERR_ARG, "few_sum_mixed_batched: astages=%d not 1 or 2", astages);
    return few::launch_sum_mixed_batched(descs, units4, nunits, max_R, ctas, astages, bstages, err, done,
                                         (cudaStream_t)stream);
}

extern "C" int few_fold_mixed(const void *W, const double *t_knots, int nseg, int R, int NN, void *Bpk, void *stream)
{
    few::clear_error();
    if (!W || !t_knots || !Bpk) return few::fail(FEW_ERR_ARG, "few_fold_mixed: null pointer");
    if (nseg < 0 || R < 1 || NN < 1) return few::fail(FEW_ERR_SIZE, "few_fold_mixed: bad sizes");
    return few::launch_fold_mixed((const double2 *)W, t_knots, nseg, R, NN, Bpk, (cudaStream_t)stream);
}

extern "C" long long few_mixed_operand_bytes(int nseg, int R, int NN)
{
    return (long long)few::mixed_bpk_bytes(nseg, R, NN);
}

extern "C" int few_sum_mixed(void *wf, const void *Bpk, const double *phase_coeffs, int N, const double *seg_info,
                             const double *t_knots, const int *units, int nunits, const int *row_m, const int *row_k,
                             int R, int nlo, int NN, double dt, int use_theta, int *err, void *stream)
{
    few::clear_error();
    if (!wf || !Bpk || !phase_coeffs || !seg_info || !t_knots || !units || !row_m || !row_k || !err)
        return few::fail(FEW_ERR_ARG, "few_sum_mixed: null pointer");
    if (N < 2 || nunits < 0 || R < 1 || R > 64 || NN < 1)
        return few::fail(FEW_ERR_SIZE, "few_sum_mixed: bad sizes (R <= 64)");
    return few::launch_sum_mixed((double2 *)wf, Bpk, phase_coeffs, N, seg_info, t_knots, units, nunits, row_m, row_k,
                                 R, nlo, NN, dt, use_theta, err, (cudaStream_t)stream);
}

