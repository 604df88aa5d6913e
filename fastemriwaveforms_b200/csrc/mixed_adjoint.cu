// Amplitude adjoint of the mixed-precision mode sum on the tcgen05 tensor
// cores, in exact integer arithmetic.
//
// Per knot segment s the gradient of L = Re sum_i g_i h_i with respect to the
// folded coefficients is the contraction over the segment's samples
//     G[r][n'][c] = sum_i tau_i^c v_{n'}(t_i) g_i u_r(t_i)
// (then scaled by h_s^c, since x^c = h_s^c tau^c), the same array the FP64
// kernel k_adj_G produces, so the unfold and the spline adjoint that follow are
// shared.  The power of tau is split between the operands, c = c_a + c_b with
// c_a in {0, 1} and c_b in {0, 2}, so each phasor is generated once per sample:
//     D[(c_a, n')][(c_b, r, re/im)] += sum_{(i, part)} A[(c_a, n')][(i, part)] B[(i, part)][(c_b, r, re/im)]
// with A = tau^c_a (Re v, Im v) and B = tau^c_b g (Re u, Im u | -Im u, Re u) for
// part 0 | 1 (the product (v)(g u) written out in real arithmetic).
//
// Precision: the phasors, g and the powers of tau are formed in FP64 (one
// FP64 sincos per phase and sample, FP64 recurrences), then every operand
// value x is scaled to an integer Y = rint(x S) with |Y| <= 127 2^24 and
// written as four signed base-256 digits (int8 planes 0..3, most significant
// first); A's scale is fixed (|A| <= 1), B's is set per block of 1024
// samples from the block's largest |g|.  The integer tensor core
// (kind::i8, s32 accumulation) multiplies digit planes i and j into the
// accumulator of level i + j (levels 0..3, ten products per K step); the
// int32 sums are exact (no rounding anywhere in the contraction), and the
// dropped levels >= 4 weigh below 2^-31 of the operands' scales.  After each
// block the four levels are combined in FP64 and added into G.  The result
// differs from the FP64 kernel only by the 2^-32 representation of the
// operands, so its gradients carry FP64-level accuracy.
//
// Shape: M = 2 x 64 n' rows per CTA (one CTA per 64 n' columns), N = (c_b, r,
// re/im) with 2R padded to 16 (both c_b per CTA while they fit one level
// accumulator of 128 TMEM columns; the four levels fill the 512 columns).  The samples are K: one CTA of 8
// warps owns one segment and loops over its samples in tiles of 32 (K = 64,
// two MMA K steps): lane = sample, and the warps share the tile's operand
// groups (16 n' of A for one c_a, or 8 rows r of B for both c_b, each written
// as whole 16-byte MN chunks, in the MN-major no-swizzle layout: core
// matrix = 8 K rows x 16 bytes, K groups 128 B apart, MN groups 1024 B apart),
// 12 warps so that every group of a tile has its own warp.  The FP64 prelude
// (phasors, tau, g) is computed once per sample, for 12 tiles at a time, into
// shared memory.  Two
// operand buffers: while the tensor core consumes tile k, the warps build tile
// k+1.  Every wait is bounded; a timeout sets the error word, drains and
// frees TMEM.
#include "few_common.cuh"
#include "few_internal.h"
#include "few_tc.cuh"

namespace few {

namespace {

constexpr int kGT = 32;              // samples per tile; K = 64 (sample x {Re, Im})
constexpr int kProd = 11;            // operand-producing warps (8 A groups + 3 B groups at R <= 24)
constexpr int kGThreads = 32 * (kProd + 1);  // + one warp that issues the MMAs
constexpr int kProdThreads = 32 * kProd;
constexpr int kGPre = kProd;         // tiles per prelude batch (one sample per producer thread)
constexpr int kStages = 2;           // operand ring
constexpr int kGFlush = 32;          // tiles per block: one B scale, int32 sums well inside 2^31
constexpr int kDigits = 4;           // base-256 digits per operand value
constexpr int kPlaneA = 8 * 1024;    // one A digit plane: 8 MN groups (2 x 64 n') x 8 K groups x 128 B
constexpr uint32_t kLBO = 128;       // K-group stride (bytes)
constexpr uint32_t kSBO = 1024;      // MN-group stride (bytes)
constexpr double kScaleA = kDigitScale;  // |A| <= 1 -> |Y| <= 127 2^24
constexpr int kLevelCols = 128;      // TMEM columns per level accumulator (N <= 128)

// Byte offset of (mn, k) in an MN-major, no-swizzle int8 tile of K = 64.
__device__ __forceinline__ uint32_t mn_off8(int mn, int k)
{
    return (uint32_t)((mn >> 4) * kSBO + (k >> 3) * kLBO + (k & 7) * 16 + (mn & 15));
}

// Per-sample values every operand group needs (FP64).
struct GPrelude {
    double2 v0;    // v_{n'} at this CTA's first n'
    double2 Er, Er8, Ep, Et;
    double2 g;     // conj of torch's upstream gradient
    double tau;
};

// Digits of four values: word[d] of digit plane d.
__device__ __forceinline__ void digit_words(const double *x, double scale, uint32_t *w)
{
    digit_words8(scaled_biased(x[0], scale), scaled_biased(x[1], scale), scaled_biased(x[2], scale),
                 scaled_biased(x[3], scale), w);
}

// Producer-only named barrier (the MMA warp does not take part).
__device__ __forceinline__ void producers_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kProdThreads) : "memory"); }


struct AdjGMixedArgs {
    const double2 *grad;   // torch upstream gradient G; g = conj(G)
    const double *pc;      // (8, N-1, 3)
    const double *seg_info;
    const double *t_knots;
    const int *seg_start;  // (nseg + 1,)
    const int *row_m;
    const int *row_k;
    double2 *G;            // (nseg, R, NN, 4)
    int *err;
    int N, R, nlo, NN, CB, ncb, NB, use_theta, tmem_cols;
    double dt;
};

// One operand group of one tile, written by a warp (lane = sample): group
// gi < nA is (16 n' block, c_a) of A, the others 8 rows r of B for both c_b.
__device__ __forceinline__ void g_group(const AdjGMixedArgs &a, int gi, int nA, int nrow0, int cbz, int lane,
                                        const GPrelude &pr, double scaleB, const int *s_rm, const int *s_rk,
                                        unsigned char *aBuf, unsigned char *bBuf)
{
    const int R = a.R, NN = a.NN, CB = a.CB, ncb = a.ncb;
    const int planeB = a.NB * 64;
    const int k0 = 16 * (lane >> 3) + (lane & 7);  // K row of part 0 (part 1: +8)
    if (gi < nA) {
        // A: tau^c_a v_{n'} for 16 n' and one c_a (MN 64 c_a + 16 blk ..): whole
        // 16-byte MN chunks for both parts
        const int blk = gi >> 1, ca = gi & 1;
        const int n0 = nrow0 + 16 * blk;
        double2 v = cmul(pr.v0, cpow_int(pr.Er8, 2 * blk));
        const double f = ca ? pr.tau : 1.0;
        uint32_t w[2][kDigits][4];  // [part][digit][word]
#pragma unroll
        for (int qb = 0; qb < 4; ++qb) {
            double re[4], im[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const bool ok = n0 + 4 * qb + e < NN;
                re[e] = ok ? f * v.x : 0.0;
                im[e] = ok ? f * v.y : 0.0;
                v = cmul(v, pr.Er);
            }
            uint32_t t4[kDigits];
            digit_words(re, kScaleA, t4);
#pragma unroll
            for (int p = 0; p < kDigits; ++p) w[0][p][qb] = t4[p];
            digit_words(im, kScaleA, t4);
#pragma unroll
            for (int p = 0; p < kDigits; ++p) w[1][p][qb] = t4[p];
        }
        const int mn = 64 * ca + 16 * blk;
#pragma unroll
        for (int p = 0; p < kDigits; ++p) {
            unsigned char *plane = aBuf + p * kPlaneA;
            *reinterpret_cast<uint4 *>(plane + mn_off8(mn, k0)) =
                make_uint4(w[0][p][0], w[0][p][1], w[0][p][2], w[0][p][3]);
            *reinterpret_cast<uint4 *>(plane + mn_off8(mn, k0 + 8)) =
                make_uint4(w[1][p][0], w[1][p][1], w[1][p][2], w[1][p][3]);
        }
        return;
    }
    // B: tau^c_b g u_r for 8 rows r, each c_b of the CTA
    const int rg = gi - nA;
    double2 u8[8];
    double2 uu = make_double2(1.0, 0.0);
    int pm = 0x7fffffff, pk = 0x7fffffff;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int r = 8 * rg + e;
        u8[e] = make_double2(0.0, 0.0);
        if (r < R) {
            const int mm = s_rm[r], kk = s_rk[r];
            if (kk == pk && mm == pm + 1) {
                uu = cmul(uu, pr.Ep);
            } else {
                uu = cpow_int(pr.Ep, mm);
                if (kk) uu = cmul(uu, cpow_int(pr.Et, kk));
            }
            pm = mm;
            pk = kk;
            u8[e] = uu;
        }
    }
    const double t2 = pr.tau * pr.tau;
    double2 gc = pr.g;
    if (cbz) gc = make_double2(gc.x * t2, gc.y * t2);
    for (int cl = 0; cl < ncb; ++cl) {
        uint32_t w0[kDigits][4], w1[kDigits][4];
#pragma unroll
        for (int qb = 0; qb < 4; ++qb) {  // rows 2 qb, 2 qb + 1
            const double2 wa = cmul(gc, u8[2 * qb]), wb = cmul(gc, u8[2 * qb + 1]);
            const uint32_t ra = scaled_biased(wa.x, scaleB), ia = scaled_biased(wa.y, scaleB);
            const uint32_t rb = scaled_biased(wb.x, scaleB), ib = scaled_biased(wb.y, scaleB);
            uint32_t t4[kDigits];
            // part 0 (Re v): (Re w, Im w); part 1 (Im v): (-Im w, Re w)
            digit_words8(ra, ia, rb, ib, t4);
#pragma unroll
            for (int p = 0; p < kDigits; ++p) w0[p][qb] = t4[p];
            digit_words8(negated_biased(ia), ra, negated_biased(ib), rb, t4);
#pragma unroll
            for (int p = 0; p < kDigits; ++p) w1[p][qb] = t4[p];
        }
        const int mn = cl * CB + 16 * rg;
#pragma unroll
        for (int p = 0; p < kDigits; ++p) {
            unsigned char *plane = bBuf + p * planeB;
            *reinterpret_cast<uint4 *>(plane + mn_off8(mn, k0)) = make_uint4(w0[p][0], w0[p][1], w0[p][2], w0[p][3]);
            *reinterpret_cast<uint4 *>(plane + mn_off8(mn, k0 + 8)) =
                make_uint4(w1[p][0], w1[p][1], w1[p][2], w1[p][3]);
        }
        gc = make_double2(gc.x * t2, gc.y * t2);
    }
}

__global__ void __launch_bounds__(kGThreads, 1) k_adj_G_mixed(AdjGMixedArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t s_full[kStages], s_empty[kStages], s_accf, s_acce, s_done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_rm[kMaxRows], s_rk[kMaxRows];
    __shared__ double s_pc[24];
    __shared__ GPrelude s_pre[kProdThreads];
    __shared__ double s_gmax[kProd];
    __shared__ double s_scaleB;
    __shared__ int s_fail;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int seg = blockIdx.x;
    const int nrow0 = 64 * blockIdx.y;   // first n' index of this CTA
    const int cbz = 2 * blockIdx.z;      // c_b of this CTA's first column block (0 or 2)
    const int R = a.R, NN = a.NN, NB = a.NB, CB = a.CB, ncb = a.ncb;
    const int lo = a.seg_start[seg], hi = a.seg_start[seg + 1];
    const double t0 = a.seg_info[3 * seg], pt0 = a.seg_info[3 * seg + 1], pw = a.seg_info[3 * seg + 2];
    const double hs = a.t_knots[seg + 1] - a.t_knots[seg];
    const long long nps = (long long)(a.N - 1) * 3;
    const int nA = 2 * ((min(64, NN - nrow0) + 15) >> 4);  // A groups: (16 n' block, c_a)
    const int ngroups = nA + (CB >> 4);                     // + B groups of 8 rows r (all c_b of the CTA)
    const int ntiles = (hi - lo + kGT - 1) / kGT;

    if (lo >= hi) {  // a segment without samples: zero gradient for this CTA's (n', c)
        for (int e = tid; e < R * 64 * 2 * ncb; e += blockDim.x) {
            const int r = e / (64 * 2 * ncb), rem = e - r * 64 * 2 * ncb;
            const int n = nrow0 + rem / (2 * ncb), q = rem % (2 * ncb);
            const int c = (q & 1) + cbz + 2 * (q >> 1);
            if (n < NN) a.G[(((long long)seg * R + r) * NN + n) * 4 + c] = make_double2(0.0, 0.0);
        }
        return;
    }

    for (int r = tid; r < R; r += blockDim.x) {
        s_rm[r] = a.row_m[r];
        s_rk[r] = a.row_k[r];
    }
    if (tid < 24) {
        const int q = tid >> 3, c = tid & 7;
        s_pc[tid] = a.pc[c * nps + (long long)seg * 3 + q];
    }
    // operand ring starts at zero: rows of A past NN and columns of B past
    // ncb * CB are never written
    const int planeB = NB * 64;                          // one B digit plane: NB/16 MN groups x 1024 B
    const int bufA = kDigits * kPlaneA, bufB = kDigits * planeB;
    for (int q = tid; q < kStages * (bufA + bufB) / 16; q += blockDim.x)
        reinterpret_cast<uint4 *>(smem_raw)[q] = make_uint4(0u, 0u, 0u, 0u);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"((uint32_t)a.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int q = 0; q < kStages; ++q) {
            mbar_init(&s_full[q], kProd);
            mbar_init(&s_empty[q], 1);
        }
        mbar_init(&s_accf, 1);
        mbar_init(&s_acce, kProd);
        mbar_init(&s_done, 1);
        s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    bool drained = true;

    if (warp == kProd) {
        // ---- MMA warp: one thread issues every tile's MMAs once its operands are in
        if (lane == 0) {
            const uint32_t idesc = idesc_s8_mn(128, NB);
            bool ok = true;
            for (int it = 0; it < ntiles && ok; ++it) {
                const int st = it % kStages;
                if (it % kGFlush == 0 && it > 0)  // the previous block's accumulators were read
                    ok = mbar_wait_bounded(&s_acce, (uint32_t)((it / kGFlush - 1) & 1));
                if (ok) ok = mbar_wait_bounded(&s_full[st], (uint32_t)((it / kStages) & 1));
                if (!ok) break;
                tc_fence_after();
                const uint32_t a0 = smem_u32(smem_raw + st * (bufA + bufB)), b0 = a0 + bufA;
                const bool fresh = (it % kGFlush) == 0;
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {  // K steps of 32 = K groups 4 ks .. 4 ks + 3
                    const uint32_t ko = ks * 4 * kLBO;
#pragma unroll
                    for (int lv = 0; lv < kDigits; ++lv) {
#pragma unroll
                        for (int i = 0; i <= lv; ++i) {
                            const uint64_t da = smem_desc(a0 + i * kPlaneA + ko, kLBO, kSBO);
                            const uint64_t db = smem_desc(b0 + (lv - i) * planeB + ko, kLBO, kSBO);
                            mma_s8(tmem + (uint32_t)(lv * kLevelCols), da, db, idesc,
                                   (fresh && ks == 0 && i == 0) ? 0u : 1u);
                        }
                    }
                }
                mma_commit(&s_empty[st]);
                if (it % kGFlush == kGFlush - 1 || it == ntiles - 1) mma_commit(&s_accf);
            }
            if (!ok) atomicExch(&s_fail, 1);
            // every MMA issued so far complete before TMEM may be freed
            mma_commit(&s_done);
            drained = mbar_wait_bounded(&s_done, 0);
        }
        __syncwarp();
    } else {
        // ---- producer warps: operands of every tile into the ring, rotating the
        // groups over the warps (each warp does every group once per prelude batch).
        // Every producer runs all ntiles iterations and reaches every named
        // barrier; after a failed (timed-out) wait a warp only skips the work.
        double scaleB = 1.0;
        bool dead = false;
        for (int it = 0; it < ntiles; ++it) {
            const int base = lo + it * kGT;
            const int st = it % kStages;
            if (it % kGFlush == 0) {
                // B's scale for this block: its largest |g|
                double gm = 0.0;
                for (int i = base + tid; i < min(hi, base + kGFlush * kGT); i += kProdThreads) {
                    const double2 Gt = a.grad[i];
                    gm = fmax(gm, sqrt(Gt.x * Gt.x + Gt.y * Gt.y));
                }
                for (int off = 16; off > 0; off >>= 1) gm = fmax(gm, __shfl_xor_sync(0xffffffffu, gm, off));
                if (lane == 0) s_gmax[warp] = gm;
                producers_sync();
                if (tid == 0) {
                    double m = s_gmax[0];
                    for (int w = 1; w < kProd; ++w) m = fmax(m, s_gmax[w]);
                    // |B| <= |g| (|u| = 1, tau <= 1); a hair of headroom for the FP64 rounding of g u
                    s_scaleB = m > 0.0 ? kScaleA / (m * (1.0 + 1e-12)) : 1.0;
                }
                producers_sync();
                scaleB = s_scaleB;
            }
            if (it % kGPre == 0) {
                // FP64 prelude for this thread's sample of the next kGPre tiles
                // (phases as interpolate.cu:626-644, phasors by FP64 sincos)
                producers_sync();  // every producer is done with the previous batch
                const int i = base + tid;
                const double t = (double)i * a.dt;
                const double s = (t - pt0) / pw;
                const double s1 = 1.0 - s;
                GPrelude pr;
                double sn, cs;
                sincos_reduced(phase_poly(s_pc + 16, s, s1), &sn, &cs);
                pr.Er = make_double2(cs, -sn);
                sincos_reduced(phase_poly(s_pc, s, s1), &sn, &cs);
                pr.Ep = make_double2(cs, -sn);
                if (a.use_theta) {
                    sincos_reduced(phase_poly(s_pc + 8, s, s1), &sn, &cs);
                    pr.Et = make_double2(cs, -sn);
                } else {
                    pr.Et = make_double2(1.0, 0.0);
                }
                pr.v0 = cpow_int(pr.Er, a.nlo + nrow0);
                double2 e8 = cmul(pr.Er, pr.Er);
                e8 = cmul(e8, e8);
                pr.Er8 = cmul(e8, e8);
                pr.tau = (t - t0) / hs;
                pr.g = make_double2(0.0, 0.0);
                if (i < hi) {
                    const double2 Gt = a.grad[i];
                    pr.g = make_double2(Gt.x, -Gt.y);
                }
                s_pre[tid] = pr;
                producers_sync();
            }
            dead = dead || *(volatile int *)&s_fail;
            // the ring stage is free once the MMAs of tile it - kStages are done
            if (!dead && it >= kStages && !mbar_wait_bounded(&s_empty[st], (uint32_t)((it / kStages - 1) & 1))) {
                atomicExch(&s_fail, 1);
                dead = true;
            }
            if (!dead) {
                const GPrelude &pr = s_pre[(it % kGPre) * kGT + lane];
                unsigned char *const aBuf = smem_raw + st * (bufA + bufB);
                for (int gi = (warp + it) % kProd; gi < ngroups; gi += kProd)
                    g_group(a, gi, nA, nrow0, cbz, lane, pr, scaleB, s_rm, s_rk, aBuf, aBuf + bufA);
            }
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&s_full[st]);
            if (it % kGFlush == kGFlush - 1 || it == ntiles - 1) {
                // block done: the four levels combined in FP64 (row (c_a, n'),
                // column (c_b, r, re/im)) and added into G (stored by the first
                // block); the MMA warp restarts the accumulators after every
                // producer warp has arrived on s_acce.  A warp reads the TMEM lanes
                // of its quarter (warp % 4); the warps of a quarter share its columns.
                if (!dead && !mbar_wait_bounded(&s_accf, (uint32_t)((it / kGFlush) & 1))) {
                    atomicExch(&s_fail, 1);
                    dead = true;
                }
                tc_fence_after();
                const bool first = it < kGFlush;
                const double unit = 1.0 / (kScaleA * scaleB) * 281474976710656.0;  // 2^48 / (S_A S_B)
                const int quad = warp & 3;
                const int nq = (kProd - 1 - quad) / 4 + 1;  // producer warps in this quarter
                const int row = 32 * quad + lane;
                const int ca = row >> 6, n = nrow0 + (row & 63);
                const uint32_t trow = tmem + ((uint32_t)(quad * 32) << 16);
                for (int j16 = warp >> 2; j16 < NB / 16 && !dead; j16 += nq) {
                    double acc[16];
#pragma unroll
                    for (int e = 0; e < 16; ++e) acc[e] = 0.0;
                    double wl = unit;
#pragma unroll
                    for (int lv = 0; lv < kDigits; ++lv) {
                        float D[16];
                        tmem_ld16(trow + (uint32_t)(lv * kLevelCols + 16 * j16), D);
                        tmem_wait_ld();
#pragma unroll
                        for (int e = 0; e < 16; ++e) acc[e] = fma((double)__float_as_int(D[e]), wl, acc[e]);
                        wl *= 0.00390625;  // 2^-8 per level
                    }
                    if (n < NN) {
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            const int col = 16 * j16 + 2 * e;
                            const int cl = col / CB, r = (col - cl * CB) >> 1;
                            if (cl < ncb && r < R) {
                                const int c = ca + cbz + 2 * cl;
                                const double hc = c == 0 ? 1.0 : (c == 1 ? hs : (c == 2 ? hs * hs : hs * hs * hs));
                                double2 *gp = a.G + (((long long)seg * R + r) * NN + n) * 4 + c;
                                double2 v = make_double2(acc[2 * e] * hc, acc[2 * e + 1] * hc);
                                if (!first) {
                                    const double2 o = *gp;
                                    v.x += o.x;
                                    v.y += o.y;
                                }
                                *gp = v;
                            }
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&s_acce);
            }
        }
    }
    // teardown: TMEM is freed only when every MMA is known to be complete
    tc_fence_before();
    const bool all_drained = __syncthreads_and(drained) != 0;
    if ((s_fail || !all_drained) && tid == 0) atomicExch(a.err, 1);
    if (all_drained && warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)a.tmem_cols)
                     : "memory");
    }
}

}  // namespace

int launch_adj_G_mixed(const double2 *grad, const double *pc, int N, const double *seg_info, const double *t_knots,
                       const int *seg_start, int nseg, const int *row_m, const int *row_k, int R, int nlo, int NN,
                       double dt, int use_theta, double2 *G, int *err, cudaStream_t st)
{
    if (nseg == 0) return FEW_OK;
    AdjGMixedArgs a;
    a.CB = (2 * R + 15) / 16 * 16;  // columns per c_b: (r, re/im), padded to 16
    // four level accumulators of kLevelCols columns each fill the 512 TMEM columns
    a.ncb = 2 * a.CB <= kLevelCols ? 2 : 1;
    if (a.ncb * a.CB > kLevelCols)
        return fail(FEW_ERR_SIZE, "few_adjoint_G_mixed: %d rows exceed the 64 the accumulators hold", R);
    a.NB = a.ncb * a.CB;
    a.grad = grad;
    a.pc = pc;
    a.seg_info = seg_info;
    a.t_knots = t_knots;
    a.seg_start = seg_start;
    a.row_m = row_m;
    a.row_k = row_k;
    a.G = G;
    a.err = err;
    a.N = N;
    a.R = R;
    a.nlo = nlo;
    a.NN = NN;
    a.use_theta = use_theta;
    a.dt = dt;
    a.tmem_cols = 512;
    const size_t smem = (size_t)kStages * (kDigits * kPlaneA + kDigits * a.NB * 64);
    FEW_CUDA_TRY(ensure_smem_attr((const void *)k_adj_G_mixed, (int)smem));
    dim3 grid(nseg, (NN + 63) / 64, 2 / a.ncb);
    k_adj_G_mixed<<<grid, kGThreads, smem, st>>>(a);
    FEW_LAUNCH_CHECK("k_adj_G_mixed");
    return FEW_OK;
}

}  // namespace few

extern "C" int few_adjoint_G_mixed(const void *grad, const double *phase_coeffs, int N, const double *seg_info,
                                   const double *t_knots, const int *seg_start, int nseg, const int *row_m,
                                   const int *row_k, int R, int nlo, int NN, double dt, int use_theta, void *G, int *err,
                                   void *stream)
{
    few::clear_error();
    if (!grad || !phase_coeffs || !seg_info || !t_knots || !seg_start || !row_m || !row_k || !G || !err)
        return few::fail(FEW_ERR_ARG, "few_adjoint_G_mixed: null pointer");
    if (N < 2 || nseg < 0 || nseg > N - 1 || R < 1 || R > 64 || NN < 1 || NN > 65535 * 64)
        return few::fail(FEW_ERR_SIZE, "few_adjoint_G_mixed: bad sizes (R <= 64)");
    return few::launch_adj_G_mixed((const double2 *)grad, phase_coeffs, N, seg_info, t_knots, seg_start, nseg, row_m,
                                   row_k, R, nlo, NN, dt, use_theta, (double2 *)G, err, (cudaStream_t)stream);
}
