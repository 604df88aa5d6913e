// Amplitude adjoint of the mixed-precision mode sum on the tcgen05 tensor cores.
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
// part 0 | 1 (the product (v)(g u) written out in real arithmetic).  M = 2 x 64
// n' rows per CTA (one CTA per 64 n' columns), N = (c_b, r, re/im) with 2R
// padded to 8 (both c_b per CTA while N <= 256).  The samples are K: one CTA of
// 8 warps owns one segment and loops over its samples in tiles of 32 (K = 64):
// lane = sample, and the warps share the tile's operand groups (8 n' of A or 4
// rows r of B, each written as 16-byte chunks of the MN-major no-swizzle layout:
// core matrix = 8 K rows x 16 bytes, K groups 128 B apart, MN groups 1024 B
// apart).  The FP64 phase prelude (phases, anchors, tau, g) is computed once per
// sample, for 8 tiles at a time, into shared memory.  Operands are split into
// bf16 hi + lo planes (three products hi*hi + hi*lo + lo*hi); FP32 accumulation
// in TMEM over at most 1024 samples, then the accumulator is added into G in
// FP64 and restarted, which keeps the FP32 rounding of long, oscillating
// (cancelling) sums small.  Two operand buffers: while the tensor core consumes
// tile k, the warps build tile k+1.  Every wait is bounded; a timeout sets the
// error word, drains and frees TMEM.
#include "few_common.cuh"
#include "few_internal.h"
#include "few_tc.cuh"

namespace few {

namespace {

constexpr int kGT = 32;            // samples per tile; K = 64 (sample x {Re, Im})
constexpr int kGThreads = 256;     // 8 warps
constexpr int kGPre = 8;           // tiles per prelude batch (kGPre * kGT = kGThreads samples)
constexpr int kGPlaneA = 16 * 1024;  // one A plane: 16 MN groups (2 x 64 n') x 8 K groups x 128 B
constexpr uint32_t kLBO = 128;     // K-group stride (bytes)
constexpr uint32_t kSBO = 1024;    // MN-group stride (bytes)
constexpr int kGFlush = 32;        // tiles accumulated in TMEM before each FP64 flush

// Byte offset of (mn, k) in an MN-major, no-swizzle tile of K = 64.
__device__ __forceinline__ uint32_t mn_off(int mn, int k)
{
    return (uint32_t)((mn >> 3) * kSBO + (k >> 3) * kLBO + (k & 7) * 16 + (mn & 7) * 2);
}

// Eight FP32 values -> one 16-byte hi chunk and one lo chunk.
__device__ __forceinline__ void split8(const float *x, uint4 &hi, uint4 &lo)
{
    uint32_t h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) split2(x[2 * e], x[2 * e + 1], h[e], l[e]);
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// (re, im) bf16 pair -> (-im, re): swap the halves, flip the new low half's
// sign (the split is sign-symmetric, so this is the split of the negated value).
__device__ __forceinline__ uint32_t rot_pair(uint32_t x) { return __byte_perm(x, 0u, 0x1032) ^ 0x8000u; }
__device__ __forceinline__ uint4 rot4(uint4 v) { return make_uint4(rot_pair(v.x), rot_pair(v.y), rot_pair(v.z), rot_pair(v.w)); }

// Per-sample values every operand group needs.
struct GPrelude {
    float2 Ep, Er, Et, g;
    float tau, pad;
    double Pr;
};

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

__global__ void __launch_bounds__(kGThreads, 1) k_adj_G_mixed(AdjGMixedArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_rm[kMaxRows], s_rk[kMaxRows];
    __shared__ double s_pc[24];
    __shared__ GPrelude s_pre[kGThreads];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int seg = blockIdx.x;
    const int nrow0 = 64 * blockIdx.y;   // first n' index of this CTA
    const int cbz = 2 * blockIdx.z;      // c_b of this CTA's first column block (0 or 2)
    const int R = a.R, NN = a.NN, NB = a.NB, CB = a.CB, ncb = a.ncb;
    const int lo = a.seg_start[seg], hi = a.seg_start[seg + 1];
    const double t0 = a.seg_info[3 * seg], pt0 = a.seg_info[3 * seg + 1], pw = a.seg_info[3 * seg + 2];
    const double hs = a.t_knots[seg + 1] - a.t_knots[seg];
    const long long nps = (long long)(a.N - 1) * 3;
    const int nA = min(8, (NN - nrow0 + 7) >> 3);  // A groups: 8 n' each (both c_a)
    const int nBg = CB >> 3;                         // B groups: 4 rows r each (all c_b of the CTA)
    const int ngroups = nA + nBg;

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
    // operand buffers start at zero: rows of A past NN and columns of B past
    // ncb * CB are never written
    const int bplane = NB * 128;                      // one B plane: NB/8 N groups x 1024 B
    const int smem_ops = 4 * kGPlaneA + 4 * bplane;
    for (int q = tid; q < smem_ops / 16; q += blockDim.x)
        reinterpret_cast<uint4 *>(smem_raw)[q] = make_uint4(0u, 0u, 0u, 0u);
    MixedPipe pp;
    mixed_setup(&s_tmem, s_bar, a.tmem_cols, pp);  // includes a __syncthreads

    unsigned char *const sA = smem_raw;                  // [buffer][plane] 16 KB each
    unsigned char *const sB = smem_raw + 4 * kGPlaneA;   // [buffer][plane] bplane each
    const uint32_t idesc = idesc_bf16(128, NB) | (1u << 15) | (1u << 16);  // A and B MN-major
    const int k0 = 16 * (lane >> 3) + (lane & 7);  // K row of part 0 (part 1: +8)
    bool failed = false;

    int it = 0;
    for (int base = lo; base < hi; base += kGT, ++it) {
        const int b = it & 1;
        if (__syncthreads_or(!pipe_drain(pp, b))) {
            failed = true;
            break;
        }
        if (it % kGPre == 0) {
            // FP64 prelude for this thread's sample of the next kGPre tiles
            // (phases as interpolate.cu:626-644, anchors reduced mod 2 pi)
            const int i = base + tid;
            const double t = (double)i * a.dt;
            const double s = (t - pt0) / pw;
            const double s1 = 1.0 - s;
            GPrelude pr;
            const double Pr = phase_poly(s_pc + 16, s, s1);
            pr.Pr = Pr;
            pr.Er = anchor(Pr);
            pr.Ep = anchor(phase_poly(s_pc, s, s1));
            pr.Et = a.use_theta ? anchor(phase_poly(s_pc + 8, s, s1)) : make_float2(1.f, 0.f);
            pr.tau = (float)((t - t0) / hs);
            pr.pad = 0.f;
            pr.g = make_float2(0.f, 0.f);
            if (i < hi) {
                const double2 Gt = a.grad[i];
                pr.g = make_float2((float)Gt.x, (float)-Gt.y);
            }
            s_pre[tid] = pr;
            __syncthreads();
        }
        const GPrelude pr = s_pre[(it % kGPre) * kGT + lane];
        unsigned char *const aH = sA + b * 2 * kGPlaneA, *const aL = aH + kGPlaneA;
        unsigned char *const bH = sB + b * 2 * bplane, *const bL = bH + bplane;
        for (int gi = warp; gi < ngroups; gi += kGThreads / 32) {
            if (gi < nA) {
                // A: tau^c_a v_{n'} for 8 n', c_a = 0 (rows 8 gi ..) and 1 (rows 64 + 8 gi ..)
                const int n0 = nrow0 + 8 * gi;
                float2 v = anchor((double)(a.nlo + n0) * pr.Pr);
                float re[8], im[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const bool ok = n0 + q < NN;
                    re[q] = ok ? v.x : 0.f;
                    im[q] = ok ? v.y : 0.f;
                    v = fcmul(v, pr.Er);
                }
                uint4 h4, l4;
#pragma unroll
                for (int ca = 0; ca < 2; ++ca) {
                    const int mn = 64 * ca + 8 * gi;
                    split8(re, h4, l4);
                    *reinterpret_cast<uint4 *>(aH + mn_off(mn, k0)) = h4;
                    *reinterpret_cast<uint4 *>(aL + mn_off(mn, k0)) = l4;
                    split8(im, h4, l4);
                    *reinterpret_cast<uint4 *>(aH + mn_off(mn, k0 + 8)) = h4;
                    *reinterpret_cast<uint4 *>(aL + mn_off(mn, k0 + 8)) = l4;
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        re[q] *= pr.tau;
                        im[q] *= pr.tau;
                    }
                }
            } else {
                // B: tau^c_b g u_r for 4 rows r, each c_b of the CTA
                const int rg = gi - nA;
                float2 u4[4];
                float2 uu = make_float2(1.f, 0.f);
                int pm = 0x7fffffff, pk = 0x7fffffff;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = 4 * rg + e;
                    u4[e] = make_float2(0.f, 0.f);
                    if (r < R) {
                        const int mm = s_rm[r], kk = s_rk[r];
                        if (kk == pk && mm == pm + 1) {
                            uu = fcmul(uu, pr.Ep);
                        } else {
                            uu = fcpow(pr.Ep, mm);
                            if (kk) uu = fcmul(uu, fcpow(pr.Et, kk));
                        }
                        pm = mm;
                        pk = kk;
                        u4[e] = uu;
                    }
                }
                const float t2 = pr.tau * pr.tau;
                float2 gc = pr.g;
                if (cbz) gc = make_float2(gc.x * t2, gc.y * t2);
                for (int cl = 0; cl < ncb; ++cl) {
                    float p0[8];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float2 w = fcmul(gc, u4[e]);
                        p0[2 * e] = w.x;      // part 0 (Re v): column (c_b, r, 0) += Re v Re w, (c_b, r, 1) += Re v Im w
                        p0[2 * e + 1] = w.y;  // part 1 (Im v) is (-Im w, Re w): rot4 of the same split
                    }
                    uint4 h4, l4;
                    split8(p0, h4, l4);
                    const int mn = cl * CB + 8 * rg;
                    *reinterpret_cast<uint4 *>(bH + mn_off(mn, k0)) = h4;
                    *reinterpret_cast<uint4 *>(bL + mn_off(mn, k0)) = l4;
                    *reinterpret_cast<uint4 *>(bH + mn_off(mn, k0 + 8)) = rot4(h4);
                    *reinterpret_cast<uint4 *>(bL + mn_off(mn, k0 + 8)) = rot4(l4);
                    gc = make_float2(gc.x * t2, gc.y * t2);
                }
            }
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a_h = smem_u32(aH), a_l = smem_u32(aL);
            const uint32_t b_h = smem_u32(bH), b_l = smem_u32(bL);
#pragma unroll
            for (int st = 0; st < 4; ++st) {  // K steps of 16 = K groups 2st, 2st+1
                const uint32_t ko = st * 2 * kLBO;
                const uint64_t da_h = smem_desc(a_h + ko, kLBO, kSBO), da_l = smem_desc(a_l + ko, kLBO, kSBO);
                const uint64_t db_h = smem_desc(b_h + ko, kLBO, kSBO), db_l = smem_desc(b_l + ko, kLBO, kSBO);
                mma_bf16(pp.tmem, da_h, db_h, idesc, ((it % kGFlush) | st) != 0);
                mma_bf16(pp.tmem, da_h, db_l, idesc, 1u);
                mma_bf16(pp.tmem, da_l, db_h, idesc, 1u);
            }
            mma_commit(&pp.bar[b]);
        }
        if (b == 0) pp.pend0 = 1;
        else pp.pend1 = 1;
        if ((it % kGFlush) == kGFlush - 1 || base + kGT >= hi) {
            // flush: every MMA done, then the accumulator (row (c_a, n'), column
            // (c_b, r, re/im)) into G in FP64, stored by the first flush and added
            // by the later ones; the next MMA restarts the accumulator.  Warps w
            // and w+4 read the same TMEM lanes (32 (w % 4) ..) and share the columns.
            const bool ok0 = pipe_drain(pp, 0), ok1 = pipe_drain(pp, 1);
            if (__syncthreads_or(!(ok0 && ok1))) {
                failed = true;
                break;
            }
            tc_fence_after();
            const bool first = it < kGFlush;
            const int quad = warp & 3;
            const int row = 32 * quad + lane;
            const int ca = row >> 6, n = nrow0 + (row & 63);
            const uint32_t trow = pp.tmem + ((uint32_t)(quad * 32) << 16);
            for (int j16 = warp >> 2; j16 < NB / 16; j16 += 2) {
                float D[16];
                tmem_ld16(trow + 16 * j16, D);
                tmem_wait_ld();
                if (n < NN) {
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int col = 16 * j16 + 2 * e;
                        const int cl = col / CB, r = (col - cl * CB) >> 1;
                        if (cl < ncb && r < R) {
                            const int c = ca + cbz + 2 * cl;
                            const double hc = c == 0 ? 1.0 : (c == 1 ? hs : (c == 2 ? hs * hs : hs * hs * hs));
                            double2 *gp = a.G + (((long long)seg * R + r) * NN + n) * 4 + c;
                            double2 v = make_double2((double)D[2 * e] * hc, (double)D[2 * e + 1] * hc);
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
            __syncthreads();
            tc_fence_after();
        }
    }
    mixed_teardown(failed, pp, a.tmem_cols, a.err);
}

}  // namespace

int launch_adj_G_mixed(const double2 *grad, const double *pc, int N, const double *seg_info, const double *t_knots,
                       const int *seg_start, int nseg, const int *row_m, const int *row_k, int R, int nlo, int NN,
                       double dt, int use_theta, double2 *G, int *err, cudaStream_t st)
{
    if (nseg == 0) return FEW_OK;
    AdjGMixedArgs a;
    a.CB = (2 * R + 7) / 8 * 8;  // columns per c_b: (r, re/im), padded to 8
    a.ncb = 2 * a.CB <= 256 ? 2 : 1;
    if (a.ncb * a.CB > 256) return fail(FEW_ERR_SIZE, "few_adjoint_G_mixed: %d rows exceed the 128 one MMA holds", R);
    a.NB = (a.ncb * a.CB + 15) / 16 * 16;
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
    int cols = 32;
    while (cols < a.NB) cols <<= 1;
    a.tmem_cols = cols;
    const size_t smem = (size_t)4 * kGPlaneA + (size_t)4 * a.NB * 128;
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
    if (N < 2 || nseg < 0 || nseg > N - 1 || R < 1 || R > 128 || NN < 1 || NN > 65535 * 64)
        return few::fail(FEW_ERR_SIZE, "few_adjoint_G_mixed: bad sizes (R <= 128)");
    return few::launch_adj_G_mixed((const double2 *)grad, phase_coeffs, N, seg_info, t_knots, seg_start, nseg, row_m,
                                   row_k, R, nlo, NN, dt, use_theta, (double2 *)G, err, (cudaStream_t)stream);
}
