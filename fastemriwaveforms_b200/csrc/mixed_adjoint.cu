// Amplitude adjoint of the mixed-precision mode sum on the tcgen05 tensor cores.
//
// Per knot segment s the gradient of L = Re sum_i g_i h_i with respect to the
// folded coefficients is the contraction over the segment's samples
//     G[r][n'][c] = sum_i u_r(t_i) b_{n',c}(t_i),   b_{n',c} = g_i tau_i^c v_{n'}(t_i)
// (then scaled by h_s^c, since x^c = h_s^c tau^c), the same array the FP64
// kernel k_adj_G produces, so the unfold and the spline adjoint that follow are
// shared.  The contraction runs over samples, so on the tensor core the samples
// are K:
//     D[(n', c)][(r, re/im)] += sum_{(i, part)} A[(n', c)][(i, part)] B[(i, part)][(r, re/im)]
// with A = (Re b, Im b) and B = (Re u, Im u | -Im u, Re u) for part 0 | 1, which
// gives D[., 2r] = Re(b u) and D[., 2r+1] = Im(b u) directly.  One CTA owns one
// segment and one tile of 32 n' columns (M = 32 n' x 4 powers of tau = 128) and
// loops over the segment's samples in tiles of 32 (K = 64): lane = sample,
// warp w = n' block of 8, so each thread's values for 8 consecutive M rows (or
// N columns) at one K row form one 16-byte chunk of the MN-major no-swizzle
// layout (core matrix = 8 K rows x 16 bytes; K groups 128 B apart, MN groups
// 1024 B apart).  Operands are split into bf16 hi + lo planes (three products
// hi*hi + hi*lo + lo*hi), FP32 accumulation in TMEM over at most 1024 samples:
// the accumulator is then added into G in FP64 and restarted, which keeps the
// FP32 rounding of long, oscillating (cancelling) sums small.
// Two operand buffers: while the tensor core consumes tile k, the threads
// build tile k+1.  Every wait is bounded; a timeout sets the error word, drains
// and frees TMEM.
#include "few_common.cuh"
#include "few_internal.h"
#include "few_tc.cuh"

namespace few {

namespace {

constexpr int kGT = 32;          // samples per tile; K = 64 (sample x {Re, Im})
constexpr int kGThreads = 128;   // 4 warps; warp w owns n' block w (8 columns) of the CTA's 32
constexpr int kGPlane = 16 * 1024;  // one A plane: 16 MN groups x 8 K groups x 128 B
constexpr uint32_t kLBO = 128;   // K-group stride (bytes)
constexpr uint32_t kSBO = 1024;  // MN-group stride (bytes)
constexpr int kGFlush = 32;      // tiles (of kGT samples) accumulated in TMEM before each FP64 flush

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
    int N, R, nlo, NN, NB, use_theta, tmem_cols;
    double dt;
};

__global__ void __launch_bounds__(kGThreads, 1) k_adj_G_mixed(AdjGMixedArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_rm[kMaxRows], s_rk[kMaxRows];
    __shared__ double s_pc[24];

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int seg = blockIdx.x;
    const int ncol0 = 32 * blockIdx.y;  // first n' index of this CTA
    const int R = a.R, NN = a.NN, NB = a.NB;
    const int lo = a.seg_start[seg], hi = a.seg_start[seg + 1];
    const double t0 = a.seg_info[3 * seg], pt0 = a.seg_info[3 * seg + 1], pw = a.seg_info[3 * seg + 2];
    const double hs = a.t_knots[seg + 1] - a.t_knots[seg];
    const long long nps = (long long)(a.N - 1) * 3;

    // the row and column of this thread's accumulator row in the epilogue
    const int j_row = w * 32 + lane;
    const int c_row = (j_row >> 3) & 3;
    const int n_row = ncol0 + 8 * w + (j_row & 7);

    if (lo >= hi) {  // a segment without samples: zero gradient
        if (n_row < NN) {
            for (int r = 0; r < R; ++r) a.G[(((long long)seg * R + r) * NN + n_row) * 4 + c_row] = make_double2(0.0, 0.0);
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
    MixedPipe pp;
    mixed_setup(&s_tmem, s_bar, a.tmem_cols, pp);  // includes a __syncthreads

    const int bplane = NB * 128;  // one B plane: NB/8 N groups x 1024 B
    unsigned char *const sA = smem_raw;                    // [buffer][plane] 16 KB each
    unsigned char *const sB = smem_raw + 4 * kGPlane;      // [buffer][plane] bplane each
    const uint32_t idesc = idesc_bf16(128, NB) | (1u << 15) | (1u << 16);  // A and B MN-major
    const int n0 = ncol0 + 8 * w;  // this thread's first n' column
    const int k0 = 16 * (lane >> 3) + (lane & 7);  // K row of part 0 (part 1: +8)
    bool failed = false;

    int it = 0;
    for (int base = lo; base < hi; base += kGT, ++it) {
        const int b = it & 1;
        if (__syncthreads_or(!pipe_drain(pp, b))) {
            failed = true;
            break;
        }
        const int i = base + lane;
        const bool valid = i < hi;
        // FP64 prelude: phases (interpolate.cu:626-644) and reduced anchors
        const double t = (double)i * a.dt;
        const double x = t - t0;
        const float tau = (float)(x / hs);
        const double s = (t - pt0) / pw;
        const double s1 = 1.0 - s;
        const double Pp = phase_poly(s_pc, s, s1);
        const double Pr = phase_poly(s_pc + 16, s, s1);
        const float2 Ep = anchor(Pp);
        const float2 Er = anchor(Pr);
        const float2 Et = a.use_theta ? anchor(phase_poly(s_pc + 8, s, s1)) : make_float2(1.f, 0.f);
        float2 g = make_float2(0.f, 0.f);
        if (valid) {
            const double2 Gt = a.grad[i];
            g = make_float2((float)Gt.x, (float)-Gt.y);
        }
        // A: b_{n', c} = g tau^c v_{n'} for this warp's 8 columns
        float2 v[8];
        v[0] = anchor((double)(a.nlo + n0) * Pr);
#pragma unroll
        for (int q = 1; q < 8; ++q) v[q] = fcmul(v[q - 1], Er);
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (n0 + q >= NN) v[q] = make_float2(0.f, 0.f);
        unsigned char *const aH = sA + b * 2 * kGPlane, *const aL = aH + kGPlane;
        float2 gc = g;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float re[8], im[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float2 z = fcmul(gc, v[q]);
                re[q] = z.x;
                im[q] = z.y;
            }
            uint4 h4, l4;
            const int mn = w * 32 + c * 8;
            split8(re, h4, l4);
            *reinterpret_cast<uint4 *>(aH + mn_off(mn, k0)) = h4;
            *reinterpret_cast<uint4 *>(aL + mn_off(mn, k0)) = l4;
            split8(im, h4, l4);
            *reinterpret_cast<uint4 *>(aH + mn_off(mn, k0 + 8)) = h4;
            *reinterpret_cast<uint4 *>(aL + mn_off(mn, k0 + 8)) = l4;
            gc.x *= tau;
            gc.y *= tau;
        }
        // B: u_r for 4 rows per N group; groups w, w+4, ...
        unsigned char *const bH = sB + b * 2 * bplane, *const bL = bH + bplane;
        for (int gn = w; gn < NB / 8; gn += 4) {
            float p0[8], p1[8];
            float2 uu = make_float2(1.f, 0.f);
            int pm = 0x7fffffff, pk = 0x7fffffff;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = 4 * gn + e;
                float2 u = make_float2(0.f, 0.f);
                if (r < R) {
                    const int mm = s_rm[r], kk = s_rk[r];
                    if (kk == pk && mm == pm + 1) {
                        uu = fcmul(uu, Ep);
                    } else {
                        uu = fcpow(Ep, mm);
                        if (kk) uu = fcmul(uu, fcpow(Et, kk));
                    }
                    pm = mm;
                    pk = kk;
                    u = uu;
                }
                p0[2 * e] = u.x;       // part 0 (Re b): column 2r += Re b Re u, 2r+1 += Re b Im u
                p0[2 * e + 1] = u.y;
                p1[2 * e] = -u.y;      // part 1 (Im b): column 2r -= Im b Im u, 2r+1 += Im b Re u
                p1[2 * e + 1] = u.x;
            }
            uint4 h4, l4;
            split8(p0, h4, l4);
            *reinterpret_cast<uint4 *>(bH + mn_off(8 * gn, k0)) = h4;
            *reinterpret_cast<uint4 *>(bL + mn_off(8 * gn, k0)) = l4;
            split8(p1, h4, l4);
            *reinterpret_cast<uint4 *>(bH + mn_off(8 * gn, k0 + 8)) = h4;
            *reinterpret_cast<uint4 *>(bL + mn_off(8 * gn, k0 + 8)) = l4;
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
            // flush: every MMA done, then this thread's accumulator row (n' block w,
            // power c_row, column n_row) into G in FP64 (stored by the first flush,
            // added by the later ones); the next MMA restarts the accumulator
            const bool ok0 = pipe_drain(pp, 0), ok1 = pipe_drain(pp, 1);
            if (__syncthreads_or(!(ok0 && ok1))) {
                failed = true;
                break;
            }
            tc_fence_after();
            const bool first = it < kGFlush;
            const uint32_t trow = pp.tmem + ((uint32_t)(w * 32) << 16);
            const double hc = c_row == 0 ? 1.0 : (c_row == 1 ? hs : (c_row == 2 ? hs * hs : hs * hs * hs));
            for (int cb = 0; cb < NB; cb += 16) {
                float D[16];
                tmem_ld16(trow + cb, D);
                tmem_wait_ld();
                if (n_row < NN) {
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int r = (cb >> 1) + e;
                        if (r < R) {
                            double2 *gp = a.G + (((long long)seg * R + r) * NN + n_row) * 4 + c_row;
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
    if (2 * R > 256) return fail(FEW_ERR_SIZE, "few_adjoint_G_mixed: %d rows exceed the 128 one MMA holds", R);
    AdjGMixedArgs a;
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
    a.NB = std::max(16, (2 * R + 15) / 16 * 16);
    a.use_theta = use_theta;
    a.dt = dt;
    int cols = 32;
    while (cols < a.NB) cols <<= 1;
    a.tmem_cols = cols;
    const size_t smem = (size_t)4 * kGPlane + (size_t)4 * a.NB * 128;
    FEW_CUDA_TRY(ensure_smem_attr((const void *)k_adj_G_mixed, (int)smem));
    dim3 grid(nseg, (NN + 31) / 32);
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
    if (N < 2 || nseg < 0 || nseg > N - 1 || R < 1 || R > 128 || NN < 1 || NN > 65535 * 32)
        return few::fail(FEW_ERR_SIZE, "few_adjoint_G_mixed: bad sizes (R <= 128)");
    return few::launch_adj_G_mixed((const double2 *)grad, phase_coeffs, N, seg_info, t_knots, seg_start, nseg, row_m,
                                   row_k, R, nlo, NN, dt, use_theta, (double2 *)G, err, (cudaStream_t)stream);
}
