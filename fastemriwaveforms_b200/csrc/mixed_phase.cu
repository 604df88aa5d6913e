// Phase adjoint of the mixed-precision mode sum on the tcgen05 tensor cores,
// in exact integer arithmetic.
//
// The gradient of L = Re sum_i g_i h_i with respect to the phase coefficients
// needs, per sample, dh/dPhi_phi = -i sum_r m'_r u_r Y_r, dh/dPhi_theta (k'_r
// weights) and dh/dPhi_r = -i sum_r u_r Z_r, with
//     Y_r(t) = sum_c tau^c sum_{n'} v_{n'}(t) W'[c][n'][r],   Z_r likewise with n' W'
// (W' = W h_s^c, tau = (t - t_s)/h_s, v = exp(-i n' Phi_r), u = exp(-i (m' Phi_phi
// + k' Phi_theta))); then e_f = Re(g dh/dPhi_f) is projected on the 8-term
// basis b_q(s) and summed per work unit, exactly as the FP64 kernel
// k_adj_phase does.  These sums cancel heavily (the coherent part of
// conj(h) dh/dPhi is imaginary), so the per-sample values need close to FP64
// accuracy: the contraction over n' runs on the integer tensor core.
//
//   A[i][(n', part)] = (Re v_{n'} | Im v_{n'})(t_i)
//   B[(n', part)][(r, q)] per segment, q = 2 (4 yz + c) + re/im: the real
//       form of w = W[c][n'][r] h_s^c (times n' for yz = 1): part Re v ->
//       (Re w, Im w), part Im v -> (-Im w, Re w)
//   D = A B  ->  Z_{c,r} and its n'-weighted twin for c = 0..3; the epilogue
//       forms Y_r = sum_c tau^c Z_{c,r} (Horner, FP64).
//
// Precision: v, u, g, tau in FP64 (FP64 sincos of each phase, FP64
// recurrences); every operand value is scaled to an integer |Y| <= 127 2^24
// (A: fixed scale, |A| <= 1; B: one scale per segment and column, from the
// column's largest value) and split into four signed base-256 digits (int8
// planes).  kind::i8 MMAs multiply digit planes i and j into the level i + j
// accumulator (levels 0..3, ten products per K step, s32, exact); the levels
// are combined in FP64 and the epilogue (tau^c, u_r, the row sums, e_f, the
// projection) runs in FP64.  The only error left is the 2^-32 representation
// of the operands.
//
// Shape: one CTA of 128 threads per work unit (<= 1024 samples of one
// segment), one sample row per thread per 128-sample tile.  The tile's A
// (K = 2 NNp: n' x {Re, Im}, in steps of 32) is generated once into shared
// memory; the rows r are then taken in passes of 4 (N = 64 columns: the four
// levels fill 256 TMEM columns, two CTAs per SM).  A pass's B (every K step of
// its rows) arrives by cp.async while the previous pass's epilogue runs; its
// MMAs are issued at once and signal an mbarrier (tcgen05.commit).  Every
// wait is bounded; a timeout sets the error word and ends the kernel after
// freeing TMEM.
#include "few_common.cuh"
#include "few_internal.h"
#include "few_tc.cuh"

namespace few {

namespace {

constexpr int kPT = 128;                            // samples per tile (MMA M)
constexpr int kKS = 32;                             // K per MMA step: 16 n' x {Re, Im}
constexpr int kDig = 4;                             // digits per operand value
constexpr int kRowsPass = 4;                        // (m', k') rows per pass
constexpr int kColsRow = 16;                        // columns per row: (Y, Z) x c = 0..3 x re/im
constexpr int kLvl = kColsRow * kRowsPass;          // TMEM columns per level (64)
constexpr int kTmemCols = kDig * kLvl;              // 256
constexpr int kAPlane = kPT * kKS;                  // A digit plane of a K step: 4 KB
constexpr int kBPlane = kLvl * kKS;                 // B digit plane of a K step and pass: 2 KB
constexpr double kScale = kDigitScale;               // |value| <= max -> |Y| <= 127 2^24
constexpr int kMaxPhaseRows = 64;
constexpr int kMaxPhaseNN = 128;                    // A of a tile (4 digits x 2 NNp x 128 B) <= 128 KB

// Byte offset of (row, kk) in a K-major, no-swizzle int8 tile of one K step
// (kk < 32): core matrices of 8 rows x 16 bytes, the two K halves 128 B apart
// (LBO), 8-row groups 256 B apart (SBO).
__host__ __device__ __forceinline__ uint32_t koff8(int row, int kk)
{
    return (uint32_t)((row >> 3) * 256 + ((kk >> 4) & 1) * 128 + (row & 7) * 16 + (kk & 15));
}

__host__ __device__ constexpr uint32_t idesc_s8_k(int M, int N)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Sixteen values -> their four digit chunks (16 bytes each, digit-plane order).
__device__ __forceinline__ void digit_chunks(const double *x, double scale, uint4 *out)
{
    uint32_t w[kDig][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t t[kDig];
        digit_words8(scaled_biased(x[4 * q], scale), scaled_biased(x[4 * q + 1], scale),
                     scaled_biased(x[4 * q + 2], scale), scaled_biased(x[4 * q + 3], scale), t);
#pragma unroll
        for (int p = 0; p < kDig; ++p) w[p][q] = t[p];
    }
#pragma unroll
    for (int p = 0; p < kDig; ++p) out[p] = make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
}

// Per segment the packed operand is one block: the NBc column scales
// (doubles), then the digit planes [K step][digit][NBc/8 column groups x 256 B].
struct PhaseDims {
    int NNp, nks, NBc;
    long long dig_bytes;  // digit bytes of one segment
    long long seg_bytes;  // the whole block of one segment (scales + digits)
};

__host__ __device__ inline PhaseDims phase_dims(int R, int NN)
{
    PhaseDims d;
    d.NNp = (NN + 15) / 16 * 16;
    d.nks = d.NNp / 16;          // K steps of 16 n' x {Re, Im}
    d.NBc = kColsRow * R;
    d.dig_bytes = (long long)d.nks * kDig * d.NBc * kKS;
    d.seg_bytes = (long long)d.NBc * 8 + d.dig_bytes;  // both multiples of 16 bytes
    return d;
}

// B operand: one CTA of 4 NNp threads per (segment, row).  A row's 16 columns
// are (yz, c, re/im) combinations of the same 4 NN complex coefficients, so the
// CTA stages the row's w = W[c][n'] h_s^c (and n' w) in shared memory, takes
// the column scales from the largest |Re w|, |Im w| per (yz, c) (both re/im
// columns of a pair see the same magnitudes), and then each thread writes the
// four digit chunks of one (column, K step, K half).
constexpr int kFoldThreads = 4 * kMaxPhaseNN;  // the largest CTA

__global__ void __launch_bounds__(kFoldThreads) k_fold_phase_s8(const double2 *__restrict__ W,
                                                                const double *__restrict__ t_knots, int nseg, int R,
                                                                int NN, int nlo, unsigned char *__restrict__ Bpk)
{
    __shared__ double2 s_w[2][kMaxPhaseNN][4];  // [yz][n'][c]
    __shared__ double s_m[kFoldThreads / 32][8];
    __shared__ double s_scale[8];               // per (yz, c)
    const PhaseDims pd = phase_dims(R, NN);
    const int s = blockIdx.x, r = blockIdx.y, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double h = t_knots[s + 1] - t_knots[s];
    unsigned char *const block = Bpk + (long long)s * pd.seg_bytes;
    const int nchunk = kColsRow * pd.nks * 2;  // (column, K step, K half) chunks of a row
    {
        // stage: thread (n', c) of n' < NNp (zero past NN); local maxima per (yz, c)
        double m0 = 0.0, m1 = 0.0;
        const int c = tid & 3, n = tid >> 2;
        if (n < pd.NNp) {
            const double hc = c == 0 ? 1.0 : (c == 1 ? h : (c == 2 ? h * h : h * h * h));
            double2 w0 = make_double2(0.0, 0.0), w1 = w0;
            if (n < NN) {
                const double2 wv = W[(((long long)s * R + r) * NN + n) * 4 + c];
                const double f1 = hc * (double)(nlo + n);
                w0 = make_double2(wv.x * hc, wv.y * hc);
                w1 = make_double2(wv.x * f1, wv.y * f1);
            }
            s_w[0][n][c] = w0;
            s_w[1][n][c] = w1;
            m0 = fmax(fabs(w0.x), fabs(w0.y));
            m1 = fmax(fabs(w1.x), fabs(w1.y));
        }
        // maxima over n' for each c: lanes with the same c are 4 apart
        for (int off = 4; off < 32; off <<= 1) {
            m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, off));
            m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, off));
        }
        if (lane < 4) {
            s_m[warp][lane] = m0;       // yz = 0, c = lane
            s_m[warp][4 + lane] = m1;   // yz = 1
        }
        __syncthreads();
        if (tid < 8) {
            double m = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, s_m[w][tid]);
            s_scale[tid] = m > 0.0 ? kScale / (m * (1.0 + 1e-12)) : 1.0;
        }
        __syncthreads();
        if (tid < kColsRow) {
            const int yz = tid >> 3, cc = (tid >> 1) & 3;
            reinterpret_cast<double *>(block)[r * kColsRow + tid] = s_scale[4 * yz + cc];
        }
        for (int q = tid; q < nchunk; q += blockDim.x) {
            const int q16 = q % kColsRow, rest = q / kColsRow;
            const int ks = rest >> 1, half = rest & 1;
            const int ri = q16 & 1, cc = (q16 >> 1) & 3, yz = q16 >> 3;
            const int j = r * kColsRow + q16;
            double x[16];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const double2 w = s_w[yz][16 * ks + 8 * half + e][cc];
                // part 0 (Re v): (Re w, Im w); part 1 (Im v): (-Im w, Re w)
                x[2 * e] = ri ? w.y : w.x;
                x[2 * e + 1] = ri ? w.x : -w.y;
            }
            uint4 ch[kDig];
            digit_chunks(x, s_scale[4 * yz + cc], ch);
#pragma unroll
            for (int p = 0; p < kDig; ++p) {
                unsigned char *dst = block + (long long)pd.NBc * 8 + ((long long)ks * kDig + p) * pd.NBc * kKS +
                                     koff8(j, 16 * half);
                *reinterpret_cast<uint4 *>(dst) = ch[p];
            }
        }
    }
}

struct PhaseArgs {
    const double2 *grad;  // torch upstream gradient G; g = conj(G)
    const unsigned char *Bpk;
    const double *pc;
    const double *seg_info;
    const double *t_knots;
    const int *units;
    const int *row_m;
    const int *row_k;
    double *partial;      // (nunits, 24)
    int *err;
    int N, R, nlo, NN, use_theta;
    double dt;
};

__global__ void __launch_bounds__(kPT, 2) k_adj_phase_s8(PhaseArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_rm[kMaxPhaseRows], s_rk[kMaxPhaseRows];
    __shared__ double s_pc[24];
    __shared__ double s_inv[kColsRow * kMaxPhaseRows];  // 2^24 / (A scale x column scale)
    __shared__ double s_e[3][kPT];
    __shared__ double s_s[kPT];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int unit = blockIdx.x;
    const int seg = a.units[3 * unit], lo = a.units[3 * unit + 1], hi = a.units[3 * unit + 2];
    const PhaseDims pd = phase_dims(a.R, a.NN);
    const int R = a.R, NN = a.NN, nks = pd.nks;
    const double t0 = a.seg_info[3 * seg], pt0 = a.seg_info[3 * seg + 1], pw = a.seg_info[3 * seg + 2];
    const double hs = a.t_knots[seg + 1] - a.t_knots[seg];
    const long long nps = (long long)(a.N - 1) * 3;

    for (int r = tid; r < R; r += blockDim.x) {
        s_rm[r] = a.row_m[r];
        s_rk[r] = a.row_k[r];
    }
    const unsigned char *const block = a.Bpk + (long long)seg * pd.seg_bytes;
    for (int j = tid; j < pd.NBc; j += blockDim.x)
        s_inv[j] = 16777216.0 / (kScale * reinterpret_cast<const double *>(block)[j]);
    if (tid < 24) {
        const int q = tid >> 3, c = tid & 7;
        s_pc[tid] = a.pc[c * nps + (long long)seg * 3 + q];
    }
    MixedPipe pp;
    mixed_setup(&s_tmem, s_bar, kTmemCols, pp);  // includes a __syncthreads

    const unsigned char *const Bseg = block + (long long)pd.NBc * 8;
    unsigned char *const sA = smem_raw;                                   // [digit][K step] planes
    unsigned char *const sB = smem_raw + (size_t)kDig * nks * kAPlane;    // [digit][K step] planes of a pass
    const int npass = (R + kRowsPass - 1) / kRowsPass;
    const bool pair_levels = nks <= 4;  // K = 32 nks <= 128: level pairs fit in int32
    const uint32_t trow = pp.tmem + ((uint32_t)(warp * 32) << 16);
    double proj[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // this lane's share of the unit's 24 outputs
    bool failed = false;

    // B of a pass: its rows of every K step and digit plane (rows x 512 bytes each)
    auto load_B = [&](int pass) {
        const int r0 = pass * kRowsPass, rows = min(kRowsPass, R - r0);
        const int per = rows * (kColsRow / 8) * 16;  // 16-byte chunks per (K step, digit)
        for (int q = tid; q < nks * kDig * per; q += blockDim.x) {
            const int kp = q / per, c = q - kp * per;  // kp = ks * kDig + digit
            const int ks = kp / kDig, p = kp - ks * kDig;
            const unsigned char *src =
                Bseg + ((long long)ks * kDig + p) * pd.NBc * kKS + (long long)r0 * kColsRow * kKS + 16 * c;
            cp_async16(sB + (p * nks + ks) * kBPlane + 16 * c, src);
        }
        cp_async_commit();
    };

    for (int base = lo; base < hi && !failed; base += kPT) {
        const int i = base + tid;
        const bool valid = i < hi;
        load_B(0);  // the buffer is free: the previous tile's MMAs were drained
        // FP64 prelude (phases as interpolate.cu:626-644)
        const double t = (double)i * a.dt;
        const double tau = (t - t0) / hs;
        const double s = (t - pt0) / pw;
        const double s1 = 1.0 - s;
        double sn, cs;
        sincos_reduced(phase_poly(s_pc, s, s1), &sn, &cs);
        const double2 Ep = make_double2(cs, -sn);
        sincos_reduced(phase_poly(s_pc + 16, s, s1), &sn, &cs);
        const double2 Er = make_double2(cs, -sn);
        double2 Et = make_double2(1.0, 0.0);
        if (a.use_theta) {
            sincos_reduced(phase_poly(s_pc + 8, s, s1), &sn, &cs);
            Et = make_double2(cs, -sn);
        }
        // A of the tile: v_{n'} for every n' (FP64 recurrence), digits into shared memory
        {
            double2 v = cpow_int(Er, a.nlo);
            for (int ks = 0; ks < nks; ++ks) {
                double x[2 * 16];
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const bool ok = valid && (16 * ks + q < NN);
                    x[2 * q] = ok ? v.x : 0.0;
                    x[2 * q + 1] = ok ? v.y : 0.0;
                    v = cmul(v, Er);
                }
#pragma unroll
                for (int half = 0; half < 2; ++half) {
                    uint4 ch[kDig];
                    digit_chunks(x + 16 * half, kScale, ch);
#pragma unroll
                    for (int p = 0; p < kDig; ++p)
                        *reinterpret_cast<uint4 *>(sA + (p * nks + ks) * kAPlane + koff8(tid, 16 * half)) = ch[p];
                }
            }
        }
        double2 Sp = make_double2(0.0, 0.0), St = Sp, Sr = Sp;
        double2 uu = make_double2(1.0, 0.0);
        int pm = 0x7fffffff, pk = 0x7fffffff;

        for (int pass = 0; pass < npass && !failed; ++pass) {
            const int r0 = pass * kRowsPass, rows = min(kRowsPass, R - r0);
            const uint32_t idesc = idesc_s8_k(kPT, kColsRow * rows);
            cp_async_wait_all();
            fence_async_smem();  // A and this pass's B visible to the tensor core
            __syncthreads();
            if (tid == 0) {
                tc_fence_after();
                const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
                for (int ks = 0; ks < nks; ++ks) {
#pragma unroll
                    for (int lv = 0; lv < kDig; ++lv) {
#pragma unroll
                        for (int ia = 0; ia <= lv; ++ia) {
                            const int jb = lv - ia;
                            const uint64_t da = smem_desc(a0 + (ia * nks + ks) * kAPlane, 128, 256);
                            const uint64_t db = smem_desc(b0 + (jb * nks + ks) * kBPlane, 128, 256);
                            mma_s8(pp.tmem + (uint32_t)(lv * kLvl), da, db, idesc, (ks == 0 && ia == 0) ? 0u : 1u);
                        }
                    }
                }
                mma_commit(&pp.bar[0]);
            }
            pp.pend0 = 1;
            if (__syncthreads_or(!pipe_drain(pp, 0))) {
                failed = true;
                break;
            }
            tc_fence_after();
            if (pass + 1 < npass) load_B(pass + 1);  // arrives while this pass's epilogue runs
            // epilogue of the pass, one row (16 columns) at a time: the four levels
            // in FP64, Y and Z by Horner in tau, u_r, and the three weighted row sums
            for (int rr = 0; rr < rows; ++rr) {
                const int r = r0 + rr;
                // the four levels of the row: four loads in flight, one wait
                float F[kDig][16];
#pragma unroll
                for (int lv = 0; lv < kDig; ++lv) tmem_ld16(trow + (uint32_t)(lv * kLvl + kColsRow * rr), F[lv]);
                tmem_wait_ld();
                int D[kDig][16];
#pragma unroll
                for (int lv = 0; lv < kDig; ++lv)
#pragma unroll
                    for (int e = 0; e < 16; ++e) D[lv][e] = __float_as_int(F[lv][e]);
                double val[16];
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    // the levels combined exactly: a level sums (level + 1) K digit
                    // products of magnitude <= 2^14, so with K <= 128 (nks <= 4) the
                    // pairs D0 2^8 + D1 and D2 2^8 + D3 stay below 2^31 in int32 and two
                    // int32 -> double steps and one FMA give the same double as four and
                    // three (every partial sum is an integer below 2^53).  int32 -> double
                    // without a conversion instruction: 2^52 + 2^31 + D in the
                    // significand, minus the offset.
                    double acc;
                    if (pair_levels) {
                        const int hi2 = D[0][q] * 256 + D[1][q], lo2 = D[2][q] * 256 + D[3][q];
                        const double dh = __hiloint2double(0x43300000, hi2 ^ 0x80000000) - 4503601774854144.0;
                        const double dl = __hiloint2double(0x43300000, lo2 ^ 0x80000000) - 4503601774854144.0;
                        acc = fma(dh, 65536.0, dl);
                    } else {
                        double lv[kDig];
#pragma unroll
                        for (int l = 0; l < kDig; ++l)
                            lv[l] = __hiloint2double(0x43300000, D[l][q] ^ 0x80000000) - 4503601774854144.0;
                        acc = fma(lv[0], 16777216.0, fma(lv[1], 65536.0, fma(lv[2], 256.0, lv[3])));
                    }
                    val[q] = acc * s_inv[kColsRow * r + q];
                }
                // q = 2 (4 yz + c) + re/im
                double2 Y = make_double2(val[6], val[7]), Z = make_double2(val[14], val[15]);
#pragma unroll
                for (int c = 2; c >= 0; --c) {
                    Y = make_double2(fma(Y.x, tau, val[2 * c]), fma(Y.y, tau, val[2 * c + 1]));
                    Z = make_double2(fma(Z.x, tau, val[8 + 2 * c]), fma(Z.y, tau, val[8 + 2 * c + 1]));
                }
                const int mm = s_rm[r], kk = s_rk[r];
                if (kk == pk && mm == pm + 1) {
                    uu = cmul(uu, Ep);
                } else {
                    uu = cpow_int(Ep, mm);
                    if (kk) uu = cmul(uu, cpow_int(Et, kk));
                }
                pm = mm;
                pk = kk;
                const double2 P = cmul(uu, Y), Q = cmul(uu, Z);
                Sp.x = fma((double)mm, P.x, Sp.x);
                Sp.y = fma((double)mm, P.y, Sp.y);
                St.x = fma((double)kk, P.x, St.x);
                St.y = fma((double)kk, P.y, St.y);
                Sr.x += Q.x;
                Sr.y += Q.y;
            }
            tc_fence_before();
            __syncthreads();  // TMEM read before the next pass's first MMA overwrites it
            tc_fence_after();
        }
        if (failed) break;
        // e_f = Re(g dh/dPhi_f) = Im(g S_f), g = conj(G)
        double ep = 0.0, et = 0.0, er = 0.0;
        if (valid) {
            const double2 Gt = a.grad[i];
            ep = Gt.x * Sp.y - Gt.y * Sp.x;
            et = Gt.x * St.y - Gt.y * St.x;
            er = Gt.x * Sr.y - Gt.y * Sr.x;
        }
        s_e[0][tid] = ep;
        s_e[1][tid] = et;
        s_e[2][tid] = er;
        s_s[tid] = s;
        __syncthreads();
        // project on b_q(s) = 1, s, s s1, s^2 s1, ... (factors s, s1 alternating):
        // warp w accumulates outputs o = w + 4k (field o / 8, term o % 8)
#pragma unroll
        for (int m = 0; m < kPT / 32; ++m) {
            const int jj = lane + 32 * m;
            const double sj = s_s[jj], s1j = 1.0 - sj;
            double bq[8];
            bq[0] = 1.0;
#pragma unroll
            for (int q = 1; q < 8; ++q) bq[q] = bq[q - 1] * ((q & 1) ? sj : s1j);
#pragma unroll
            for (int kq = 0; kq < 6; ++kq) {
                const int o = warp + 4 * kq;
                const int f = o >> 3, q = o & 7;
                double bsel = bq[0];
#pragma unroll
                for (int qq = 1; qq < 8; ++qq) bsel = (q == qq) ? bq[qq] : bsel;
                proj[kq] = fma(bsel, s_e[f][jj], proj[kq]);
            }
        }
        __syncthreads();  // s_e, s_s read before the next tile writes them
    }
    if (!failed) {
#pragma unroll
        for (int kq = 0; kq < 6; ++kq) {
            double v = proj[kq];
            for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            if (lane == 0) a.partial[(long long)unit * 24 + warp + 4 * kq] = v;
        }
    }
    cp_async_wait_all();
    mixed_teardown(failed, pp, kTmemCols, a.err);
}

}  // namespace

size_t phase_operand_bytes(int nseg, int R, int NN)
{
    if (R > kMaxPhaseRows) return 0;
    return (size_t)nseg * (size_t)phase_dims(R, NN).seg_bytes;
}

}  // namespace few

extern "C" long long few_mixed_adjoint_operand_bytes(int nseg, int R, int NN)
{
    if (nseg < 0 || R < 1 || NN < 1) return 0;
    return (long long)few::phase_operand_bytes(nseg, R, NN);
}

extern "C" int few_fold_mixed_adjoint(const void *W, const double *t_knots, int nseg, int R, int nlo, int NN, void *Bpk,
                                      void *stream)
{
    few::clear_error();
    if (!W || !t_knots || !Bpk) return few::fail(FEW_ERR_ARG, "few_fold_mixed_adjoint: null pointer");
    if (nseg < 0 || R < 1 || R > few::kMaxPhaseRows || NN < 1)
        return few::fail(FEW_ERR_SIZE, "few_fold_mixed_adjoint: bad sizes (R <= %d)", few::kMaxPhaseRows);
    if (nseg == 0) return FEW_OK;
    if (NN > few::kMaxPhaseNN)
        return few::fail(FEW_ERR_SIZE, "few_fold_mixed_adjoint: NN=%d > %d", NN, few::kMaxPhaseNN);
    const dim3 grid(nseg, R);
    few::k_fold_phase_s8<<<grid, 4 * few::phase_dims(R, NN).NNp, 0, (cudaStream_t)stream>>>(
        (const double2 *)W, t_knots, nseg, R, NN, nlo, (unsigned char *)Bpk);
    FEW_LAUNCH_CHECK("k_fold_phase_s8");
    return FEW_OK;
}

extern "C" int few_adjoint_phase_mixed(const void *grad, const void *Bpk, const double *phase_coeffs, int N,
                                       const double *seg_info, const double *t_knots, const int *units, int nunits,
                                       const int *row_m, const int *row_k, int R, int nlo, int NN, double dt,
                                       int use_theta, double *partial, int *err, void *stream)
{
    few::clear_error();
    if (!grad || !Bpk || !phase_coeffs || !seg_info || !t_knots || !units || !row_m || !row_k || !partial || !err)
        return few::fail(FEW_ERR_ARG, "few_adjoint_phase_mixed: null pointer");
    if (N < 2 || nunits < 0 || R < 1 || R > few::kMaxPhaseRows || NN < 1 || NN > few::kMaxPhaseNN)
        return few::fail(FEW_ERR_SIZE, "few_adjoint_phase_mixed: bad sizes (R <= %d, NN <= %d)", few::kMaxPhaseRows,
                         few::kMaxPhaseNN);
    if (nunits == 0) return FEW_OK;
    few::PhaseArgs a;
    a.grad = (const double2 *)grad;
    a.Bpk = (const unsigned char *)Bpk;
    a.pc = phase_coeffs;
    a.seg_info = seg_info;
    a.t_knots = t_knots;
    a.units = units;
    a.row_m = row_m;
    a.row_k = row_k;
    a.partial = partial;
    a.err = err;
    a.N = N;
    a.R = R;
    a.nlo = nlo;
    a.NN = NN;
    a.use_theta = use_theta;
    a.dt = dt;
    const int smem = few::kDig * few::phase_dims(R, NN).nks * (few::kAPlane + few::kBPlane);
    FEW_CUDA_TRY(few::ensure_smem_attr((const void *)few::k_adj_phase_s8, smem));
    few::k_adj_phase_s8<<<nunits, few::kPT, smem, (cudaStream_t)stream>>>(a);
    FEW_LAUNCH_CHECK("k_adj_phase_s8");
    return FEW_OK;
}
