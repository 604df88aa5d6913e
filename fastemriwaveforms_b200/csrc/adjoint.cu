// Adjoint of the interpolated mode sum: dL/d(amplitude knots) and
// dL/d(phase coefficients) for L = Re sum_i g_i h_i, with g supplied.
//
// The forward map is  knots y --spline--> coefficients a --fold--> W --sum--> h,
// phases Phi(s) = sum_q b_q(s) coef_q (the 8-term basis of
// src/few/cutils/interpolate.cu:642-644).  Its adjoint runs the chain backwards:
//
//   k_adj_phase   per sample, the forward-like sums dh/dPhi_phi, dh/dPhi_r,
//                 dh/dPhi_theta (phasors recomputed, not stored), projected on
//                 the basis b_q(s) and reduced per work unit; k_adj_phase_reduce
//                 adds the unit partials per segment in unit order.
//   k_adj_G       per segment, G[key][c] = sum_i g_i x_i^c P_key(t_i): one CTA
//                 per segment, per-sample phasor tables staged in shared memory,
//                 each thread owning a few keys (deterministic, no atomics).
//   k_adj_joint   both of the above from one pass: per key and work unit the
//                 moments sum_i sigma_i^p g_i P_key(t_i), p = 0..10, from which
//                 G and the phase-coefficient gradients follow (used when both
//                 gradients are wanted); k_adj_joint_reduce(_G) add the units.
//   k_unfold      the transpose of the fold: dL/da per mode and coefficient.
//   k_spline_adjoint  the transpose of the spline build: solves with A^T, the
//                 transposed not-a-knot matrix.  With M the row operations that
//                 remove the two non-dominant rows (row1 -= row0,
//                 row[N-2] -= row[N-1]) and M A = A~, A^{-T} = M^T A~^{-T}: the
//                 first and last columns of A~ each hold one entry, and the
//                 interior block is the transpose of a row-dominant tridiagonal
//                 matrix (column-dominant), so elimination without pivoting is
//                 stable there too.
//
// With torch's convention the upstream gradient of a complex output is
// G = dL/dRe h + i dL/dIm h, so g = conj(G).  Gradients with respect to real
// inputs are plain derivatives; for complex inputs d/dRe + i d/dIm.
#include "few_common.cuh"
#include "few_internal.h"

namespace few {

namespace {

constexpr int kAdjThreads = 256;
constexpr int kSmemBudget = 200 * 1024;

struct AdjPhaseArgs {
    const double2 *grad;  // (out_len,) torch upstream gradient G; g = conj(G)
    const double2 *W;
    const double *pc;     // (8, N-1, 3)
    const double *seg_info;
    const int *units;
    const int *row_m;
    const int *row_k;
    double *partial;      // (nunits, 24): unit partials of dL/dcoef[field][q], field 0 phi, 1 theta, 2 r
    int N, R, nlo, NN, rows_per_pass, use_theta;
    double dt;
};

// dL/dPhi at every sample of the unit, projected on the phase basis.
//
// Shared memory holds the folded coefficients of this pass's rows in blocks of
// RB rows (rows past R zero-filled), each block laid out (n', row, c): the
// 4 RB double2 values one column n' needs are contiguous, so every load of the
// key loop is at an immediate offset from one pointer.  The per-row factors
// (u_r, m'_r, k'_r) are formed once per block.  s_e (after the blocks) holds
// dL/dPhi_f per sample of the unit for the fields in use (phi, r, and theta).
template <int RB, bool THETA>
__global__ void __launch_bounds__(kAdjThreads, 2) k_adj_phase(AdjPhaseArgs a)
{
    constexpr int NF = THETA ? 3 : 2;  // fields: 0 phi, 1 r, 2 theta
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_rm[kMaxRows + 8], s_rk[kMaxRows + 8];
    __shared__ double s_pc[24];

    const int u = blockIdx.x;
    const int seg = a.units[3 * u], lo = a.units[3 * u + 1];
    const int hi = min(a.units[3 * u + 2], lo + 1024);  // units hold at most 1024 samples (checked on the host)
    const double t0 = a.seg_info[3 * seg], pt0 = a.seg_info[3 * seg + 1], pw = a.seg_info[3 * seg + 2];
    const int R = a.R, NN = a.NN, nlo = a.nlo;
    const int rpp = a.rows_per_pass;  // a multiple of RB
    double2 *sW = reinterpret_cast<double2 *>(smem_raw);
    double (*s_e)[1024] = reinterpret_cast<double (*)[1024]>(smem_raw + (size_t)rpp * NN * 4 * sizeof(double2));
    const long long nps = (long long)(a.N - 1) * 3;
    const int Rp = (R + RB - 1) / RB * RB;
    for (int r = threadIdx.x; r < Rp; r += blockDim.x) {
        s_rm[r] = r < R ? a.row_m[r] : 0;  // padded rows: u = 1 against zero coefficients
        s_rk[r] = r < R ? a.row_k[r] : 0;
    }
    if (threadIdx.x < 24) {
        const int q = threadIdx.x >> 3, c = threadIdx.x & 7;
        s_pc[threadIdx.x] = a.pc[c * nps + (long long)seg * 3 + q];
    }
    for (int q = threadIdx.x; q < hi - lo; q += blockDim.x)
#pragma unroll
        for (int f = 0; f < NF; ++f) s_e[f][q] = 0.0;

    for (int r0 = 0; r0 < Rp; r0 += rpp) {
        const int nrp = min(rpp, Rp - r0);  // a multiple of RB
        __syncthreads();
        {
            // (row, n', c) in global order -> (block, n', row in block, c) in shared
            const double2 *src = a.W + ((long long)seg * R + r0) * NN * 4;
            const int count = nrp * NN * 4;
            for (int e = threadIdx.x; e < count; e += blockDim.x) {
                const int rr = e / (NN * 4), rem = e - rr * (NN * 4);
                const int n = rem >> 2, c = rem & 3;
                const int blk = rr / RB, q = rr - blk * RB;
                sW[(((long long)blk * NN + n) * RB + q) * 4 + c] = (r0 + rr < R) ? src[e] : make_double2(0.0, 0.0);
            }
        }
        __syncthreads();
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const double t = rmul(a.dt, (double)i);
            const double x = rsub(t, t0);
            const double s = __ddiv_rn(rsub(t, pt0), pw);
            const double s1 = rsub(1.0, s);
            const double Pp = phase_poly(s_pc, s, s1);
            const double Pr = phase_poly(s_pc + 16, s, s1);
            double sn, cs;
            sincos(Pp, &sn, &cs);
            const double2 Ep = make_double2(cs, -sn);
            sincos(Pr, &sn, &cs);
            const double2 Er = make_double2(cs, -sn);
            double2 Et = make_double2(1.0, 0.0);
            if (THETA) {
                sincos(phase_poly(s_pc + 8, s, s1), &sn, &cs);
                Et = make_double2(cs, -sn);
            }
            const double2 V0 = cpow_int(Er, nlo);
            double2 Dp = make_double2(0.0, 0.0), Dr = Dp, Dt = Dp;
            for (int rb = 0; rb < nrp; rb += RB) {
                double2 U[RB];
                double mq[RB], kq[RB];
#pragma unroll
                for (int q = 0; q < RB; ++q) {
                    const int mm = s_rm[r0 + rb + q], kk = s_rk[r0 + rb + q];
                    double2 uu = cpow_int(Ep, mm);
                    if (THETA && kk) uu = cmul(uu, cpow_int(Et, kk));
                    U[q] = uu;
                    mq[q] = (double)mm;
                    kq[q] = (double)kk;
                }
                double2 v = V0;
                double dn = (double)nlo;
                const double2 *wb = sW + (long long)rb * NN * 4;  // block (rb / RB): (n', row, c)
                for (int n = 0; n < NN; ++n) {
                    const double2 *wn = wb + n * (RB * 4);
                    double2 T = make_double2(0.0, 0.0), Tm = T, Tk = T;
#pragma unroll
                    for (int q = 0; q < RB; ++q) {
                        const double2 w0 = wn[4 * q], w1 = wn[4 * q + 1], w2 = wn[4 * q + 2], w3 = wn[4 * q + 3];
                        double2 Wx;
                        Wx.x = fma(fma(fma(w3.x, x, w2.x), x, w1.x), x, w0.x);
                        Wx.y = fma(fma(fma(w3.y, x, w2.y), x, w1.y), x, w0.y);
                        const double2 P = cmul(U[q], Wx);
                        T.x += P.x;
                        T.y += P.y;
                        Tm.x = fma(mq[q], P.x, Tm.x);
                        Tm.y = fma(mq[q], P.y, Tm.y);
                        if (THETA) {
                            Tk.x = fma(kq[q], P.x, Tk.x);
                            Tk.y = fma(kq[q], P.y, Tk.y);
                        }
                    }
                    const double2 vT = cmul(v, T);
                    const double2 vTm = cmul(v, Tm);
                    Dp.x += vTm.x;
                    Dp.y += vTm.y;
                    Dr.x = fma(dn, vT.x, Dr.x);
                    Dr.y = fma(dn, vT.y, Dr.y);
                    if (THETA) {
                        const double2 vTk = cmul(v, Tk);
                        Dt.x += vTk.x;
                        Dt.y += vTk.y;
                    }
                    v = cmul(v, Er);
                    dn += 1.0;
                }
            }
            // dh/dPhi = -i D; dL/dPhi = Re(g (-i D)) = Im(g D) with g = conj(G)
            const double2 G = a.grad[i];
            // partial over this pass's rows; passes add in a fixed order
            s_e[0][i - lo] += G.x * Dp.y - G.y * Dp.x;
            s_e[1][i - lo] += G.x * Dr.y - G.y * Dr.x;
            if (THETA) s_e[2][i - lo] += G.x * Dt.y - G.y * Dt.x;
        }
    }
    __syncthreads();
    // project on the basis b_q(s) = 1, s, s s1, s^2 s1, s^2 s1^2, s^3 s1^2, s^3 s1^3,
    // s^4 s1^3: warp w produces outputs w, w+8, w+16 (24 = 3 fields x 8 terms;
    // output field order phi, theta, r)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int o = warp; o < 24; o += nwarp) {
        const int f = o >> 3, q = o & 7;
        const int fe = f == 0 ? 0 : (f == 2 ? 1 : 2);  // s_e row of output field f
        double v = 0.0;
        if (fe < NF) {
            for (int j = lane; j < hi - lo; j += 32) {
                const double t = rmul(a.dt, (double)(lo + j));
                const double s = __ddiv_rn(rsub(t, pt0), pw);
                const double s1 = rsub(1.0, s);
                double b = 1.0;
                // b_q: alternate factors s, s1 starting with s
                for (int k = 0; k < q; ++k) b *= (k & 1) ? s1 : s;
                v = fma(s_e[fe][j], b, v);
            }
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        }
        if (lane == 0) a.partial[(long long)u * 24 + o] = v;
    }
}

// Sum the unit partials of each segment (units of a segment are consecutive) into
// grad_pc (N-1, 3, 8) (the layout of phase_interp_coeffs).
__global__ void k_adj_phase_reduce(const double *__restrict__ partial, const int *__restrict__ seg_units, int nseg,
                                   double *__restrict__ grad_pc)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nseg * 24) return;
    const int s = idx / 24, e = idx - s * 24;
    double v = 0.0;
    for (int u = seg_units[s]; u < seg_units[s + 1]; ++u) v += partial[(long long)u * 24 + e];
    grad_pc[idx] = v;  // (s, field, q) with e = field*8 + q
}

// G[s][key][c] = sum_{i in segment s} g_i x_i^c P_key(t_i).
struct AdjGArgs {
    const double2 *grad;
    const double *pc;
    const double *seg_info;
    const int *seg_start;  // (nseg+1,) first output sample of each segment (clamped)
    const int *row_m;
    const int *row_k;
    double2 *G;            // (nseg, R, NN, 4)
    int N, R, nlo, NN, use_theta, key_base, nkeys_pass;
    double dt;
};

constexpr int kGThreads = 384;
constexpr int kGPhase = kGThreads;  // samples whose phase data is staged at once (one per thread)
constexpr int kGTile = 64;    // samples per phasor-table tile
constexpr int kGCols = 64;    // n' columns per CTA (one per thread of a row block)
constexpr int kGRowBlocks = kGThreads / kGCols;  // 6 row blocks per CTA

constexpr int kGPow = 16;     // per tile sample and phasor: E^0..E^7, then E^0, E^8, ..., E^56

// Dynamic shared memory of k_adj_G<RB>: the phasor tables of one tile, the
// small power tables of its samples, and the phase data of kGPhase samples.
constexpr size_t adj_g_smem(int rb)
{
    return (size_t)kGTile * kGRowBlocks * rb * sizeof(double2)  // g u_r
           + (size_t)kGTile * kGCols * sizeof(double2)          // v_{n'}
           + (size_t)kGTile * 2 * kGPow * sizeof(double2)       // powers of e^{-i Phi_phi}, e^{-i Phi_r}
           + (size_t)kGPhase * 5 * sizeof(double2)              // Ep, Er, Et, g, v at this CTA's first n'
           + (size_t)kGPhase * 4 * sizeof(double);              // 1, x, x^2, x^3
}

// E^p from a sample's power table (E^0..E^7, E^0, E^8, ..., E^56): two factors
// for |p| < 64 (a power by squaring past that), the conjugate for p < 0.
__device__ __forceinline__ double2 pow_from_table(const double2 *T, int p)
{
    const int q = p < 0 ? -p : p;
    double2 z = q < 64 ? cmul(T[8 + (q >> 3)], T[q & 7]) : cpow_int(T[1], q);
    if (p < 0) z.y = -z.y;
    return z;
}

// grid (nseg, row groups of 6*RB rows, column groups of 64), 384 threads (12
// warps per SM at <= 170 registers): thread (row block rb, column c) owns keys
// (r = group*6*RB + rb*RB + q, n' = c) for q < RB and
// accumulates their four x^c sums over every sample of the segment.  Every
// thread first evaluates the phases, sincos, g and v at the CTA's first n' of
// one of the next kGPhase samples; then, per tile of kGTile samples, 2 kGTile
// threads build each sample's small power tables of e^{-i Phi_phi} and
// e^{-i Phi_r} (E^0..E^7 and E^8k), the CTA fills the row factors g_i u_r(t_i)
// and the column phasors v_{n'}(t_i) from them (each entry two or three
// independent complex products, no long dependent chains), and each thread
// reads its column phasor once per sample and uses it for RB rows (the row
// factors are warp-wide broadcasts).  Samples are added in order:
// deterministic.
template <int RB>
__global__ void __launch_bounds__(kGThreads, 1) k_adj_G(AdjGArgs a)
{
    constexpr int RG = kGRowBlocks * RB;  // rows per CTA
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 (*s_gu)[RG] = reinterpret_cast<double2 (*)[RG]>(smem_raw);
    double2 (*s_v)[kGCols] = reinterpret_cast<double2 (*)[kGCols]>(smem_raw + (size_t)kGTile * RG * sizeof(double2));
    double2 (*s_P)[2][kGPow] =  // [tile sample][phi, r][power]
        reinterpret_cast<double2 (*)[2][kGPow]>(smem_raw + (size_t)kGTile * (RG + kGCols) * sizeof(double2));
    double2 (*s_E)[5] = reinterpret_cast<double2 (*)[5]>(smem_raw + (size_t)kGTile * (RG + kGCols + 2 * kGPow) *
                                                                         sizeof(double2));
    double (*s_x)[4] = reinterpret_cast<double (*)[4]>(
        smem_raw + (size_t)(kGTile * (RG + kGCols + 2 * kGPow) + kGPhase * 5) * sizeof(double2));
    __shared__ int s_rm[RG], s_rk[RG];
    __shared__ double s_pc[24];

    const int R = a.R, NN = a.NN;
    const int seg = blockIdx.x;
    const int r0 = blockIdx.y * RG, c0 = blockIdx.z * kGCols;
    const int lo = a.seg_start[seg], hi = a.seg_start[seg + 1];
    const double t0 = a.seg_info[3 * seg], pt0 = a.seg_info[3 * seg + 1], pw = a.seg_info[3 * seg + 2];
    const long long nps = (long long)(a.N - 1) * 3;
    const int tid = threadIdx.x;
    const int col = tid % kGCols, rb = tid / kGCols;
    for (int r = tid; r < RG; r += blockDim.x) {
        s_rm[r] = (r0 + r < R) ? a.row_m[r0 + r] : 0;
        s_rk[r] = (r0 + r < R) ? a.row_k[r0 + r] : 0;
    }
    if (tid < 24) {
        const int q = tid >> 3, c = tid & 7;
        s_pc[tid] = a.pc[c * nps + (long long)seg * 3 + q];
    }
    double acc[RB][4][2];
#pragma unroll
    for (int q = 0; q < RB; ++q)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[q][c][0] = acc[q][c][1] = 0.0;

    for (int p0 = lo; p0 < hi; p0 += kGPhase) {
        const int np = min(kGPhase, hi - p0);
        __syncthreads();  // s_pc and the row tables are written; the previous batch's readers are done
        if (tid < np) {
            const int i = p0 + tid;
            const double t = rmul(a.dt, (double)i);
            const double x = rsub(t, t0);
            const double s = __ddiv_rn(rsub(t, pt0), pw);
            const double s1 = rsub(1.0, s);
            double sn, cs;
            sincos(phase_poly(s_pc, s, s1), &sn, &cs);
            s_E[tid][0] = make_double2(cs, -sn);
            sincos(phase_poly(s_pc + 16, s, s1), &sn, &cs);
            s_E[tid][1] = make_double2(cs, -sn);
            if (a.use_theta) {
                sincos(phase_poly(s_pc + 8, s, s1), &sn, &cs);
                s_E[tid][2] = make_double2(cs, -sn);
            } else {
                s_E[tid][2] = make_double2(1.0, 0.0);
            }
            const double2 G = a.grad[i];
            s_E[tid][3] = make_double2(G.x, -G.y);  // g = conj(G)
            s_E[tid][4] = cpow_int(s_E[tid][1], a.nlo + c0);
            s_x[tid][0] = 1.0;
            s_x[tid][1] = x;
            s_x[tid][2] = x * x;
            s_x[tid][3] = x * x * x;
        }
        for (int i0 = 0; i0 < np; i0 += kGTile) {
            const int ns = min(kGTile, np - i0);
            __syncthreads();  // phase data written; the previous tile's readers are done
            // small power tables of each sample's e^{-i Phi_phi} (f = 0) and e^{-i Phi_r} (f = 1)
            if (tid < 2 * ns) {
                const int j = tid >> 1, f = tid & 1;
                const double2 E = s_E[i0 + j][f];
                double2 *T = s_P[j][f];
                double2 z = make_double2(1.0, 0.0);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    T[q] = z;
                    z = cmul(z, E);
                }
                const double2 E8 = z;
                z = make_double2(1.0, 0.0);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    T[8 + q] = z;
                    z = cmul(z, E8);
                }
            }
            __syncthreads();
            // tables: g u_r for this CTA's rows, v_{n'} = v_{c0} E_r^{n' - c0} for its columns
            for (int w = tid; w < ns * RG; w += blockDim.x) {
                const int j = w / RG, r = w - j * RG;
                double2 uu = pow_from_table(s_P[j][0], s_rm[r]);
                if (s_rk[r]) uu = cmul(uu, cpow_int(s_E[i0 + j][2], s_rk[r]));
                s_gu[j][r] = cmul(s_E[i0 + j][3], uu);
            }
            for (int w = tid; w < ns * kGCols; w += blockDim.x) {
                const int j = w / kGCols, c = w - j * kGCols;
                const double2 *T = s_P[j][1];
                s_v[j][c] = cmul(s_E[i0 + j][4], cmul(T[8 + (c >> 3)], T[c & 7]));
            }
            __syncthreads();
            for (int j = 0; j < ns; ++j) {
                const double2 v = s_v[j][col];
                const double x1 = s_x[i0 + j][1], x2 = s_x[i0 + j][2], x3 = s_x[i0 + j][3];
#pragma unroll
                for (int q = 0; q < RB; ++q) {
                    const double2 z = cmul(s_gu[j][rb * RB + q], v);
                    acc[q][0][0] += z.x;
                    acc[q][0][1] += z.y;
                    acc[q][1][0] = fma(x1, z.x, acc[q][1][0]);
                    acc[q][1][1] = fma(x1, z.y, acc[q][1][1]);
                    acc[q][2][0] = fma(x2, z.x, acc[q][2][0]);
                    acc[q][2][1] = fma(x2, z.y, acc[q][2][1]);
                    acc[q][3][0] = fma(x3, z.x, acc[q][3][0]);
                    acc[q][3][1] = fma(x3, z.y, acc[q][3][1]);
                }
            }
        }
    }
    const int n = c0 + col;
    if (n < NN) {
#pragma unroll
        for (int q = 0; q < RB; ++q) {
            const int r = r0 + rb * RB + q;
            if (r < R) {
                double2 *g = a.G + (((long long)seg * R + r) * NN + n) * 4;
#pragma unroll
                for (int c = 0; c < 4; ++c) g[c] = make_double2(acc[q][c][0], acc[q][c][1]);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Joint FP64 adjoint: G and the phase-coefficient gradients from one pass.
//
// For key (r, n') let z_i = g_i u_r(t_i) v_n(t_i) (n = nlo + n') and let
// sigma_i = x_i / w (x = t - t0, w the phase step of the segment).  The kernel
// accumulates per key the eleven moments M_p = sum_i sigma_i^p z_i, p = 0..10,
// over the samples of a work unit (part of one segment); both gradients are
// linear in them, so the units of a segment combine by plain sums:
//   G[c] = w^c M_c  (c = 0..3), and
//   dL/dcoef_{f,q} = sum_keys wt_f Im( sum_c W_c w^c sum_j beta_qj M_{j+c} ),
// with wt_f = m', k' or n for the fields phi, theta, r, W_c the forward's folded
// coefficients and beta_qj the coefficients of the basis term b_q(s) as a
// polynomial in sigma (s = sigma - (pt0 - t0) / w).  The second line holds
// because dL/dPhi_f(t_i) = Im(g_i D_f(t_i)) with D_f = sum_keys wt_f u v^n W(x),
// and b_q(s) x^c is a polynomial of degree q + c <= 10 in sigma.  Per (key,
// sample) that is one complex product and eleven complex accumulations (26 FP64
// operations) where the two separate kernels take 12 (G) plus about 17 (the
// per-sample phase sums), and the phasors are formed once.
// ---------------------------------------------------------------------------
constexpr int kJMom = 11;  // moments sigma^0 .. sigma^10

struct AdjJointArgs {
    const double2 *grad;
    const double2 *W;      // (nseg, R, NN, 4) the forward's folded coefficients
    const double *pc;
    const double *seg_info;
    const int *units;      // (nunits, 3): segment, first sample, end sample (<= 1024 samples)
    const int *row_m;
    const int *row_k;
    double2 *Gpart;        // (nunits, R, NN, 4) each unit's share of G, or null
    double *partial;       // (nunits * blocks per unit, 24) or null
    int N, R, nlo, NN, use_theta;
    double dt;
};

// Dynamic shared memory of k_adj_joint: the tile tables of k_adj_G plus the
// powers sigma^1..sigma^10 of the tile's samples and sigma of the staged ones
// (nrb row blocks of rb rows by cols columns; nrb * cols samples staged).
constexpr size_t adj_joint_smem(int nrb, int rb, int cols, int tile)
{
    return (size_t)tile * nrb * rb * sizeof(double2)           // g u_r
           + (size_t)tile * cols * sizeof(double2)              // v_{n'}
           + (size_t)tile * 2 * kGPow * sizeof(double2)         // powers of e^{-i Phi_phi}, e^{-i Phi_r}
           + (size_t)nrb * cols * 5 * sizeof(double2)           // Ep, Er, Et, g, v at this CTA's first n'
           + (size_t)tile * 5 * sizeof(double2)                 // (sigma^(2h+1), sigma^(2h+2)), h < 5
           + (size_t)nrb * cols * sizeof(double);               // sigma
}

// grid (work units, row groups of NRB*RB rows, column groups of COLS),
// NRB*COLS threads.  A work unit is at most 1024 samples of one segment, so
// the CTAs are of like size whatever the knot spacing.  The work split and the
// per-tile tables are k_adj_G's (the power tables built two threads per sample
// and phasor); each thread keeps the 11 moments of its RB keys in registers,
// samples added in order (deterministic).  The epilogue writes the unit's
// share of G and reduces the keys' phase terms over the CTA into one row of 24
// partials (field-major: phi, theta, r; 8 basis terms each).
template <int NRB, int RB, int COLS, int UNR, int TILE, int NMOM>
__global__ void __launch_bounds__(NRB * COLS, 1) k_adj_joint(AdjJointArgs a)
{
    constexpr int NT = NRB * COLS;  // threads; also the samples staged per phase batch
    constexpr int RG = NRB * RB;    // rows per CTA
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char *sp = smem_raw;
    double2 (*s_gu)[RG] = reinterpret_cast<double2 (*)[RG]>(sp);
    sp += (size_t)TILE * RG * sizeof(double2);
    double2 (*s_v)[COLS] = reinterpret_cast<double2 (*)[COLS]>(sp);
    sp += (size_t)TILE * COLS * sizeof(double2);
    double2 (*s_P)[2][kGPow] = reinterpret_cast<double2 (*)[2][kGPow]>(sp);
    sp += (size_t)TILE * 2 * kGPow * sizeof(double2);
    double2 (*s_E)[5] = reinterpret_cast<double2 (*)[5]>(sp);
    sp += (size_t)NT * 5 * sizeof(double2);
    double2 (*s_sig)[5] = reinterpret_cast<double2 (*)[5]>(sp);
    sp += (size_t)TILE * 5 * sizeof(double2);
    double *s_sx = reinterpret_cast<double *>(sp);
    __shared__ int s_rm[RG], s_rk[RG];
    __shared__ double s_pc[24];
    __shared__ double s_beta[8][8];
    __shared__ double s_red[NT / 32][24];

    const int R = a.R, NN = a.NN;
    const int u = blockIdx.x;
    const int seg = a.units[3 * u], lo = a.units[3 * u + 1], hi = a.units[3 * u + 2];
    const int r0 = blockIdx.y * RG, c0 = blockIdx.z * COLS;
    const double t0 = a.seg_info[3 * seg], pt0 = a.seg_info[3 * seg + 1], pw = a.seg_info[3 * seg + 2];
    const long long nps = (long long)(a.N - 1) * 3;
    const int tid = threadIdx.x;
    const int col = tid % COLS, rb = tid / COLS;
    for (int r = tid; r < RG; r += blockDim.x) {
        s_rm[r] = (r0 + r < R) ? a.row_m[r0 + r] : 0;
        s_rk[r] = (r0 + r < R) ? a.row_k[r0 + r] : 0;
    }
    if (tid < 24) {
        const int q = tid >> 3, c = tid & 7;
        s_pc[tid] = a.pc[c * nps + (long long)seg * 3 + q];
    }
    if (tid == 32) {
        // b_q = prod_{k < q} (k even ? s : s1) as polynomials in sigma, with
        // s = sigma - d and s1 = (1 + d) - sigma
        const double d = (pt0 - t0) / pw;
        double b[8] = {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int q = 0; q < 8; ++q) {
#pragma unroll
            for (int j = 0; j < 8; ++j) s_beta[q][j] = b[j];
            const double al = (q & 1) ? -1.0 : 1.0, ga = (q & 1) ? 1.0 + d : -d;
#pragma unroll
            for (int j = 7; j >= 0; --j) b[j] = ga * b[j] + (j ? al * b[j - 1] : 0.0);
        }
    }
    // NMOM = 11 moments for both gradients, 5 for G alone (moments 0..3 used)
    static_assert(NMOM == kJMom || NMOM == 5, "11 moments, or 5 for G alone");
    constexpr bool PHASE = NMOM == kJMom;
    double2 acc[RB][NMOM];
#pragma unroll
    for (int q = 0; q < RB; ++q)
#pragma unroll
        for (int p = 0; p < NMOM; ++p) acc[q][p] = make_double2(0.0, 0.0);

    for (int p0 = lo; p0 < hi; p0 += NT) {
        const int np = min(NT, hi - p0);
        __syncthreads();  // s_pc and the row tables are written; the previous batch's readers are done
        if (tid < np) {
            const int i = p0 + tid;
            const double t = rmul(a.dt, (double)i);
            const double x = rsub(t, t0);
            const double s = __ddiv_rn(rsub(t, pt0), pw);
            const double s1 = rsub(1.0, s);
            double sn, cs;
            sincos(phase_poly(s_pc, s, s1), &sn, &cs);
            s_E[tid][0] = make_double2(cs, -sn);
            sincos(phase_poly(s_pc + 16, s, s1), &sn, &cs);
            s_E[tid][1] = make_double2(cs, -sn);
            if (a.use_theta) {
                sincos(phase_poly(s_pc + 8, s, s1), &sn, &cs);
                s_E[tid][2] = make_double2(cs, -sn);
            } else {
                s_E[tid][2] = make_double2(1.0, 0.0);
            }
            const double2 G = a.grad[i];
            s_E[tid][3] = make_double2(G.x, -G.y);  // g = conj(G)
            s_E[tid][4] = cpow_int(s_E[tid][1], a.nlo + c0);
            s_sx[tid] = __ddiv_rn(x, pw);
        }
        for (int i0 = 0; i0 < np; i0 += TILE) {
            const int ns = min(TILE, np - i0);
            __syncthreads();  // phase data written; the previous tile's readers are done
            // power tables (two work items per sample and phasor: half h writes
            // E^{4h..4h+3} and E^{8 (4h..4h+3)}, every entry at most seven products
            // from E), then the sigma powers (one item per sample)
            for (int k = tid; k < 5 * ns; k += NT) {
                if (k < 4 * ns) {
                    const int j = k >> 2, f = (k >> 1) & 1, h = k & 1;
                    const double2 E = s_E[i0 + j][f];
                    double2 *T = s_P[j][f];
                    const double2 E2 = cmul(E, E), E4 = cmul(E2, E2), E8 = cmul(E4, E4);
                    const double2 E16 = cmul(E8, E8), E32 = cmul(E16, E16);
                    const double2 b1 = h ? E4 : make_double2(1.0, 0.0), b8 = h ? E32 : make_double2(1.0, 0.0);
                    T[4 * h] = b1;
                    T[4 * h + 1] = h ? cmul(b1, E) : E;
                    T[4 * h + 2] = h ? cmul(b1, E2) : E2;
                    T[4 * h + 3] = cmul(h ? cmul(b1, E2) : E2, E);
                    T[8 + 4 * h] = b8;
                    T[8 + 4 * h + 1] = h ? cmul(b8, E8) : E8;
                    T[8 + 4 * h + 2] = h ? cmul(b8, E16) : E16;
                    T[8 + 4 * h + 3] = cmul(h ? cmul(b8, E16) : E16, E8);
                } else {
                    const int j = k - 4 * ns;
                    const double sg = s_sx[i0 + j];
                    double *row = reinterpret_cast<double *>(s_sig[j]);
                    double pp = sg;
#pragma unroll
                    for (int q = 0; q < 10; ++q) {
                        row[q] = pp;
                        pp *= sg;
                    }
                }
            }
            __syncthreads();
            {
                // written through restrict pointers, so the loads of one entry need
                // not wait for the stores of the previous one
                const double2 *__restrict__ tP = &s_P[0][0][0];
                const double2 *__restrict__ tE = &s_E[i0][0];
                double2 *__restrict__ tgu = &s_gu[0][0];
                double2 *__restrict__ tv = &s_v[0][0];
                for (int w = tid; w < ns * RG; w += NT) {
                    const int j = w / RG, r = w - j * RG;
                    double2 uu = pow_from_table(tP + (2 * j) * kGPow, s_rm[r]);
                    if (s_rk[r]) uu = cmul(uu, cpow_int(tE[5 * j + 2], s_rk[r]));
                    tgu[w] = cmul(tE[5 * j + 3], uu);
                }
                for (int w = tid; w < ns * COLS; w += NT) {
                    const int j = w / COLS, c = w - j * COLS;
                    const double2 *T = tP + (2 * j + 1) * kGPow;
                    tv[w] = cmul(tE[5 * j + 4], cmul(T[8 + (c >> 3)], T[c & 7]));
                }
            }
            __syncthreads();
#pragma unroll UNR
            for (int j = 0; j < ns; ++j) {
                const double2 v = s_v[j][col];
                double2 z[RB];
#pragma unroll
                for (int q = 0; q < RB; ++q) {
                    z[q] = cmul(s_gu[j][rb * RB + q], v);
                    acc[q][0].x += z[q].x;
                    acc[q][0].y += z[q].y;
                }
#pragma unroll
                for (int h = 0; h < (NMOM - 1) / 2; ++h) {
                    const double2 sg = s_sig[j][h];
#pragma unroll
                    for (int q = 0; q < RB; ++q) {
                        acc[q][2 * h + 1].x = fma(sg.x, z[q].x, acc[q][2 * h + 1].x);
                        acc[q][2 * h + 1].y = fma(sg.x, z[q].y, acc[q][2 * h + 1].y);
                        acc[q][2 * h + 2].x = fma(sg.y, z[q].x, acc[q][2 * h + 2].x);
                        acc[q][2 * h + 2].y = fma(sg.y, z[q].y, acc[q][2 * h + 2].y);
                    }
                }
            }
        }
    }

    __syncthreads();  // the row and basis tables are visible even to a segment without samples
    // epilogue: G, then this thread's phase terms
    const double w1 = pw, w2 = pw * pw, w3 = w2 * pw;
    const int n = c0 + col;
    double ph[3][8];
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int q = 0; q < 8; ++q) ph[f][q] = 0.0;
#pragma unroll
    for (int q = 0; q < RB; ++q) {
        const int r = r0 + rb * RB + q;
        if (r >= R || n >= NN) continue;
        const long long key = ((long long)seg * R + r) * NN + n;
        if (a.Gpart) {  // this unit's share of G; k_adj_joint_reduce_G adds a segment's units
            double2 *g = a.Gpart + (((long long)u * R + r) * NN + n) * 4;
            g[0] = acc[q][0];
            g[1] = make_double2(acc[q][1].x * w1, acc[q][1].y * w1);
            g[2] = make_double2(acc[q][2].x * w2, acc[q][2].y * w2);
            g[3] = make_double2(acc[q][3].x * w3, acc[q][3].y * w3);
        }
        if constexpr (PHASE) if (a.partial) {
            const double2 *Wk = a.W + key * 4;
            const double2 W0 = Wk[0], W1 = Wk[1], W2 = Wk[2], W3 = Wk[3];
            const double2 om[4] = {W0, make_double2(W1.x * w1, W1.y * w1), make_double2(W2.x * w2, W2.y * w2),
                                   make_double2(W3.x * w3, W3.y * w3)};
            double iq[8];  // Im sum_c om_c M_{j+c}
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                double v = 0.0;
#pragma unroll
                for (int c = 0; c < 4; ++c) v = fma(om[c].x, acc[q][j + c].y, fma(om[c].y, acc[q][j + c].x, v));
                iq[j] = v;
            }
            const double wm = (double)s_rm[rb * RB + q];
            const double wk = a.use_theta ? (double)s_rk[rb * RB + q] : 0.0;
            const double wn = (double)(a.nlo + n);
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                double y = 0.0;
#pragma unroll
                for (int j = 0; j <= b; ++j) y = fma(s_beta[b][j], iq[j], y);
                ph[0][b] = fma(wm, y, ph[0][b]);
                ph[1][b] = fma(wk, y, ph[1][b]);
                ph[2][b] = fma(wn, y, ph[2][b]);
            }
        }
    }
    if (!PHASE || !a.partial) return;
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            double v = ph[f][q];
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0) s_red[warp][f * 8 + q] = v;
        }
    __syncthreads();
    if (tid < 24) {
        double v = 0.0;
        for (int w = 0; w < NT / 32; ++w) v += s_red[w][tid];
        const long long cta = ((long long)blockIdx.x * gridDim.y + blockIdx.y) * gridDim.z + blockIdx.z;
        a.partial[cta * 24 + tid] = v;
    }
}

// grad_pc[s][e] = sum over the segment's units and their CTAs of the partials,
// in order.
__global__ void k_adj_joint_reduce(const double *__restrict__ partial, const int *__restrict__ seg_units, int nblk,
                                   int nseg, double *__restrict__ grad_pc)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nseg * 24) return;
    const int s = idx / 24, e = idx - s * 24;
    double v = 0.0;
    for (long long b = (long long)seg_units[s] * nblk; b < (long long)seg_units[s + 1] * nblk; ++b)
        v += partial[b * 24 + e];
    grad_pc[idx] = v;
}

// G[s][key][c] = sum of the segment's unit shares, in unit order.
__global__ void k_adj_joint_reduce_G(const double2 *__restrict__ Gpart, const int *__restrict__ seg_units, int nseg,
                                     long long per_unit, double2 *__restrict__ G)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nseg * per_unit) return;
    const int s = (int)(idx / per_unit);
    const long long e = idx - (long long)s * per_unit;
    double2 v = make_double2(0.0, 0.0);
    for (int u = seg_units[s]; u < seg_units[s + 1]; ++u) {
        const double2 g = Gpart[(long long)u * per_unit + e];
        v.x += g.x;
        v.y += g.y;
    }
    G[idx] = v;
}

// Transpose of the fold: dL/d coefficient (4, N, 2K); knots >= nseg get 0.
__global__ void k_unfold(const double2 *__restrict__ G, const double2 *__restrict__ ylms,
                         const int *__restrict__ key_plus, const int *__restrict__ key_minus, int K, int N, int nseg,
                         int nkeys, double *__restrict__ gcoef)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)N * K) return;
    const int s = (int)(idx / K), j = (int)(idx - (long long)s * K);
    const long long plane = (long long)N * 2 * K;
    double gre[4] = {0.0, 0.0, 0.0, 0.0}, gim[4] = {0.0, 0.0, 0.0, 0.0};
    if (s < nseg) {
        const double2 Yp = ylms[j];
        const double2 *gp = G + ((long long)s * nkeys + key_plus[j]) * 4;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const double2 z = cmul(gp[c], Yp);
            gre[c] = z.x;    // dL/dRe a = Re(G Y+)
            gim[c] = -z.y;   // dL/dIm a = -Im(G Y+)
        }
        if (key_minus[j] >= 0) {
            const double2 Ym = ylms[K + j];
            const double2 *gm = G + ((long long)s * nkeys + key_minus[j]) * 4;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const double2 z = cmul(gm[c], Ym);
                gre[c] += z.x;   // Re(G Y-)
                gim[c] += z.y;   // +Im(G Y-)
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        gcoef[c * plane + (long long)s * 2 * K + j] = gre[c];
        gcoef[c * plane + (long long)s * 2 * K + K + j] = gim[c];
    }
}

// Transpose of k_spline_build for one series per thread.  gc (4, N, ni) knot
// major is consumed (overwritten as scratch); gy receives dL/dy through the same
// strided view the build reads y with (accumulated with += when `accumulate`).
struct SplineAdjArgs {
    const double *t;
    long long t_rs;
    double *gc;
    double *gy;
    long long sk, sp, off2;
    int split, ni, N, accumulate;
};

__global__ void __launch_bounds__(128) k_spline_adjoint(SplineAdjArgs a)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.ni) return;
    const int N = a.N;
    const double *x = a.t + (long long)p * a.t_rs;
    double *gyb = (p < a.split) ? a.gy + (long long)p * a.sp : a.gy + a.off2 + (long long)(p - a.split) * a.sp;
    const long long sk = a.sk, ni = a.ni;
    const long long plane = (long long)N * ni;
    double *g0 = a.gc + p;
    double *g1 = g0 + plane;
    double *g2 = g1 + plane;
    double *g3 = g2 + plane;

    const double x0 = x[0], x1 = x[1], x2 = x[2];
    const double h0 = x1 - x0, h1 = x2 - x1, d0 = x2 - x0;
    const double xa = x[N - 3], xb = x[N - 2], xc = x[N - 1];
    const double hA = xb - xa, hB = xc - xb, dE = xc - xa;

    // gradient of the extrapolated last-knot coefficients, folded into segment N-2
    const long long oE = (long long)(N - 1) * ni;
    const double gE1 = g1[oE], gE2 = g2[oE], gE3 = g3[oE];
    const double gy_last0 = g0[oE];

    // Pass F: slopes' gradient gs_i and the forward sweep of A~^T (interior block).
    // Stored at knot i: g1 <- c'_i, g2 <- r'_i, g3 <- direct dL/d delta_i.
    double gs_carry = 0.0;  // contribution to gs_i from segment i-1
    double w0 = 0.0, wE = 0.0;
    double cprev = 0.0, rprev = 0.0;
    for (int i = 0; i <= N - 2; ++i) {
        const long long o = (long long)i * ni;
        const double h = x[i + 1] - x[i];
        double a1 = g1[o], a2 = g2[o], a3 = g3[o];
        if (i == N - 2) {
            a1 += gE1;
            a2 += 2 * h * gE1 + gE2;
            a3 += 3 * h * h * gE1 + 3 * h * gE2 + gE3;
        }
        const double gtt = -a2 + a3 / h;
        const double gdel = a2 / h - 2.0 * gtt / h;
        const double gs_i = gs_carry + a1 - a2 / h + gtt / h;
        gs_carry = gtt / h;
        g3[o] = gdel;
        if (i == 0) {
            w0 = gs_i / h1;
        } else {
            // row i of A~^T restricted to the interior block
            double rhs = gs_i;
            if (i == 1) rhs -= d0 * w0;
            if (i == N - 2) {
                wE = gs_carry / hA;  // gs_{N-1} is complete: only segment N-2 feeds it
                rhs -= dE * wE;
            }
            const double dg = 2 * (x[i] - x[i - 1] + h) - (i == 1 ? d0 : 0.0) - (i == N - 2 ? dE : 0.0);
            const double lo = (i >= 2) ? (x[i - 1] - x[i - 2]) : 0.0;  // A~^T[i][i-1] = h_{i-2}
            const double up = (i <= N - 3) ? (x[i + 2] - x[i + 1]) : 0.0;  // A~^T[i][i+1] = h_{i+1}
            const double den = dg - lo * cprev;
            const double cp = up / den;
            const double rp = (rhs - lo * rprev) / den;
            g1[o] = cp;
            g2[o] = rp;
            cprev = cp;
            rprev = rp;
        }
    }

    // Pass B: w (= z on the interior), z_0 = w0 - w1, z_{N-1} = wE - w_{N-2};
    // gb = z feeds d delta; then dL/dy.
    const double w_last = rprev;              // w_{N-2}
    const double zE = wE - w_last;            // z_{N-1}
    // row N-1 of b: delta_{N-3} and delta_{N-2}
    const double rE_a = zE * hB * hB / dE;
    const double rE_b = zE * (2 * dE + hB) * hA / dE;
    double w_ip1 = 0.0;           // w_{i+1}
    double gdel_ip1 = 0.0;        // final d delta_{i+1}
    double pend_from_next = 0.0;  // row i+1's contribution 3 h_{i+1} z_{i+1} to d delta_i
    auto put = [&](long long knot, double v) {
        double *dst = gyb + knot * sk;
        *dst = a.accumulate ? *dst + v : v;
    };
    for (int i = N - 2; i >= 1; --i) {
        const long long o = (long long)i * ni;
        const double w_i = (i == N - 2) ? w_last : (g2[o] - g1[o] * w_ip1);
        const double hl = x[i] - x[i - 1];  // h_{i-1}
        const double hr = x[i + 1] - x[i];  // h_i
        // d delta_i: direct + row i (3 h_{i-1} z_i) + row i+1 + boundary rows
        double gdel_i = g3[o] + 3.0 * hl * w_i + pend_from_next;
        if (i == N - 2) gdel_i += rE_b;
        if (i == N - 3) gdel_i += rE_a;
        if (i == 1) gdel_i += (w0 - w_i) * h0 * h0 / d0;
        // dL/dy_{i+1} = c0 gradient + d delta_i / h_i - d delta_{i+1} / h_{i+1}
        double gy_ip1 = ((i + 1 == N - 1) ? gy_last0 : g0[o + ni]) + gdel_i / hr;
        if (i + 1 <= N - 2) gy_ip1 -= gdel_ip1 / (x[i + 2] - x[i + 1]);
        put(i + 1, gy_ip1);
        pend_from_next = 3.0 * hr * w_i;
        gdel_ip1 = gdel_i;
        w_ip1 = w_i;
        if (i == 1) {
            // delta_0: direct + row 1 + row 0 (z_0 = w_0 - w_1); then y_1 and y_0
            const double z0 = w0 - w_i;
            const double gdel0 = g3[0] + pend_from_next + z0 * (h0 + 2 * d0) * h1 / d0;
            put(1, g0[ni] + gdel0 / h0 - gdel_i / hr);
            put(0, g0[0] - gdel0 / h0);
        }
    }
}

// k_spline_adjoint for knots shared by every series, from the host
// factorization (few_spline_factor, columns 5-9 and 12-13 and the boundary
// row); loads batched ahead of the recurrences as in k_spline_build_factored.
constexpr int kAdjBatch = 8;

// Transpose of the shared-knot build, in scan form (the sweeps of the
// transposed interior block are linear recurrences with knot-only factors, as
// in k_spline_build_factored): rows 1..N-2 are cut into kScanChunks chunks,
// one warp each, lane = series (32 per CTA).
//   pass 1  dL/d slopes (gs) and dL/d delta (direct part, parked in g3), and the
//           forward sweep of A~^T from a zero carry (parked in g2); row 0 and
//           the extrapolated last knot's gradient are folded in as in the
//           sequential form; the neighbour row each chunk reads (the previous
//           segment's contribution to gs) is loaded before any warp writes;
//   carry   chained through shared memory with the chunk products (table
//           columns 12 and 13);
//   pass 2  corrected forward values and the back substitution from a zero
//           carry (parked in g2);
//   pass 3  w = corrected back substitution, dL/d delta and dL/dy for the
//           chunk's knots; the two rows past the chunk end come from the next
//           chunks' parked values and carries.
__global__ void __launch_bounds__(32 * kScanChunks) k_spline_adjoint_factored(
    const double *__restrict__ fac, double *__restrict__ gc, double *__restrict__ gy, long long sk, long long sp,
    int split, long long off2, int ni, int N, int accumulate)
{
    constexpr int W = kFacWidth;
    constexpr int P = kScanChunks;
    __shared__ double s_end[P][32];
    __shared__ double s_carry[P + 1][32];
    __shared__ double s_w0[32], s_wE[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int p0 = blockIdx.x * 32 + lane;
    const bool live = p0 < ni;
    const int p = live ? p0 : ni - 1;  // idle lanes compute on a valid series and store nothing
    double *gyb = (p < split) ? gy + (long long)p * sp : gy + off2 + (long long)(p - split) * sp;
    const long long nil = ni, plane = (long long)N * ni;
    double *g0 = gc + p;
    double *g1 = g0 + plane;
    double *g2 = g1 + plane;
    double *g3 = g2 + plane;
    const double *bnd = fac + (long long)W * N;
    const double gam0 = __ldg(bnd + 0), gam1 = __ldg(bnd + 1), d0 = __ldg(bnd + 2), h1 = __ldg(bnd + 3);
    const double e0 = __ldg(bnd + 4), e1 = __ldg(bnd + 5), dE = __ldg(bnd + 6), hA = __ldg(bnd + 7);
    const int L = (N - 2 + P - 1) / P;
    const int a = 1 + w * L, e = min(a + L, N - 1);  // rows [a, e)
    auto fa = [&](long long i, int col) { return __ldg(fac + (long long)W * i + col); };

    // neighbour row a-1 (its gtt feeds gs_a); row 0 also gives w0 and its direct term
    double carry = 0.0, w0 = 0.0, vd0 = 0.0;
    if (a < e) {
        const long long o = (long long)(a - 1) * nil;
        const double a1 = g1[o], a2 = g2[o], a3 = g3[o];
        const double ih = fa(a - 1, 6);
        const double gtt = -a2 + a3 * ih;
        carry = gtt * ih;
        if (a == 1) {
            w0 = (a1 - a2 * ih + gtt * ih) / h1;  // gs_0 has no previous segment
            vd0 = a2 * ih - 2.0 * gtt * ih;
        }
    }
    __syncthreads();
    if (w == 0) {
        s_w0[lane] = w0;
        if (live) g3[0] = vd0;
    }

    // pass 1
    double rho = 0.0, wE = 0.0;
    if (a < e) {
        const long long oE = (long long)(N - 1) * nil;
        for (int i0 = a; i0 < e; i0 += kAdjBatch) {
            double v1[kAdjBatch], v2[kAdjBatch], v3[kAdjBatch], fh[kAdjBatch], fih[kAdjBatch], flt[kAdjBatch],
                fidt[kAdjBatch];
#pragma unroll
            for (int q = 0; q < kAdjBatch; ++q) {
                const int i = min(i0 + q, e - 1);
                const long long o = (long long)i * nil;
                v1[q] = g1[o];
                v2[q] = g2[o];
                v3[q] = g3[o];
                fh[q] = fa(i, 5);
                fih[q] = fa(i, 6);
                flt[q] = fa(i, 7);
                fidt[q] = fa(i, 8);
            }
#pragma unroll
            for (int q = 0; q < kAdjBatch; ++q) {
                const int i = i0 + q;
                if (i < e) {
                    const long long o = (long long)i * nil;
                    double a1 = v1[q], a2 = v2[q], a3 = v3[q];
                    const double h = fh[q], ih = fih[q];
                    if (i == N - 2) {  // the extrapolated last knot depends on segment N-2
                        const double gE1 = g1[oE], gE2 = g2[oE], gE3 = g3[oE];
                        a1 += gE1;
                        a2 += 2 * h * gE1 + gE2;
                        a3 += 3 * h * h * gE1 + 3 * h * gE2 + gE3;
                    }
                    const double gtt = -a2 + a3 * ih;
                    double rhs = carry + a1 - a2 * ih + gtt * ih;
                    carry = gtt * ih;
                    if (live) g3[o] = a2 * ih - 2.0 * gtt * ih;  // direct dL/d delta_i
                    if (i == 1) rhs -= d0 * w0;
                    if (i == N - 2) {
                        wE = carry / hA;
                        rhs -= dE * wE;
                    }
                    rho = (rhs - flt[q] * rho) * fidt[q];
                    if (live) g2[o] = rho;
                }
            }
        }
    }
    s_end[w][lane] = rho;
    if (e == N - 1) s_wE[lane] = wE;
    __syncthreads();
    if (w == 0) {
        double c = 0.0;
        for (int q = 0; q < P; ++q) {
            s_carry[q][lane] = c;
            const int aq = 1 + q * L, eq = min(aq + L, N - 1);
            if (aq < eq) c = s_end[q][lane] + fa(eq - 1, 12) * c;
        }
    }
    __syncthreads();
    const double cf = s_carry[w][lane];

    // pass 2
    double sig = 0.0;
    if (a < e) {
        for (int i0 = e - 1; i0 >= a; i0 -= kAdjBatch) {
            double rv[kAdjBatch], fp[kAdjBatch], fct[kAdjBatch];
#pragma unroll
            for (int q = 0; q < kAdjBatch; ++q) {
                const int i = max(i0 - q, a);
                rv[q] = g2[(long long)i * nil];
                fp[q] = fa(i, 12);
                fct[q] = fa(i, 9);
            }
#pragma unroll
            for (int q = 0; q < kAdjBatch; ++q) {
                const int i = i0 - q;
                if (i >= a) {
                    const double r = fma(fp[q], cf, rv[q]);
                    sig = r - fct[q] * sig;
                    if (live) g2[(long long)i * nil] = sig;
                }
            }
        }
    }
    __syncthreads();
    s_end[w][lane] = sig;
    __syncthreads();
    if (w == 0) {
        double c = 0.0;
        for (int q = P - 1; q >= 0; --q) {
            s_carry[q][lane] = c;
            const int aq = 1 + q * L, eq = min(aq + L, N - 1);
            if (aq < eq) c = s_end[q][lane] + fa(aq, 13) * c;
        }
        s_carry[P][lane] = c;
    }
    __syncthreads();
    if (a >= e || !live) return;

    // pass 3
    const double w0v = s_w0[lane];
    const double w_last = g2[(long long)(N - 2) * nil];  // the last row's product factor is 0
    const double zE = s_wE[lane] - w_last;
    const double rE_a = zE * e0, rE_b = zE * e1;
    auto w_at = [&](int j) {  // w_j for any interior row j
        const int cj = (j - 1) / L;
        return fma(fa(j, 13), s_carry[cj][lane], g2[(long long)j * nil]);
    };
    auto gdel_at = [&](int j, double wj, double wj1) {  // dL/d delta_j given w_j, w_{j+1}
        double gd = g3[(long long)j * nil] + 3.0 * fa(j - 1, 5) * wj;
        if (j + 1 <= N - 2) gd += 3.0 * fa(j + 1, 5) * wj1;
        if (j == N - 2) gd += rE_b;
        if (j == N - 3) gd += rE_a;
        if (j == 1) gd += (w0v - wj) * gam1;
        return gd;
    };
    auto put = [&](long long knot, double v) {
        double *dst = gyb + knot * sk;
        *dst = accumulate ? *dst + v : v;
    };
    const double cb = s_carry[w][lane];
    double w_ip1 = 0.0, gdel_ip1 = 0.0;
    if (e <= N - 2) {
        w_ip1 = cb;  // w at row e
        const double w_e1 = (e + 1 <= N - 2) ? w_at(e + 1) : 0.0;
        gdel_ip1 = gdel_at(e, w_ip1, w_e1);
    }
    for (int i0 = e - 1; i0 >= a; i0 -= kAdjBatch) {
        double vs[kAdjBatch], vd[kAdjBatch], vn[kAdjBatch], fq[kAdjBatch], fhl[kAdjBatch], fhr[kAdjBatch],
            fih[kAdjBatch];
#pragma unroll
        for (int q = 0; q < kAdjBatch; ++q) {
            const int i = max(i0 - q, a);
            const long long o = (long long)i * nil;
            vs[q] = g2[o];
            vd[q] = g3[o];
            vn[q] = g0[o + nil];
            fq[q] = fa(i, 13);
            fhl[q] = fa(i - 1, 5);
            fhr[q] = fa(i + 1, 5);
            fih[q] = fa(i, 6);
        }
#pragma unroll
        for (int q = 0; q < kAdjBatch; ++q) {
            const int i = i0 - q;
            if (i >= a) {
                const double w_i = fma(fq[q], cb, vs[q]);
                double gdel_i = vd[q] + 3.0 * fhl[q] * w_i;
                if (i + 1 <= N - 2) gdel_i += 3.0 * fhr[q] * w_ip1;
                if (i == N - 2) gdel_i += rE_b;
                if (i == N - 3) gdel_i += rE_a;
                if (i == 1) gdel_i += (w0v - w_i) * gam1;
                double gy_ip1 = vn[q] + gdel_i * fih[q];
                if (i + 1 <= N - 2) gy_ip1 -= gdel_ip1 * fa(i + 1, 6);
                put(i + 1, gy_ip1);
                w_ip1 = w_i;
                gdel_ip1 = gdel_i;
            }
        }
    }
    if (w == 0) {
        // knots 1 and 0 from row 0 (after the loop: w_ip1 = w_1, gdel_ip1 = gdel_1)
        const double ih0 = fa(0, 6);
        const double gdel0 = g3[0] + 3.0 * fa(1, 5) * w_ip1 + (w0v - w_ip1) * gam0;
        put(1, g0[nil] + gdel0 * ih0 - gdel_ip1 * fa(1, 6));
        put(0, g0[0] - gdel0 * ih0);
    }
}

}  // namespace

int launch_spline_adjoint_factored(const double *fac, double *gc, double *gy, long long sk, long long sp, int split,
                                   long long off2, int ni, int N, int accumulate, cudaStream_t st)
{
    k_spline_adjoint_factored<<<(ni + 31) / 32, 32 * kScanChunks, 0, st>>>(fac, gc, gy, sk, sp, split, off2, ni, N,
                                                                          accumulate);
    FEW_LAUNCH_CHECK("k_spline_adjoint_factored");
    return FEW_OK;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
int launch_adj_phase(const double2 *grad, const double2 *W, const double *pc, int N, const double *seg_info,
                     const int *units, int nunits, const int *row_m, const int *row_k, int R, int nlo, int NN,
                     double dt, int use_theta, double *partial, cudaStream_t st)
{
    if (nunits == 0) return FEW_OK;
    AdjPhaseArgs a;
    a.grad = grad;
    a.W = W;
    a.pc = pc;
    a.seg_info = seg_info;
    a.units = units;
    a.row_m = row_m;
    a.row_k = row_k;
    a.partial = partial;
    a.N = N;
    a.R = R;
    a.nlo = nlo;
    a.NN = NN;
    a.use_theta = use_theta;
    a.dt = dt;
    // rows in blocks of 7 or 8 (the one that pads R less; 8 on a tie), as many
    // blocks per pass as fit beside the per-sample field array
    const long long row_bytes = (long long)NN * 4 * sizeof(double2);
    const int rb = ((R + 6) / 7 * 7 < (R + 7) / 8 * 8) ? 7 : 8;
    const int Rp = (R + rb - 1) / rb * rb;
    const long long e_bytes = (long long)(use_theta ? 3 : 2) * 1024 * sizeof(double);
    const int blocks = (int)std::min<long long>(Rp / rb, (kSmemBudget - e_bytes) / (row_bytes * rb));
    if (blocks < 1) return fail(FEW_ERR_SIZE, "adjoint: NN=%d too large for one row block in shared memory", NN);
    a.rows_per_pass = blocks * rb;
    const size_t smem = (size_t)(a.rows_per_pass * row_bytes + e_bytes);
    auto go = [&](auto kern) -> int {
        FEW_CUDA_TRY(ensure_smem_attr((const void *)kern, (int)smem));
        kern<<<nunits, kAdjThreads, smem, st>>>(a);
        FEW_LAUNCH_CHECK("k_adj_phase");
        return FEW_OK;
    };
    if (rb == 7) return use_theta ? go(k_adj_phase<7, true>) : go(k_adj_phase<7, false>);
    return use_theta ? go(k_adj_phase<8, true>) : go(k_adj_phase<8, false>);
}

int launch_adj_phase_reduce(const double *partial, const int *seg_units, int nseg, double *grad_pc, cudaStream_t st)
{
    if (nseg == 0) return FEW_OK;
    const int threads = 256;
    k_adj_phase_reduce<<<(nseg * 24 + threads - 1) / threads, threads, 0, st>>>(partial, seg_units, nseg, grad_pc);
    FEW_LAUNCH_CHECK("k_adj_phase_reduce");
    return FEW_OK;
}

int launch_adj_G(const double2 *grad, const double *pc, int N, const double *seg_info, const int *seg_start, int nseg,
                 const int *row_m, const int *row_k, int R, int nlo, int NN, double dt, int use_theta, double2 *G,
                 cudaStream_t st)
{
    if (nseg == 0) return FEW_OK;
    AdjGArgs a;
    a.grad = grad;
    a.pc = pc;
    a.seg_info = seg_info;
    a.seg_start = seg_start;
    a.row_m = row_m;
    a.row_k = row_k;
    a.G = G;
    a.N = N;
    a.R = R;
    a.nlo = nlo;
    a.NN = NN;
    a.use_theta = use_theta;
    a.key_base = 0;
    a.nkeys_pass = R * NN;
    a.dt = dt;
    const int colg = (NN + kGCols - 1) / kGCols;
    // rows per CTA = 6 row blocks x RB; take the RB with the least padding
    int best = 4, best_pad = 1 << 30;
    for (int rb : {2, 4, 6, 8}) {
        const int rg = kGRowBlocks * rb;
        const int pad = (R + rg - 1) / rg * rg - R;
        if (pad < best_pad || (pad == best_pad && rb > best)) {
            best = rb;
            best_pad = pad;
        }
    }
    const int rg = kGRowBlocks * best;
    dim3 grid(nseg, (R + rg - 1) / rg, colg);
    const size_t smem = adj_g_smem(best);
    if (best == 2) {
        FEW_CUDA_TRY(ensure_smem_attr((const void *)k_adj_G<2>, (int)smem));
        k_adj_G<2><<<grid, kGThreads, smem, st>>>(a);
    } else if (best == 4) {
        FEW_CUDA_TRY(ensure_smem_attr((const void *)k_adj_G<4>, (int)smem));
        k_adj_G<4><<<grid, kGThreads, smem, st>>>(a);
    } else if (best == 6) {
        FEW_CUDA_TRY(ensure_smem_attr((const void *)k_adj_G<6>, (int)smem));
        k_adj_G<6><<<grid, kGThreads, smem, st>>>(a);
    } else {
        FEW_CUDA_TRY(ensure_smem_attr((const void *)k_adj_G<8>, (int)smem));
        k_adj_G<8><<<grid, kGThreads, smem, st>>>(a);
    }
    FEW_LAUNCH_CHECK("k_adj_G");
    return FEW_OK;
}

// Shape of the joint adjoint's CTA: NRB row blocks of RB rows by COLS columns,
// the candidate that pads the (row, column) keys least, the first listed on a
// tie.  With fewer columns per CTA the row and column tables cover fewer
// entries per key (12 x 32: 24 + 32 per sample for 768 keys; 6 x 64: 12 + 64
// for 768 keys).  Three rows per thread (7 x 3 rows x 32 columns, 224 threads,
// no padding at R = 21) took 10.74 ms against 9.86 ms for 11 x 2 x 32: seven
// warps per SM were too few.
struct JointShape {
    int nrb, rb, cols;
};
constexpr JointShape kJointShapes[] = {{12, 2, 32}, {11, 2, 32}, {6, 2, 64}, {5, 2, 64}};

static JointShape joint_shape(int R, int NN)
{
    JointShape best = kJointShapes[0];
    long long best_keys = -1;
    for (const JointShape &c : kJointShapes) {
        const int rg = c.rb * c.nrb;
        const long long keys = (long long)((R + rg - 1) / rg * rg) * ((NN + c.cols - 1) / c.cols * c.cols);
        if (best_keys < 0 || keys < best_keys) {
            best = c;
            best_keys = keys;
        }
    }
    return best;
}

long long adj_joint_blocks(int R, int NN)
{
    const JointShape sh = joint_shape(R, NN);
    const int rg = sh.rb * sh.nrb;
    return (long long)((R + rg - 1) / rg) * ((NN + sh.cols - 1) / sh.cols);
}

long long adj_joint_scratch(int nunits, int R, int NN)
{
    // each unit's share of G (R NN 4 complex), then the CTAs' phase partials
    return (long long)nunits * R * NN * 8 + (long long)nunits * adj_joint_blocks(R, NN) * 24;
}

int launch_adj_joint(const double2 *grad, const double2 *W, const double *pc, int N, const double *seg_info,
                     const int *units, int nunits, const int *seg_units, int nseg, const int *row_m, const int *row_k,
                     int R, int nlo, int NN, double dt, int use_theta, double2 *G, double *grad_pc, double *scratch,
                     cudaStream_t st)
{
    if (nunits == 0 || nseg == 0) return FEW_OK;
    double2 *Gpart = reinterpret_cast<double2 *>(scratch);
    double *partial = scratch + (long long)nunits * R * NN * 8;
    AdjJointArgs a;
    a.grad = grad;
    a.W = W;
    a.pc = pc;
    a.seg_info = seg_info;
    a.units = units;
    a.row_m = row_m;
    a.row_k = row_k;
    a.Gpart = G ? Gpart : nullptr;
    a.partial = grad_pc ? partial : nullptr;
    a.N = N;
    a.R = R;
    a.nlo = nlo;
    a.NN = NN;
    a.use_theta = use_theta;
    a.dt = dt;
    if (!grad_pc) {
        // G alone: five moments per key (0..3 used), 6 row blocks of 4 rows x 64
        // columns, 64-sample tiles
        dim3 grid(nunits, (R + 23) / 24, (NN + 63) / 64);
        const size_t smem = adj_joint_smem(6, 4, 64, 64);
        auto kern = k_adj_joint<6, 4, 64, 2, 64, 5>;
        FEW_CUDA_TRY(ensure_smem_attr((const void *)kern, (int)smem));
        kern<<<grid, 384, smem, st>>>(a);
        FEW_LAUNCH_CHECK("k_adj_joint");
        return launch_reduce_unit_G(Gpart, seg_units, nseg, (long long)R * NN * 4, G, st);
    }
    const JointShape sh = joint_shape(R, NN);
    const int rg = sh.rb * sh.nrb, nt = sh.nrb * sh.cols;
    dim3 grid(nunits, (R + rg - 1) / rg, (NN + sh.cols - 1) / sh.cols);
    // 128-sample tiles (half the table barriers per sample: 9.85 against 9.93 ms at
    // the one-year waveform) where their tables fit shared memory, else 64
    const int tile = adj_joint_smem(sh.nrb, sh.rb, sh.cols, 128) + 4096 <= 227 * 1024 ? 128 : 64;
    const size_t smem = adj_joint_smem(sh.nrb, sh.rb, sh.cols, tile);
    auto go = [&](auto kern) -> int {
        FEW_CUDA_TRY(ensure_smem_attr((const void *)kern, (int)smem));
        kern<<<grid, nt, smem, st>>>(a);
        FEW_LAUNCH_CHECK("k_adj_joint");
        return FEW_OK;
    };
    int rc;
    if (tile == 64) {
        if (sh.nrb == 12)
            rc = go(k_adj_joint<12, 2, 32, 2, 64, kJMom>);
        else if (sh.nrb == 11)
            rc = go(k_adj_joint<11, 2, 32, 2, 64, kJMom>);
        else if (sh.nrb == 6)
            rc = go(k_adj_joint<6, 2, 64, 2, 64, kJMom>);
        else
            rc = go(k_adj_joint<5, 2, 64, 2, 64, kJMom>);
    } else {
        if (sh.nrb == 12)
            rc = go(k_adj_joint<12, 2, 32, 2, 128, kJMom>);
        else if (sh.nrb == 11)
            rc = go(k_adj_joint<11, 2, 32, 2, 128, kJMom>);
        else if (sh.nrb == 6)
            rc = go(k_adj_joint<6, 2, 64, 2, 128, kJMom>);
        else
            rc = go(k_adj_joint<5, 2, 64, 2, 128, kJMom>);
    }
    if (rc != FEW_OK) return rc;
    const int threads = 256;
    if (G) {
        const int rg_ = launch_reduce_unit_G(Gpart, seg_units, nseg, (long long)R * NN * 4, G, st);
        if (rg_ != FEW_OK) return rg_;
    }
    if (grad_pc) {
        const int nblk = (int)(grid.y * grid.z);
        k_adj_joint_reduce<<<(nseg * 24 + threads - 1) / threads, threads, 0, st>>>(partial, seg_units, nblk, nseg,
                                                                                  grad_pc);
        FEW_LAUNCH_CHECK("k_adj_joint_reduce");
    }
    return FEW_OK;
}

int launch_reduce_unit_G(const double2 *Gpart, const int *seg_units, int nseg, long long per_unit, double2 *G,
                         cudaStream_t st)
{
    const long long total = (long long)nseg * per_unit;
    if (total == 0) return FEW_OK;
    const int threads = 256;
    k_adj_joint_reduce_G<<<(unsigned)((total + threads - 1) / threads), threads, 0, st>>>(Gpart, seg_units, nseg,
                                                                                         per_unit, G);
    FEW_LAUNCH_CHECK("k_adj_joint_reduce_G");
    return FEW_OK;
}

int launch_unfold(const double2 *G, const double2 *ylms, const int *key_plus, const int *key_minus, int K, int N,
                  int nseg, int nkeys, double *gcoef, cudaStream_t st)
{
    const long long total = (long long)N * K;
    const int threads = 256;
    k_unfold<<<(unsigned)((total + threads - 1) / threads), threads, 0, st>>>(G, ylms, key_plus, key_minus, K, N, nseg,
                                                                             nkeys, gcoef);
    FEW_LAUNCH_CHECK("k_unfold");
    return FEW_OK;
}

int launch_spline_adjoint(const double *t, long long t_rs, double *gc, double *gy, long long sk, long long sp,
                          int split, long long off2, int ni, int N, int accumulate, cudaStream_t st)
{
    SplineAdjArgs a;
    a.t = t;
    a.t_rs = t_rs;
    a.gc = gc;
    a.gy = gy;
    a.sk = sk;
    a.sp = sp;
    a.off2 = off2;
    a.split = split;
    a.ni = ni;
    a.N = N;
    a.accumulate = accumulate;
    const int threads = 128;
    k_spline_adjoint<<<(ni + threads - 1) / threads, threads, 0, st>>>(a);
    FEW_LAUNCH_CHECK("k_spline_adjoint");
    return FEW_OK;
}

}  // namespace few

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int few_adjoint_phase(const void *grad, const void *W, const double *phase_coeffs, int N,
                                 const double *seg_info, const int *units, int nunits, const int *row_m,
                                 const int *row_k, int R, int nlo, int NN, double dt, int use_theta, double *partial,
                                 void *stream)
{
    few::clear_error();
    if (!grad || !W || !phase_coeffs || !seg_info || !units || !row_m || !row_k || !partial)
        return few::fail(FEW_ERR_ARG, "few_adjoint_phase: null pointer");
    if (N < 2 || nunits < 0 || R < 1 || R > few::kMaxRows || NN < 1)
        return few::fail(FEW_ERR_SIZE, "few_adjoint_phase: bad sizes");
    return few::launch_adj_phase((const double2 *)grad, (const double2 *)W, phase_coeffs, N, seg_info, units, nunits,
                                 row_m, row_k, R, nlo, NN, dt, use_theta, partial, (cudaStream_t)stream);
}

extern "C" int few_adjoint_phase_reduce(const double *partial, const int *seg_units, int nseg, double *grad_pc,
                                        void *stream)
{
    few::clear_error();
    if (!partial || !seg_units || !grad_pc) return few::fail(FEW_ERR_ARG, "few_adjoint_phase_reduce: null pointer");
    if (nseg < 0) return few::fail(FEW_ERR_SIZE, "few_adjoint_phase_reduce: bad sizes");
    return few::launch_adj_phase_reduce(partial, seg_units, nseg, grad_pc, (cudaStream_t)stream);
}

extern "C" int few_adjoint_G(const void *grad, const double *phase_coeffs, int N, const double *seg_info,
                             const int *seg_start, int nseg, const int *row_m, const int *row_k, int R, int nlo, int NN,
                             double dt, int use_theta, void *G, void *stream)
{
    few::clear_error();
    if (!grad || !phase_coeffs || !seg_info || !seg_start || !row_m || !row_k || !G)
        return few::fail(FEW_ERR_ARG, "few_adjoint_G: null pointer");
    if (N < 2 || nseg < 0 || nseg > N - 1 || R < 1 || R > few::kMaxRows || NN < 1)
        return few::fail(FEW_ERR_SIZE, "few_adjoint_G: bad sizes");
    return few::launch_adj_G((const double2 *)grad, phase_coeffs, N, seg_info, seg_start, nseg, row_m, row_k, R, nlo,
                             NN, dt, use_theta, (double2 *)G, (cudaStream_t)stream);
}

extern "C" long long few_adjoint_joint_scratch(int nunits, int R, int NN)
{
    if (nunits < 1 || R < 1 || NN < 1) return 0;
    return few::adj_joint_scratch(nunits, R, NN);
}

extern "C" int few_adjoint_joint(const void *grad, const void *W, const double *phase_coeffs, int N,
                                 const double *seg_info, const int *units, int nunits, const int *seg_units, int nseg,
                                 const int *row_m, const int *row_k, int R, int nlo, int NN, double dt, int use_theta,
                                 void *G, double *grad_pc, double *scratch, void *stream)
{
    few::clear_error();
    if (!grad || !phase_coeffs || !seg_info || !units || !seg_units || !row_m || !row_k || !scratch)
        return few::fail(FEW_ERR_ARG, "few_adjoint_joint: null pointer");
    if (!G && !grad_pc) return few::fail(FEW_ERR_ARG, "few_adjoint_joint: neither G nor grad_pc given");
    if (grad_pc && !W) return few::fail(FEW_ERR_ARG, "few_adjoint_joint: grad_pc needs W");
    if (N < 2 || nunits < 0 || nseg < 0 || nseg > N - 1 || R < 1 || R > few::kMaxRows || NN < 1)
        return few::fail(FEW_ERR_SIZE, "few_adjoint_joint: bad sizes");
    return few::launch_adj_joint((const double2 *)grad, (const double2 *)W, phase_coeffs, N, seg_info, units, nunits,
                                 seg_units, nseg, row_m, row_k, R, nlo, NN, dt, use_theta, (double2 *)G, grad_pc,
                                 scratch, (cudaStream_t)stream);
}

extern "C" int few_unfold(const void *G, const void *ylms, const int *key_plus, const int *key_minus, int K, int N,
                          int nseg, int nkeys, double *gcoef, void *stream)
{
    few::clear_error();
    if (!G || !ylms || !key_plus || !key_minus || !gcoef) return few::fail(FEW_ERR_ARG, "few_unfold: null pointer");
    if (K < 1 || N < 2 || nseg < 0 || nseg > N - 1 || nkeys < 1) return few::fail(FEW_ERR_SIZE, "few_unfold: bad sizes");
    return few::launch_unfold((const double2 *)G, (const double2 *)ylms, key_plus, key_minus, K, N, nseg, nkeys, gcoef,
                              (cudaStream_t)stream);
}

extern "C" int few_spline_adjoint_factored(const double *fac, double *gcoeffs, double *gy, long long y_knot_stride,
                                           long long y_interp_stride, int y_split, long long y_split_offset,
                                           int ninterps, int length, int accumulate, void *stream)
{
    few::clear_error();
    if (!fac || !gcoeffs || !gy) return few::fail(FEW_ERR_ARG, "few_spline_adjoint_factored: null pointer");
    if (ninterps < 1) return few::fail(FEW_ERR_SIZE, "few_spline_adjoint_factored: ninterps=%d < 1", ninterps);
    if (length < 4) return few::fail(FEW_ERR_SIZE, "few_spline_adjoint_factored: length=%d < 4", length);
    if (y_split < 0 || y_split > ninterps) return few::fail(FEW_ERR_ARG, "few_spline_adjoint_factored: bad y_split");
    return few::launch_spline_adjoint_factored(fac, gcoeffs, gy, y_knot_stride, y_interp_stride, y_split,
                                               y_split_offset, ninterps, length, accumulate, (cudaStream_t)stream);
}

extern "C" int few_spline_adjoint(const double *t, long long t_row_stride, double *gcoeffs, double *gy,
                                  long long y_knot_stride, long long y_interp_stride, int y_split,
                                  long long y_split_offset, int ninterps, int length, int accumulate, void *stream)
{
    few::clear_error();
    if (!t || !gcoeffs || !gy) return few::fail(FEW_ERR_ARG, "few_spline_adjoint: null pointer");
    if (ninterps < 1) return few::fail(FEW_ERR_SIZE, "few_spline_adjoint: ninterps=%d < 1", ninterps);
    if (length < 4) return few::fail(FEW_ERR_SIZE, "few_spline_adjoint: length=%d < 4", length);
    if (y_split < 0 || y_split > ninterps) return few::fail(FEW_ERR_ARG, "few_spline_adjoint: bad y_split");
    return few::launch_spline_adjoint(t, t_row_stride, gcoeffs, gy, y_knot_stride, y_interp_stride, y_split,
                                      y_split_offset, ninterps, length, accumulate, (cudaStream_t)stream);
}
