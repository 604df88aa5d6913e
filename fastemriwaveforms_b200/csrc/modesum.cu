// Folded FP64 mode sum.
//
// The reference (src/few/cutils/interpolate.cu:444-689) evaluates, for every
// output sample and every mode, a complex exponential of the rounded phase
// fl(m*Phi_phi + k*Phi_theta + n*Phi_r), the cubic amplitude, and two complex
// products, one launch per knot segment with FP64 atomics.
//
// Here the sum is regrouped without changing its value:
//   * Fold.  The phase of a term depends on its key (m', k', n') only, so per
//     knot segment s every amplitude term sharing a key is summed once:
//     W[s][key][c] = sum Y+_j a_c(j) (the +m term of mode j) and
//     sum Y-_j conj(a_c(j)) for the -m term, whose key is (-m, -k, -n) because
//     conj(exp(-i fl(phase))) = exp(-i fl(-phase)).  (k_fold_coeffs)
//   * Phasors by recurrence.  Per sample, e^{-i Phi_phi}, e^{-i Phi_r}
//     (and e^{-i Phi_theta} if used) come from one FP64 sincos each; every key
//     phasor is built from them by complex multiplication: rows (m', k') by
//     binary powering, columns n' by a running product along the n' grid.
//   * Rounding replay (FEW_SUM_FAITHFUL).  The reference rounds the combined
//     phase; the recurrence does not.  The exact difference is recovered with
//     error-free transformations: m'*Phi = p + e exactly (e = fma(m', Phi, -p)),
//     and a + b = fl(a+b) + TwoSum error.  With eps the sum of the five errors,
//     e^{-i fl(phase)} = e^{-i phase} e^{+i eps}, and |eps| < 1e-8 rad, so the
//     factor is applied as (1 + i eps).  Row-only and column-only errors are
//     folded into the row and column phasors; the one error that depends on
//     both (rounding fl(s12 + p3)) costs one TwoSum per key and sample.
//   * Per sample: h = sum_{n'} v_{n'} sum_{r} u_r (sum_c x^c W[r][n'][c]),
//     10 DFMA per key in FEW_SUM_EXACT, 18 FP64 operations per key in
//     FEW_SUM_FAITHFUL.
// One CTA owns a run of at most `chunk` samples of one segment (a work unit),
// stages that segment's W block in shared memory (broadcast reads), and each
// thread writes its own samples: no atomics, deterministic, coalesced stores.
#include <algorithm>
#include <cstdio>
#include <cstdlib>

#include "few_common.cuh"
#include "few_internal.h"

namespace few {

namespace {

constexpr int kSumThreads = 256;
constexpr int kRowBlock = 8;                   // rows held in registers at once
constexpr int kSmemBudget = 200 * 1024;        // dynamic shared memory for W per CTA

// ---------------------------------------------------------------------------
// Fold: thread per (segment, key), contributors in mode order (deterministic).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_fold_coeffs(const double *__restrict__ coeffs,
                                                     const double2 *__restrict__ ylms,
                                                     const int *__restrict__ key_ptr,
                                                     const int *__restrict__ key_list, int K, int N,
                                                     int nseg, int nkeys, double2 *__restrict__ W)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nseg * nkeys) return;
    const int s = (int)(idx / nkeys);
    const int q = (int)(idx - (long long)s * nkeys);
    const long long plane = (long long)N * 2 * K;
    const double *cs = coeffs + (long long)s * 2 * K;
    double2 acc[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] = make_double2(0.0, 0.0);
    const int b = key_ptr[q], e = key_ptr[q + 1];
    for (int it = b; it < e; ++it) {
        const int code = key_list[it];
        const int j = code >> 1;
        const bool minus = code & 1;
        const double2 Y = minus ? ylms[K + j] : ylms[j];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const double ar = cs[c * plane + j];
            const double ai = minus ? -cs[c * plane + K + j] : cs[c * plane + K + j];
            acc[c].x = fma(Y.x, ar, fma(-Y.y, ai, acc[c].x));
            acc[c].y = fma(Y.x, ai, fma(Y.y, ar, acc[c].y));
        }
    }
    double2 *w = W + idx * 4;
#pragma unroll
    for (int c = 0; c < 4; ++c) w[c] = acc[c];
}

// ---------------------------------------------------------------------------
// Sum.
// ---------------------------------------------------------------------------
struct SumArgs {
    double2 *wf;
    const double2 *W;
    const double *pc;  // (8, N-1, 3)
    const double *seg_info;
    const int *units;
    const int *row_m;
    const int *row_k;
    int N, R, nlo, NN;
    int rows_per_pass;
    int use_theta;
    double dt;
};

// Rows per pass of the folded sum: all R when their blocks of RB rows fit in
// smem_bytes, else the most whole blocks that fit (0 if not even one does).
__host__ __device__ inline int sum_rows_per_pass(int R, int NN, int RB, int smem_bytes)
{
    const int fit = smem_bytes / (NN * 4 * (int)sizeof(double2));  // rows whose coefficients fit
    if ((R + RB - 1) / RB * RB <= fit) return R;
    return fit / RB * RB;
}

// One work unit (samples [lo, hi) of segment seg) of the folded sum; the
// block's shared memory holds the segment's W rows.  Each thread carries SPT
// samples (i, i + blockDim, ...) through the key loop together, so every
// shared-memory read of W feeds SPT samples and the samples' dependency chains
// interleave.  Phi_theta is used when THETA && a.use_theta; THETA = false
// (no row with k' != 0) drops it and its phasor from the registers at compile
// time, with the same result as a.use_theta = 0.  Ends with a barrier so the
// caller may reuse shared memory.
template <int RB, bool FAITHFUL, int SPT, bool THETA>
__device__ __forceinline__ void sum_unit(const SumArgs &a, int seg, int lo, int hi, double2 *sW, int *s_rm, int *s_rk,
                                         double *s_pc)
{
    const double t0 = a.seg_info[3 * seg], pt0 = a.seg_info[3 * seg + 1], pw = a.seg_info[3 * seg + 2];
    const int R = a.R, NN = a.NN, nlo = a.nlo;
    const long long nps = (long long)(a.N - 1) * 3;
    const bool theta = THETA && a.use_theta;
    // The faithful form parks Phi_phi and e^{-i Phi_phi}, needed only at each
    // row block's start, in per-thread shared-memory slots (volatile reads, so
    // they are not kept in registers) and recomputes e^{-i nlo Phi_r} per row
    // block: the registers freed go to the key loop's schedule (8.67 -> 7.18 ms
    // on B200 at the one-year 3843-mode waveform, identical bits).  The exact
    // form is faster with them in registers.
    __shared__ double2 s_park_ep[FAITHFUL ? SPT * kSumThreads : 1];
    __shared__ double s_park_pp[FAITHFUL ? SPT * kSumThreads : 1];
    const volatile double *park_ep = reinterpret_cast<const volatile double *>(s_park_ep);
    const volatile double *park_pp = s_park_pp;

    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        s_rm[r] = a.row_m[r];
        s_rk[r] = a.row_k[r];
    }
    if (threadIdx.x < 24) {
        const int q = threadIdx.x >> 3, c = threadIdx.x & 7;  // q: 0 phi, 1 theta, 2 r
        s_pc[threadIdx.x] = a.pc[c * nps + (long long)seg * 3 + q];
    }

    for (int r0 = 0; r0 < R; r0 += a.rows_per_pass) {
        const int nrp = min(a.rows_per_pass, R - r0);
        __syncthreads();  // previous pass finished reading sW
        {
            // rows (row, n', c) in global order -> blocks of RB rows, each laid out
            // (n', row in block, c): the 4 RB coefficients one column needs are
            // contiguous (the last block of a pass may be partly unused)
            const double2 *src = a.W + ((long long)seg * R + r0) * NN * 4;
            const int count = nrp * NN * 4;
            for (int e = threadIdx.x; e < count; e += blockDim.x) {
                const int rr = e / (NN * 4), rem = e - rr * (NN * 4);
                const int blk = rr / RB, q = rr - blk * RB;
                sW[((blk * NN) + (rem >> 2)) * (RB * 4) + q * 4 + (rem & 3)] = src[e];
            }
        }
        __syncthreads();
        for (int ib = lo + threadIdx.x; ib < hi; ib += SPT * blockDim.x) {
            double x[SPT], Pp[SPT], Pr[SPT], Pt[SPT];
            double2 Ep[SPT], Er[SPT], Et[SPT], V0[SPT], h[SPT];
#pragma unroll
            for (int sm = 0; sm < SPT; ++sm) {
                // a sample past the end repeats the first one; its result is dropped
                const int i = (ib + sm * (int)blockDim.x < hi) ? ib + sm * (int)blockDim.x : ib;
                // Sample time and phases exactly as interpolate.cu:626-644.
                const double t = rmul(a.dt, (double)i);
                x[sm] = rsub(t, t0);
                const double s = __ddiv_rn(rsub(t, pt0), pw);
                const double s1 = rsub(1.0, s);
                Pp[sm] = phase_poly(s_pc, s, s1);
                Pr[sm] = phase_poly(s_pc + 16, s, s1);
                Pt[sm] = theta ? phase_poly(s_pc + 8, s, s1) : 0.0;
                double sn, cs;
                sincos(Pp[sm], &sn, &cs);
                Ep[sm] = make_double2(cs, -sn);
                if (FAITHFUL) {
                    s_park_ep[sm * kSumThreads + threadIdx.x] = Ep[sm];
                    s_park_pp[sm * kSumThreads + threadIdx.x] = Pp[sm];
                }
                sincos(Pr[sm], &sn, &cs);
                Er[sm] = make_double2(cs, -sn);
                Et[sm] = make_double2(1.0, 0.0);
                if (theta) {
                    sincos(Pt[sm], &sn, &cs);
                    Et[sm] = make_double2(cs, -sn);
                }
                if (!FAITHFUL) V0[sm] = cpow_int(Er[sm], nlo);
                h[sm] = make_double2(0.0, 0.0);
            }

            for (int rb = 0; rb < nrp; rb += RB) {
                double2 U[SPT][RB];
                double S12[SPT][RB];
                double2 Epb[SPT];
                double Ppb[SPT];
#pragma unroll
                for (int sm = 0; sm < SPT; ++sm) {
                    const int slot = sm * kSumThreads + threadIdx.x;
                    Epb[sm] = FAITHFUL ? make_double2(park_ep[2 * slot], park_ep[2 * slot + 1]) : Ep[sm];
                    Ppb[sm] = FAITHFUL ? park_pp[slot] : Pp[sm];
                }
#pragma unroll
                for (int q = 0; q < RB; ++q) {
#pragma unroll
                    for (int sm = 0; sm < SPT; ++sm) {
                        U[sm][q] = make_double2(0.0, 0.0);
                        S12[sm][q] = 0.0;
                    }
                    if (rb + q < nrp) {
                        const int mm = s_rm[r0 + rb + q], kk = s_rk[r0 + rb + q];
#pragma unroll
                        for (int sm = 0; sm < SPT; ++sm) {
                            double2 uu = cpow_int(Epb[sm], mm);
                            if (theta && kk) uu = cmul(uu, cpow_int(Et[sm], kk));
                            if (FAITHFUL) {
                                const double dm = (double)mm;
                                const double p1 = rmul(dm, Ppb[sm]);
                                const double e1 = fma(dm, Ppb[sm], -p1);
                                if (THETA) {
                                    const double dk = (double)kk;
                                    const double p2 = rmul(dk, Pt[sm]);
                                    const double e2 = fma(dk, Pt[sm], -p2);
                                    const double s12 = radd(p1, p2);
                                    const double e12 = two_sum_err(p1, p2, s12);
                                    uu = crot_small(uu, (e1 + e2) + e12);
                                    S12[sm][q] = s12;
                                } else {
                                    // fl(p1 + 0) = p1 and its TwoSum error is 0
                                    uu = crot_small(uu, e1);
                                    S12[sm][q] = p1;
                                }
                            }
                            U[sm][q] = uu;
                        }
                    }
                }
                double2 v[SPT];
#pragma unroll
                for (int sm = 0; sm < SPT; ++sm) v[sm] = FAITHFUL ? cpow_int(Er[sm], nlo) : V0[sm];
                const double2 *wrow = sW + (long long)rb * NN * 4;
                for (int c = 0; c < NN; ++c) {
                    double2 vv[SPT], T[SPT];
                    double p3[SPT];
#pragma unroll
                    for (int sm = 0; sm < SPT; ++sm) {
                        vv[sm] = v[sm];
                        p3[sm] = 0.0;
                        if (FAITHFUL) {
                            const double dn = (double)(nlo + c);
                            p3[sm] = rmul(dn, Pr[sm]);
                            vv[sm] = crot_small(v[sm], fma(dn, Pr[sm], -p3[sm]));
                        }
                        T[sm] = make_double2(0.0, 0.0);
                    }
                    const double2 *wc = wrow + c * (RB * 4);
#pragma unroll
                    for (int q = 0; q < RB; ++q) {
                        if (rb + q < nrp) {
                            const double2 *w = wc + q * 4;
                            const double2 w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3];
#pragma unroll
                            for (int sm = 0; sm < SPT; ++sm) {
                                double2 Wx;
                                Wx.x = fma(fma(fma(w3.x, x[sm], w2.x), x[sm], w1.x), x[sm], w0.x);
                                Wx.y = fma(fma(fma(w3.y, x[sm], w2.y), x[sm], w1.y), x[sm], w0.y);
                                if (FAITHFUL) {
                                    const double sp = radd(S12[sm][q], p3[sm]);
                                    Wx = crot_small(Wx, two_sum_err(S12[sm][q], p3[sm], sp));
                                }
                                T[sm].x = fma(U[sm][q].x, Wx.x, fma(-U[sm][q].y, Wx.y, T[sm].x));
                                T[sm].y = fma(U[sm][q].x, Wx.y, fma(U[sm][q].y, Wx.x, T[sm].y));
                            }
                        }
                    }
#pragma unroll
                    for (int sm = 0; sm < SPT; ++sm) {
                        h[sm].x = fma(vv[sm].x, T[sm].x, fma(-vv[sm].y, T[sm].y, h[sm].x));
                        h[sm].y = fma(vv[sm].x, T[sm].y, fma(vv[sm].y, T[sm].x, h[sm].y));
                        v[sm] = cmul(v[sm], Er[sm]);
                    }
                }
            }
#pragma unroll
            for (int sm = 0; sm < SPT; ++sm) {
                const int i = ib + sm * (int)blockDim.x;
                if (i < hi) {
                    double2 o = a.wf[i];
                    o.x += h[sm].x;
                    o.y += h[sm].y;
                    a.wf[i] = o;
                }
            }
        }
    }
    __syncthreads();
}

template <int RB, bool FAITHFUL, int SPT, bool THETA>
__global__ void __launch_bounds__(kSumThreads, (SPT == 1 || RB <= 4) ? 2 : 1) k_sum_folded(SumArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_rm[kMaxRows], s_rk[kMaxRows];
    __shared__ double s_pc[24];
    const int u = blockIdx.x;
    sum_unit<RB, FAITHFUL, SPT, THETA>(a, a.units[3 * u], a.units[3 * u + 1], a.units[3 * u + 2],
                                reinterpret_cast<double2 *>(smem_raw), s_rm, s_rk, s_pc);
}

// Persistent form: CTAs stride over the work units of many waveforms; unit u
// is {waveform, segment, first sample, end sample}.  The shared-memory budget
// is fixed at launch; rows per pass follow each waveform's NN; Phi_theta
// follows each waveform's use_theta.
template <int RB, bool FAITHFUL, int SPT>
__global__ void __launch_bounds__(kSumThreads, (SPT == 1 || RB <= 4) ? 2 : 1) k_sum_folded_batched(const few_wave_desc *__restrict__ descs,
                                                                       const int *__restrict__ units4, int nunits,
                                                                       int smem_bytes,
                                                                       unsigned long long *__restrict__ done)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_rm[kMaxRows], s_rk[kMaxRows];
    __shared__ double s_pc[24];
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int w = units4[4 * u];
        const few_wave_desc d = descs[w];
        SumArgs a;
        a.wf = (double2 *)d.wf;
        a.W = (const double2 *)d.W;
        a.pc = d.phase_coeffs;
        a.seg_info = d.seg_info;
        a.units = nullptr;
        a.row_m = d.row_m;
        a.row_k = d.row_k;
        a.N = d.N;
        a.R = d.R;
        a.nlo = d.nlo;
        a.NN = d.NN;
        a.use_theta = d.use_theta;
        a.dt = d.dt;
        a.rows_per_pass = sum_rows_per_pass(d.R, d.NN, RB, smem_bytes);
        sum_unit<RB, FAITHFUL, SPT, true>(a, units4[4 * u + 1], units4[4 * u + 2], units4[4 * u + 3],
                                    reinterpret_cast<double2 *>(smem_raw), s_rm, s_rk, s_pc);
        if (done) {  // completion time of the waveform: the latest of its units
            __syncthreads();
            if (threadIdx.x == 0) atomicMax(done + w, global_ns());
        }
    }
}

template <int RB, bool F, int SPT>
int launch_sum_t(const SumArgs &a, int nunits, size_t smem, cudaStream_t st)
{
    if (a.use_theta) {
        FEW_CUDA_TRY(ensure_smem_attr((const void *)k_sum_folded<RB, F, SPT, true>, kSmemBudget));
        k_sum_folded<RB, F, SPT, true><<<nunits, kSumThreads, smem, st>>>(a);
        FEW_LAUNCH_CHECK("k_sum_folded");
        return FEW_OK;
    }
    FEW_CUDA_TRY(ensure_smem_attr((const void *)k_sum_folded<RB, F, SPT, false>, kSmemBudget));
    k_sum_folded<RB, F, SPT, false><<<nunits, kSumThreads, smem, st>>>(a);
    FEW_LAUNCH_CHECK("k_sum_folded");
    return FEW_OK;
}

// Shape of the FP64 sum: rows held in registers (RB) x samples per thread (SPT).
struct SumShape {
    int rb, spt;
};

// Measured on B200 at the one-year 3843-mode waveform: faithful 8 rows x 2
// samples per thread (8.65 ms vs 9.17 ms for 8x1), exact 4 rows x 1 sample
// (6.32 ms vs 7.15 ms).  FEW_B200_SUM_SHAPE="RBxSPT" overrides both.
SumShape sum_shape(int mode)
{
    static const SumShape forced = [] {
        SumShape sh{0, 0};
        const char *v = getenv("FEW_B200_SUM_SHAPE");
        if (v) {
            int rb = 0, spt = 0;
            if (sscanf(v, "%dx%d", &rb, &spt) == 2 && (rb == 4 || rb == 8) && (spt == 1 || spt == 2)) sh = {rb, spt};
        }
        return sh;
    }();
    if (forced.rb) return forced;
    return mode == FEW_SUM_FAITHFUL ? SumShape{8, 2} : SumShape{4, 1};
}

template <int RB, bool F, int SPT>
int launch_batched_t(const few_wave_desc *descs, const int *units4, int nunits, int smem_bytes, int ctas,
                     unsigned long long *done,
                     cudaStream_t st)
{
    FEW_CUDA_TRY(ensure_smem_attr((const void *)k_sum_folded_batched<RB, F, SPT>, kSmemBudget));
    k_sum_folded_batched<RB, F, SPT><<<ctas, kSumThreads, smem_bytes, st>>>(descs, units4, nunits, smem_bytes, done);
    FEW_LAUNCH_CHECK("k_sum_folded_batched");
    return FEW_OK;
}

}  // namespace

int launch_sum_folded_batched(const few_wave_desc *descs, const int *units4, int nunits, int smem_bytes, int mode,
                              int ctas, unsigned long long *done, cudaStream_t st)
{
    if (nunits == 0) return FEW_OK;
    if (smem_bytes < 64 || smem_bytes > kSmemBudget)
        return fail(FEW_ERR_SIZE, "few_sum_batched: shared memory %d out of range", smem_bytes);
    if (ctas <= 0) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        ctas = 2 * sms;
    }
    ctas = std::min(ctas, nunits);
    // the same shape as the single-waveform kernel, so both give the same bits
    const SumShape sh = sum_shape(mode);
    const bool F = mode == FEW_SUM_FAITHFUL;
    if (sh.rb == 4 && sh.spt == 2)
        return F ? launch_batched_t<4, true, 2>(descs, units4, nunits, smem_bytes, ctas, done, st)
                 : launch_batched_t<4, false, 2>(descs, units4, nunits, smem_bytes, ctas, done, st);
    if (sh.rb == 8 && sh.spt == 2)
        return F ? launch_batched_t<8, true, 2>(descs, units4, nunits, smem_bytes, ctas, done, st)
                 : launch_batched_t<8, false, 2>(descs, units4, nunits, smem_bytes, ctas, done, st);
    if (sh.rb == 4)
        return F ? launch_batched_t<4, true, 1>(descs, units4, nunits, smem_bytes, ctas, done, st)
                 : launch_batched_t<4, false, 1>(descs, units4, nunits, smem_bytes, ctas, done, st);
    return F ? launch_batched_t<8, true, 1>(descs, units4, nunits, smem_bytes, ctas, done, st)
             : launch_batched_t<8, false, 1>(descs, units4, nunits, smem_bytes, ctas, done, st);
}

int launch_fold(const double *coeffs, const double2 *ylms, const int *key_ptr, const int *key_list, int K, int N,
                int nseg, int R, int NN, double2 *W, cudaStream_t st)
{
    const int nkeys = R * NN;
    const long long total = (long long)nseg * nkeys;
    if (total == 0) return FEW_OK;
    const int threads = 256;
    const long long blocks = (total + threads - 1) / threads;
    k_fold_coeffs<<<(unsigned)blocks, threads, 0, st>>>(coeffs, ylms, key_ptr, key_list, K, N, nseg, nkeys, W);
    FEW_LAUNCH_CHECK("k_fold_coeffs");
    return FEW_OK;
}

int launch_sum_folded(double2 *wf, const double2 *W, const double *pc, int N, const double *seg_info,
                      const int *units, int nunits, const int *row_m, const int *row_k, int R, int nlo, int NN,
                      double dt, int mode, int use_theta, cudaStream_t st)
{
    if (nunits == 0) return FEW_OK;
    SumArgs a;
    a.wf = wf;
    a.W = W;
    a.pc = pc;
    a.seg_info = seg_info;
    a.units = units;
    a.row_m = row_m;
    a.row_k = row_k;
    a.N = N;
    a.R = R;
    a.nlo = nlo;
    a.NN = NN;
    a.use_theta = use_theta;
    a.dt = dt;
    const long long row_bytes = (long long)NN * 4 * sizeof(double2);
    const SumShape sh = sum_shape(mode);
    const int rpp = sum_rows_per_pass(R, NN, sh.rb, kSmemBudget);
    if (rpp < 1)
        return fail(FEW_ERR_SIZE, "few_sum_folded: NN=%d too large for one row block in shared memory", NN);
    a.rows_per_pass = rpp;
    const size_t smem = (size_t)((rpp + sh.rb - 1) / sh.rb * sh.rb) * row_bytes;
    if (sh.rb == 4 && sh.spt == 2)
        return mode == FEW_SUM_FAITHFUL ? launch_sum_t<4, true, 2>(a, nunits, smem, st)
                                        : launch_sum_t<4, false, 2>(a, nunits, smem, st);
    if (sh.rb == 8 && sh.spt == 2)
        return mode == FEW_SUM_FAITHFUL ? launch_sum_t<8, true, 2>(a, nunits, smem, st)
                                        : launch_sum_t<8, false, 2>(a, nunits, smem, st);
    if (sh.rb == 4)
        return mode == FEW_SUM_FAITHFUL ? launch_sum_t<4, true, 1>(a, nunits, smem, st)
                                        : launch_sum_t<4, false, 1>(a, nunits, smem, st);
    return mode == FEW_SUM_FAITHFUL ? launch_sum_t<8, true, 1>(a, nunits, smem, st)
                                    : launch_sum_t<8, false, 1>(a, nunits, smem, st);
}

}  // namespace few

extern "C" int few_fold_coeffs(const double *coeffs, const void *ylms, const int *key_ptr, const int *key_list,
                               int K, int N, int nseg, int R, int NN, void *W, void *stream)
{
    few::clear_error();
    if (!coeffs || !ylms || !key_ptr || !key_list || !W) return few::fail(FEW_ERR_ARG, "few_fold_coeffs: null pointer");
    if (K < 1 || N < 2 || nseg < 0 || nseg > N - 1 || R < 1 || NN < 1)
        return few::fail(FEW_ERR_SIZE, "few_fold_coeffs: bad sizes");
    return few::launch_fold(coeffs, (const double2 *)ylms, key_ptr, key_list, K, N, nseg, R, NN, (double2 *)W,
                            (cudaStream_t)stream);
}

extern "C" int few_sum_batched(const few_wave_desc *descs, int nwave, const int *units4, int nunits, int smem_bytes,
                               int mode, int ctas, unsigned long long *done, void *stream)
{
    few::clear_error();
    if (!descs || !units4) return few::fail(FEW_ERR_ARG, "few_sum_batched: null pointer");
    if (nwave < 1 || nunits < 0) return few::fail(FEW_ERR_SIZE, "few_sum_batched: bad sizes");
    if (mode != FEW_SUM_FAITHFUL && mode != FEW_SUM_EXACT) return few::fail(FEW_ERR_ARG, "few_sum_batched: bad mode");
    return few::launch_sum_folded_batched(descs, units4, nunits, smem_bytes, mode, ctas, done, (cudaStream_t)stream);
}

extern "C" int few_sum_folded(void *wf, const void *W, const double *phase_coeffs, int N, const double *seg_info,
                              const int *units, int nunits, const int *row_m, const int *row_k, int R, int nlo,
                              int NN, double dt, int mode, int use_theta, void *stream)
{
    few::clear_error();
    if (!wf || !W || !phase_coeffs || !seg_info || !units || !row_m || !row_k)
        return few::fail(FEW_ERR_ARG, "few_sum_folded: null pointer");
    if (N < 2 || nunits < 0 || R < 1 || R > few::kMaxRows || NN < 1)
        return few::fail(FEW_ERR_SIZE, "few_sum_folded: bad sizes (R must be <= %d)", few::kMaxRows);
    if (mode != FEW_SUM_FAITHFUL && mode != FEW_SUM_EXACT) return few::fail(FEW_ERR_ARG, "few_sum_folded: bad mode");
    return few::launch_sum_folded((double2 *)wf, (const double2 *)W, phase_coeffs, N, seg_info, units, nunits, row_m,
                                  row_k, R, nlo, NN, dt, mode, use_theta, (cudaStream_t)stream);
}

namespace few {
namespace {
__global__ void k_stamp(unsigned long long *dst) { *dst = global_ns(); }
}  // namespace
}  // namespace few

extern "C" int few_stamp(unsigned long long *dst, void *stream)
{
    few::clear_error();
    if (!dst) return few::fail(FEW_ERR_ARG, "few_stamp: null pointer");
    few::k_stamp<<<1, 1, 0, (cudaStream_t)stream>>>(dst);
    FEW_LAUNCH_CHECK("k_stamp");
    return FEW_OK;
}
