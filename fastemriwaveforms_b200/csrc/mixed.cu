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
// (LBO) and 256 B between 8-row groups (SBO).  One CTA of 128 threads owns a
// work unit (<= 1024 samples of one segment); each thread owns one sample row of
// a 128-sample tile.  K runs in chunks of 32 (16 n' x {Re, Im}); two stages:
// while the tensor cores run chunk k's MMAs (2 K-steps x 3 split products per
// group of <= 256 columns), the threads write chunk k+1 of A and its B chunk
// arrives by cp.async; an mbarrier per stage (tcgen05.commit) gates reuse.
// Every wait is bounded and a timeout sets an error word and ends the kernel
// after freeing TMEM.
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

// One work unit (samples [lo, hi) of segment seg) on the tensor cores.
// Returns false (for every thread) if a tensor-core wait timed out.
__device__ bool mixed_unit(const MixedArgs &a, int seg, int lo, int hi, unsigned char *smem_raw, MixedPipe &pp,
                           int *s_rm, int *s_rk, double *s_pc)
{
    const int tid = threadIdx.x, warp = tid >> 5;
    const int NB = a.NB;
    const int bchunk = 2 * NB * kKC * 2;               // one B chunk: hi then lo planes
    const int stage = kAStage + bchunk;
    const double t0 = a.seg_info[3 * seg], pt0 = a.seg_info[3 * seg + 1], pw = a.seg_info[3 * seg + 2];
    const double hs = a.t_knots[seg + 1] - a.t_knots[seg];
    const int R = a.R, NN = a.NN, nlo = a.nlo, nch = a.nchunks;
    const long long nps = (long long)(a.N - 1) * 3;

    for (int r = tid; r < R; r += blockDim.x) {
        s_rm[r] = a.row_m[r];
        s_rk[r] = a.row_k[r];
    }
    if (tid < 24) {
        const int q = tid >> 3, c = tid & 7;
        s_pc[tid] = a.pc[c * nps + (long long)seg * 3 + q];
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const __nv_bfloat16 *Bseg = a.Bpk + (long long)seg * nch * 2 * NB * kKC;
    bool failed = false;

    for (int base = lo; base < hi && !failed; base += kMT) {
        const int i = base + tid;
        const bool valid = i < hi;
        // FP64 prelude: phases (interpolate.cu:626-644) and anchors
        const double t = (double)i * a.dt;
        const double x = t - t0;
        const float tau = (float)(x / hs);
        const double s = (t - pt0) / pw;
        const double s1 = 1.0 - s;
        const double Pp = phase_poly(s_pc, s, s1);
        const double Pr = phase_poly(s_pc + 16, s, s1);
        const double Pt = a.use_theta ? phase_poly(s_pc + 8, s, s1) : 0.0;
        const float2 Ep = anchor(Pp);
        const float2 Er = anchor(Pr);
        const float2 Et = a.use_theta ? anchor(Pt) : make_float2(1.f, 0.f);
        const float2 Er2 = fcmul(Er, Er);
        float2 v[16];

        for (int k = 0; k < nch && !failed; ++k) {
            const int b = k & 1;
            const int nblk = k;
            // stage b is free once the MMAs of chunk k-2 are done
            if (__syncthreads_or(!pipe_drain(pp, b))) {
                failed = true;
                break;
            }
            unsigned char *const sAb = smem_raw + b * stage;
            unsigned char *const sBb = sAb + kAStage;
            {
                const unsigned char *src = reinterpret_cast<const unsigned char *>(Bseg + (long long)k * 2 * NB * kKC);
                for (int q = tid; q < bchunk / 16; q += blockDim.x) cp_async16(sBb + 16 * q, src + 16 * q);
                cp_async_commit();
            }
            {
                // two interleaved chains (even and odd n') stepping by Er^2: half the
                // dependent depth of one chain, and 8 FP32 steps from the anchor at most
                v[0] = anchor((double)(nlo + 16 * nblk) * Pr);
                v[1] = fcmul(v[0], Er);
#pragma unroll
                for (int q = 2; q < 16; ++q) v[q] = fcmul(v[q - 2], Er2);
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    if (!valid || 16 * nblk + q >= NN) v[q] = make_float2(0.f, 0.f);
            }
            unsigned char *const aH = sAb, *const aL = sAb + kMT * kKC * 2;
#pragma unroll
            for (int g = 0; g < 4; ++g) {  // 4 groups of 4 complex = 8 bf16 = 16 bytes
                uint32_t h4[4], l4[4];
#pragma unroll
                for (int e2 = 0; e2 < 4; ++e2) {
                    const float2 z = v[4 * g + e2];
                    split2(z.x, z.y, h4[e2], l4[e2]);
                }
                const uint32_t off = tile_off(tid, 8 * g, kMT / 8);
                *reinterpret_cast<uint4 *>(aH + off) = make_uint4(h4[0], h4[1], h4[2], h4[3]);
                *reinterpret_cast<uint4 *>(aL + off) = make_uint4(l4[0], l4[1], l4[2], l4[3]);
            }
            cp_async_wait_all();
            fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                tc_fence_after();
                const uint32_t a_h = smem_u32(aH), a_l = smem_u32(aL);
                const uint32_t b_h = smem_u32(sBb), b_l = b_h + NB * kKC * 2;
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
                        const uint32_t d = pp.tmem + (uint32_t)n0;
                        mma_bf16(d, da_h, db_h, idesc, (k | st) != 0);
                        mma_bf16(d, da_h, db_l, idesc, 1u);
                        mma_bf16(d, da_l, db_h, idesc, 1u);
                    }
                }
                mma_commit(&pp.bar[b]);
            }
            if (b == 0) pp.pend0 = 1;
            else pp.pend1 = 1;
        }
        if (failed) break;
        // all MMAs of the tile done before the accumulator is read
        const bool ok0 = pipe_drain(pp, 0), ok1 = pipe_drain(pp, 1);
        if (__syncthreads_or(!(ok0 && ok1))) {
            failed = true;
            break;
        }
        // epilogue: this thread's accumulator row (TMEM lane = tid); two (m', k')
        // rows of 8 columns per 16-column load; u_r by one multiplication when m'
        // steps by one
        tc_fence_after();
        const uint32_t trow = pp.tmem + ((uint32_t)(warp * 32) << 16);
        float2 uu = make_float2(1.f, 0.f);
        int pm = 0x7fffffff, pk = 0x7fffffff;
        float2 Sp = make_float2(0.f, 0.f);
        for (int c0 = 0; c0 < NB; c0 += 16) {
            float D[16];
            tmem_ld16(trow + c0, D);
            tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int r = (c0 >> 3) + q;
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
                    const float *d8 = D + 8 * q;
                    // Y = sum_c tau^c Z_c (Horner)
                    const float yr = fmaf(fmaf(fmaf(d8[6], tau, d8[4]), tau, d8[2]), tau, d8[0]);
                    const float yi = fmaf(fmaf(fmaf(d8[7], tau, d8[5]), tau, d8[3]), tau, d8[1]);
                    Sp.x = fmaf(uu.x, yr, fmaf(-uu.y, yi, Sp.x));
                    Sp.y = fmaf(uu.x, yi, fmaf(uu.y, yr, Sp.y));
                }
            }
        }
        if (valid) {
            double2 o = a.wf[i];
            o.x += (double)Sp.x;
            o.y += (double)Sp.y;
            a.wf[i] = o;
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    cp_async_wait_all();
    return !failed;
}

__global__ void __launch_bounds__(kMT, 1) k_sum_mixed(MixedArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_rm[kMaxRows], s_rk[kMaxRows];
    __shared__ double s_pc[24];
    MixedPipe pp;
    mixed_setup(&s_tmem, s_bar, a.tmem_cols, pp);
    const int u = blockIdx.x;
    const bool ok =
        mixed_unit(a, a.units[3 * u], a.units[3 * u + 1], a.units[3 * u + 2], smem_raw, pp, s_rm, s_rk, s_pc);
    mixed_teardown(!ok, pp, a.tmem_cols, a.err);
}

// Persistent form over many waveforms: TMEM and the mbarriers are set up once
// per CTA; units {waveform, segment, first, end} are taken in stride.
__global__ void __launch_bounds__(kMT, 1) k_sum_mixed_batched(const few_wave_desc *__restrict__ descs,
                                                              const int *__restrict__ units4, int nunits,
                                                              int tmem_cols, int *err,
                                                              unsigned long long *__restrict__ done)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_rm[kMaxRows], s_rk[kMaxRows];
    __shared__ double s_pc[24];
    MixedPipe pp;
    mixed_setup(&s_tmem, s_bar, tmem_cols, pp);
    bool ok = true;
    for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
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
        ok = mixed_unit(a, units4[4 * u + 1], units4[4 * u + 2], units4[4 * u + 3], smem_raw, pp, s_rm, s_rk, s_pc);
        if (done && ok && threadIdx.x == 0) atomicMax(done + units4[4 * u], global_ns());  // unit complete
    }
    mixed_teardown(!ok, pp, tmem_cols, err);
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

size_t mixed_smem_bytes(int NB) { return (size_t)2 * (kAStage + 2 * NB * kKC * 2); }

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
    const size_t smem = mixed_smem_bytes(a.NB);
    FEW_CUDA_TRY(ensure_smem_attr((const void *)k_sum_mixed, (int)smem));
    k_sum_mixed<<<nunits, kMT, smem, st>>>(a);
    FEW_LAUNCH_CHECK("k_sum_mixed");
    return FEW_OK;
}

int launch_sum_mixed_batched(const few_wave_desc *descs, const int *units4, int nunits, int max_R, int ctas, int *err,
                             unsigned long long *done, cudaStream_t st)
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
    const size_t smem = mixed_smem_bytes(NB);
    FEW_CUDA_TRY(ensure_smem_attr((const void *)k_sum_mixed_batched, (int)smem));
    k_sum_mixed_batched<<<ctas, kMT, smem, st>>>(descs, units4, nunits, cols, err, done);
    FEW_LAUNCH_CHECK("k_sum_mixed_batched");
    return FEW_OK;
}

}  // namespace few

extern "C" int few_sum_mixed_batched(const few_wave_desc *descs, int nwave, const int *units4, int nunits, int max_R,
                                     int ctas, int *err, unsigned long long *done, void *stream)
{
    few::clear_error();
    if (!descs || !units4 || !err) return few::fail(FEW_ERR_ARG, "few_sum_mixed_batched: null pointer");
    if (nwave < 1 || nunits < 0 || max_R < 1 || max_R > 64)
        return few::fail(FEW_ERR_SIZE, "few_sum_mixed_batched: bad sizes (max_R <= 64)");
    return few::launch_sum_mixed_batched(descs, units4, nunits, max_R, ctas, err, done, (cudaStream_t)stream);
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

