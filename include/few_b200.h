/*
 * few_b200.h -- C ABI of the B200-native interpolated mode sum
 * (libfew_b200.so, built from fastemriwaveforms_b200/csrc).
 *
 * The reference reaches its native code through a Cython pointer shim
 * (src/few/cutils/pyinterp.pyx:25-61) that passes raw addresses to
 * interpolate_arrays and get_waveform (src/few/cutils/interpolate.hh:27-31).
 * This header is the replacement boundary: plain pointers and sizes, no
 * Python or torch types.  Differences from the reference's functions:
 *   - every entry point returns an int status (FEW_OK or a negative FEW_ERR_*)
 *     instead of calling exit() on a CUDA error (global.h:49-57);
 *     few_last_error() gives the message of the last failure on this thread;
 *   - every device entry point takes the CUDA stream to run on (void *, a
 *     cudaStream_t; NULL is the legacy default stream) and returns without
 *     synchronising, unless its comment says otherwise;
 *   - pointers marked [device] are device memory, [host] host memory.
 * Complex arrays are interleaved (re, im) double pairs, i.e. complex128.
 */
#ifndef FEW_B200_H
#define FEW_B200_H

#if defined(__GNUC__)
#define FEW_API __attribute__((visibility("default")))
#else
#define FEW_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define FEW_OK 0
#define FEW_ERR_ARG (-1)      /* null pointer or invalid argument value          */
#define FEW_ERR_SIZE (-2)     /* size out of the supported range                 */
#define FEW_ERR_CUDA (-3)     /* a CUDA runtime call failed                      */
#define FEW_ERR_KNOTS (-4)    /* knots unusable (see the function's comment)     */
#define FEW_ERR_NOMEM (-5)    /* host or device allocation failed                */

/* Sum precision modes (few_sum_folded `mode`). */
#define FEW_SUM_FAITHFUL 0 /* FP64; replays the reference's rounding of m*Phi_phi+k*Phi_theta+n*Phi_r */
#define FEW_SUM_EXACT 1    /* FP64; mode phasors by recurrence, the combined phase never rounded     */

/* Coefficient layouts of few_spline_build. */
#define FEW_LAYOUT_KNOT_MAJOR 0   /* (4, length, ninterps): CubicSplineInterpolant.interp_array */
#define FEW_LAYOUT_INTERP_MAJOR 1 /* (4, ninterps, length): interpolate_arrays' in-place layout */

/* One waveform of a batched (persistent) launch: device pointers to its
 * arrays, as the single-waveform entry points take them. */
typedef struct few_wave_desc {
    void *wf;                   /* (out_len,) complex, accumulated                     */
    const void *W;              /* folded coefficients (few_fold_coeffs)               */
    const void *Bpk;            /* tensor-core operand (few_fold_mixed), NULL if FP64  */
    const double *phase_coeffs; /* (8, N-1, 3)                                         */
    const double *seg_info;     /* (3*(N-1),) from few_segment_plan                    */
    const double *t_knots;      /* (N,) amplitude knots                                */
    const int *row_m;           /* (R,) fold rows                                      */
    const int *row_k;           /* (R,)                                                */
    int N, R, nlo, NN, use_theta, reserved;
    double dt;
} few_wave_desc;

/* Message of the last failed call on the calling thread ("" if none). */
FEW_API const char *few_last_error(void);

/* ABI version, bumped on any signature change. */
FEW_API int few_abi_version(void);

/* ------------------------------------------------------------------------ */
/* Reference-shaped entry points                                            */
/* ------------------------------------------------------------------------ */

/* Replaces interpolate_arrays (src/few/cutils/interpolate.hh:27,
 * interpolate.cu:284-325): not-a-knot cubic splines of `ninterps` series.
 * t_arr [device] (ninterps*length): knots, one row per interpolant.
 * interp_array [device] (4, ninterps, length): row 0 holds y on entry; rows
 * 1..3 receive c1, c2, c3 (and row 0 is rewritten with the same y).
 * B, upper_diag, diag, lower_diag [device]: the reference's caller scratch;
 * accepted for signature compatibility and not touched.
 * Requires length >= 4 (the reference reads out of bounds at length 2 and its
 * system is singular at length 3); knots strictly increasing. */
FEW_API int few_interpolate_arrays(const double *t_arr, double *interp_array, int ninterps, int length,
                           double *B, double *upper_diag, double *diag, double *lower_diag,
                           void *stream);

/* Replaces get_waveform (src/few/cutils/interpolate.hh:29-31,
 * interpolate.cu:726-797): accumulates the interpolated mode sum into
 * d_waveform.
 * d_waveform [device] (out_len,) complex: h[i] += sum over modes (caller zeroes).
 * interp_array [device] (4, init_len, 2K): CubicSplineInterpolant.interp_array.
 * phase_interp_t [host] (init_len,); h_t [host] (init_len,): knot times, read
 * on the host as in the reference.
 * phase_interp_coeffs [device] (8, init_len-1, 3) flat.
 * d_m, d_k, d_n [device] (K,) int32; d_Ylms [device] (2K,) complex, the -m
 * half already multiplied by (-1)^l.  dev: the CUDA device to use.
 * This entry point copies m, k, n to the host and synchronises `stream`
 * before it returns (the reference synchronises after every launch).
 * Uses FEW_SUM_FAITHFUL.  FEW_ERR_KNOTS when no knot reaches the last
 * output sample (undefined in the reference). */
FEW_API int few_get_waveform(void *d_waveform, const double *interp_array, const double *phase_interp_t,
                     const double *phase_interp_coeffs, const int *d_m, const int *d_k,
                     const int *d_n, int init_len, int out_len, int num_teuk_modes,
                     const void *d_Ylms, double delta_t, const double *h_t, int dev, void *stream);

/* Size of the fixed device scratch of few_get_waveform_noalloc. */
#define FEW_NOALLOC_SCRATCH_BYTES (8u << 20)

/* few_get_waveform without any device memory allocation.  No counterpart in
 * the reference: it exists for callers that cannot call cudaMalloc (or
 * cudaMallocAsync) -- a host framework that owns all device memory through
 * its own pool, an application held to a fixed device memory budget, or a
 * pipeline that must not let the CUDA driver block or synchronise inside an
 * allocation.  Arguments, layouts and results are those of few_get_waveform.
 * Its scratch is one device array of FEW_NOALLOC_SCRATCH_BYTES (8 MiB) inside
 * the library, which every GPU that loads the library holds until the process
 * exits; the waveform is built in batches of knot segments that fit it.
 * Sizes where a single knot segment's folded coefficients do not fit
 * (R * NN * 64 bytes plus the fold tables, R the (m, k) rows and NN the n
 * range of the mode list) are rejected with FEW_ERR_SIZE and a message.
 * The first call on each device looks up the array's device address (with
 * that device made current) and keeps it for the life of the process; do not
 * call the entry point on a device again after a cudaDeviceReset of it.  The
 * caller's current device is restored on return.
 * All calls on a device share the array, so calls that overlap on the GPU
 * (other threads, other streams) race and must be serialised by the caller;
 * each call writes every scratch byte it reads, so nothing needs clearing.
 * Synchronises `stream` before returning, like few_get_waveform. */
FEW_API int few_get_waveform_noalloc(void *d_waveform, const double *interp_array, const double *phase_interp_t,
                                     const double *phase_interp_coeffs, const int *d_m, const int *d_k,
                                     const int *d_n, int init_len, int out_len, int num_teuk_modes,
                                     const void *d_Ylms, double delta_t, const double *h_t, int dev,
                                     void *stream);

/* ------------------------------------------------------------------------ */
/* Spline build and evaluation (CubicSplineInterpolant)                     */
/* ------------------------------------------------------------------------ */

/* Not-a-knot cubic splines of ninterps series of `length` knots
 * (CubicSplineInterpolant.__init__, src/few/summation/interpolatedmodesum.py:35-107).
 * t [device]: knots; interpolant p uses t + p*t_row_stride (0 = shared knots).
 * y [device]: value i of interpolant p is
 *     y[i*y_knot_stride + p*y_interp_stride]                         for p <  y_split,
 *     y[y_split_offset + i*y_knot_stride + (p-y_split)*y_interp_stride] for p >= y_split
 *   (a (ninterps, length) array: strides (1, length), y_split = ninterps; the
 *   real/imaginary halves of a (length, K) complex array: strides (2K, 2),
 *   y_split = K, y_split_offset = 1).
 * coeffs [device]: (4, ...) in `layout`; must not overlap y.
 * Requires length >= 4; knots strictly increasing. */
FEW_API int few_spline_build(const double *t, long long t_row_stride, const double *y, long long y_knot_stride,
                     long long y_interp_stride, int y_split, long long y_split_offset, int ninterps,
                     int length, double *coeffs, int layout, void *stream);

/* Width of a row of few_spline_factor's table. */
#define FEW_FAC_WIDTH 16

/* Host factorization of the not-a-knot system (and of its transpose) for knots
 * t [host] (N,), shared by every series on those knots: fac [host]
 * ((N+1)*FEW_FAC_WIDTH,) (row layout in fastemriwaveforms_b200/csrc/plan.cpp).
 * FEW_ERR_KNOTS unless t increases strictly. */
FEW_API int few_spline_factor(const double *t, int N, double *fac);

/* few_spline_build for knots shared by all series, from their factorization
 * (few_spline_factor, copied to the device: fac [device]).  Same y view,
 * layouts and results as few_spline_build (to rounding); no division per
 * series. */
FEW_API int few_spline_build_factored(const double *fac, const double *y, long long y_knot_stride,
                                      long long y_interp_stride, int y_split, long long y_split_offset,
                                      int ninterps, int length, double *coeffs, int layout, void *stream);

/* Spline evaluation (CubicSplineInterpolant.__call__, interpolatedmodesum.py:161-257).
 * t [device]: knots, interpolant p uses t + p*t_row_stride (0 = shared).
 * coeffs [device] (4, length, ninterps).  tnew [device]: point j of
 * interpolant p is tnew[p*tnew_row_stride + j] (0 = shared points).
 * out [device] (ninterps, M).  flags [device] int[2]: flags[0] is set to 1 if
 * any point lies left of the first knot, flags[1] if right of the last
 * (deriv_order 0 fills those with the edge values; the caller raises for
 * derivatives, as the reference does).  deriv_order 0..3. */
FEW_API int few_spline_eval(const double *t, long long t_row_stride, const double *coeffs, int ninterps,
                    int length, const double *tnew, long long tnew_row_stride, int M, int deriv_order,
                    double *out, int *flags, void *stream);

/* ------------------------------------------------------------------------ */
/* Host planners (pure host code, no GPU)                                   */
/* ------------------------------------------------------------------------ */

/* Fold plan of the mode list.  Term (+) of mode j has phase key
 * (m_j, k_j, n_j); term (-) (m_j != 0) has key (-m_j, -k_j, -n_j).  Keys are
 * laid on a dense grid: rows = distinct (m', k') pairs sorted ascending,
 * columns n' = nlo .. nlo+NN-1.
 * Outputs: row_m, row_k [host] (max_rows,): the rows; dims [host] int[3] =
 * {R, nlo, NN}; key_ptr [host] (max_rows*NN_max+1 -- pass max_keys+1 entries)
 * and key_list [host] (2K,): contributors of key q are
 * key_list[key_ptr[q] .. key_ptr[q+1]), each 2*j (+ term) or 2*j+1 (- term),
 * in mode order.  FEW_ERR_SIZE if R > max_rows or R*NN > max_keys. */
FEW_API int few_fold_plan(const int *m, const int *k, const int *n, int K, int max_rows, int max_keys,
                  int *row_m, int *row_k, int *dims, int *key_ptr, int *key_list);

/* Segment plan (find_start_inds, interpolate.cu:694-723) and work units.
 * h_t, phase_t [host] (init_len,).  Segment j owns output samples
 * [seg_start[j], seg_start[j+1]).  seg_start [host] (init_len,);
 * seg_info [host] (3*(init_len-1),): per segment {h_t[j], phase_t[j],
 * phase_t[j+1]-phase_t[j]}; units [host] (3*max_units,): {segment, first
 * sample, end sample} for runs of at most `chunk` samples; counts [host]
 * int[2] = {segments used, units}.  FEW_ERR_KNOTS when no knot reaches the
 * last output sample; FEW_ERR_SIZE when max_units is too small
 * (init_len + out_len/chunk + 1 always suffices). */
FEW_API int few_segment_plan(const double *h_t, const double *phase_t, int init_len, int out_len, double dt,
                     int chunk, int max_units, int *seg_start, double *seg_info, int *units,
                     int *counts);

/* ------------------------------------------------------------------------ */
/* Mode-sum kernels                                                         */
/* ------------------------------------------------------------------------ */

/* Folds the amplitude splines over the modes sharing a phase key, per segment:
 * W[s][r][c'][c] = sum over contributors of Y+_j a_c(j)  (+ term)
 *                                       or Y-_j conj(a_c(j)) (- term),
 * a_c(j) = coeffs[c][s][j] + i coeffs[c][s][K+j] (spline coefficient c of
 * mode j at knot s).  coeffs [device] (4, N, 2K); ylms [device] (2K,) complex
 * (-m half times (-1)^l); key_ptr, key_list [device] from few_fold_plan;
 * W [device] (nseg, R, NN, 4) complex. */
FEW_API int few_fold_coeffs(const double *coeffs, const void *ylms, const int *key_ptr, const int *key_list,
                    int K, int N, int nseg, int R, int NN, void *W, void *stream);

/* Accumulates the folded sum into wf [device] (out_len,) complex:
 * wf[i] += sum_{r,c'} (sum_c x^c W[s][r][c'][c]) exp(-i phase_{r,c'}(t_i)),
 * t_i = i*dt, x = t_i - seg_info[s].t0, phases from the 8-term polynomials
 * phase_coeffs [device] (8, N-1, 3) at s = (t_i - pt0)/pw.
 * seg_info [device] (3*(N-1),), units [device] (3*nunits,) from
 * few_segment_plan; row_m, row_k [device] (R,); nlo, NN: the n' grid.
 * mode: FEW_SUM_FAITHFUL or FEW_SUM_EXACT.  use_theta: nonzero if any row
 * has k' != 0 (Phi_theta is then evaluated). */
FEW_API int few_sum_folded(void *wf, const void *W, const double *phase_coeffs, int N, const double *seg_info,
                   const int *units, int nunits, const int *row_m, const int *row_k, int R, int nlo,
                   int NN, double dt, int mode, int use_theta, void *stream);

/* Persistent form of few_sum_folded over many waveforms (no counterpart in
 * the reference, which launches one kernel per knot segment of one waveform):
 * descs [device] (nwave,); units4 [device] (4*nunits,) = {waveform, segment,
 * first sample, end sample}, segments' samples as few_segment_plan makes
 * them (units of one waveform must not overlap).  smem_bytes: dynamic shared
 * memory per CTA (<= 200 KiB; the largest R*NN*64 of the batch, capped);
 * ctas: persistent CTAs (0: two per SM).  mode FEW_SUM_FAITHFUL or FEW_SUM_EXACT.
 * done [device] (nwave,) or NULL: each waveform's completion time, the
 * %globaltimer nanoseconds after its last work unit, merged with atomicMax
 * (zero it first). */
FEW_API int few_sum_batched(const few_wave_desc *descs, int nwave, const int *units4, int nunits, int smem_bytes,
                            int mode, int ctas, unsigned long long *done, void *stream);

/* Writes the GPU's %globaltimer (nanoseconds) into dst [device] when the
 * stream reaches it: a time stamp that a CUDA graph can hold. */
FEW_API int few_stamp(unsigned long long *dst, void *stream);

/* ------------------------------------------------------------------------ */
/* Mixed-precision sum on tcgen05 tensor cores (no counterpart in the        */
/* reference, which computes in FP64 only)                                  */
/* ------------------------------------------------------------------------ */

/* Bytes of the tensor-core B operand for nseg segments of an R x NN fold grid
 * (0 if R > 64). */
FEW_API long long few_mixed_operand_bytes(int nseg, int R, int NN);

/* Packs the folded coefficients W (few_fold_coeffs) into the split-BF16 B
 * operand Bpk [device] (few_mixed_operand_bytes bytes): per segment the
 * coefficients are rescaled by h_s^c (h_s = t_knots[s+1] - t_knots[s]) and laid
 * out in the tensor-core tile order, 8 columns per (m', k') row (the powers of
 * tau x re/im).  t_knots [device] (N,). */
FEW_API int few_fold_mixed(const void *W, const double *t_knots, int nseg, int R, int NN, void *Bpk, void *stream);

/* Mixed-precision sum into wf [device] (out_len,) complex (accumulated):
 * FP64 phases, anchors and mod-2pi reduction; FP32 phasor recurrence
 * re-anchored every 16 n' steps; the per-segment contraction over n' on
 * tcgen05 in split BF16 with FP32 accumulation, the powers of tau and the row
 * phasors in the FP32 epilogue.  Arguments as few_sum_folded plus
 * t_knots [device] (N,) and err [device] int (set to 1 if a tensor-core wait
 * timed out; the kernel then stops early).  R <= 64. */
FEW_API int few_sum_mixed(void *wf, const void *Bpk, const double *phase_coeffs, int N, const double *seg_info,
                          const double *t_knots, const int *units, int nunits, const int *row_m, const int *row_k,
                          int R, int nlo, int NN, double dt, int use_theta, int *err, void *stream);

/* Persistent form of few_sum_mixed over many waveforms: descs [device]
 * (nwave,) with Bpk set (few_fold_mixed per waveform); units4 [device]
 * (4*nunits,) = {waveform, segment, first sample, end sample}; max_R: the
 * largest R in the batch (<= 64, sizes shared memory and TMEM); ctas:
 * persistent CTAs (0: two per SM); astages: A-operand stages per producer half
 * (1 or 2; 0: 1); bstages: depth of the B-operand ring, 2..4 bulk-copy slots
 * (0: as many as keep two CTAs per SM); err [device] int as in few_sum_mixed;
 * done as in few_sum_batched.  Results do not depend on the stage counts. */
FEW_API int few_sum_mixed_batched(const few_wave_desc *descs, int nwave, const int *units4, int nunits, int max_R,
                                  int ctas, int astages, int bstages, int *err, unsigned long long *done,
                                  void *stream);

/* ------------------------------------------------------------------------ */
/* Adjoint (no counterpart in the reference: it has no gradients)           */
/* ------------------------------------------------------------------------ */
/* For L = Re sum_i g_i h_i.  `grad` [device] (out_len,) complex is torch's
 * upstream gradient of the waveform, G = dL/dRe h + i dL/dIm h (so g = conj(G)).
 * Phasors are recomputed from the phase polynomials, not stored.  All other
 * arguments are the forward's. */

/* dL/d(phase coefficients), per work unit (units of at most 1024 samples, as
 * few_segment_plan makes them with chunk <= 1024): partial [device] (nunits, 24) =
 * sum over the unit's samples of dL/dPhi_f(t_i) b_q(s_i), f = phi, theta, r,
 * b_q the 8-term basis (1, s, s s1, s^2 s1, s^2 s1^2, s^3 s1^2, s^3 s1^3, s^4 s1^3). */
FEW_API int few_adjoint_phase(const void *grad, const void *W, const double *phase_coeffs, int N,
                              const double *seg_info, const int *units, int nunits, const int *row_m,
                              const int *row_k, int R, int nlo, int NN, double dt, int use_theta, double *partial,
                              void *stream);

/* Sums the unit partials per segment in unit order: seg_units [device]
 * (nseg+1,) = first unit of each segment; grad_pc [device] (nseg, 3, 8), the
 * layout of phase_interp_coeffs. */
FEW_API int few_adjoint_phase_reduce(const double *partial, const int *seg_units, int nseg, double *grad_pc,
                                     void *stream);

/* G [device] (nseg, R, NN, 4) complex: G[s][key][c] = sum over segment s's
 * samples of g_i x_i^c exp(-i phase_key(t_i)).  seg_start [device] (nseg+1,). */
FEW_API int few_adjoint_G(const void *grad, const double *phase_coeffs, int N, const double *seg_info,
                          const int *seg_start, int nseg, const int *row_m, const int *row_k, int R, int nlo, int NN,
                          double dt, int use_theta, void *G, void *stream);

/* Both FP64 adjoints from one pass over the samples.  Per key and work unit
 * the kernel sums the moments M_p = sum_i sigma_i^p g_i exp(-i phase_key(t_i)),
 * p = 0..10, sigma = x / (phase step); G[c] = step^c M_c, and the phase
 * gradients are the keys' moments contracted with the folded coefficients W
 * [device] (nseg, R, NN, 4) and the basis terms written as polynomials in
 * sigma.  units [device] (nunits, 3) and seg_units [device] (nseg+1,) as for
 * few_adjoint_phase and few_adjoint_phase_reduce (units of at most 1024
 * samples, those of a segment consecutive).  G [device] as few_adjoint_G, or
 * null; grad_pc [device] (nseg, 3, 8) as few_adjoint_phase_reduce writes it,
 * or null (not both null); scratch [device] few_adjoint_joint_scratch(nunits,
 * R, NN) doubles (each unit's share of G and the CTAs' phase partials, summed
 * per segment in a fixed order).  With grad_pc null the kernel keeps only the
 * moments G needs (the form the amplitude-only backward uses).  Agrees with the
 * two separate kernels to rounding (the sums are regrouped). */
FEW_API long long few_adjoint_joint_scratch(int nunits, int R, int NN);
FEW_API int few_adjoint_joint(const void *grad, const void *W, const double *phase_coeffs, int N,
                              const double *seg_info, const int *units, int nunits, const int *seg_units, int nseg,
                              const int *row_m, const int *row_k, int R, int nlo, int NN, double dt, int use_theta,
                              void *G, double *grad_pc, double *scratch, void *stream);

/* Tensor-core adjoint (no counterpart in the reference).  Same quantities as
 * few_adjoint_G and few_adjoint_phase, with the contractions on the tcgen05
 * integer tensor cores in exact arithmetic: FP64 operands (phasors, g, powers
 * of tau, folded coefficients) scaled to 32-bit integers and split into four
 * signed base-256 int8 digits, digit products summed in int32 per level and
 * combined in FP64; the results differ from the FP64 kernels by the 2^-32
 * representation of the operands only.  err [device] int is set to 1 if a tensor-core wait timed out. */

/* few_adjoint_G on the tensor cores: the contraction over each segment's
 * samples with K = samples.  t_knots [device] (N,).  R <= 64. */
FEW_API int few_adjoint_G_mixed(const void *grad, const double *phase_coeffs, int N, const double *seg_info,
                                const double *t_knots, const int *seg_start, int nseg, const int *row_m,
                                const int *row_k, int R, int nlo, int NN, double dt, int use_theta, void *G, int *err,
                                void *stream);

/* Bytes of the packed operand of the tensor-core phase adjoint (0 if R > 64):
 * per segment the column scales and the int8 digit planes. */
FEW_API long long few_mixed_adjoint_operand_bytes(int nseg, int R, int NN);

/* Packs W into the phase adjoint's operand: per (m', k') row 8 columns, the
 * real form of W[c] h^c for c = c_a + {0, 2} (Y) and of n' W[c] h^c (Z,
 * n' = nlo + column), each column scaled by its largest value and split into
 * four int8 digits. */
FEW_API int few_fold_mixed_adjoint(const void *W, const double *t_knots, int nseg, int R, int nlo, int NN, void *Bpk,
                                   void *stream);

/* few_adjoint_phase on the tensor cores: the contraction over n' against the
 * packed (Y, Z) operand, dL/dPhi per sample in an FP64 epilogue, projected on
 * the basis per work unit into partial [device] (nunits, 24).  R <= 64. */
FEW_API int few_adjoint_phase_mixed(const void *grad, const void *Bpk, const double *phase_coeffs, int N,
                                    const double *seg_info, const double *t_knots, const int *units, int nunits,
                                    const int *row_m, const int *row_k, int R, int nlo, int NN, double dt,
                                    int use_theta, double *partial, int *err, void *stream);

/* Transpose of few_fold_coeffs: gcoef [device] (4, N, 2K) = dL/d(spline
 * coefficients) (zero at knots >= nseg).  key_plus, key_minus [device] (K,):
 * key index of each mode's + and - term (-1: none). */
FEW_API int few_unfold(const void *G, const void *ylms, const int *key_plus, const int *key_minus, int K, int N,
                       int nseg, int nkeys, double *gcoef, void *stream);

/* Transpose of few_spline_build (knot-major coefficients): gcoeffs [device]
 * (4, length, ninterps) = dL/d(coefficients), overwritten as scratch; gy
 * [device] receives dL/dy through the y view of few_spline_build (written, or
 * added to when accumulate != 0). */
FEW_API int few_spline_adjoint(const double *t, long long t_row_stride, double *gcoeffs, double *gy,
                               long long y_knot_stride, long long y_interp_stride, int y_split,
                               long long y_split_offset, int ninterps, int length, int accumulate, void *stream);

/* few_spline_adjoint for knots shared by every series, from their
 * factorization (few_spline_factor copied to the device: fac [device]). */
FEW_API int few_spline_adjoint_factored(const double *fac, double *gcoeffs, double *gy, long long y_knot_stride,
                                        long long y_interp_stride, int y_split, long long y_split_offset,
                                        int ninterps, int length, int accumulate, void *stream);

/* ------------------------------------------------------------------------ */
/* Amplitudes: tensor-product B-spline grids (the producer of teuk_modes)    */
/* ------------------------------------------------------------------------ */

/* Drop-in for interp2D_wrap (src/few/cutils/AmpInterp2D.hh:6-8, kernel
 * AmpInterp2D.cu:86-208): z [device] (num_indiv_c, mx) = each coefficient grid
 * c [device] (num_indiv_c, len_indiv_c) evaluated at the points (x[i], y[i])
 * [device] (mx,) as a B-spline of degrees kx, ky (1..5) with knots tx [device]
 * (nx,), ty [device] (ny,); len_indiv_c = (nx-kx-1)(ny-ky-1); points outside
 * the knots are clamped as FITPACK does.  mx must equal my.  The values equal
 * the reference's CPU path bit for bit. */
FEW_API int few_interp2d(double *z, const double *tx, int nx, const double *ty, int ny, const double *c, int kx,
                         int ky, const double *x, int mx, const double *y, int my, int num_indiv_c, int len_indiv_c,
                         void *stream);

/* The amplitudes directly in the mode sum's layout (what AmpInterp2D.__call__,
 * src/few/amplitude/ampinterp2d.py:127-189, assembles on the host): out
 * [device] (m, nmodes) complex128, out[i][j] = grid 2 mode_j + i grid 2 mode_j + 1
 * at (x[i], y[i]), with c [device] (num_teuk_modes, 2, len_indiv_c) and
 * mode_j = mode_idx[j] [device] (nmodes,), or j when mode_idx is null. */
FEW_API int few_amp_interp2d(void *out, const double *tx, int nx, const double *ty, int ny, const double *c, int kx,
                             int ky, const double *x, const double *y, int m, const int *mode_idx, int nmodes,
                             int len_indiv_c, void *stream);

/* ------------------------------------------------------------------------ */
/* Frequency-domain sum (FDInterpolatedModeSum, fdinterp.py:92-542)         */
/* ------------------------------------------------------------------------ */

/* Kerr geodesic fundamental frequencies (get_fundamental_frequencies,
 * src/few/utils/geodesic.py:470-535, and its kernels geodesic.py:157-451):
 * for i < n, (a[i*a_stride], p[i], e[i], x[i]) [device] -> o_phi, o_theta,
 * o_r [device] (n,), each divided by denom (1 for the dimensionless
 * frequencies, 2 pi M MTSUN_SI for Hz); abs_phi != 0 stores |o_phi| (the
 * frequency-domain sum's convention).  a_stride is 0 (one spin) or 1.
 * status [device] int (may be NULL) gets bit 1 OR-ed in when an elliptic
 * modulus falls outside [0, 1] (the reference raises ValueError there). */
FEW_API int few_fundamental_frequencies(const double *a, int a_stride, const double *p, const double *e,
                                        const double *x, int n, double denom, int abs_phi, double *o_phi,
                                        double *o_theta, double *o_r, int *status, void *stream);

/* Size in bytes of one per-mode turnover record of few_fd_plan_extrema. */
FEW_API int few_fd_turn_bytes(void);

/* Turnover search of fdinterp.py:262-376 for every mode: fdense [device]
 * (3, D) = the frequency splines at the dense grid t_j = j*tn_step + tn_start
 * (j < D-1), t_{D-1} = tn_stop (numpy.linspace); t [device] (N,) knots;
 * fcoef [device] (4, N, 3) the frequency splines' coefficients (knot-major);
 * m, k, n [device] (K,).  turns [device] (K, 2) records (few_fd_turn_bytes
 * each): for the maximum and the minimum of each mode's frequency, whether it
 * is an interior turnover, its segment and the frequency at the root of the
 * cubic's derivative.  flags [device] int[2], zeroed by the caller: flags[0]
 * bit 1 some root was kept, bit 2 a segment kept both roots, bit 4 a
 * discriminant below -1e10 (the reference stops at a breakpoint() for 2 and
 * 4), bit 8 a NaN; flags[1] the number of interior turnovers (the reference
 * widens a segment only when there is exactly one, fdinterp.py:367-376). */
FEW_API int few_fd_plan_extrema(const double *fdense, int D, double tn_start, double tn_step, double tn_stop,
                                const double *t, int N, const double *fcoef, const int *m, const int *k, const int *n,
                                int K, void *turns, int *flags, void *stream);

/* Bin ranges of every (mode, segment) (fdinterp.py:271-430): fknots [device]
 * (3, N) the frequencies at the knots; turns/flags from few_fd_plan_extrema;
 * f0 = frequency[0], df = frequency[1] - frequency[0]; has_farr selects the
 * user-grid rule for positive frequencies with fpos1 = frequency[zero_index+1].
 * Outputs [device] (K*(N-1),), entry mode*(N-1)+seg: start32/end32 the
 * reference's int32 seg_start_inds/seg_end_inds; lo and count the bins its
 * kernel visits, [lo, lo+count) within [0, L). */
FEW_API int few_fd_plan_bins(const double *fknots, const int *m, const int *k, const int *n, int K, int N,
                             const void *turns, const int *flags, double f0, double df, int has_farr, double fpos1,
                             int zero_index, int L, int *start32, int *end32, int *lo, long long *count,
                             void *stream);

/* prefix [device] (E+1,) = exclusive prefix sums of count [device] (E,);
 * scratch [device] 1024 long longs. */
FEW_API int few_fd_scan(const long long *count, long long E, long long *prefix, long long *scratch, void *stream);

/* f [device] (L,) = the default two-sided grid (j - L/2) / Ldt, Ldt = L*dt
 * (fdinterp.py:398-403). */
FEW_API int few_fd_frequency_grid(double *f, int L, double Ldt, void *stream);

/* The stationary-phase sum (make_generic_kerr_waveform_fd,
 * interpolate.cu:1141-1520) over the planned bins: wf [device] (L,) complex,
 * accumulated; freq [device] (L,).  Amplitude spline coefficient q of series p
 * (0..2K-1: real parts then imaginary parts) at knot j is
 * amp[q*aq + p*ap + j*aj]; the frequency splines' (series 0..2 = f_phi,
 * f_theta, f_r) fco[q*fq + p*fp + j*fj]; phase coefficient c (0..7) of field
 * (Phi_phi, Phi_theta, Phi_r) on segment s is pc[c*pcc + field*pcf + s*pcs].
 * ylms [device] (2K) complex, the -m half already times (-1)^l.  lo, prefix
 * [device] from few_fd_plan_bins / few_fd_scan.  blocks: CTAs of 256 threads
 * (<= 0: 32 per SM); ctas_per_sm: the register budget the kernel is built for
 * (1, 2 or 3 resident CTAs per SM; <= 0: 2).  Accumulation is by FP64
 * atomics: sums are reproducible to rounding, not bit for bit. */
FEW_API int few_fd_sum(void *wf, int L, const double *freq, int zero_index, int include_minus_m, const double *amp,
                       long long aq, long long ap, long long aj, const double *fco, long long fq, long long fp,
                       long long fj, const double *pc, long long pcc, long long pcf, long long pcs,
                       const double *phase_t, const double *t, int N, const int *m, const int *k, const int *n, int K,
                       const void *ylms, const int *lo, const long long *prefix, int blocks, int ctas_per_sm,
                       void *stream);

/* (h+, hx) from the two-sided sum (fdinterp.py:518-536): out [device]
 * (2, count) complex, rows h+ and hx at bins first .. first+count-1. */
FEW_API int few_fd_finalize(const void *wf, int L, int first, int count, void *out, void *stream);

/* Drop-in for get_waveform_generic_fd (src/few/cutils/interpolate.hh:33-38):
 * the reference's argument list and layouts (interp_array (4, 2K+3, N),
 * phase_interp_coeffs (8, 3, N-1), seg_start/end_inds (K, N-1)), all
 * [device], plus the stream.  separate_modes != 0 is refused (FEW_ERR_ARG):
 * the reference kernel writes mode_i * data_length + i into a buffer of
 * data_length elements. */
FEW_API int few_get_waveform_fd(void *waveform, const double *interp_array, const double *phase_interp_t,
                                const double *phase_interp_coeffs, const int *m, const int *k, const int *n,
                                int num_teuk_modes, double delta_t, const double *old_time_arr, int init_length,
                                int data_length, const double *frequencies, const int *seg_start_inds,
                                const int *seg_end_inds, int num_segments, const void *Ylm_all, int zero_index,
                                int include_minus_m, int separate_modes, void *stream);

/* ------------------------------------------------------------------------ */
/* Harmonics and mode selection (the producers of ylms and the mode list)   */
/* ------------------------------------------------------------------------ */

/* -2 spin-weighted spherical harmonics (GetYlms, src/few/utils/ylm.py:278-365):
 * out [device] (n,) complex = Y_{l[i], m[i]}(theta, phi) for l, m [device]
 * (n,) int; with include_minus_m != 0, out holds 2n values, the second half
 * Y_{l[i], -m[i]}.  Requires 2 <= l <= 64, |m| <= l; other entries give NaN and
 * OR 1 into status [device] int (may be NULL). */
FEW_API int few_ylm(const int *l, const int *m, int n, int include_minus_m, double theta, double phi, void *out,
                    int *status, void *stream);

/* Per-mode power estimate of ModeSelector's threshold form
 * (src/few/utils/modeselector.py:393-423): teuk [device] (N, K) complex,
 * ylms [device] complex, minus_index [device] (K,) int: the ylms index of mode
 * j's -m harmonic or -1 (m = 0), psd [device] (N, K) or NULL, t [device]
 * (N,).  snr2 [device] (K,) = sum_{n<N-1} (|A Y|^2 + |conj(A) Y^-|^2) / psd
 * * (t[n+1] - t[n]), summed in knot order. */
FEW_API int few_mode_snr2(const void *teuk, int N, int K, const void *ylms, const int *minus_index,
                          const double *psd, const double *t, double *snr2, void *stream);

/* The keep rule (modeselector.py:428-434) on estimates sorted descending:
 * keep [device] (K,) int, keep[0] = 1, keep[i] = cumsum[i-1] < total
 * (1 - threshold)^2, with the cumulative sum taken in order. */
FEW_API int few_mode_keep(const double *sorted_desc, int K, double threshold, int *keep, void *stream);

/* ------------------------------------------------------------------------ */
/* Direct mode sum (DirectModeSum, src/few/summation/directmodesum.py)       */
/* ------------------------------------------------------------------------ */

/* out [device] (N,) complex = sum_j Y_j A_ij e^{-i phi_ij} + sum_{m_j > 0}
 * (-1)^l_j Y_{K+j} conj(A_ij) e^{+i phi_ij}, phi_ij = (m_j Phi_phi,i +
 * k_j Phi_theta,i) + n_j Phi_r,i (directmodesum.py:101-131): teuk [device]
 * (N, K) complex, ylms [device] (2K) complex, phases [device] (3, N), l, m, k,
 * n [device] (K,) int. */
FEW_API int few_direct_sum(const void *teuk, const void *ylms, const double *phases, const int *l, const int *m,
                           const int *k, const int *n, int N, int K, void *out, void *stream);

/* ------------------------------------------------------------------------ */
/* AAK summation (AAKSummation, src/few/summation/aakwave.py:12-196)         */
/* ------------------------------------------------------------------------ */

/* Drop-in for get_waveform of src/few/cutils/gpuAAK.hh:6-10 (kernel
 * gpuAAK.cu:181-482): waveform [device] (out_len,) complex, hI - i hII on the
 * samples the trajectory covers (segment j owns [ceil(t_j/dt), ceil(t_j+1/dt))
 * up to T = (out_len-1) dt, as gpuAAK.cu:495-519); interp_array [device]
 * (8, init_len-1, 6) = dense-output coefficients of (p, e, Y, Phi_phi,
 * Phi_theta, Phi_r); h_t [host] (init_len,).  Plus the stream; returns after
 * the kernel has finished (the reference synchronises too).  A trajectory
 * that ends before T leaves the later samples untouched (the reference reads
 * past its arrays there). */
FEW_API int few_aak_waveform(void *waveform, const double *interp_array, double M_phys, double S_phys, double mu,
                             double qS, double phiS, double qK, double phiK, double dist, int nmodes, int mich,
                             int init_len, int out_len, double delta_t, const double *h_t, void *stream);

/* The same kernel on device tables, asynchronous and without allocation:
 * waveform [device]; coef [device] (8, cstride, 6); t_knots [device] (nseg+1,);
 * first [device] (nseg+1,) the first sample of each segment by the rule above
 * (first[nseg] = one past the last sample); total = first[nseg]. */
FEW_API int few_aak_sum(void *waveform, const double *coef, int cstride, const double *t_knots, const int *first,
                        int nseg, int total, double M_phys, double S_phys, double mu, double qS, double phiS,
                        double qK, double phiK, double dist, int nmodes, int mich, double delta_t, void *stream);

/* ------------------------------------------------------------------------ */
/* Trajectory dense output (DOPR853), the producer of phase_interp_coeffs    */
/* ------------------------------------------------------------------------ */

/* One phase of DOPR853.prep_evaluate (src/few/trajectory/dopr853.py:621-758)
 * over a batch of nsys steps of a node-component system; all pointers
 * [device].  The basis of each step needs f at the step's end and at three
 * extra stages, which the caller evaluates between the phases (the ODE is the
 * trajectory's, not this library's):
 *   phase 0: in x0, h0, y0, y1 (node, nsys), dydx1 = f(x1, y1), stages
 *            (10, node, nsys) = k1..k10 as take_step leaves them (slots 2
 *            and 3 hold stages 11 and 12); out rcont[..., 0..3], the stored
 *            stages' part of rcont[..., 4..7], arg = stage 14's argument,
 *            xarg (nsys,) its time;
 *   phase 1: in k14 = f(xarg, arg); out arg, xarg of stage 15;
 *   phase 2: in k14, k15; out arg, xarg of stage 16;
 *   phase 3: in k14, k15, k16; completes rcont[..., 4..7].
 * rcont (nsys, node, 8) is the reference's layout; its components 3..5 of a
 * trajectory (Phi_phi, Phi_theta, Phi_r) are InterpolatedModeSum's
 * phase_interp_coeffs.  Sums are rounded in the reference's order. */
FEW_API int few_dopr853_dense(const double *x0, const double *h0, const double *x1, const double *y0,
                              const double *y1, const double *dydx1, const double *stages, const double *k14,
                              const double *k15, const double *k16, double *arg, double *xarg, double *rcont,
                              int node, int nsys, int phase, void *stream);

/* DOPR853.eval (order 0) and eval_derivative (orders 1..3)
 * (dopr853.py:760-875): out [device] (npts, node) at t_new [device] (npts,)
 * from coeffs [device] (nold-1, node, 8) on the knots t_old [device] (nold,).
 * t_new must lie in [t_old[0], t_old[nold-1]] (the Python layer checks and
 * raises ValueError as the reference does). */
FEW_API int few_dopr853_eval(const double *t_new, int npts, const double *t_old, int nold, const double *coeffs,
                             int node, int order, double *out, void *stream);

/* ------------------------------------------------------------------------ */
/* Measurement                                                              */
/* ------------------------------------------------------------------------ */

/* FP64 FMA throughput probe (no counterpart in the reference): `blocks` CTAs
 * of 256 threads, each thread 8 independent FMA chains of `iters` steps,
 * 16*iters flops per thread.  out [device] (blocks*256,) receives the chain
 * sums.  Used to measure the FP64 pipe peak that bounds the sum kernels. */
FEW_API int few_probe_fp64_fma(double *out, int blocks, int iters, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FEW_B200_H */
