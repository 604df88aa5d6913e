// Host-side internals shared by the translation units of libfew_b200.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "few_b200.h"

namespace few {

// Records the message of a failed call for few_last_error() and returns code.
int fail(int code, const char *fmt, ...);

// Clears the message at the start of a call.
void clear_error();

// Checks a CUDA runtime result; on failure records it and returns FEW_ERR_CUDA.
#define FEW_CUDA_TRY(expr)                                                                   \
    do {                                                                                     \
        cudaError_t few_err_ = (expr);                                                       \
        if (few_err_ != cudaSuccess)                                                         \
            return ::few::fail(FEW_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,                 \
                               cudaGetErrorString(few_err_), __FILE__, __LINE__);            \
    } while (0)

// After a kernel launch: report launch-configuration errors.
#define FEW_LAUNCH_CHECK(name)                                                               \
    do {                                                                                     \
        cudaError_t few_err_ = cudaGetLastError();                                           \
        if (few_err_ != cudaSuccess)                                                         \
            return ::few::fail(FEW_ERR_CUDA, "launch of %s failed: %s", name,                 \
                               cudaGetErrorString(few_err_));                                \
    } while (0)

// Raises a kernel's dynamic shared-memory limit once per device (not during a
// stream capture after the first call).
cudaError_t ensure_smem_attr(const void *kernel, int bytes);

// Host-side fold plan and segment plan (plan.cpp), also used by the
// reference-shaped entry point.
int fold_plan(const int *m, const int *k, const int *n, int K, int max_rows, int max_keys, int *row_m,
              int *row_k, int *dims, int *key_ptr, int *key_list);
int spline_factor(const double *x, int N, double *fac);
int segment_plan(const double *h_t, const double *phase_t, int init_len, int out_len, double dt,
                 int chunk, int max_units, int *seg_start, double *seg_info, int *units, int *counts);

// Kernel launchers (no argument validation beyond what the kernels need).
int launch_spline_build(const double *t, long long t_rs, const double *y, long long sk, long long sp,
                        int split, long long off2, int ni, int N, double *out, int layout,
                        cudaStream_t st);
int launch_fold(const double *coeffs, const double2 *ylms, const int *key_ptr, const int *key_list,
                int K, int N, int nseg, int R, int NN, double2 *W, cudaStream_t st);
int launch_sum_folded(double2 *wf, const double2 *W, const double *pc, int N, const double *seg_info,
                      const int *units, int nunits, const int *row_m, const int *row_k, int R,
                      int nlo, int NN, double dt, int mode, int use_theta, cudaStream_t st);

int launch_adj_phase(const double2 *grad, const double2 *W, const double *pc, int N, const double *seg_info,
                     const int *units, int nunits, const int *row_m, const int *row_k, int R, int nlo, int NN,
                     double dt, int use_theta, double *partial, cudaStream_t st);
int launch_adj_phase_reduce(const double *partial, const int *seg_units, int nseg, double *grad_pc, cudaStream_t st);
int launch_adj_G(const double2 *grad, const double *pc, int N, const double *seg_info, const int *seg_start, int nseg,
                 const int *row_m, const int *row_k, int R, int nlo, int NN, double dt, int use_theta, double2 *G,
                 cudaStream_t st);
long long adj_joint_blocks(int R, int NN);
long long adj_joint_scratch(int nunits, int R, int NN);
int launch_adj_joint(const double2 *grad, const double2 *W, const double *pc, int N, const double *seg_info,
                     const int *units, int nunits, const int *seg_units, int nseg, const int *row_m, const int *row_k,
                     int R, int nlo, int NN, double dt, int use_theta, double2 *G, double *grad_pc, double *scratch,
                     cudaStream_t st);
// G[s] = sum of the per-unit shares Gpart[u] (per_unit complex values each) over
// the segment's units seg_units[s] .. seg_units[s+1]-1, in unit order.
int launch_reduce_unit_G(const double2 *Gpart, const int *seg_units, int nseg, long long per_unit, double2 *G,
                         cudaStream_t st);
int launch_unfold(const double2 *G, const double2 *ylms, const int *key_plus, const int *key_minus, int K, int N,
                  int nseg, int nkeys, double *gcoef, cudaStream_t st);
int launch_spline_adjoint(const double *t, long long t_rs, double *gc, double *gy, long long sk, long long sp,
                          int split, long long off2, int ni, int N, int accumulate, cudaStream_t st);

int launch_spline_adjoint_factored(const double *fac, double *gc, double *gy, long long sk, long long sp, int split,
                                   long long off2, int ni, int N, int accumulate, cudaStream_t st);

constexpr int kFacWidth = 16;       // doubles per row of the shared spline factorization
constexpr int kScanChunks = 8;      // knot chunks of the scan form of the spline sweeps (warps per CTA)
constexpr int kMaxRows = 256;        // distinct (m', k') rows of a fold plan
constexpr int kMaxBStages = 4;       // B-operand bulk-copy slots of the tensor-core sum
constexpr int kDefaultChunk = 1024;  // output samples per work unit of the sum

}  // namespace few
