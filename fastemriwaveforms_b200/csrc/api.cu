// Error reporting and the reference-shaped entry points of libfew_b200.so.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "few_common.cuh"
#include "few_internal.h"

namespace few {

namespace {
thread_local char g_last_error[512] = "";
}

int fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

void clear_error() { g_last_error[0] = '\0'; }

cudaError_t ensure_smem_attr(const void *kernel, int bytes)
{
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> done;  // (kernel, device) -> bytes set
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_pair(kernel, dev);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done[key] = bytes;
    return e;
}

}  // namespace few

extern "C" const char *few_last_error(void) { return few::g_last_error; }

extern "C" int few_abi_version(void) { return 4; }

extern "C" int few_interpolate_arrays(const double *t_arr, double *interp_array, int ninterps, int length, double *B,
                                      double *upper_diag, double *diag, double *lower_diag, void *stream)
{
    (void)B;
    (void)upper_diag;
    (void)diag;
    (void)lower_diag;
    few::clear_error();
    if (!t_arr || !interp_array) return few::fail(FEW_ERR_ARG, "few_interpolate_arrays: null pointer");
    if (ninterps < 1) return few::fail(FEW_ERR_SIZE, "few_interpolate_arrays: ninterps=%d < 1", ninterps);
    if (length < 4)
        return few::fail(FEW_ERR_SIZE, "few_interpolate_arrays: length=%d; not-a-knot splines need at least 4 knots",
                         length);
    // y is row 0 of interp_array, read in place; rows 1..3 receive c1..c3.
    return few::launch_spline_build(t_arr, length, interp_array, 1, length, ninterps, 0, ninterps, length,
                                    interp_array, FEW_LAYOUT_INTERP_MAJOR, (cudaStream_t)stream);
}

extern "C" int few_get_waveform(void *d_waveform, const double *interp_array, const double *phase_interp_t,
                                const double *phase_interp_coeffs, const int *d_m, const int *d_k, const int *d_n,
                                int init_len, int out_len, int num_teuk_modes, const void *d_Ylms, double delta_t,
                                const double *h_t, int dev, void *stream)
{
    few::clear_error();
    if (!d_waveform || !interp_array || !phase_interp_t || !phase_interp_coeffs || !d_m || !d_k || !d_n || !d_Ylms ||
        !h_t)
        return few::fail(FEW_ERR_ARG, "few_get_waveform: null pointer");
    if (init_len < 2 || out_len < 1 || num_teuk_modes < 1)
        return few::fail(FEW_ERR_SIZE, "few_get_waveform: bad sizes");
    const int K = num_teuk_modes;
    cudaStream_t st = (cudaStream_t)stream;
    FEW_CUDA_TRY(cudaSetDevice(dev));

    std::vector<int> m(K), k(K), n(K);
    FEW_CUDA_TRY(cudaMemcpyAsync(m.data(), d_m, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
    FEW_CUDA_TRY(cudaMemcpyAsync(k.data(), d_k, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
    FEW_CUDA_TRY(cudaMemcpyAsync(n.data(), d_n, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
    FEW_CUDA_TRY(cudaStreamSynchronize(st));

    // Fold plan.
    int mmax = 0, kmax = 0, nmax = 0;
    for (int j = 0; j < K; ++j) {
        mmax = std::max(mmax, std::abs(m[j]));
        kmax = std::max(kmax, std::abs(k[j]));
        nmax = std::max(nmax, std::abs(n[j]));
    }
    const int max_rows = few::kMaxRows;
    const long long max_keys_ll = (long long)max_rows * (2LL * nmax + 1);
    if (max_keys_ll > (1 << 24)) return few::fail(FEW_ERR_SIZE, "few_get_waveform: mode grid too large");
    const int max_keys = (int)max_keys_ll;
    std::vector<int> row_m(max_rows), row_k(max_rows), key_ptr(max_keys + 1), key_list(2 * K);
    int dims[3];
    int rc = few::fold_plan(m.data(), k.data(), n.data(), K, max_rows, max_keys, row_m.data(), row_k.data(), dims,
                            key_ptr.data(), key_list.data());
    if (rc) return rc;
    const int R = dims[0], nlo = dims[1], NN = dims[2];
    int use_theta = 0;
    for (int r = 0; r < R; ++r) use_theta |= (row_k[r] != 0);

    // Segment plan.
    const int chunk = few::kDefaultChunk;
    const int max_units = init_len + out_len / chunk + 1;
    std::vector<int> seg_start(init_len), units(3 * (size_t)max_units);
    std::vector<double> seg_info(3 * (size_t)(init_len - 1));
    int counts[2];
    rc = few::segment_plan(h_t, phase_interp_t, init_len, out_len, delta_t, chunk, max_units, seg_start.data(),
                           seg_info.data(), units.data(), counts);
    if (rc) return rc;
    const int nseg = counts[0], nunits = counts[1];

    // One stream-ordered workspace: tables, then W.
    const size_t nkeys = (size_t)R * NN;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (bytes + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_rm = take(sizeof(int) * R), o_rk = take(sizeof(int) * R);
    const size_t o_kp = take(sizeof(int) * (nkeys + 1)), o_kl = take(sizeof(int) * 2 * K);
    const size_t o_si = take(sizeof(double) * 3 * (size_t)std::max(nseg, 1));
    const size_t o_un = take(sizeof(int) * 3 * (size_t)std::max(nunits, 1));
    const size_t o_W = take(sizeof(double2) * 4 * nkeys * (size_t)std::max(nseg, 1));
    char *ws = nullptr;
    FEW_CUDA_TRY(cudaMallocAsync((void **)&ws, off, st));
    int status = FEW_OK;
    auto put = [&](size_t o, const void *src, size_t bytes) {
        if (status == FEW_OK && bytes) {
            cudaError_t e = cudaMemcpyAsync(ws + o, src, bytes, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) status = few::fail(FEW_ERR_CUDA, "few_get_waveform: upload failed: %s", cudaGetErrorString(e));
        }
    };
    put(o_rm, row_m.data(), sizeof(int) * R);
    put(o_rk, row_k.data(), sizeof(int) * R);
    put(o_kp, key_ptr.data(), sizeof(int) * (nkeys + 1));
    put(o_kl, key_list.data(), sizeof(int) * (size_t)key_ptr[nkeys]);
    put(o_si, seg_info.data(), sizeof(double) * 3 * (size_t)nseg);
    put(o_un, units.data(), sizeof(int) * 3 * (size_t)nunits);
    if (status == FEW_OK)
        status = few::launch_fold(interp_array, (const double2 *)d_Ylms, (const int *)(ws + o_kp),
                                  (const int *)(ws + o_kl), K, init_len, nseg, R, NN, (double2 *)(ws + o_W), st);
    if (status == FEW_OK)
        status = few::launch_sum_folded((double2 *)d_waveform, (const double2 *)(ws + o_W), phase_interp_coeffs,
                                        init_len, (const double *)(ws + o_si), (const int *)(ws + o_un), nunits,
                                        (const int *)(ws + o_rm), (const int *)(ws + o_rk), R, nlo, NN, delta_t,
                                        FEW_SUM_FAITHFUL, use_theta, st);
    cudaError_t e1 = cudaFreeAsync(ws, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (status != FEW_OK) return status;
    if (e1 != cudaSuccess) return few::fail(FEW_ERR_CUDA, "few_get_waveform: free failed: %s", cudaGetErrorString(e1));
    if (e2 != cudaSuccess) return few::fail(FEW_ERR_CUDA, "few_get_waveform: %s", cudaGetErrorString(e2));
    return FEW_OK;
}
