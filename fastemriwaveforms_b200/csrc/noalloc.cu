// few_get_waveform_noalloc: the interpolated mode sum without any device
// memory allocation.
//
// Who needs it: few_get_waveform takes a stream-ordered workspace from
// cudaMallocAsync for its plan tables and the folded coefficients.  Some hosts
// cannot allow that: a framework that owns all device memory through its own
// pool and forbids outside allocations, an application holding a hard device
// memory budget, or a real-time pipeline in which an allocation (which may
// block or synchronise inside the CUDA driver) is not acceptable on the
// calling thread.  Those callers use this entry point instead.
//
// How: the scratch lives in one file-scope device array, kNoAllocScratchBytes
// (8 MiB) long, that every GPU which loads the library holds until the
// process exits.  Host code cannot use the array's name as a device address
// (in host code it names a host-side stand-in), so the first call on each
// device looks the address up once with cudaGetSymbolAddress, with that
// device current, and passes it to the kernels.  The address is kept for the
// life of the process: after a cudaDeviceReset on that device (which unloads
// the library's device code) the entry point must not be called again.  The
// waveform is then built in batches of knot segments: for each batch the
// folded coefficients of its segments are written into the array and consumed
// by the sum kernel before the next batch reuses the space, all in order on
// the caller's stream.  The caller's current device is restored on return.
//
// The kernels are the same ones few_get_waveform launches (k_fold_coeffs,
// k_sum_folded); only where their scratch lives differs.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "few_common.cuh"
#include "few_internal.h"

namespace few {

namespace {

constexpr size_t kNoAllocScratchBytes = FEW_NOALLOC_SCRATCH_BYTES;
static_assert(kNoAllocScratchBytes == (size_t(8) << 20), "the header states an 8 MiB scratch");
constexpr int kMaxDevices = 64;

// The one scratch array shared by every call on a device.  No byte of it needs
// to start at zero: each call writes every byte it later reads.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_addr_mutex;
void *g_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on `dev` (looked up once per device).
int scratch_address(int dev, unsigned char **out)
{
    if (dev < 0 || dev >= kMaxDevices) return fail(FEW_ERR_ARG, "few_get_waveform_noalloc: device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(FEW_ERR_CUDA, "few_get_waveform_noalloc: cudaGetSymbolAddress failed: %s",
                        cudaGetErrorString(e));
        g_addr[dev] = p;
    }
    *out = (unsigned char *)g_addr[dev];
    return FEW_OK;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// The body of few_get_waveform_noalloc, run with `dev` current.
int get_waveform_noalloc(void *d_waveform, const double *interp_array, const double *phase_interp_t,
                         const double *phase_interp_coeffs, const int *d_m, const int *d_k, const int *d_n,
                         int init_len, int out_len, int num_teuk_modes, const void *d_Ylms, double delta_t,
                         const double *h_t, int dev, void *stream)
{
    const int K = num_teuk_modes;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned char *scratch = nullptr;
    int rc = scratch_address(dev, &scratch);
    if (rc) return rc;

    std::vector<int> m(K), k(K), n(K);
    FEW_CUDA_TRY(cudaMemcpyAsync(m.data(), d_m, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
    FEW_CUDA_TRY(cudaMemcpyAsync(k.data(), d_k, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
    FEW_CUDA_TRY(cudaMemcpyAsync(n.data(), d_n, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
    FEW_CUDA_TRY(cudaStreamSynchronize(st));

    // Fold plan and segment plan, exactly as few_get_waveform makes them.
    int nmax = 0;
    for (int j = 0; j < K; ++j) nmax = std::max(nmax, std::abs(n[j]));
    const int max_rows = kMaxRows;
    const long long max_keys_ll = (long long)max_rows * (2LL * nmax + 1);
    if (max_keys_ll > (1 << 24)) return fail(FEW_ERR_SIZE, "few_get_waveform_noalloc: mode grid too large");
    const int max_keys = (int)max_keys_ll;
    std::vector<int> row_m(max_rows), row_k(max_rows), key_ptr(max_keys + 1), key_list(2 * K);
    int dims[3];
    rc = fold_plan(m.data(), k.data(), n.data(), K, max_rows, max_keys, row_m.data(), row_k.data(), dims,
                   key_ptr.data(), key_list.data());
    if (rc) return rc;
    const int R = dims[0], nlo = dims[1], NN = dims[2];
    int use_theta = 0;
    for (int r = 0; r < R; ++r) use_theta |= (row_k[r] != 0);
    const int chunk = kDefaultChunk;
    const int max_units = init_len + out_len / chunk + 1;
    std::vector<int> seg_start(init_len), units(3 * (size_t)max_units);
    std::vector<double> seg_info(3 * (size_t)(init_len - 1));
    int counts[2];
    rc = segment_plan(h_t, phase_interp_t, init_len, out_len, delta_t, chunk, max_units, seg_start.data(),
                      seg_info.data(), units.data(), counts);
    if (rc) return rc;
    const int nseg = counts[0], nunits = counts[1];

    // Fixed part of the scratch: fold tables.
    const size_t nkeys = (size_t)R * NN;
    const size_t o_rm = 0;
    const size_t o_rk = o_rm + align256(sizeof(int) * R);
    const size_t o_kp = o_rk + align256(sizeof(int) * R);
    const size_t o_kl = o_kp + align256(sizeof(int) * (nkeys + 1));
    const size_t fixed = o_kl + align256(sizeof(int) * 2 * (size_t)K);
    const size_t w_per_seg = sizeof(double2) * 4 * nkeys;
    const size_t per_unit = sizeof(int) * 3;
    // A batch of one segment needs its W block, its seg_info and at most
    // ceil(out_len/chunk)+1 units; refuse what cannot fit even that.
    const size_t max_units_one_seg = (size_t)out_len / chunk + 2;
    if (fixed + align256(sizeof(double) * 3) + align256(per_unit * max_units_one_seg) + align256(w_per_seg) >
        kNoAllocScratchBytes)
        return fail(FEW_ERR_SIZE,
                    "few_get_waveform_noalloc: one segment needs %zu bytes of scratch (%d rows x %d columns of "
                    "folded coefficients) but the fixed scratch holds %zu bytes; use few_get_waveform",
                    fixed + w_per_seg + per_unit * max_units_one_seg, R, NN, kNoAllocScratchBytes);

    int status = FEW_OK;
    auto put = [&](size_t o, const void *src, size_t bytes) {
        if (status == FEW_OK && bytes) {
            cudaError_t e = cudaMemcpyAsync(scratch + o, src, bytes, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess)
                status = fail(FEW_ERR_CUDA, "few_get_waveform_noalloc: upload failed: %s", cudaGetErrorString(e));
        }
    };
    put(o_rm, row_m.data(), sizeof(int) * R);
    put(o_rk, row_k.data(), sizeof(int) * R);
    put(o_kp, key_ptr.data(), sizeof(int) * (nkeys + 1));
    put(o_kl, key_list.data(), sizeof(int) * (size_t)key_ptr[nkeys]);

    // Batches of consecutive segments; units are renumbered relative to the
    // batch's first segment and the per-segment inputs are offset to match.
    std::vector<int> bunits;
    int u = 0, s0 = 0;
    const long long seg_stride = 2LL * K;  // coefficients of one knot inside a (4, N, 2K) plane
    while (status == FEW_OK && s0 < nseg) {
        int s1 = s0;
        size_t units_in = 0;
        int u_end = u;
        for (;;) {
            if (s1 >= nseg) break;
            int ue = u_end;
            while (ue < nunits && units[3 * (size_t)ue] == s1) ++ue;
            const size_t need = fixed + align256(sizeof(double) * 3 * (size_t)(s1 + 1 - s0)) +
                                align256(per_unit * (units_in + (ue - u_end))) +
                                align256(w_per_seg * (size_t)(s1 + 1 - s0));
            if (need > kNoAllocScratchBytes && s1 > s0) break;
            units_in += (size_t)(ue - u_end);
            u_end = ue;
            ++s1;
        }
        const int bs = s1 - s0, bu = u_end - u;
        const size_t o_si = fixed;
        const size_t o_un = o_si + align256(sizeof(double) * 3 * (size_t)bs);
        const size_t o_W = o_un + align256(per_unit * (size_t)bu);
        bunits.assign(units.begin() + 3 * (size_t)u, units.begin() + 3 * (size_t)u_end);
        for (int q = 0; q < bu; ++q) bunits[3 * (size_t)q] -= s0;
        put(o_si, seg_info.data() + 3 * (size_t)s0, sizeof(double) * 3 * (size_t)bs);
        put(o_un, bunits.data(), per_unit * (size_t)bu);
        if (status == FEW_OK)
            status = launch_fold(interp_array + (size_t)s0 * seg_stride, (const double2 *)d_Ylms,
                                 (const int *)(scratch + o_kp), (const int *)(scratch + o_kl), K, init_len, bs, R, NN,
                                 (double2 *)(scratch + o_W), st);
        if (status == FEW_OK)
            status = launch_sum_folded((double2 *)d_waveform, (const double2 *)(scratch + o_W),
                                       phase_interp_coeffs + (size_t)s0 * 3, init_len, (const double *)(scratch + o_si),
                                       (const int *)(scratch + o_un), bu, (const int *)(scratch + o_rm),
                                       (const int *)(scratch + o_rk), R, nlo, NN, delta_t, FEW_SUM_FAITHFUL, use_theta,
                                       st);
        u = u_end;
        s0 = s1;
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (status != FEW_OK) return status;
    if (e != cudaSuccess) return fail(FEW_ERR_CUDA, "few_get_waveform_noalloc: %s", cudaGetErrorString(e));
    return FEW_OK;
}

}  // namespace
}  // namespace few

extern "C" int few_get_waveform_noalloc(void *d_waveform, const double *interp_array, const double *phase_interp_t,
                                        const double *phase_interp_coeffs, const int *d_m, const int *d_k,
                                        const int *d_n, int init_len, int out_len, int num_teuk_modes,
                                        const void *d_Ylms, double delta_t, const double *h_t, int dev, void *stream)
{
    using namespace few;
    clear_error();
    if (!d_waveform || !interp_array || !phase_interp_t || !phase_interp_coeffs || !d_m || !d_k || !d_n || !d_Ylms ||
        !h_t)
        return fail(FEW_ERR_ARG, "few_get_waveform_noalloc: null pointer");
    if (init_len < 2 || out_len < 1 || num_teuk_modes < 1)
        return fail(FEW_ERR_SIZE, "few_get_waveform_noalloc: bad sizes");
    // the work runs with `dev` current; the caller's current device is restored on return
    int prev = 0;
    FEW_CUDA_TRY(cudaGetDevice(&prev));
    FEW_CUDA_TRY(cudaSetDevice(dev));
    const int rc = get_waveform_noalloc(d_waveform, interp_array, phase_interp_t, phase_interp_coeffs, d_m, d_k, d_n,
                                        init_len, out_len, num_teuk_modes, d_Ylms, delta_t, h_t, dev, stream);
    const cudaError_t e = cudaSetDevice(prev);
    if (rc != FEW_OK) return rc;
    if (e != cudaSuccess)
        return fail(FEW_ERR_CUDA, "few_get_waveform_noalloc: restoring device %d: %s", prev, cudaGetErrorString(e));
    return FEW_OK;
}
