// Teukolsky amplitudes from bicubic (generally bi-degree kx, ky <= 5) tensor-
// product B-splines: the producer of the mode sum's teuk_modes
// (src/few/amplitude/ampinterp2d.py:127-189, kernel src/few/cutils/AmpInterp2D.cu:86-208).
//
// Every coefficient grid c_g (len_indiv_c = (nx-kx-1)(ny-ky-1) values) is
// evaluated at the same points (x_i, y_i):
//     z_g(x_i, y_i) = sum_{a<=kx} sum_{b<=ky} c_g[(lx_i + a)(ny-ky-1) + ly_i + b] wx_i[a] wy_i[b]
// where lx_i, wx_i (and ly_i, wy_i) are the knot interval and the kx+1
// non-zero B-spline values at x_i: FITPACK's interval search on the clamped
// argument and its de Boor-Cox recurrence (Dierckx, "Curve and surface fitting
// with splines", fpbspl/fpbisp).  The basis depends on the point only, so it is
// computed once per point and shared by all grids (the reference recomputes it
// per grid and point).  Every operation is explicitly rounded in the order
// the reference's C code writes it (no contraction), so the values equal the
// reference's CPU path bit for bit.
//
// Layouts.  few_interp2d: the reference's z (num_indiv_c, m) (interp2D_wrap,
// AmpInterp2D.hh:6-8).  few_amp_interp2d: the amplitudes directly in the mode
// sum's (m, nmodes) complex128 layout, grid 2j (real part) and 2j+1 (imaginary
// part) of mode mode_idx[j] (the transpose and complex assembly that
// AmpInterp2D.__call__ does on the host, ampinterp2d.py:186-189, fused into
// the kernel: a CTA evaluates a tile of 32 points x 32 modes, lane = point,
// and writes each output row through a shared-memory transpose).
#include "few_common.cuh"
#include "few_internal.h"

namespace few {

namespace {

constexpr int kMaxDeg = 5;       // largest spline degree (FITPACK's fpbspl work array)
constexpr int kTileP = 32;       // points per CTA
constexpr int kTileM = 32;       // modes per CTA (fused layout) / grids per CTA (reference layout)
constexpr int kAmpThreads = 256; // 8 warps

// Interval and the k+1 non-zero B-splines of degree k at x (clamped to the
// spline's base interval), as FITPACK: l is the first index in [k+1, n-k-1]
// with x < t[l] (or n-k-1), then de Boor-Cox.  Returns l - (k+1).
__device__ __forceinline__ int bspline_basis(const double *__restrict__ t, int n, int k, double x, double *h)
{
    const int k1 = k + 1, nk1 = n - k1;
    const double tb = t[k1 - 1], te = t[nk1];
    double arg = x;
    if (arg < tb) arg = tb;
    if (arg > te) arg = te;
    // smallest l in [k1, nk1] with arg < t[l] (binary search; t is non-decreasing)
    int lo = k1, hi = nk1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (arg < t[mid]) hi = mid;
        else lo = mid + 1;
    }
    const int l = lo;
    double hh[kMaxDeg];
    h[0] = 1.0;
    for (int j = 1; j <= k; ++j) {
        for (int i = 0; i < k; ++i) hh[i] = h[i];
        h[0] = 0.0;
        for (int i = 0; i < j; ++i) {
            const int li = l + i, lj = li - j;
            const double f = __ddiv_rn(hh[i], __dsub_rn(t[li], t[lj]));
            h[i] = __dadd_rn(h[i], __dmul_rn(f, __dsub_rn(t[li], arg)));
            h[i + 1] = __dmul_rn(f, __dsub_rn(arg, t[lj]));
        }
    }
    return l - k1;
}

struct Interp2DArgs {
    const double *tx, *ty;
    const double *c;
    const double *x, *y;
    const int *mode_idx;  // fused layout: grids 2 mode_idx[j], 2 mode_idx[j] + 1; null = identity
    void *out;
    int nx, ny, kx, ky, m, ngrid_or_modes, len_indiv_c;
};

// The per-point basis of this CTA's points into shared memory, point index
// fastest (s_w[dim][q][point]) so a warp's reads of one weight hit distinct banks.
__device__ __forceinline__ void tile_basis(const Interp2DArgs &a, int p0, double (*s_w)[kMaxDeg + 1][kTileP],
                                           int (*s_l)[kTileP])
{
    const int t = threadIdx.x;
    if (t < 2 * kTileP) {
        const int p = t >> 1, dim = t & 1;
        const int i = min(p0 + p, a.m - 1);
        double h[kMaxDeg + 1];
        const int l = dim == 0 ? bspline_basis(a.tx, a.nx, a.kx, a.x[i], h)
                               : bspline_basis(a.ty, a.ny, a.ky, a.y[i], h);
        const int kk = dim == 0 ? a.kx : a.ky;
        for (int q = 0; q <= kk; ++q) s_w[dim][q][p] = h[q];
        s_l[dim][p] = l;
    }
    __syncthreads();
}

// One grid at one point, summed in the reference's order (fpbisp): degrees
// known at compile time, weights in registers.
template <int KX, int KY>
__device__ __forceinline__ double eval_grid_k(const double *__restrict__ cg, int nky1, int lx, int ly,
                                              const double (&wx)[KX + 1], const double (&wy)[KY + 1])
{
    double sp = 0.0;
#pragma unroll
    for (int i1 = 0; i1 <= KX; ++i1) {
        const double *row = cg + (lx + i1) * nky1 + ly;
#pragma unroll
        for (int j1 = 0; j1 <= KY; ++j1) sp = __dadd_rn(sp, __dmul_rn(__dmul_rn(row[j1], wx[i1]), wy[j1]));
    }
    return sp;
}

// The same for run-time degrees.
__device__ __forceinline__ double eval_grid(const double *__restrict__ cg, int nky1, int kx, int ky, int lx, int ly,
                                            const double *wx, const double *wy)
{
    double sp = 0.0;
    int l1 = lx * nky1 + ly;
    for (int i1 = 0; i1 <= kx; ++i1) {
        int l2 = l1;
        for (int j1 = 0; j1 <= ky; ++j1) {
            sp = __dadd_rn(sp, __dmul_rn(__dmul_rn(cg[l2], wx[i1]), wy[j1]));
            ++l2;
        }
        l1 += nky1;
    }
    return sp;
}

// Reference layout: z[g * m + i]; grid (blockIdx.y), points by tile.
__global__ void __launch_bounds__(kAmpThreads) k_interp2d(Interp2DArgs a)
{
    __shared__ double s_w[2][kMaxDeg + 1][kTileP];
    __shared__ int s_l[2][kTileP];
    const int p0 = blockIdx.x * kTileP;
    tile_basis(a, p0, s_w, s_l);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i = p0 + lane;
    const int nky1 = a.ny - a.ky - 1;
    double *z = static_cast<double *>(a.out);
    double wx[kMaxDeg + 1], wy[kMaxDeg + 1];
    for (int q = 0; q <= kMaxDeg; ++q) {
        wx[q] = s_w[0][q][lane];
        wy[q] = s_w[1][q][lane];
    }
    for (int gl = warp; gl < kTileM; gl += kAmpThreads / 32) {
        const int g = blockIdx.y * kTileM + gl;
        if (g >= a.ngrid_or_modes || i >= a.m) continue;
        const double *cg = a.c + (long long)g * a.len_indiv_c;
        z[(long long)g * a.m + i] = eval_grid(cg, nky1, a.kx, a.ky, s_l[0][lane], s_l[1][lane], wx, wy);
    }
}

// Fused layout: out[i * nmodes + j] = z_{2 mode_j}(i) + i z_{2 mode_j + 1}(i).
// KX = KY = 0: run-time degrees.
template <int KX, int KY>
__global__ void __launch_bounds__(kAmpThreads) k_amp_interp2d(Interp2DArgs a)
{
    __shared__ double s_w[2][kMaxDeg + 1][kTileP];
    __shared__ int s_l[2][kTileP];
    __shared__ double2 s_out[kTileP][kTileM + 1];
    const int p0 = blockIdx.x * kTileP, j0 = blockIdx.y * kTileM;
    tile_basis(a, p0, s_w, s_l);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nky1 = a.ny - a.ky - 1;
    const int nmodes = a.ngrid_or_modes;
    const int lx = s_l[0][lane], ly = s_l[1][lane];
    const bool live = p0 + lane < a.m;
    if constexpr (KX > 0) {
        double wx[KX + 1], wy[KY + 1];
#pragma unroll
        for (int q = 0; q <= KX; ++q) wx[q] = s_w[0][q][lane];
#pragma unroll
        for (int q = 0; q <= KY; ++q) wy[q] = s_w[1][q][lane];
        // each warp's modes jl = warp + 8 r, unrolled: independent chains interleave
#pragma unroll
        for (int r = 0; r < kTileM / (kAmpThreads / 32); ++r) {
            const int jl = warp + r * (kAmpThreads / 32), j = j0 + jl;
            double2 v = make_double2(0.0, 0.0);
            if (j < nmodes && live) {
                const int mode = a.mode_idx ? a.mode_idx[j] : j;
                const double *cg = a.c + (long long)mode * 2 * a.len_indiv_c;
                v.x = eval_grid_k<KX, KY>(cg, nky1, lx, ly, wx, wy);
                v.y = eval_grid_k<KX, KY>(cg + a.len_indiv_c, nky1, lx, ly, wx, wy);
            }
            s_out[lane][jl] = v;
        }
    } else {
        double wx[kMaxDeg + 1], wy[kMaxDeg + 1];
        for (int q = 0; q <= kMaxDeg; ++q) {
            wx[q] = s_w[0][q][lane];
            wy[q] = s_w[1][q][lane];
        }
        for (int jl = warp; jl < kTileM; jl += kAmpThreads / 32) {
            const int j = j0 + jl;
            double2 v = make_double2(0.0, 0.0);
            if (j < nmodes && live) {
                const int mode = a.mode_idx ? a.mode_idx[j] : j;
                const double *cg = a.c + (long long)mode * 2 * a.len_indiv_c;
                v.x = eval_grid(cg, nky1, a.kx, a.ky, lx, ly, wx, wy);
                v.y = eval_grid(cg + a.len_indiv_c, nky1, a.kx, a.ky, lx, ly, wx, wy);
            }
            s_out[lane][jl] = v;
        }
    }
    __syncthreads();
    double2 *out = static_cast<double2 *>(a.out);
    for (int pl = warp; pl < kTileP; pl += kAmpThreads / 32) {
        const int i = p0 + pl, j = j0 + lane;
        if (i < a.m && j < nmodes) out[(long long)i * nmodes + j] = s_out[pl][lane];
    }
}

int check_interp2d(const char *who, const double *tx, int nx, const double *ty, int ny, const double *c, int kx,
                   int ky, const double *x, const double *y, int m, int n, int len_indiv_c, const void *out)
{
    if (!tx || !ty || !c || !x || !y || !out) return fail(FEW_ERR_ARG, "%s: null pointer", who);
    if (kx < 1 || ky < 1 || kx > kMaxDeg || ky > kMaxDeg)
        return fail(FEW_ERR_SIZE, "%s: spline degrees kx=%d ky=%d outside 1..%d", who, kx, ky, kMaxDeg);
    if (nx < 2 * (kx + 1) || ny < 2 * (ky + 1))
        return fail(FEW_ERR_SIZE, "%s: nx=%d, ny=%d knots too few for degrees %d, %d", who, nx, ny, kx, ky);
    if ((long long)(nx - kx - 1) * (ny - ky - 1) != (long long)len_indiv_c)
        return fail(FEW_ERR_SIZE, "%s: len_indiv_c=%d != (nx-kx-1)(ny-ky-1)", who, len_indiv_c);
    if (m < 0 || n < 0) return fail(FEW_ERR_SIZE, "%s: negative sizes", who);
    return FEW_OK;
}

}  // namespace

}  // namespace few

extern "C" int few_interp2d(double *z, const double *tx, int nx, const double *ty, int ny, const double *c, int kx,
                            int ky, const double *x, int mx, const double *y, int my, int num_indiv_c,
                            int len_indiv_c, void *stream)
{
    few::clear_error();
    if (mx != my) return few::fail(FEW_ERR_SIZE, "few_interp2d: mx and my must be the same value");
    int rc = few::check_interp2d("few_interp2d", tx, nx, ty, ny, c, kx, ky, x, y, mx, num_indiv_c, len_indiv_c, z);
    if (rc) return rc;
    if (mx == 0 || num_indiv_c == 0) return FEW_OK;
    few::Interp2DArgs a{tx, ty, c, x, y, nullptr, z, nx, ny, kx, ky, mx, num_indiv_c, len_indiv_c};
    dim3 grid((mx + few::kTileP - 1) / few::kTileP, (num_indiv_c + few::kTileM - 1) / few::kTileM);
    if (grid.y > 65535) return few::fail(FEW_ERR_SIZE, "few_interp2d: too many grids");
    few::k_interp2d<<<grid, few::kAmpThreads, 0, (cudaStream_t)stream>>>(a);
    FEW_LAUNCH_CHECK("k_interp2d");
    return FEW_OK;
}

extern "C" int few_amp_interp2d(void *out, const double *tx, int nx, const double *ty, int ny, const double *c,
                                int kx, int ky, const double *x, const double *y, int m, const int *mode_idx,
                                int nmodes, int len_indiv_c, void *stream)
{
    few::clear_error();
    int rc = few::check_interp2d("few_amp_interp2d", tx, nx, ty, ny, c, kx, ky, x, y, m, nmodes, len_indiv_c, out);
    if (rc) return rc;
    if (m == 0 || nmodes == 0) return FEW_OK;
    few::Interp2DArgs a{tx, ty, c, x, y, mode_idx, out, nx, ny, kx, ky, m, nmodes, len_indiv_c};
    dim3 grid((m + few::kTileP - 1) / few::kTileP, (nmodes + few::kTileM - 1) / few::kTileM);
    if (grid.y > 65535) return few::fail(FEW_ERR_SIZE, "few_amp_interp2d: too many modes");
    if (kx == 3 && ky == 3)
        few::k_amp_interp2d<3, 3><<<grid, few::kAmpThreads, 0, (cudaStream_t)stream>>>(a);
    else
        few::k_amp_interp2d<0, 0><<<grid, few::kAmpThreads, 0, (cudaStream_t)stream>>>(a);
    FEW_LAUNCH_CHECK("k_amp_interp2d");
    return FEW_OK;
}
