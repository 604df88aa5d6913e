// Host planners: the mode fold map and the segment / work-unit tables.
//
// segment_plan restates find_start_inds (src/few/cutils/interpolate.cu:694-723):
// segment j owns output samples [ceil(t_j/dt), ceil(t_{j+1}/dt)), the first
// segment starts at sample 0, and the first knot at or past the last output
// time T = (out_len-1)*dt closes the plan.  Differences, all on inputs the
// reference leaves undefined: knots must increase strictly (otherwise segments
// would overlap), sample indices are clamped to [0, out_len), and a knot list
// that never reaches T is refused instead of read past its end.
#include <algorithm>
#include <cmath>
#include <map>
#include <utility>
#include <vector>

#include "few_internal.h"

namespace few {

int fold_plan(const int *m, const int *k, const int *n, int K, int max_rows, int max_keys, int *row_m, int *row_k,
              int *dims, int *key_ptr, int *key_list)
{
    if (!m || !k || !n || !row_m || !row_k || !dims || !key_ptr || !key_list)
        return fail(FEW_ERR_ARG, "few_fold_plan: null pointer");
    if (K < 1) return fail(FEW_ERR_SIZE, "few_fold_plan: K=%d < 1", K);
    const long long bound = 1 << 20;
    std::map<std::pair<int, int>, int> rows;
    int nlo = 0, nhi = 0;
    bool first = true;
    auto see = [&](int mm, int kk, int nn) {
        rows.emplace(std::make_pair(mm, kk), 0);
        if (first || nn < nlo) nlo = nn;
        if (first || nn > nhi) nhi = nn;
        first = false;
    };
    for (int j = 0; j < K; ++j) {
        if (std::llabs(m[j]) > bound || std::llabs(k[j]) > bound || std::llabs(n[j]) > bound)
            return fail(FEW_ERR_ARG, "few_fold_plan: mode index out of range at j=%d", j);
        see(m[j], k[j], n[j]);
        if (m[j] != 0) see(-m[j], -k[j], -n[j]);
    }
    const int R = (int)rows.size();
    const int NN = nhi - nlo + 1;
    if (R > max_rows) return fail(FEW_ERR_SIZE, "few_fold_plan: %d (m,k) rows exceed %d", R, max_rows);
    if ((long long)R * NN > max_keys)
        return fail(FEW_ERR_SIZE, "few_fold_plan: %d x %d keys exceed %d", R, NN, max_keys);
    int r = 0;
    for (auto &kv : rows) {
        kv.second = r;
        row_m[r] = kv.first.first;
        row_k[r] = kv.first.second;
        ++r;
    }
    const int nkeys = R * NN;
    std::vector<int> count(nkeys + 1, 0);
    auto key_of = [&](int mm, int kk, int nn) { return rows[std::make_pair(mm, kk)] * NN + (nn - nlo); };
    for (int j = 0; j < K; ++j) {
        count[key_of(m[j], k[j], n[j]) + 1]++;
        if (m[j] != 0) count[key_of(-m[j], -k[j], -n[j]) + 1]++;
    }
    for (int q = 0; q < nkeys; ++q) count[q + 1] += count[q];
    for (int q = 0; q <= nkeys; ++q) key_ptr[q] = count[q];
    std::vector<int> fillp(count.begin(), count.end() - 1);
    for (int j = 0; j < K; ++j) {
        key_list[fillp[key_of(m[j], k[j], n[j])]++] = 2 * j;
        if (m[j] != 0) key_list[fillp[key_of(-m[j], -k[j], -n[j])]++] = 2 * j + 1;
    }
    dims[0] = R;
    dims[1] = nlo;
    dims[2] = NN;
    return FEW_OK;
}

int segment_plan(const double *h_t, const double *phase_t, int init_len, int out_len, double dt, int chunk,
                 int max_units, int *seg_start, double *seg_info, int *units, int *counts)
{
    if (!h_t || !phase_t || !seg_start || !seg_info || !units || !counts)
        return fail(FEW_ERR_ARG, "few_segment_plan: null pointer");
    if (init_len < 2 || out_len < 1 || chunk < 1) return fail(FEW_ERR_SIZE, "few_segment_plan: bad sizes");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(FEW_ERR_ARG, "few_segment_plan: dt must be positive");
    for (int i = 1; i < init_len; ++i)
        if (!(h_t[i] > h_t[i - 1]))
            return fail(FEW_ERR_KNOTS, "few_segment_plan: knot times must increase strictly (index %d)", i);
    // find_start_inds (interpolate.cu:694-723)
    const double T = (out_len - 1) * dt;
    seg_start[0] = 0;
    int nseg = -1;
    for (int i = 1; i < init_len; ++i) {
        const double t = h_t[i];
        if (t < T) {
            double c = std::ceil(t / dt);
            seg_start[i] = (int)std::min<double>(std::max<double>(c, 0.0), (double)out_len);
        } else {
            seg_start[i] = out_len;
            nseg = i;
            break;
        }
    }
    if (nseg < 0)
        return fail(FEW_ERR_KNOTS, "few_segment_plan: the last knot (%g s) is before the last output sample (%g s)",
                    h_t[init_len - 1], T);
    int nu = 0;
    for (int j = 0; j < nseg; ++j) {
        const int a = std::max(seg_start[j], 0), b = std::min(seg_start[j + 1], out_len);
        seg_info[3 * j] = h_t[j];
        seg_info[3 * j + 1] = phase_t[j];
        seg_info[3 * j + 2] = phase_t[j + 1] - phase_t[j];
        if (a < b && !(phase_t[j + 1] > phase_t[j]))
            return fail(FEW_ERR_KNOTS, "few_segment_plan: phase knot times must increase (segment %d)", j);
        for (int u = a; u < b; u += chunk) {
            if (nu >= max_units) return fail(FEW_ERR_SIZE, "few_segment_plan: more than %d work units", max_units);
            units[3 * nu] = j;
            units[3 * nu + 1] = u;
            units[3 * nu + 2] = std::min(u + chunk, b);
            ++nu;
        }
    }
    counts[0] = nseg;
    counts[1] = nu;
    return FEW_OK;
}

// Factorization of the not-a-knot system shared by every series on knots t
// (the elimination k_spline_build performs per thread, done once), and of the
// interior block of its transpose for the adjoint (k_spline_adjoint_factored).
// fac (N+1, kFacWidth = 16), row i:
//   0 lo_i, 1 1/den_i, 2 c'_i, 3 alpha_i, 4 beta_i  (rows 1..N-2; forward sweep
//     r'_i = (alpha_i delta_{i-1} + beta_i delta_i - lo_i r'_{i-1}) / den_i, the
//     two boundary rows' right-hand sides folded into rows 1 and N-2)
//   5 h_i, 6 1/h_i                                   (rows 0..N-2)
//   7 lo~_i = h_{i-2}, 8 1/den~_i, 9 c~_i           (rows 1..N-2; transposed block)
//   10, 11  products of the sweep factors -lo_j/den_j over [chunk start, i] and of
//           -c'_j over [i, chunk end), 12, 13 the same for the transposed block
//           (-lo~_j/den~_j and -c~_j): the interior rows 1..N-2 are cut into
//           kScanChunks chunks of ceil((N-2)/kScanChunks) rows, and a chunk's
//           sweeps, run with a zero carry-in, are corrected by carry x product.
// Row N: gamma0, gamma1 (b0 = gamma0 delta_0 + gamma1 delta_1), d0 = x2 - x0, h1,
// eps0, eps1 (bE = eps0 delta_{N-3} + eps1 delta_{N-2}), dE = x_{N-1} - x_{N-3},
// hA = x_{N-2} - x_{N-3}.
int spline_factor(const double *x, int N, double *fac)
{
    const int W = kFacWidth;
    if (!x || !fac) return fail(FEW_ERR_ARG, "few_spline_factor: null pointer");
    if (N < 4) return fail(FEW_ERR_SIZE, "few_spline_factor: length=%d; not-a-knot splines need at least 4 knots", N);
    for (int i = 1; i < N; ++i)
        if (!(x[i] > x[i - 1])) return fail(FEW_ERR_KNOTS, "few_spline_factor: knots must increase strictly");
    for (int q = 0; q < W * (N + 1); ++q) fac[q] = 0.0;
    for (int i = 0; i <= N - 2; ++i) {
        const double h = x[i + 1] - x[i];
        fac[W * i + 5] = h;
        fac[W * i + 6] = 1.0 / h;
    }
    const double h0 = x[1] - x[0], h1 = x[2] - x[1], d0 = x[2] - x[0];
    const double hA = x[N - 2] - x[N - 3], hB = x[N - 1] - x[N - 2], dE = x[N - 1] - x[N - 3];
    const double g0 = (h0 + 2 * d0) * h1 / d0, g1 = h0 * h0 / d0;
    const double e0 = hB * hB / dE, e1 = (2 * dE + hB) * hA / dE;
    double cprev = 0.0, ctprev = 0.0;
    for (int i = 1; i <= N - 2; ++i) {
        const double hl = x[i] - x[i - 1], hr = x[i + 1] - x[i];
        double lo = hr, dg = 2 * (hl + hr), up = hl, alpha = 3.0 * hr, beta = 3.0 * hl;
        if (i == 1) {
            dg -= d0;
            lo = 0.0;
            alpha -= g0;
            beta -= g1;
        }
        if (i == N - 2) {
            dg -= dE;
            up = 0.0;
            alpha -= e0;
            beta -= e1;
        }
        const double den = dg - lo * cprev;
        const double cp = up / den;
        fac[W * i + 0] = lo;
        fac[W * i + 1] = 1.0 / den;
        fac[W * i + 2] = cp;
        fac[W * i + 3] = alpha;
        fac[W * i + 4] = beta;
        cprev = cp;
        // transposed interior block: row i has h_{i-2} left (i >= 2), the same
        // diagonal, and h_{i+1} right (i <= N-3)
        const double lot = (i >= 2) ? (x[i - 1] - x[i - 2]) : 0.0;
        const double upt = (i <= N - 3) ? (x[i + 2] - x[i + 1]) : 0.0;
        const double dent = dg - lot * ctprev;
        const double ct = upt / dent;
        fac[W * i + 7] = lot;
        fac[W * i + 8] = 1.0 / dent;
        fac[W * i + 9] = ct;
        ctprev = ct;
    }
    // chunk products for the scan form of both sweeps
    const int M = N - 2, L = (M + kScanChunks - 1) / kScanChunks;
    for (int a = 1; a <= N - 2; a += L) {
        const int e = std::min(a + L, N - 1);  // rows [a, e)
        double pf = 1.0, pft = 1.0;
        for (int i = a; i < e; ++i) {
            pf *= -fac[W * i + 0] * fac[W * i + 1];
            pft *= -fac[W * i + 7] * fac[W * i + 8];
            fac[W * i + 10] = pf;
            fac[W * i + 12] = pft;
        }
        double pb = 1.0, pbt = 1.0;
        for (int i = e - 1; i >= a; --i) {
            pb *= -fac[W * i + 2];
            pbt *= -fac[W * i + 9];
            fac[W * i + 11] = pb;
            fac[W * i + 13] = pbt;
        }
    }
    double *b = fac + (size_t)W * N;
    b[0] = g0;
    b[1] = g1;
    b[2] = d0;
    b[3] = h1;
    b[4] = e0;
    b[5] = e1;
    b[6] = dE;
    b[7] = hA;
    return FEW_OK;
}

}  // namespace few

extern "C" int few_spline_factor(const double *t, int N, double *fac)
{
    few::clear_error();
    return few::spline_factor(t, N, fac);
}

extern "C" int few_fold_plan(const int *m, const int *k, const int *n, int K, int max_rows, int max_keys, int *row_m,
                             int *row_k, int *dims, int *key_ptr, int *key_list)
{
    few::clear_error();
    return few::fold_plan(m, k, n, K, max_rows, max_keys, row_m, row_k, dims, key_ptr, key_list);
}

extern "C" int few_segment_plan(const double *h_t, const double *phase_t, int init_len, int out_len, double dt,
                                int chunk, int max_units, int *seg_start, double *seg_info, int *units, int *counts)
{
    few::clear_error();
    return few::segment_plan(h_t, phase_t, init_len, out_len, dt, chunk, max_units, seg_start, seg_info, units,
                             counts);
}
