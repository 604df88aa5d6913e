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

}  // namespace few

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
