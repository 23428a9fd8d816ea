// Host-side preprocessing of a species matrix (see prepare.h).
//
// Scaling follows the engine's published recipe: Ruiz equilibration by
// infinity norms, then one Pock-Chambolle (alpha = 1) step by absolute sums
// (Pock & Chambolle, ICCV 2011 -- the metric the reference builds at
// `src/gpu_pdhg_corrector.py:183-200`), then a power-iteration estimate of the
// scaled spectral norm for a constant PDHG step.
#include "prepare.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace fbalp {

bool canonical_csr(int32_t rows, int32_t cols, const int64_t* indptr, const int32_t* indices,
                   const double* values, Csr* out, std::string* err) {
    if (rows < 0 || cols < 1) {
        *err = "matrix needs rows >= 0 and cols >= 1";
        return false;
    }
    if (rows > 0 && (indptr == nullptr)) {
        *err = "row pointer is NULL";
        return false;
    }
    if (indptr && indptr[0] != 0) {
        *err = "row pointer must start at 0";
        return false;
    }
    Csr a;
    a.rows = rows;
    a.cols = cols;
    a.ptr.assign(rows + 1, 0);
    std::vector<std::pair<int32_t, double>> row;
    for (int32_t i = 0; i < rows; ++i) {
        int64_t b = indptr[i], e = indptr[i + 1];
        if (e < b) {
            *err = "row pointer is not monotone";
            return false;
        }
        row.clear();
        for (int64_t k = b; k < e; ++k) {
            int32_t j = indices[k];
            double v = values[k];
            if (j < 0 || j >= cols) {
                *err = "column index out of range";
                return false;
            }
            if (!std::isfinite(v)) {
                *err = "matrix values must be finite";
                return false;
            }
            row.emplace_back(j, v);
        }
        std::stable_sort(row.begin(), row.end(),
                         [](const auto& x, const auto& y) { return x.first < y.first; });
        size_t p = 0;
        while (p < row.size()) {
            int32_t j = row[p].first;
            double s = 0.0;
            while (p < row.size() && row[p].first == j) s += row[p++].second;
            if (s != 0.0) {
                a.idx.push_back(j);
                a.val.push_back(s);
            }
        }
        a.ptr[i + 1] = static_cast<int64_t>(a.idx.size());
    }
    if (a.idx.size() >= static_cast<size_t>(INT32_MAX)) {
        *err = "too many nonzeros";
        return false;
    }
    *out = std::move(a);
    return true;
}

Csr transpose(const Csr& a) {
    Csr t;
    t.rows = a.cols;
    t.cols = a.rows;
    t.ptr.assign(a.cols + 1, 0);
    for (int32_t j : a.idx) t.ptr[j + 1]++;
    for (int32_t j = 0; j < a.cols; ++j) t.ptr[j + 1] += t.ptr[j];
    t.idx.resize(a.idx.size());
    t.val.resize(a.val.size());
    std::vector<int64_t> fill(t.ptr.begin(), t.ptr.end() - 1);
    for (int32_t i = 0; i < a.rows; ++i)
        for (int64_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
            int64_t p = fill[a.idx[k]]++;
            t.idx[p] = i;  // rows ascending inside each column
            t.val[p] = a.val[k];
        }
    return t;
}

static std::vector<double> power_start(int32_t n) {
    std::vector<double> v(n);
    for (int32_t j = 0; j < n; ++j) {
        uint64_t h = (static_cast<uint64_t>(j) * 2654435761ull) % (1ull << 32);
        v[j] = static_cast<double>(h) / 4294967296.0 + 0.5;
    }
    return v;
}

Scaling scale_matrix(const Csr& a, int ruiz_iterations, int power_iterations, double step_safety) {
    const int32_t m = a.rows, n = a.cols;
    Scaling s;
    s.dr.assign(m, 1.0);
    s.dc.assign(n, 1.0);
    std::vector<double> rmax(m), cmax(n);
    for (int it = 0; it < ruiz_iterations; ++it) {
        std::fill(rmax.begin(), rmax.end(), 0.0);
        std::fill(cmax.begin(), cmax.end(), 0.0);
        for (int32_t i = 0; i < m; ++i)
            for (int64_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
                double cur = std::fabs(a.val[k]) * s.dr[i] * s.dc[a.idx[k]];
                rmax[i] = std::max(rmax[i], cur);
                cmax[a.idx[k]] = std::max(cmax[a.idx[k]], cur);
            }
        for (int32_t i = 0; i < m; ++i) s.dr[i] = s.dr[i] / (rmax[i] > 0 ? std::sqrt(rmax[i]) : 1.0);
        for (int32_t j = 0; j < n; ++j) s.dc[j] = s.dc[j] / (cmax[j] > 0 ? std::sqrt(cmax[j]) : 1.0);
    }
    std::fill(rmax.begin(), rmax.end(), 0.0);
    std::fill(cmax.begin(), cmax.end(), 0.0);
    for (int32_t i = 0; i < m; ++i)
        for (int64_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
            double cur = std::fabs(a.val[k]) * s.dr[i] * s.dc[a.idx[k]];
            rmax[i] += cur;
            cmax[a.idx[k]] += cur;
        }
    for (int32_t i = 0; i < m; ++i) s.dr[i] = s.dr[i] / (rmax[i] > 0 ? std::sqrt(rmax[i]) : 1.0);
    for (int32_t j = 0; j < n; ++j) s.dc[j] = s.dc[j] / (cmax[j] > 0 ? std::sqrt(cmax[j]) : 1.0);

    // scaled matrix values, then power iteration on A~^T A~
    std::vector<double> sv(a.val.size());
    for (int32_t i = 0; i < m; ++i)
        for (int64_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) sv[k] = a.val[k] * s.dr[i] * s.dc[a.idx[k]];
    std::vector<double> v = power_start(n), av(m), w(n);
    double nv = 0.0;
    for (double t : v) nv += t * t;
    nv = std::sqrt(nv);
    for (double& t : v) t /= nv;
    double lam = 0.0;
    for (int it = 0; it < power_iterations; ++it) {
        for (int32_t i = 0; i < m; ++i) {
            double acc = 0.0;
            for (int64_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) acc += sv[k] * v[a.idx[k]];
            av[i] = acc;
        }
        std::fill(w.begin(), w.end(), 0.0);
        for (int32_t i = 0; i < m; ++i)
            for (int64_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) w[a.idx[k]] += sv[k] * av[i];
        double nw = 0.0;
        for (double t : w) nw += t * t;
        nw = std::sqrt(nw);
        lam = nw;
        if (!(nw > 0.0)) break;
        for (int32_t j = 0; j < n; ++j) v[j] = w[j] / nw;
    }
    s.sigma_max = lam > 0.0 ? std::sqrt(lam) : 0.0;
    s.eta = s.sigma_max > 0.0 ? step_safety / s.sigma_max : 1.0;
    return s;
}

Sell build_sell(const Csr& a, const std::vector<int32_t>& row_order,
                const std::vector<int32_t>& col_rename, const std::vector<double>& row_scale,
                const std::vector<double>& col_scale, int32_t pad_index, int32_t long_cut) {
    Sell s;
    const int32_t rows = a.rows;
    auto len = [&](int32_t r) { return static_cast<int32_t>(a.ptr[row_order[r] + 1] - a.ptr[row_order[r]]); };
    auto is_long = [&](int32_t r) { return long_cut > 0 && len(r) > long_cut; };
    s.nslices = (rows + 31) / 32;
    s.off.assign(s.nslices + 1, 0);
    s.length.assign(s.nslices, 0);
    s.lmask.assign(s.nslices, 0u);
    s.long_off.assign(1, 0);
    for (int32_t sl = 0; sl < s.nslices; ++sl) {
        int32_t L = 0;
        for (int32_t lane = 0; lane < 32; ++lane) {
            int32_t r = sl * 32 + lane;
            if (r >= rows) break;
            if (is_long(r)) {
                s.lmask[sl] |= 1u << lane;
                continue;
            }
            L = std::max<int32_t>(L, len(r));
        }
        s.length[sl] = L;
        s.off[sl + 1] = s.off[sl] + 32 * L;
    }
    s.idx.assign(s.off[s.nslices], pad_index);
    s.val.assign(s.off[s.nslices], 0.0);
    for (int32_t sl = 0; sl < s.nslices; ++sl)
        for (int32_t lane = 0; lane < 32; ++lane) {
            int32_t r = sl * 32 + lane;
            if (r >= rows) break;
            int32_t o = row_order[r];
            if (is_long(r)) {
                for (int64_t p = a.ptr[o]; p < a.ptr[o + 1]; ++p) {
                    s.long_idx.push_back(col_rename[a.idx[p]]);
                    s.long_val.push_back(a.val[p] * row_scale[o] * col_scale[a.idx[p]]);
                }
                s.long_line.push_back(r);
                s.long_off.push_back(static_cast<int32_t>(s.long_idx.size()));
                continue;
            }
            int32_t k = 0;
            for (int64_t p = a.ptr[o]; p < a.ptr[o + 1]; ++p, ++k) {
                int32_t e = s.off[sl] + k * 32 + lane;
                s.idx[e] = col_rename[a.idx[p]];
                s.val[e] = a.val[p] * row_scale[o] * col_scale[a.idx[p]];
            }
        }
    return s;
}

void warp_schedule(const Sell& s, int warps, std::vector<int32_t>* sched_off,
                   std::vector<int32_t>* sched) {
    std::vector<int32_t> order(s.nslices);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t x, int32_t y) { return s.length[x] > s.length[y]; });
    std::vector<int64_t> load(warps, 0);
    std::vector<std::vector<int32_t>> lists(warps);
    for (int32_t sl : order) {
        int w = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
        lists[w].push_back(sl);
        load[w] += s.length[sl] + 4;  // +4: the per-slice elementwise update
    }
    sched_off->assign(warps + 1, 0);
    sched->clear();
    for (int w = 0; w < warps; ++w) {
        std::sort(lists[w].begin(), lists[w].end());
        for (int32_t sl : lists[w]) sched->push_back(sl);
        (*sched_off)[w + 1] = static_cast<int32_t>(sched->size());
    }
}

void warp_schedule_split(const Sell& s, int warps, std::vector<int32_t>* sched_off, std::vector<int32_t>* sched,
                         std::vector<int32_t>* long_sched_off, std::vector<int32_t>* long_sched) {
    std::vector<int64_t> load(warps, 0);
    std::vector<std::vector<int32_t>> lists(warps), llists(warps);
    const int32_t nlong = static_cast<int32_t>(s.long_line.size());
    std::vector<int32_t> lorder(nlong);
    std::iota(lorder.begin(), lorder.end(), 0);
    auto llen = [&](int32_t q) { return s.long_off[q + 1] - s.long_off[q]; };
    std::stable_sort(lorder.begin(), lorder.end(), [&](int32_t x, int32_t y) { return llen(x) > llen(y); });
    for (int32_t q : lorder) {
        int w = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
        llists[w].push_back(q);
        load[w] += (llen(q) + 31) / 32 + 8;
    }
    std::vector<int32_t> order(s.nslices);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t x, int32_t y) { return s.length[x] > s.length[y]; });
    for (int32_t sl : order) {
        int w = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
        lists[w].push_back(sl);
        load[w] += s.length[sl] + 4;
    }
    sched_off->assign(warps + 1, 0);
    long_sched_off->assign(warps + 1, 0);
    sched->clear();
    long_sched->clear();
    for (int w = 0; w < warps; ++w) {
        std::sort(lists[w].begin(), lists[w].end());
        for (int32_t sl : lists[w]) sched->push_back(sl);
        (*sched_off)[w + 1] = static_cast<int32_t>(sched->size());
        std::sort(llists[w].begin(), llists[w].end());
        for (int32_t q : llists[w]) long_sched->push_back(q);
        (*long_sched_off)[w + 1] = static_cast<int32_t>(long_sched->size());
    }
}

}  // namespace fbalp
