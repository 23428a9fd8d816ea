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

namespace {

// Shared-memory wavefronts of one step k of a slice: the lanes gather
// target[lane] (an element index).  Paired kernel: float2 targets, 16
// lanes (half a warp) per 128-byte wavefront, 16 bank pairs; single
// kernel: float targets, 32 lanes, 32 banks.  Per group the count is the
// largest number of DISTINCT targets sharing a bank (equal targets are one
// broadcast).
int step_wavefronts(const int32_t* t) {
    // per bank, the distinct targets seen so far (a target is compared only
    // with the targets of its own bank)
    int total = 0;
    int32_t seen[32][32];
    int cnt[32];
    for (int g = 0; g < 32; g += 16) {  // float2: two half-warps, 16 bank pairs
        int worst = 0;
        for (int c = 0; c < 16; ++c) cnt[c] = 0;
        for (int q = g; q < g + 16; ++q) {
            const int c = t[q] & 15;
            bool dup = false;
            for (int r = 0; r < cnt[c] && !dup; ++r) dup = seen[c][r] == t[q];
            if (!dup) {
                seen[c][cnt[c]++] = t[q];
                worst = std::max(worst, cnt[c]);
            }
        }
        total += worst;
    }
    int worst = 0;
    for (int c = 0; c < 32; ++c) cnt[c] = 0;
    for (int q = 0; q < 32; ++q) {  // float: one warp, 32 banks
        const int c = t[q] & 31;
        bool dup = false;
        for (int r = 0; r < cnt[c] && !dup; ++r) dup = seen[c][r] == t[q];
        if (!dup) {
            seen[c][cnt[c]++] = t[q];
            worst = std::max(worst, cnt[c]);
        }
    }
    return total + worst;
}

}  // namespace

void spread_banks(Sell* s, int32_t pad_index, int rounds) {
    std::vector<int32_t> grid;   // [k][lane] targets of one slice
    std::vector<double> gval;
    std::vector<int> cost;
    for (int32_t sl = 0; sl < s->nslices; ++sl) {
        const int32_t L = s->length[sl];
        if (L < 2) continue;
        const int32_t base = s->off[sl];
        // greedy: step by step, each lane with entries left places the one
        // whose bank is least used by the distinct targets placed so far
        std::vector<std::vector<std::pair<int32_t, double>>> left(32);
        for (int lane = 0; lane < 32; ++lane)
            for (int32_t k = 0; k < L; ++k) {
                const int32_t e = base + k * 32 + lane;
                if (s->idx[e] != pad_index) left[lane].emplace_back(s->idx[e], s->val[e]);
            }
        grid.assign(static_cast<size_t>(L) * 32, pad_index);
        gval.assign(static_cast<size_t>(L) * 32, 0.0);
        for (int32_t k = 0; k < L; ++k) {
            int32_t* t = &grid[static_cast<size_t>(k) * 32];
            for (int g = 0; g < 32; g += 16) {
                int cnt[16] = {0};
                for (int lane = g; lane < g + 16; ++lane) {
                    auto& cand = left[lane];
                    if (cand.empty()) continue;
                    size_t best = 0;
                    int best_cost = 1 << 30;
                    for (size_t c = 0; c < cand.size(); ++c) {
                        bool dup = false;
                        for (int r = g; r < lane && !dup; ++r) dup = t[r] == cand[c].first;
                        const int cc = dup ? 0 : cnt[cand[c].first & 15] + 1;
                        if (cc < best_cost) {
                            best_cost = cc;
                            best = c;
                        }
                    }
                    bool dup = false;
                    for (int r = g; r < lane && !dup; ++r) dup = t[r] == cand[best].first;
                    if (!dup) ++cnt[cand[best].first & 15];
                    t[lane] = cand[best].first;
                    gval[static_cast<size_t>(k) * 32 + lane] = cand[best].second;
                    cand.erase(cand.begin() + static_cast<std::ptrdiff_t>(best));
                }
            }
        }
        // local search: swap two positions of one lane (an entry with a
        // hole included) while that lowers the two steps' wavefronts
        cost.assign(L, 0);
        for (int32_t k = 0; k < L; ++k) cost[k] = step_wavefronts(&grid[static_cast<size_t>(k) * 32]);
        for (int round = 0; round < rounds; ++round) {
            bool improved = false;
            for (int lane = 0; lane < 32; ++lane) {
                if ((s->lmask[sl] >> lane) & 1u) continue;
                for (int32_t a = 0; a < L; ++a)
                    for (int32_t b = a + 1; b < L; ++b) {
                        int32_t& ta = grid[static_cast<size_t>(a) * 32 + lane];
                        int32_t& tb = grid[static_cast<size_t>(b) * 32 + lane];
                        if (ta == tb) continue;
                        std::swap(ta, tb);
                        const int ca = step_wavefronts(&grid[static_cast<size_t>(a) * 32]);
                        const int cb = step_wavefronts(&grid[static_cast<size_t>(b) * 32]);
                        if (ca + cb < cost[a] + cost[b]) {
                            cost[a] = ca;
                            cost[b] = cb;
                            std::swap(gval[static_cast<size_t>(a) * 32 + lane], gval[static_cast<size_t>(b) * 32 + lane]);
                            improved = true;
                        } else {
                            std::swap(ta, tb);
                        }
                    }
            }
            if (!improved) break;
        }
        for (int32_t k = 0; k < L; ++k)
            for (int lane = 0; lane < 32; ++lane) {
                const int32_t e = base + k * 32 + lane;
                s->idx[e] = grid[static_cast<size_t>(k) * 32 + lane];
                s->val[e] = gval[static_cast<size_t>(k) * 32 + lane];
            }
    }
}

int64_t gather_wavefronts(const Sell& s) {
    int64_t total = 0;
    for (int32_t sl = 0; sl < s.nslices; ++sl)
        for (int32_t k = 0; k < s.length[sl]; ++k) total += step_wavefronts(&s.idx[s.off[sl] + k * 32]);
    return total;
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
