// Host check of the bank-spreading entry order (spread_banks): on seeded
// random sparse matrices shaped like the metabolic models (row lengths
// 1-18 plus a few hub rows above the long-line cut), every row keeps its
// entries (index and value pairs, as a multiset), padding keeps the padding
// index, long lines are untouched, and the gather wavefront count does not
// rise.  Prints the wavefront totals before and after.
#include <algorithm>
#include <cstdio>
#include <numeric>
#include <random>
#include <vector>

#include "prepare.h"

using namespace fbalp;

static std::vector<std::vector<std::pair<int32_t, double>>> rows_of(const Sell& s, int32_t rows, int32_t pad) {
    std::vector<std::vector<std::pair<int32_t, double>>> out(rows);
    for (int32_t sl = 0; sl < s.nslices; ++sl)
        for (int32_t k = 0; k < s.length[sl]; ++k)
            for (int lane = 0; lane < 32; ++lane) {
                const int32_t r = sl * 32 + lane, e = s.off[sl] + k * 32 + lane;
                if (s.idx[e] == pad) continue;
                if (r >= rows) return {};
                out[r].emplace_back(s.idx[e], s.val[e]);
            }
    for (auto& v : out) std::sort(v.begin(), v.end());
    return out;
}

int main() {
    int bad = 0;
    int64_t before_total = 0, after_total = 0;
    for (int seed = 0; seed < 6; ++seed) {
        std::mt19937 rng(seed);
        const int32_t m = 700 + 150 * seed, n = 2 * m;
        Csr a;
        a.rows = m;
        a.cols = n;
        a.ptr.assign(m + 1, 0);
        for (int32_t i = 0; i < m; ++i) {
            int len = 1 + static_cast<int>(rng() % 18);
            if (i % 97 == 0) len = 40 + static_cast<int>(rng() % 40);  // hub rows
            std::vector<int32_t> cols(n);
            std::iota(cols.begin(), cols.end(), 0);
            for (int k = 0; k < len; ++k) std::swap(cols[k], cols[k + rng() % (n - k)]);
            std::sort(cols.begin(), cols.begin() + len);
            for (int k = 0; k < len; ++k) {
                a.idx.push_back(cols[k]);
                a.val.push_back(0.5 + static_cast<double>(rng() % 1000) / 100.0);
            }
            a.ptr[i + 1] = static_cast<int64_t>(a.idx.size());
        }
        std::vector<int32_t> order(m), rename(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
            return a.ptr[x + 1] - a.ptr[x] > a.ptr[y + 1] - a.ptr[y];
        });
        std::iota(rename.begin(), rename.end(), 0);
        const std::vector<double> ones_m(m, 1.0), ones_n(n, 1.0);
        Sell s = build_sell(a, order, rename, ones_m, ones_n, n, kLongCut);
        Sell t = s;
        spread_banks(&t, n);
        const int64_t w0 = gather_wavefronts(s), w1 = gather_wavefronts(t);
        before_total += w0;
        after_total += w1;
        if (w1 > w0) { bad++; printf("seed %d: wavefronts rose %ld -> %ld\n", seed, (long)w0, (long)w1); }
        const auto r0 = rows_of(s, m, n), r1 = rows_of(t, m, n);
        if (r0.empty() || r0 != r1) { bad++; printf("seed %d: row contents changed\n", seed); }
        if (s.off != t.off || s.length != t.length || s.lmask != t.lmask || s.long_idx != t.long_idx ||
            s.long_val != t.long_val || s.long_off != t.long_off || s.long_line != t.long_line) {
            bad++;
            printf("seed %d: slice shape or long lines changed\n", seed);
        }
        for (int32_t sl = 0; sl < t.nslices; ++sl)
            for (int lane = 0; lane < 32; ++lane)
                if ((t.lmask[sl] >> lane) & 1u)
                    for (int32_t k = 0; k < t.length[sl]; ++k)
                        if (t.idx[t.off[sl] + k * 32 + lane] != n) { bad++; printf("long lane not padding\n"); }
    }
    printf("wavefronts before %ld after %ld bad %d\n", (long)before_total, (long)after_total, bad);
    return bad ? 1 : 0;
}
