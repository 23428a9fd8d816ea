// Host-side check of the shared-memory layout planner: every region starts on
// a 16-byte boundary, regions never overlap, and the plan respects its cap.
#include "fbalp_internal.h"
#include <cstdio>
#include <vector>
#include <algorithm>
// Check alignment AND that no two regions of a layout overlap.
int main() {
  int bad = 0, total = 0;
  for (int w : {1, 4, 8, 16, 32})
    for (int n : {1, 2, 260, 650, 2600, 6800})
      for (int m : {0, 1, 120, 300, 1200, 3400})
        for (int esz : {4, 8})
          for (long cap : {8192L, 100000L, 230000L}) {
            int an = (m+31)/32, atn = (n+31)/32;
            long ae = 37L*an*32/3, ate = 11L*atn*32/3;
            auto P = fbalp::plan_layout(n, m, w, an, atn, ae, ate, esz, cap, true);
            auto& L = P.layout; total++;
            struct R { long b, e; int slab; };
            std::vector<R> rs = {{L.sched_a_off, L.sched_a_off + 4*(w+1), 0}, {L.sched_at_off, L.sched_at_off + 4*(w+1), 0},
                                 {L.list_a, L.list_a + 16L*an, 0}, {L.list_at, L.list_at + 16L*atn, 0}};
            if (L.mat_smem) { rs.push_back({L.mat_a_idx, L.mat_a_idx + 2*ae, 0}); rs.push_back({L.mat_at_idx, L.mat_at_idx + 2*ate, 0});
                              rs.push_back({L.mat_a_val, L.mat_a_val + esz*ae, 0}); rs.push_back({L.mat_at_val, L.mat_at_val + esz*ate, 0}); }
            long e[fbalp::kArrayCount]; fbalp::array_elems(n, m, e);
            for (int a = 0; a < fbalp::kArrayCount; ++a) rs.push_back({L.arr[a], L.arr[a] + esz*e[a], ((L.smem_mask>>a)&1) ? 0 : 1});
            bool ok = fbalp::layout_aligned(L);
            for (auto& r : rs) { if (r.slab == 0 && r.e > P.smem_bytes) ok = false; if (r.slab == 1 && r.e > P.slab_bytes) ok = false; }
            for (size_t i = 0; i < rs.size(); ++i) for (size_t j = i+1; j < rs.size(); ++j)
              if (rs[i].slab == rs[j].slab && rs[i].b < rs[j].e && rs[j].b < rs[i].e && rs[i].e > rs[i].b && rs[j].e > rs[j].b) ok = false;
            if (P.smem_bytes > cap) ok = false;
            if (!ok) { bad++; if (bad < 5) printf("bad w=%d n=%d m=%d esz=%d cap=%ld\n", w, n, m, esz, cap); }
          }
  printf("layouts checked %d, bad %d\n", total, bad);
  return bad != 0;
}
