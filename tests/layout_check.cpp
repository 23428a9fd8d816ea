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
  // re-centred layouts (single, staged or streamed; paired): operand lists,
  // long-line lists and masks, packed words, FP32 / float2 vectors; disjoint,
  // inside the cap, every staged index (an element offset of a gather target
  // in 4- or 8-byte units) within 16 bits
  for (int w : {1, 8, 16, 32})
    for (int n : {1, 2, 260, 900, 1800, 2700, 6800})
      for (int m : {0, 1, 120, 950, 1400, 3400})
        for (int neqf : {0, 1, 2})
          for (int nl : {0, 1, 12})
            for (long cap : {8192L, 100000L, 225000L})
              for (int kind : {0, 1, 2, 3}) {  // 0 staged, 1 streamed, 2 paired, 3 staged with FP32 values
                const int neq = neqf == 0 ? m : (neqf == 1 ? m / 2 : 0);
                fbalp::LinesShape sa, sat;
                sa.nslices = (m+31)/32; sat.nslices = (n+31)/32;
                sa.elems = 37L*sa.nslices*32/3; sat.elems = 11L*sat.nslices*32/3;
                sa.nlong = std::min(nl, m); sat.nlong = std::min(nl, n);
                sa.long_elems = 70L*sa.nlong; sat.long_elems = 45L*sat.nlong;
                auto P = kind == 2 ? fbalp::plan_layout_pair(n, m, neq, w, sa, sat, cap)
                                   : fbalp::plan_layout_recentred(n, m, w, sa, sat, cap, kind != 1, kind == 3);
                auto& L = P.layout; total++;
                if (!L.recentred) continue;
                const long u = kind == 2 ? 8 : 4;  // vector element bytes
                struct R { long b, e; };
                std::vector<R> rs = {{L.sched_a_off, L.sched_a_off + 4*(w+1)}, {L.sched_at_off, L.sched_at_off + 4*(w+1)},
                                     {L.lsched_a_off, L.lsched_a_off + 4*(w+1)}, {L.lsched_at_off, L.lsched_at_off + 4*(w+1)},
                                     {L.list_a, L.list_a + 16L*sa.nslices}, {L.list_at, L.list_at + 16L*sat.nslices},
                                     {L.llist_a, L.llist_a + 16L*sa.nlong}, {L.llist_at, L.llist_at + 16L*sat.nlong},
                                     {L.lmask_a, L.lmask_a + 4L*sa.nslices}, {L.lmask_at, L.lmask_at + 4L*sat.nslices},
                                     {L.arr[fbalp::kXbar], L.arr[fbalp::kXbar] + u*(n+1)}, {L.arr[fbalp::kY], L.arr[fbalp::kY] + u*(m+1)},
                                     {L.arr[fbalp::kC], L.arr[fbalp::kC] + u*n}, {L.arr[fbalp::kL], L.arr[fbalp::kL] + u*n},
                                     {L.arr[fbalp::kU], L.arr[fbalp::kU] + u*n}, {L.arr[fbalp::kB], L.arr[fbalp::kB] + u*m},
                                     {L.arr[fbalp::kYa], L.arr[fbalp::kYa] + (kind == 2 ? u*(m-neq) : u*m)}};
                if (kind != 2) rs.push_back({L.arr[fbalp::kX], L.arr[fbalp::kX] + u*n});
                if (L.mat_smem && kind != 3) {
                  rs.push_back({L.mat_a_idx, L.mat_a_idx + 4*sa.elems}); rs.push_back({L.mat_at_idx, L.mat_at_idx + 4*sat.elems});
                  rs.push_back({L.mat_a_long, L.mat_a_long + 4*sa.long_elems}); rs.push_back({L.mat_at_long, L.mat_at_long + 4*sat.long_elems});
                }
                if (L.mat_smem && kind == 3) {
                  rs.push_back({L.mat_a_idx, L.mat_a_idx + 2*sa.elems}); rs.push_back({L.mat_at_idx, L.mat_at_idx + 2*sat.elems});
                  rs.push_back({L.mat_a_long, L.mat_a_long + 2*sa.long_elems}); rs.push_back({L.mat_at_long, L.mat_at_long + 2*sat.long_elems});
                  rs.push_back({L.mat_a_val, L.mat_a_val + 4*sa.elems}); rs.push_back({L.mat_at_val, L.mat_at_val + 4*sat.elems});
                  rs.push_back({L.mat_a_lval, L.mat_a_lval + 4*sa.long_elems}); rs.push_back({L.mat_at_lval, L.mat_at_lval + 4*sat.long_elems});
                }
                bool ok = fbalp::layout_aligned(L) && P.smem_bytes <= cap && L.recentred == (kind == 2 ? 2 : 1) &&
                          L.f32_values == (kind == 3 ? 1 : 0);
                for (auto& r : rs) if (r.e > P.smem_bytes) ok = false;
                for (size_t i = 0; i < rs.size(); ++i) for (size_t j = i+1; j < rs.size(); ++j)
                  if (rs[i].b < rs[j].e && rs[j].b < rs[i].e && rs[i].e > rs[i].b && rs[j].e > rs[j].b) ok = false;
                if (L.mat_smem && (L.arr[fbalp::kY] / u + m > 65535 || L.arr[fbalp::kXbar] / u + n > 65535)) ok = false;
                if (!ok) { bad++; if (bad < 5) printf("bad recentred kind=%d w=%d n=%d m=%d neq=%d nl=%d cap=%ld\n", kind, w, n, m, neq, nl, cap); }
              }
  printf("layouts checked %d, bad %d\n", total, bad);
  return bad != 0;
}
