// Host-side preprocessing of one species matrix: canonical CSR, Ruiz +
// Pock-Chambolle scaling, spectral step, SELL-32 slicing, warp schedules.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace fbalp {

struct Csr {
    int32_t rows = 0, cols = 0;
    std::vector<int64_t> ptr;
    std::vector<int32_t> idx;
    std::vector<double> val;
};

// Canonicalise: sort columns inside every row, sum duplicates, drop zeros.
// Returns false (with a message) on out-of-range indices, a non-monotone row
// pointer or non-finite values.
bool canonical_csr(int32_t rows, int32_t cols, const int64_t* indptr, const int32_t* indices,
                   const double* values, Csr* out, std::string* err);

Csr transpose(const Csr& a);

struct Scaling {
    std::vector<double> dr, dc;  // original row / column order
    double sigma_max = 0.0;      // ||Dr A Dc||_2 estimate
    double eta = 1.0;            // step size
};

Scaling scale_matrix(const Csr& a, int ruiz_iterations, int power_iterations, double step_safety);

// SELL-32 slices of a matrix whose rows are visited in `row_order` (new ->
// old) and whose column indices are renamed by `col_rename` (old -> new).
// Padding entries point at `pad_index` with value 0.
struct Sell {
    int32_t nslices = 0;
    std::vector<int32_t> off;    // nslices + 1, in elements
    std::vector<int32_t> idx;
    std::vector<double> val;
    std::vector<int32_t> length; // slice lengths
    // long lines (build_sell with a cut): rows longer than the cut are left
    // out of the slices (their lanes are empty, flagged in lmask) and stored
    // unpadded, one after another, for a warp to walk together
    std::vector<uint32_t> lmask;    // per slice: bit `lane` set = a long line
    std::vector<int32_t> long_line; // new index of each long line
    std::vector<int32_t> long_off;  // long lines + 1, in elements
    std::vector<int32_t> long_idx;
    std::vector<double> long_val;
};

Sell build_sell(const Csr& a, const std::vector<int32_t>& row_order,
                const std::vector<int32_t>& col_rename, const std::vector<double>& row_scale,
                const std::vector<double>& col_scale, int32_t pad_index, int32_t long_cut = 0);

// Reorder the entries inside each row of a slice (padding slots included:
// a row's entries may sit at any of the slice's steps) so that the lanes
// of one step gather from distinct shared-memory banks: a greedy placement
// step by step, then `rounds` passes of pairwise swaps within a lane.  The
// cost of a step is its gather wavefronts in the paired kernel (float2
// targets, per half-warp, 16 bank pairs) plus in the single-instance kernel
// (float targets, per warp, 32 banks).  Row sums are unchanged; only the
// FP32 accumulation order moves.
void spread_banks(Sell* s, int32_t pad_index, int rounds = 3);

// The same cost summed over every step of every slice (both kernels).
int64_t gather_wavefronts(const Sell& s);

// Rows longer than this many entries are long lines (walked by a whole warp
// in the re-centred kernels): one warp step covers 32 of their entries.
constexpr int32_t kLongCut = 32;

// Greedy longest-first assignment of slices to `warps` warps.
void warp_schedule(const Sell& s, int warps, std::vector<int32_t>* sched_off,
                   std::vector<int32_t>* sched);

// The same with the long lines of a cut Sell: long lines first (cost
// ceil(len / 32) + 8: strided loads, a shuffle reduction and one lane's
// update), then the slices (cost len + 4).
void warp_schedule_split(const Sell& s, int warps, std::vector<int32_t>* sched_off, std::vector<int32_t>* sched,
                         std::vector<int32_t>* long_sched_off, std::vector<int32_t>* long_sched);

}  // namespace fbalp
