// Constants and helpers shared by the host engine and the kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pdhg_kernel.cuh"

namespace fbalp {

constexpr int kMetrics = 8;
constexpr int kRedSums = 10;
constexpr int kMaxThreads = 1024;

constexpr int kStatusOptimal = 0;
constexpr int kStatusIterationLimit = 1;
constexpr int kStatusNumerical = 2;
constexpr int kStatusInvalid = 3;
constexpr int kStatusNotRun = 4;
constexpr int kStatusHandoff = 5;

// Restart rule of the Halpern scheme (Lu & Yang; cuPDLPx) and the PDLP
// primal-weight smoothing (a solve parameter, primal_weight_smoothing).
constexpr double kBetaSufficient = 0.2;
constexpr double kBetaNecessary = 0.8;
constexpr double kBetaArtificial = 0.36;
// the FP32 phase only hands off on a stall once its error is below this
constexpr double kStallFloor = 1.0;

// Element counts of the per-instance arrays (gather targets carry a zero
// slot at index n / m), in shared-memory priority order.
inline void array_elems(int n, int m, int64_t* s) {
    const int64_t v[kArrayCount] = {n + 1, m + 1, n, n, m, n, n, n, m, n + 1, m + 1, 0};
    for (int a = 0; a < kArrayCount; ++a) s[a] = v[a];
}

inline int64_t align_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

// Host-side layout planner: decide, for one species and one precision, what
// lives in the CTA's shared memory (schedule lists always; the two gather
// targets; then the matrix slices with 16-bit indices; then the remaining
// arrays in priority order) and what spills to the CTA's global slab.
struct LayoutPlan {
    Layout layout;
    int64_t smem_bytes;  // dynamic shared memory used
    int64_t slab_bytes;  // per-CTA global slab bytes
};

inline LayoutPlan plan_layout(int n, int m, int warps, int a_nslices, int at_nslices,
                              int64_t a_elems, int64_t at_elems, int esz, int64_t smem_cap,
                              bool allow_matrix) {
    LayoutPlan P{};
    Layout& L = P.layout;
    int64_t off = 0;
    L.sched_a_off = off;
    off += 4 * (warps + 1);
    L.sched_at_off = off;
    off += 4 * (warps + 1);
    off = align_up(off, 16);  // int4 slice lists need 16-byte alignment
    L.list_a = off;
    off += static_cast<int64_t>(sizeof(int4)) * a_nslices;
    L.list_at = off;
    off += static_cast<int64_t>(sizeof(int4)) * at_nslices;
    off = align_up(off, 16);
    int64_t slab = 0;
    int64_t e[kArrayCount];
    array_elems(n, m, e);
    L.smem_mask = 0;
    auto place = [&](int a) {
        const int64_t bytes = align_up(e[a] * esz, 16);
        if (off + bytes <= smem_cap) {
            L.arr[a] = off;
            L.smem_mask |= 1 << a;
            off += bytes;
        } else {
            L.arr[a] = slab;
            slab += bytes;
        }
    };
    place(0);  // xbar
    place(1);  // y
    const int64_t mat = align_up(2 * a_elems, 16) + align_up(2 * at_elems, 16) +
                        align_up(esz * a_elems, 16) + align_up(esz * at_elems, 16);
    L.mat_smem = 0;
    if (allow_matrix && n + 1 < 65536 && m + 1 < 65536 && off + mat <= smem_cap) {
        L.mat_smem = 1;
        L.mat_a_idx = off;
        off += align_up(2 * a_elems, 16);
        L.mat_at_idx = off;
        off += align_up(2 * at_elems, 16);
        L.mat_a_val = off;
        off += align_up(esz * a_elems, 16);
        L.mat_at_val = off;
        off += align_up(esz * at_elems, 16);
    }
    for (int a = 2; a < kArrayCount; ++a) place(a);
    P.smem_bytes = off;
    P.slab_bytes = slab;
    return P;
}

// FP64 layout with the unscaled FP32 matrix staged: schedule lists, the two
// FP64 gather targets z (n+1) and w (m+1), the matrix slices (16-bit indices,
// FP32 values), then x, xa and the remaining arrays while they fit.  Returns
// a plan with unscaled = 0 when the targets and the matrix do not fit.
inline LayoutPlan plan_layout_unscaled(int n, int m, int warps, int a_nslices, int at_nslices,
                                       int64_t a_elems, int64_t at_elems, int64_t smem_cap) {
    LayoutPlan P{};
    Layout& L = P.layout;
    int64_t off = 0;
    L.sched_a_off = off;
    off += 4 * (warps + 1);
    L.sched_at_off = off;
    off += 4 * (warps + 1);
    off = align_up(off, 16);
    L.list_a = off;
    off += static_cast<int64_t>(sizeof(int4)) * a_nslices;
    L.list_at = off;
    off += static_cast<int64_t>(sizeof(int4)) * at_nslices;
    off = align_up(off, 16);
    const int esz = 8;
    const int64_t need = align_up((int64_t(n) + 1) * esz, 16) + align_up((int64_t(m) + 1) * esz, 16) +
                         align_up(2 * a_elems, 16) + align_up(2 * at_elems, 16) + align_up(4 * a_elems, 16) +
                         align_up(4 * at_elems, 16);
    const int64_t max_word = (int64_t(1) << 16) - 1;
    if (off + need > smem_cap || (off + need) / esz > max_word) return P;  // unscaled stays 0
    L.unscaled = 1;
    L.mat_smem = 1;
    L.smem_mask = 0;
    int64_t e[kArrayCount];
    array_elems(n, m, e);
    e[kW] = m + 1;
    auto put = [&](int a) {
        L.arr[a] = off;
        L.smem_mask |= 1 << a;
        off += align_up(e[a] * esz, 16);
    };
    put(kXbar);
    put(kW);
    L.mat_a_idx = off;
    off += align_up(2 * a_elems, 16);
    L.mat_at_idx = off;
    off += align_up(2 * at_elems, 16);
    L.mat_a_val = off;
    off += align_up(4 * a_elems, 16);
    L.mat_at_val = off;
    off += align_up(4 * at_elems, 16);
    int64_t slab = 0;
    const int order[] = {kX, kXa, kY, kYa, kC, kL, kU, kB, kXs, kYs};
    for (int a : order) {
        const int64_t bytes = align_up(e[a] * esz, 16);
        if (off + bytes <= smem_cap) {
            L.arr[a] = off;
            L.smem_mask |= 1 << a;
            off += bytes;
        } else {
            L.arr[a] = slab;
            slab += bytes;
        }
    }
    P.smem_bytes = off;
    P.slab_bytes = slab;
    return P;
}

// Sizes of one re-centred operand (DevLines) for the layout planners.
struct LinesShape {
    int32_t nslices = 0, nlong = 0;
    int64_t elems = 0, long_elems = 0;
};

// The part of a re-centred layout that describes the operands: slice and
// long-line schedule offsets, slice lists, long-line lists and per-slice
// long-lane masks of A and A^T.  Returns the next free offset (16-aligned).
inline int64_t place_recentred_lists(Layout& L, int warps, const LinesShape& a, const LinesShape& at) {
    int64_t off = 0;
    L.sched_a_off = off;
    off += 4 * (warps + 1);
    L.sched_at_off = off;
    off += 4 * (warps + 1);
    L.lsched_a_off = off;
    off += 4 * (warps + 1);
    L.lsched_at_off = off;
    off += 4 * (warps + 1);
    off = align_up(off, 16);
    L.list_a = off;
    off += static_cast<int64_t>(sizeof(int4)) * a.nslices;
    L.list_at = off;
    off += static_cast<int64_t>(sizeof(int4)) * at.nslices;
    L.llist_a = off;
    off += static_cast<int64_t>(sizeof(int4)) * a.nlong;
    L.llist_at = off;
    off += static_cast<int64_t>(sizeof(int4)) * at.nlong;
    L.lmask_a = off;
    off += 4 * static_cast<int64_t>(a.nslices);
    L.lmask_at = off;
    off += 4 * static_cast<int64_t>(at.nslices);
    return align_up(off, 16);
}

// Re-centred FP32 layout: everything the iteration touches in shared memory
// (the operand lists; the FP32 gather targets dxbar (n+1) and dy (m+1); the
// matrix as packed words (16-bit index, BF16 value) -- slices, then long
// lines; dx, d, l - x^, u - x^ (n each); r and the inequality bound -y^ (m
// each)), and in the CTA's global slab the two FP64 point buffers of x and
// y, the FP32 reduced cost / residual of the last evaluated candidate, and
// the instance's scaled FP64 objective, bounds and right-hand side.  Returns
// recentred = 0 when the shared part does not fit.  With `stage` false the
// matrix is not staged (it is streamed from L2 every iteration) and only the
// lists and vectors need to fit.
inline LayoutPlan plan_layout_recentred(int n, int m, int warps, const LinesShape& sa, const LinesShape& sat,
                                        int64_t smem_cap, bool stage = true, bool f32_values = false) {
    LayoutPlan P{};
    Layout& L = P.layout;
    int64_t off = place_recentred_lists(L, warps, sa, sat);
    if (n + 1 >= 65536 || m + 1 >= 65536) return P;
    const int64_t e[kArrayCount] = {n + 1, m + 1, n, 0, m, n, n, n, m, 0, 0, 0};
    L.smem_mask = 0;
    auto put = [&](int a) {
        L.arr[a] = off;
        L.smem_mask |= 1 << a;
        off += align_up(e[a] * 4, 16);
    };
    put(kXbar);
    put(kY);
    if (stage && !f32_values) {  // packed 32-bit words (16-bit index | BF16 value)
        L.mat_a_idx = off;
        off += align_up(4 * sa.elems, 16);
        L.mat_at_idx = off;
        off += align_up(4 * sat.elems, 16);
        L.mat_a_long = off;
        off += align_up(4 * sa.long_elems, 16);
        L.mat_at_long = off;
        off += align_up(4 * sat.long_elems, 16);
        L.mat_a_val = L.mat_a_idx;
        L.mat_at_val = L.mat_at_idx;
    } else if (stage) {  // 16-bit indices and FP32 values in separate arrays
        for (auto* pr : {&L.mat_a_idx, &L.mat_at_idx, &L.mat_a_long, &L.mat_at_long}) {
            const int64_t cnt = pr == &L.mat_a_idx ? sa.elems : pr == &L.mat_at_idx ? sat.elems
                                : pr == &L.mat_a_long ? sa.long_elems : sat.long_elems;
            *pr = off;
            off += align_up(2 * cnt, 16);
        }
        for (auto* pr : {&L.mat_a_val, &L.mat_at_val, &L.mat_a_lval, &L.mat_at_lval}) {
            const int64_t cnt = pr == &L.mat_a_val ? sa.elems : pr == &L.mat_at_val ? sat.elems
                                : pr == &L.mat_a_lval ? sa.long_elems : sat.long_elems;
            *pr = off;
            off += align_up(4 * cnt, 16);
        }
    }
    L.f32_values = f32_values ? 1 : 0;
    for (int a : {kX, kC, kL, kU, kB, kYa}) put(a);
    if (off > smem_cap) return P;
    // every staged 16-bit index is an element offset from the start of
    // shared memory
    if (stage && off / 4 > (int64_t(1) << 16) - 1) return P;
    L.mat_smem = stage ? 1 : 0;
    L.recentred = 1;
    int64_t slab = 0;
    for (int b = 0; b < 2; ++b) {
        L.pt_x[b] = slab;
        slab += align_up((int64_t(n) + 1) * 8, 16);
        L.pt_y[b] = slab;
        slab += align_up((int64_t(m) + 1) * 8, 16);
    }
    L.dcand = slab;
    slab += align_up(int64_t(n) * 4, 16);
    L.rcand = slab;
    slab += align_up(int64_t(m) * 4, 16);
    for (int64_t* o : {&L.sc_c, &L.sc_l, &L.sc_u}) {
        *o = slab;
        slab += align_up(int64_t(n) * 8, 16);
    }
    L.sc_b = slab;
    slab += align_up(int64_t(m) * 8, 16);
    P.smem_bytes = off;
    P.slab_bytes = slab;
    return P;
}

// Paired re-centred FP32 layout: two instances of one species share one CTA
// and one staged copy of the species' packed matrix words.  Their vectors
// are interleaved as float2 (component s = instance slot s): the gather
// targets dxbar (n+1) and dy (m+1), then the packed words (16-bit index =
// float2 element offset of the gather target from the start of shared
// memory | BF16 value; slices, then long lines), then d, l - x^, u - x^ (n
// each), r (m) and the inequality bound -y^ of the rows at and beyond neq
// (m - neq).  The Halpern iterate x is not stored: with reflection 1 it
// equals w xbar, with w the previous iteration's Halpern weight.  The slab
// holds ONE instance's FP64 data (the re-centred slab); a CTA uses two
// consecutive slabs.  Returns recentred = 0 when the shared part does not
// fit.
inline LayoutPlan plan_layout_pair(int n, int m, int neq, int warps, const LinesShape& sa, const LinesShape& sat,
                                   int64_t smem_cap) {
    LayoutPlan P{};
    Layout& L = P.layout;
    int64_t off = place_recentred_lists(L, warps, sa, sat);
    if (n + 1 >= 65536 || m + 1 >= 65536 || neq < 0 || neq > m) return P;
    L.smem_mask = 0;
    auto put = [&](int a, int64_t elems) {
        L.arr[a] = off;
        L.smem_mask |= 1 << a;
        off += align_up(elems * 8, 16);
    };
    put(kXbar, int64_t(n) + 1);
    put(kY, int64_t(m) + 1);
    // every staged 16-bit index is a float2 element offset of a gather
    // target from the start of shared memory
    if (off / 8 > (int64_t(1) << 16) - 1) return P;
    L.mat_a_idx = off;
    off += align_up(4 * sa.elems, 16);
    L.mat_at_idx = off;
    off += align_up(4 * sat.elems, 16);
    L.mat_a_long = off;
    off += align_up(4 * sa.long_elems, 16);
    L.mat_at_long = off;
    off += align_up(4 * sat.long_elems, 16);
    L.mat_a_val = L.mat_a_idx;
    L.mat_at_val = L.mat_at_idx;
    put(kC, n);
    put(kL, n);
    put(kU, n);
    put(kB, m);
    put(kYa, int64_t(m) - neq);
    if (off > smem_cap) return P;
    L.mat_smem = 1;
    L.recentred = 2;
    int64_t slab = 0;
    for (int b = 0; b < 2; ++b) {
        L.pt_x[b] = slab;
        slab += align_up((int64_t(n) + 1) * 8, 16);
        L.pt_y[b] = slab;
        slab += align_up((int64_t(m) + 1) * 8, 16);
    }
    L.dcand = slab;
    slab += align_up(int64_t(n) * 4, 16);
    L.rcand = slab;
    slab += align_up(int64_t(m) * 4, 16);
    for (int64_t* o : {&L.sc_c, &L.sc_l, &L.sc_u}) {
        *o = slab;
        slab += align_up(int64_t(n) * 8, 16);
    }
    L.sc_b = slab;
    slab += align_up(int64_t(m) * 8, 16);
    P.smem_bytes = off;
    P.slab_bytes = slab;
    return P;
}

// Every region must start on a 16-byte boundary (int4 lists, FP64 arrays).
inline bool layout_aligned(const Layout& L) {
    const int64_t offs[] = {L.list_a, L.list_at, L.mat_a_idx, L.mat_at_idx, L.mat_a_val, L.mat_at_val,
                            L.llist_a, L.llist_at, L.mat_a_long, L.mat_at_long, L.mat_a_lval, L.mat_at_lval};
    for (int64_t o : offs)
        if (o % 16 != 0) return false;
    for (int a = 0; a < kArrayCount; ++a)
        if (L.arr[a] % 16 != 0) return false;
    for (int64_t o : {L.sched_a_off, L.sched_at_off, L.lsched_a_off, L.lsched_at_off, L.lmask_a, L.lmask_at})
        if (o % 4 != 0) return false;
    return true;
}

const void* kernel_symbol(bool fp64, int threads, bool fast);
const void* recentred_symbol(int threads, bool staged, bool patched, bool f32_values = false);
cudaError_t launch_recentred(bool staged, bool patched, int grid, int threads, size_t smem, cudaStream_t stream,
                             const KernelParams& p, bool f32_values = false);
const void* pair_symbol(int threads);
cudaError_t launch_pair(int grid, int threads, size_t smem, cudaStream_t stream, const KernelParams& p);
cudaError_t launch_pdhg(bool fp64, bool fast, int grid, int threads, size_t smem, cudaStream_t stream,
                        const KernelParams& p);

}  // namespace fbalp
