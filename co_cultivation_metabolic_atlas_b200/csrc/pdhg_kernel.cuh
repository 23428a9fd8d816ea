// Persistent, instance-resident restarted Halpern PDHG for batches of LPs
// that share one matrix per species (sm_100a).
//
// One CTA owns one LP instance at a time.  Its iterates, anchors and scaled
// bounds live in shared memory; so do the species' SELL-32 matrix slices
// (16-bit indices) whenever they fit beside them, otherwise the slices are
// streamed from L2.  Arrays that do not fit spill to a per-CTA global slab.
// Every convergence test, restart decision and primal-weight update happens
// inside the kernel.  When an instance finishes (certified, budget exhausted,
// or invalid) the CTA writes its results and pulls the next instance from an
// atomic work queue, so instances of different species and different
// iteration counts share one launch without host round trips.  Consecutive
// instances of the same species reuse the staged matrix.
//
// Arithmetic (per instance, scaled space; oracle/pdhg.py restates it):
//   xn = clip(x - tau (c - A^T y), l, u)             tau = eta/omega
//   yn = P_Y(y + sigma (b - A (2 xn - x)))          sigma = eta*omega
//   x  = w ((1+rho) xn - rho x) + (1-w) xa          w = (k+1)/(k+2)
//   y  = w ((1+rho) yn - rho y) + (1-w) ya
// The reference iterates plain PDHG with a fixed diagonal metric
// (`src/gpu_pdhg_corrector.py:334-358`, `src/gpu_pdhg_workspace.py:122-134`);
// the projections keep its NaN-preserving form (a NaN is never clipped).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fbalp {

constexpr int kMaxWarps = 32;
constexpr int kRed = 16;  // reduced quantities per convergence check
constexpr int kArrayCount = 12;
constexpr int kMaxPatches = 8;  // per-instance matrix entries per species

// Array order: xbar, y, x, xa, ya, c, l, u, b, xs, ys, w.  In the unscaled
// FP64 layout xbar holds z = dc * xbar (the gather target of the A pass) and
// w = dr * y is the gather target of the A^T pass.
enum ArrayId { kXbar = 0, kY, kX, kXa, kYa, kC, kL, kU, kB, kXs, kYs, kW };

// One operand of the re-centred kernels (A for the dual pass, A^T for the
// primal pass): SELL-32 slices whose long lines (more than 32 entries) are
// left out -- their lanes are empty and flagged in `lmask` -- and the long
// lines stored unpadded, each walked by a whole warp.
struct DevLines {
    int32_t nslices, nlong;
    int64_t elems, long_elems;
    const int4* list;             // slices in warp-schedule order {slice, base, len, patched}
    const int32_t* sched_off;     // [warps + 1] ranges of `list` per warp
    const uint32_t* lmask;        // per slice: lanes whose line is long
    const int4* long_list;        // long lines in warp order {line, base, len, 0}
    const int32_t* long_sched_off;  // [warps + 1] ranges of `long_list` per warp
    const uint32_t* pk;           // packed slice words (16-bit index | BF16 value)
    const int32_t* idx;           // slice indices (pad -> n or m)
    const double* v64;            // slice FP64 scaled values
    const float* v32;             // slice FP32 scaled values
    const uint32_t* long_pk;      // long-line words
    const int32_t* long_idx;
    const double* long_v64;
    const float* long_v32;
};

struct DevSpecies {
    int32_t m, n, neq, pad_;
    int32_t a_nslices, at_nslices;
    int64_t a_elems, at_elems;
    const int4* a_list;           // per slice in warp-schedule order: {slice, base, len, 0}
    const int4* at_list;
    const int32_t* a_sched_off;   // [warps + 1] ranges of a_list per warp
    const int32_t* at_sched_off;
    const int32_t* a_idx;         // SELL-32 column indices (new numbering); pad -> n
    const float* a_v32;
    const double* a_v64;
    const int32_t* at_idx;        // pad -> m
    const float* at_v32;
    const double* at_v64;
    const int32_t* row_perm;      // new -> original row
    const int32_t* col_perm;      // new -> original column
    const double* dr;             // new order
    const double* dc;             // new order
    double eta;
    // unscaled values in the same SELL slices: FP32 part (exact for the
    // usual stoichiometric coefficients) and, per new-numbered row of A /
    // A^T, the FP64 remainders of entries FP32 cannot hold exactly
    const float* a_hi;
    const float* at_hi;
    const int32_t* lo_a_ptr;
    const int32_t* lo_a_idx;
    const double* lo_a_val;
    const int32_t* lo_at_ptr;
    const int32_t* lo_at_idx;
    const double* lo_at_val;
    const double* inv_dr;         // 1 / dr, new order
    const double* inv_dc;         // 1 / dc, new order
    // the re-centred phase's operands (long lines split off): the scaled
    // matrix as packed 32-bit words, the 16-bit index in the low half, the
    // value rounded to BF16 in the high half (pk null when n or m exceeds
    // 16-bit indices), with FP64 values for its convergence tests
    DevLines ra, rat;
    // per-instance matrix entries: instance i's matrix is A + sum_p
    // delta_ip e_{row p} e_{col p}^T (new numbering; the slices holding a
    // patched row / column carry w = 1 in their schedule entries); the scaled
    // delta is delta * patch_scale (dr_row dc_col)
    int32_t npatch, pad2_;
    int32_t patch_row[kMaxPatches];
    int32_t patch_col[kMaxPatches];
    double patch_scale[kMaxPatches];
    double patch_base[kMaxPatches];  // scaled template value at each patched entry
    double patch_col_f2;             // sum of squares of the patched columns' other entries (scaled)
    double sigma_max;             // ||A~||_2 estimate of the shared matrix
};

// Byte offsets of one species' working set inside the CTA's dynamic shared
// memory (or its global slab for arrays whose bit in smem_mask is clear).
struct Layout {
    int64_t sched_a_off, sched_at_off, list_a, list_at;
    int32_t mat_smem, smem_mask;
    int32_t unscaled, recentred;
    int64_t mat_a_idx, mat_at_idx, mat_a_val, mat_at_val;
    int64_t arr[kArrayCount];
    // re-centred layouts only: the long lines' schedule offsets [warps + 1],
    // lists (int4), per-slice lane masks (uint32) and packed words
    int64_t lsched_a_off, lsched_at_off, llist_a, llist_at, lmask_a, lmask_at, mat_a_long, mat_at_long;
    // re-centred layouts with FP32 matrix values (f32_values = 1): the
    // staged 16-bit indices sit at mat_*_idx (slices) and mat_*_long (long
    // lines), the FP32 values at mat_*_val and mat_*_lval
    int64_t mat_a_lval, mat_at_lval;
    int32_t f32_values, pad4_;
    // re-centred FP32 layout only (slab offsets): the two FP64 point buffers
    // of x (n+1) and y (m+1) -- base and candidate, roles swapped at every
    // re-centring -- and the FP32 reduced cost / primal residual of the last
    // evaluated candidate
    int64_t pt_x[2], pt_y[2], dcand, rcand;
    // and the instance's scaled FP64 objective and bounds (new column order)
    // and scaled right-hand side (new row order)
    int64_t sc_c, sc_l, sc_u, sc_b;
};

struct KernelParams {
    const DevSpecies* species;
    const Layout* layouts;        // per species, for this launch's precision
    int32_t count;
    const int32_t* order;         // work order (instance ids)
    const int32_t* inst_species;
    const int64_t* col_off;
    const int64_t* row_off;
    const double* lower;
    const double* upper;
    const double* cost;
    const double* rhs;            // may be null (zero)
    const double* warm_x;         // may be null
    const double* warm_y;         // may be null
    const double* warm_omega;     // may be null
    const int32_t* prior_iters;   // may be null: added to the reported count
    double* out_x;
    double* out_y;
    double* out_obj;
    double* out_metrics;
    double* out_omega;            // may be null
    int32_t* out_status;
    int32_t* out_iters;
    int32_t* queue;
    unsigned char* spill;         // per-CTA global slabs (may be null)
    int64_t spill_stride;         // bytes per CTA
    int32_t max_iters;
    int32_t check_every;
    double tol_p, tol_d, tol_g;
    double rho;
    int32_t restarts;
    int32_t final_status;
    int32_t clip_output;          // clip reported x to the original bounds
    int32_t stall_checks;         // >0: stall rule after this many
                                  // non-improving convergence tests
    double floor_tol;             // FP64 phase: tolerance accepted after a stall
    double gate_p, gate_d, gate_g;  // ... where the point also passes the
                                    // original-LP certificate gate
    double omega_smoothing;       // primal-weight update at a restart
    double passthrough_tol;       // FP32 phase: warm starts with error <= this
                                  // skip the phase unchanged (0 = never)
    int32_t fallback_iters;       // warm starts not converged after this many
                                  // iterations restart once cold (0 = never)
    // re-centred FP32 phase followed by an FP64 phase: instances the first
    // phase does not certify are appended to `handoff_list` (count in
    // `handoff_count`) with their point in hand_x / hand_y / hand_omega and
    // iteration count in hand_iters; certified ones go straight to out_*.
    // The FP64 phase then reads its work list size from `count_dev`.
    int32_t* handoff_list;        // may be null: every instance goes to out_*
    int32_t* handoff_count;
    double* hand_x;
    double* hand_y;
    double* hand_omega;
    int32_t* hand_iters;          // may be null; iterations of this phase
    const int32_t* count_dev;     // may be null: use `count`
    int32_t handoff_on_stall;     // >0: a re-centred solve whose KKT error has
                                  // not halved for this many full tests hands
                                  // off to the FP64 phase (0 = never)
    const double* patch_values;   // may be null: per instance, npatch deltas
                                  // (original units) at patch_stride apart
    int32_t patch_stride, pad3_;
    const int32_t* hint_iters;    // may be null: per instance, the iteration
                                  // count of its previous solve; an instance
                                  // whose hint is >= check_every skips the
                                  // early termination tests (8, 16, 32, ...)
};

}  // namespace fbalp
