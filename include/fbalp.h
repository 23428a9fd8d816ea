/*
 * fbalp.h -- C ABI of the B200 batched flux-balance LP engine.
 *
 * The engine solves batches of independent LPs
 *
 *     minimize    c.x
 *     subject to  A[:neq] x  = b[:neq]
 *                 A[neq:] x <= b[neq:]
 *                 l <= x <= u
 *
 * where every instance of a "species" shares that species' matrix A (the
 * stoichiometric matrix S of a flux-balance model) and carries its own
 * bounds l, u, objective c and right-hand side b.  Row duals follow the HiGHS
 * convention (inequality duals <= 0, reduced cost c - A^T y).
 *
 * It replaces the reference project's batched GPU LP backend call (the
 * `solve_batch` service used by the dFBA rollout):
 *   - `src/temporal_gpu_lp.py:86-199`  TemporalGpuLPBackend.solve_batch
 *   - `src/gpu_pdhg_corrector.py:99-218`  GpuPdhgCorrector.__init__ (setup)
 *   - `src/gpu_pdhg_corrector.py:273-438` GpuPdhgCorrector.solve (iterations)
 *   - `src/gpu_pdhg_workspace.py:55-384`  GpuPdhgWorkspace (resident loop)
 *   - `src/gpu_block_lp.py:52-132`        certify_blocks_device (certificate)
 *
 * Conventions: all functions return FBALP_OK (0) or an FBALP_ERR_* code;
 * fbalp_last_error() gives the message of the calling thread's last failure.
 * Invalid arguments are rejected before any state changes.  Species matrices
 * are HOST arrays (copied at creation); instance data, warm starts and
 * outputs are caller-owned DEVICE arrays.  One engine has one owner: calls on
 * the same engine must be serialised (as `src/gpu_pdhg_workspace.py:11-12`
 * and `src/cpu_repeated_lp.py:7` require of the reference services).
 */
#ifndef FBALP_H
#define FBALP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* return codes */
#define FBALP_OK 0
#define FBALP_ERR_INVALID 1   /* invalid argument; nothing was changed       */
#define FBALP_ERR_CUDA 2      /* CUDA runtime error                          */
#define FBALP_ERR_ALLOC 3     /* device or host allocation failed            */
#define FBALP_ERR_STATE 4     /* call out of order (e.g. solve before set)   */

/* per-instance solver status */
#define FBALP_STATUS_OPTIMAL 0          /* FP64 tolerances met (tight, or the
                                           floor tolerance after a stall)    */
#define FBALP_STATUS_ITERATION_LIMIT 1  /* budget exhausted; fails closed     */
#define FBALP_STATUS_NUMERICAL 2        /* NaN/Inf met in the iteration       */
#define FBALP_STATUS_INVALID_INPUT 3    /* l > u, NaN bound, non-finite c / b */
#define FBALP_STATUS_NOT_RUN 4
#define FBALP_STATUS_HANDOFF 5          /* FP32 phase met its tolerances      */

/* precision schedules */
#define FBALP_PRECISION_FP64 0   /* FP64 iterates throughout                  */
#define FBALP_PRECISION_MIXED 1  /* FP32 iterates, then FP64 refinement phase */
#define FBALP_PRECISION_FP32 2   /* FP32 phase only (diagnostic)              */

/* out_metrics row layout (FBALP_METRICS doubles per instance) */
#define FBALP_METRICS 8

/* most per-instance matrix entries one species may declare */
#define FBALP_MAX_PATCHES 8
#define FBALP_M_PRIMAL_RESIDUAL 0   /* max |A_eq x-b|, (A_ub x-b)+, bound viol. */
#define FBALP_M_DUAL_VIOLATION 1    /* y_ub+, reduced-cost sign on inf. bounds  */
#define FBALP_M_RELATIVE_KKT_GAP 2  /* complementarity / max(1,|c.x|)           */
#define FBALP_M_OBJECTIVE 3         /* c.x                                      */
#define FBALP_M_DUAL_OBJECTIVE 4    /* b.y + sum_j min_{[l_j,u_j]} r_j x_j      */
#define FBALP_M_RELATIVE_GAP 5      /* |c.x - dual| / (1 + |c.x| + |dual|)      */
#define FBALP_M_X_INF 6             /* max |x_j|                                */
#define FBALP_M_OMEGA 7             /* final primal weight                      */

typedef struct fbalp_engine fbalp_engine;

/* Setup options (per engine).  Replaces the constructor arguments of
 * `src/gpu_pdhg_corrector.py:92-99` (step_safety, primal_weight); the
 * diagonal metric of `:183-200` becomes Ruiz + Pock-Chambolle scaling with a
 * spectral step. */
typedef struct fbalp_options {
    int32_t ruiz_iterations;   /* default 10                                 */
    int32_t power_iterations;  /* default 256 (||A~||_2 estimate)            */
    double step_safety;        /* default 0.99 (eta = safety / ||A~||_2)     */
    int32_t warps_per_block;   /* default 16, at most 32                     */
    int32_t blocks_per_sm;     /* default 0 = derive from occupancy          */
    int32_t max_dynamic_smem;  /* bytes of shared memory per CTA for instance
                                  arrays; 0 = device limit.  Arrays that do not
                                  fit live in a per-CTA global slab.        */
    int32_t stage_matrix;      /* 1 (default): stage the species matrix into
                                  shared memory when it fits; 0: stream it
                                  from L2 every iteration                   */
    int32_t fp64_max_dynamic_smem; /* cap for the FP64 phase (0 = same as
                                  max_dynamic_smem); a smaller cap spills the
                                  cold arrays and fits more CTAs per SM     */
    int32_t pair_instances;    /* 1 (default): the re-centred phase runs two
                                  instances of a species per CTA (one staged
                                  matrix, interleaved vectors) when every
                                  species fits that layout, the reflection is
                                  1, no entries are patched and the batch has
                                  at least two instances per CTA; 0: one
                                  instance per CTA.  Same results.          */
    int32_t spread_banks;      /* 1 (default): the re-centred kernels' matrix
                                  entries are ordered inside each row so that
                                  one step's gathers hit distinct shared-memory
                                  banks (fewer conflicts; only the FP32
                                  accumulation order changes); 0: column
                                  order                                     */
} fbalp_options;

/* Solve parameters.  Replaces `iterations` / `check_interval` of
 * `src/gpu_pdhg_corrector.py:273-281`; the acceptance gate of
 * `src/gpu_block_lp.py:84` is evaluated on the returned metrics. */
typedef struct fbalp_solve_params {
    int32_t precision;           /* FBALP_PRECISION_*                         */
    int32_t max_iterations;      /* FP64 phase budget per instance            */
    int32_t fp32_max_iterations; /* FP32 phase budget (MIXED / FP32)          */
    int32_t check_every;         /* convergence / restart test period         */
    double tol_primal;           /* primal <= tol*(1+|x|_inf)   (FP64 phase)  */
    double tol_dual;             /* dual viol. <= tol*(1+|c|_inf)             */
    double tol_gap;              /* relative gap and relative KKT gap (default
                                    1e-7, the reference's gate)              */
    double fp32_tol_primal;      /* hand-off tolerances of the FP32 phase     */
    double fp32_tol_dual;
    double fp32_tol_gap;
    double reflection;           /* Halpern reflection rho in [0,1], default 1 */
    int32_t restarts;            /* 1 = adaptive restarts, 0 = none           */
    int32_t fp32_stall_checks;   /* FP32 phase hands off after this many tests
                                    without halving its KKT error (0 = never) */
    int32_t fp64_stall_checks;   /* FP64 phase: after this many such tests a
                                    point meeting floor_tol is accepted as
                                    OPTIMAL (an FP64 rounding floor above the
                                    tight tolerances; 0 = never)             */
    double floor_tol;            /* default 1e-7 = the reference's gap gate   */
    double fp32_passthrough_tol; /* MIXED: a warm start whose FP64 KKT error is
                                    already <= this skips the FP32 phase
                                    unchanged (default 1e-3; 0 = never)      */
    int32_t fallback_iterations; /* a warm-started FP64 solve not converged
                                    after this many iterations restarts once
                                    from the cold point (default 4096; 0 =
                                    never): cold PDHG is the fallback of every
                                    seed                                     */
    int32_t fp32_recentre;       /* MIXED (default 1): the FP32 phase iterates
                                    on differences from an FP64 base point that
                                    moves to the iterate at every restart, so
                                    FP32 iterations reach the FP64 tolerances;
                                    instances it does not certify (a stall)
                                    continue in the FP64 phase.  Used when the
                                    batch's species fit the shared-memory
                                    layout, else the plain schedule below.
                                    0: plain schedule -- FP32 iterates to the
                                    fp32_* tolerances, then FP64 iterates    */
    int32_t fp32_values_phase;   /* MIXED re-centred schedule: 1 (default) --
                                    instances the re-centred phase hands off
                                    (its matrix words hold BF16 values)
                                    continue in a re-centred phase with FP32
                                    matrix values (same budget, no stall rule)
                                    where the species fit it; 0: the
                                    hand-offs continue in the FP64 phase;
                                    2: continuation -- every instance runs in
                                    the FP32-valued phase from the warm point
                                    (no BF16 phase, no cold fallback); for
                                    iterates an earlier call stopped at its
                                    cap; as 1 where the species do not fit  */
    /* the original-LP certificate gate a point accepted by the stall-floor
       rule must also pass: absolute primal residual, absolute dual
       violation, relative KKT gap (default 1e-5 / 1e-7 / 1e-7, the
       reference's gate); floor_tol is relative to |x|_inf, which open 1000
       bounds make large                                                    */
    double gate_primal;
    double gate_dual;
    double gate_gap;
    double primal_weight_smoothing; /* theta of the primal-weight update at a
                                    restart, log w <- theta log(|dy| / |dx|)
                                    + (1 - theta) log w, in [0, 1] (default
                                    0.5, PDLP's; 0 keeps the weight fixed)   */
} fbalp_solve_params;

void fbalp_default_options(fbalp_options* options);
void fbalp_default_solve_params(fbalp_solve_params* params);

/* Create an engine for `num_species` matrices (HOST CSR arrays; int64 row
 * pointers, int32 column indices, double values; duplicates are summed and
 * zeros dropped, as `_problem` does at `src/cpu_repeated_lp.py:141`).
 * `stream` is a cudaStream_t (NULL = legacy default stream).
 * Replaces: GpuPdhgCorrector.__init__ (`src/gpu_pdhg_corrector.py:99-218`)
 * and GpuPdhgWorkspace.__init__ (`src/gpu_pdhg_workspace.py:55-155`). */
int fbalp_engine_create(int32_t num_species, const int32_t* rows, const int32_t* cols,
                        const int32_t* neq, const int64_t* const* indptr,
                        const int32_t* const* indices, const double* const* values,
                        const fbalp_options* options, void* stream, fbalp_engine** out);

/* Bind a batch of `count` instances.  `species_id` is a HOST array.  The
 * DEVICE arrays `lower`, `upper`, `cost` (and `rhs`, NULL = zero) are flat:
 * instance i occupies columns [col_offset[i], col_offset[i] + n_{species[i]})
 * and rows [row_offset[i], row_offset[i] + m_{species[i]}), offsets being the
 * prefix sums in instance order.  The pointers are kept (not copied) and must
 * stay valid until the next set_instances / destroy.
 * Replaces: the per-call host assembly and copies of
 * `src/gpu_pdhg_corrector.py:140-184` and GpuPdhgWorkspace.update_problem
 * (`src/gpu_pdhg_workspace.py:209-267`). */
int fbalp_engine_set_instances(fbalp_engine* engine, int64_t count, const int32_t* species_id,
                               const double* lower, const double* upper, const double* cost,
                               const double* rhs);

/* Re-point the bound batch at new DEVICE arrays of the same layout (same
 * count, species and offsets) without recomputing it: the per-step call of a
 * caller whose bounds change every step in place or in alternating buffers.
 * Replaces: GpuPdhgWorkspace.update_problem (`src/gpu_pdhg_workspace.py:
 * 209-267`), which keeps its pointers and rewrites their values. */
int fbalp_engine_set_instance_data(fbalp_engine* engine, const double* lower, const double* upper,
                                   const double* cost, const double* rhs);

/* Optional per-instance iteration hints (DEVICE int32[count], e.g. the
 * iteration counts of the previous solve; NULL clears): in the re-centred
 * phase an instance whose hint is >= check_every skips the early
 * termination-only tests at iterations 8, 16, 32, ... (each costs a few
 * iterations' time); results are unaffected except that such an instance
 * cannot stop before its first full test.  The pointer is kept until the next
 * set_instances / set_iteration_hints.  No counterpart in the reference (its
 * certificate period is fixed, `src/gpu_pdhg_corrector.py:278-279`). */
int fbalp_engine_set_iteration_hints(fbalp_engine* engine, const int32_t* hints);

/* Per-instance matrix entries: declare up to 8 entries (original row and
 * column indices) of species `species` whose value differs per instance;
 * instance i's matrix is then A + sum_q delta_iq e_{rows[q]} e_{cols[q]}^T
 * with the deltas bound by fbalp_engine_set_patch_values.  For LPs whose
 * coefficients change with the state, e.g. the cooperative community LP's
 * biomass-weighted rows (`src/community_solver.py:1084-1151`).  Solves of a
 * batch with patched entries use the re-centred mixed schedule (and have no
 * FP64 hand-off phase).  count = 0 clears.  The step size of each instance
 * is shrunk to stay below 1/(||A~|| + ||scaled deltas||_F). */
int fbalp_engine_set_patches(fbalp_engine* engine, int32_t species, int32_t count, const int32_t* rows,
                             const int32_t* cols);

/* Bind the per-instance deltas of the patched entries: DEVICE double
 * [count * stride], instance i's deltas at [i*stride, i*stride + npatch);
 * NULL clears (every instance uses A).  Kept until the next
 * set_instances / set_patch_values. */
int fbalp_engine_set_patch_values(fbalp_engine* engine, const double* values, int32_t stride);

/* Certificate of the ORIGINAL LPs of a batch from solutions of their
 * diagonally scaled copies, in one launch on `stream` (asynchronous).
 * Instance i solved  A_i w (=,<=) b_i, l_i <= w <= u_i, min c_i.w  with
 * A_i = A + sum_q deltas[i*npatch+q] e_{patch_rows[q]} e_{patch_cols[q]}^T
 * (A: `rows` x `cols` DEVICE CSR a_ptr/a_idx/a_val with its transpose
 * at_ptr/at_idx/at_val, rows [0, neq) equalities), and A_i = R A_orig D^-1,
 * b_i = R b_orig, w = D v, c_i = D^-1 c_orig, where row r is scaled by
 * scale_table[i*groups + row_group[r]] and column j by
 * scale_table[i*groups + col_group[j]].  x, cost, lower, upper are DEVICE
 * [count*cols], y and rhs [count*rows].  Writes per instance the original
 * LP's primal residual, dual violation and relative KKT gap (the formulas of
 * out_metrics, in the original units; NaN if any input is NaN) to DEVICE
 * out_primal/out_dual/out_gap [count].  Indices must lie inside the matrix.
 * Replaces certify_blocks_device (`src/gpu_block_lp.py:52-132`) applied to
 * the cooperative stage LPs, whose coefficients the reference scales by the
 * biomass (`src/community_solver.py:1084-1151, 116-204`). */
int fbalp_scaled_certificate(int32_t count, int32_t rows, int32_t cols, int32_t neq, const int32_t* a_ptr,
                             const int32_t* a_idx, const double* a_val, const int32_t* at_ptr,
                             const int32_t* at_idx, const double* at_val, int32_t npatch,
                             const int32_t* patch_rows, const int32_t* patch_cols, const double* deltas,
                             const double* x, const double* y, const double* cost, const double* lower,
                             const double* upper, const double* rhs, const int32_t* row_group,
                             const int32_t* col_group, int32_t groups, const double* scale_table,
                             double* out_primal, double* out_dual, double* out_gap, void* stream);

/* Solve every bound instance.  Warm starts (`warm_x`, `warm_y`: flat DEVICE,
 * original units; `warm_omega`: per instance) may be NULL (cold start).
 * Outputs are DEVICE arrays: status[count], objective[count],
 * x[total columns], y[total rows], iterations[count],
 * metrics[count * FBALP_METRICS]; `out_omega` (may be NULL) receives the
 * final primal weight per instance.  Asynchronous on the engine's stream.
 * Replaces: GpuPdhgCorrector.solve (`src/gpu_pdhg_corrector.py:273-438`),
 * GpuPdhgWorkspace.run / set_accepted (`src/gpu_pdhg_workspace.py:295-367`)
 * and certify_blocks_device (`src/gpu_block_lp.py:52-132`). */
int fbalp_engine_solve(fbalp_engine* engine, const double* warm_x, const double* warm_y,
                       const double* warm_omega, const fbalp_solve_params* params,
                       int32_t* out_status, double* out_objective, double* out_x, double* out_y,
                       int32_t* out_iterations, double* out_metrics, double* out_omega);

/* Allocation-free solve.  No counterpart in the reference: it exists for
 * callers that cannot allocate device memory at solve time -- real-time
 * loops that forbid allocator calls once running, and hosts whose device
 * memory is owned and budgeted by another allocator (a caching pool or a
 * fixed arena), where a cudaMalloc behind its back fails or breaks its
 * accounting.  They create the engine (which allocates its species data) up
 * front; this call then allocates nothing: besides the caller's inputs and
 * outputs it uses one library-wide scratch array of 32 MiB in device memory
 * (held by every GPU that loads the library until the process exits).
 * Limits: one-species engine, FP64 precision only (params->precision must be
 * FBALP_PRECISION_FP64), instances laid out uniformly (instance i at columns
 * [i*n, (i+1)*n) and rows [i*m, (i+1)*m)), and a batch whose metadata and
 * per-CTA spill slabs fit in the scratch; larger requests fail with
 * FBALP_ERR_INVALID before any work is queued.  The current device must be
 * the engine's device (FBALP_ERR_INVALID otherwise).  The first call on each
 * device looks up the scratch address with cudaGetSymbolAddress, so make it
 * before any stream capture.  All calls share the scratch, which keeps the
 * last call's contents: calls whose kernels overlap on the GPU race.
 * Outputs and their meaning are those of fbalp_engine_solve; the phase
 * queries (fbalp_engine_phase_times / _iterations) do not cover this call. */
int fbalp_engine_solve_noalloc(fbalp_engine* engine, int64_t count, const double* lower,
                               const double* upper, const double* cost, const double* rhs,
                               const double* warm_x, const double* warm_y, const double* warm_omega,
                               const fbalp_solve_params* params, int32_t* out_status,
                               double* out_objective, double* out_x, double* out_y,
                               int32_t* out_iterations, double* out_metrics, double* out_omega);

/* Release the engine's device memory.  Replaces the reference services'
 * close()/release paths (`src/cpu_repeated_lp.py:820-831`). */
int fbalp_engine_destroy(fbalp_engine* engine);

/* Change the stream later calls are queued on (cudaStream_t). */
int fbalp_engine_set_stream(fbalp_engine* engine, void* stream);

/* HOST query: total columns/rows of the bound batch and the per-instance
 * offsets (arrays of `count` int64, may be NULL). */
int fbalp_engine_layout(const fbalp_engine* engine, int64_t* total_cols, int64_t* total_rows,
                        int64_t* col_offsets, int64_t* row_offsets);

/* HOST-only preprocessing of one matrix, for inspection and tests: the Ruiz +
 * Pock-Chambolle scalings (dr[rows], dc[cols], original order), the spectral
 * norm estimate of the scaled matrix and the step size.  Replaces the metric
 * computed at `src/gpu_pdhg_corrector.py:183-200`. */
int fbalp_prepare_matrix(int32_t rows, int32_t cols, const int64_t* indptr,
                         const int32_t* indices, const double* values,
                         const fbalp_options* options, double* dr, double* dc,
                         double* sigma_max, double* eta);

/* Device time (ms) of the last solve's FP32 and FP64 phase launches (0 for a
 * phase that did not run); waits for the last launch to finish.  Timing
 * instrumentation for benchmarks; the reference reports per-phase seconds in
 * its `timing` dicts (`src/gpu_pdhg_corrector.py:392-405`). */
int fbalp_engine_phase_times(fbalp_engine* engine, float* ms_fp32, float* ms_fp64);

/* Kernel kinds the last fbalp_engine_solve launched for its first (FP32 /
 * re-centred) and FP64 phases: FBALP_KERNEL_* or -1 for a phase that did not
 * run; the second phase of the mixed re-centred schedule is the FP32-valued
 * re-centred kernel (FBALP_KERNEL_RECENTRED_F32_*) or the FP64 kernel.
 * Instrumentation for tests and benchmarks. */
#define FBALP_KERNEL_FP32 0
#define FBALP_KERNEL_FP64 1
#define FBALP_KERNEL_RECENTRED_STAGED 2
#define FBALP_KERNEL_RECENTRED_STREAMED 3
#define FBALP_KERNEL_RECENTRED_PAIRED 4
#define FBALP_KERNEL_RECENTRED_F32_STAGED 5
#define FBALP_KERNEL_RECENTRED_F32_STREAMED 6
int fbalp_engine_phase_kernels(fbalp_engine* engine, int32_t* fp32_kind, int32_t* fp64_kind);

/* Timing slots (benchmark instrumentation): create `slots` (0..64) pairs of
 * CUDA events per precision phase (previous slots are destroyed).  While a
 * slot is selected with fbalp_engine_use_timing_slot (-1 selects none), every
 * phase launch of fbalp_engine_solve is bracketed by that slot's events;
 * under stream capture they become external event nodes of the graph, so
 * each replay of the graph re-records them.  fbalp_engine_slot_times waits
 * for the slot's last recorded launch and returns its device times (0 for a
 * phase the slot never bracketed).  Lets a benchmark time the PDHG launches
 * of graph-replayed solves without leaving the graph. */
int fbalp_engine_timing_slots(fbalp_engine* engine, int32_t slots);
int fbalp_engine_use_timing_slot(fbalp_engine* engine, int32_t slot);
int fbalp_engine_slot_times(fbalp_engine* engine, int32_t slot, float* ms_fp32, float* ms_fp64);

/* After a MIXED solve: copy the per-instance FP32-phase iteration counts into
 * the DEVICE array `out_fp32_iterations[count]` (asynchronous). */
int fbalp_engine_phase_iterations(fbalp_engine* engine, int32_t* out_fp32_iterations);

const char* fbalp_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* FBALP_H */
