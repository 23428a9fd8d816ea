// Internal state of an engine (shared by the entry points in engine.cu and
// noalloc.cu).  Not part of the C ABI.
#pragma once

#include <algorithm>
#include <cmath>
#include <exception>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/fbalp.h"
#include "fbalp_internal.h"
#include "prepare.h"

namespace fbalp_detail {

inline thread_local std::string g_last_error;

inline int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

struct CudaError : std::exception {
    std::string msg;
    explicit CudaError(std::string m) : msg(std::move(m)) {}
    const char* what() const noexcept override { return msg.c_str(); }
};

inline void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T> inline T* dev_upload(const std::vector<T>& h, std::vector<void*>& owned) {
    T* d = nullptr;
    size_t bytes = std::max<size_t>(1, h.size()) * sizeof(T);
    check(cudaMalloc(&d, bytes), "cudaMalloc");
    owned.push_back(d);
    if (!h.empty()) check(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy");
    return d;
}

struct SpeciesHost {
    int32_t m = 0, n = 0, neq = 0;
    fbalp::Scaling scaling;
    std::vector<int32_t> row_perm, col_perm;  // new -> old
    fbalp::Sell A, AT;
    fbalp::Sell Araw, ATraw;  // same slices, unscaled values
    std::vector<int32_t> a_sched_off, a_sched, at_sched_off, at_sched;
    std::vector<int4> alist, atlist;  // schedule entries as uploaded (w: patched slice)
    int4* d_alist = nullptr;           // their device copies
    int4* d_atlist = nullptr;
    // the re-centred kernels' operands: slices without the long lines, the
    // long lines, their schedules and uploaded lists
    fbalp::Sell Ar, ATr;
    std::vector<int32_t> ra_sched_off, ra_sched, ra_lsched_off, ra_lsched;
    std::vector<int32_t> rat_sched_off, rat_sched, rat_lsched_off, rat_lsched;
    std::vector<int4> ralist, ratlist;
    int4* d_ralist = nullptr;
    int4* d_ratlist = nullptr;
    fbalp::LinesShape shape_a() const {
        return {Ar.nslices, static_cast<int32_t>(Ar.long_line.size()), Ar.off.back(), Ar.long_off.back()};
    }
    fbalp::LinesShape shape_at() const {
        return {ATr.nslices, static_cast<int32_t>(ATr.long_line.size()), ATr.off.back(), ATr.long_off.back()};
    }
};

struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    void ensure(size_t want) {
        if (want <= bytes) return;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        check(cudaMalloc(&ptr, std::max<size_t>(want, 256)), "cudaMalloc workspace");
        bytes = std::max<size_t>(want, 256);
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

// Checks of the solve parameters shared by every solve entry point.
inline bool valid_params(const fbalp_solve_params& q, std::string* err) {
    if (q.precision < 0 || q.precision > 2) return *err = "precision must be FP64, MIXED or FP32", false;
    if (q.max_iterations < 0 || q.fp32_max_iterations < 0) return *err = "iteration budgets must be non-negative", false;
    if (q.check_every < 1) return *err = "check_every must be positive", false;
    for (double t : {q.tol_primal, q.tol_dual, q.tol_gap, q.fp32_tol_primal, q.fp32_tol_dual, q.fp32_tol_gap})
        if (!(t >= 0.0) || !std::isfinite(t)) return *err = "tolerances must be finite and non-negative", false;
    if (!(q.reflection >= 0.0 && q.reflection <= 1.0)) return *err = "reflection must be in [0,1]", false;
    if (q.restarts != 0 && q.restarts != 1) return *err = "restarts must be 0 or 1", false;
    if (q.fp32_stall_checks < 0 || q.fp64_stall_checks < 0) return *err = "stall checks must be non-negative", false;
    if (!(q.floor_tol >= 0.0) || !std::isfinite(q.floor_tol)) return *err = "floor_tol must be finite and non-negative", false;
    for (double t : {q.gate_primal, q.gate_dual, q.gate_gap})
        if (!(t >= 0.0) || !std::isfinite(t)) return *err = "certificate gates must be finite and non-negative", false;
    if (!(q.primal_weight_smoothing >= 0.0 && q.primal_weight_smoothing <= 1.0))
        return *err = "primal_weight_smoothing must be in [0, 1]", false;
    if (q.fallback_iterations < 0) return *err = "fallback_iterations must be non-negative", false;
    if (q.fp32_recentre != 0 && q.fp32_recentre != 1) return *err = "fp32_recentre must be 0 or 1", false;
    if (!(q.fp32_passthrough_tol >= 0.0) || !std::isfinite(q.fp32_passthrough_tol))
        return *err = "fp32_passthrough_tol must be finite and non-negative", false;
    if (q.fp32_values_phase < 0 || q.fp32_values_phase > 2)
        return *err = "fp32_values_phase must be 0, 1 or 2", false;
    return true;
}

}  // namespace fbalp_detail

using namespace fbalp_detail;

struct fbalp_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 0;
    int smem_optin = 0;
    fbalp_options opt{};
    std::vector<SpeciesHost> species;
    std::vector<fbalp::DevSpecies> dev_species_host;
    fbalp::DevSpecies* dev_species = nullptr;
    std::vector<void*> owned;  // species allocations
    // bound batch
    int64_t count = 0, total_cols = 0, total_rows = 0;
    std::vector<int32_t> h_species;
    std::vector<int64_t> h_coloff, h_rowoff;
    const double *lower = nullptr, *upper = nullptr, *cost = nullptr, *rhs = nullptr;
    const int32_t* hints = nullptr;  // per-instance iteration hints (device), may be null
    const double* patch_values = nullptr;  // per-instance patched-entry deltas (device), may be null
    int32_t patch_stride = 0;
    Buffer inst_species, col_off, row_off, order;
    bool bound = false;
    // workspace
    Buffer queue, mid_x, mid_y, mid_omega, mid_iters, mid_status, mid_obj, mid_metrics, spill;
    Buffer hand_list, hand_count;  // re-centred phase -> next phase work list
    Buffer layout32_buf, layout64_buf;
    // device copies of the launch layouts, one per kernel kind (plain FP32,
    // FP64, re-centred staged, re-centred streamed, paired re-centred),
    // uploaded only when their
    // content changes: a solve that reuses them issues no host-to-device
    // copy, so it can be captured in a CUDA graph
    Buffer layout_dev[7];
    std::vector<fbalp::Layout> layout_host[7];
    std::vector<fbalp::Layout> layouts32, layouts64;
    // per phase of the last solve (first, FP64, FP32-valued middle phase)
    int last_grid[3] = {0, 0, 0};
    // largest static shared memory of each kernel family at this engine's
    // block size (persistent, re-centred, paired; -1 until queried)
    int64_t static_smem[3] = {-1, -1, -1};
    int last_kind[3] = {-1, -1, -1};  // kernel kind (the layout_dev index)
    int64_t last_smem[3] = {0, 0, 0};
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // phase start/stop: fp32, fp64
    bool ran[2] = {false, false};
    // timing slots: per slot the same four events, recorded around the
    // phase launches while the slot is selected -- as external event nodes
    // when the launches are captured into a CUDA graph, so that every replay
    // of that graph re-records them
    std::vector<cudaEvent_t> slot_ev;
    std::vector<char> slot_ran;  // per slot and phase: events recorded (or captured)
    int slot = -1;               // selected slot (-1: none)
    ~fbalp_engine() {
        for (cudaEvent_t& v : ev)
            if (v) cudaEventDestroy(v);
        for (cudaEvent_t& v : slot_ev)
            if (v) cudaEventDestroy(v);
        for (void* p : owned) cudaFree(p);
        for (Buffer* b : {&inst_species, &col_off, &row_off, &order, &queue, &mid_x, &mid_y, &mid_omega,
                          &mid_iters, &mid_status, &mid_obj, &mid_metrics, &spill, &layout32_buf,
                          &layout64_buf, &hand_list, &hand_count, &layout_dev[0], &layout_dev[1],
                          &layout_dev[2], &layout_dev[3], &layout_dev[4], &layout_dev[5], &layout_dev[6]})
            b->release();
    }
};
