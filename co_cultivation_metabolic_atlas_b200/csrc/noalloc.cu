// Allocation-free solve entry point (fbalp_engine_solve_noalloc).
//
// Some callers cannot allocate device memory at solve time: real-time
// control loops that forbid allocator calls once they have started, and
// hosts whose device memory is owned and budgeted by another allocator (a
// framework's caching pool, a fixed-size arena) so that a cudaMalloc behind
// its back either fails or breaks its accounting.  They create the engine
// (which allocates its species data) at start-up and then call this entry
// point, which uses only the caller's inputs/outputs and the scratch array
// below: the work-queue counter, the per-instance metadata of a
// single-species batch, the layout record and the per-CTA spill slabs of the
// FP64 PDHG kernel.
//
// The scratch is a file-scope __device__ array of kNoallocScratchBytes
// (32 MiB); every GPU that loads the library holds it until the process
// exits.  Host code must not use the array's name as a device address: on
// the first call on each device (with that device current, which must be
// the engine's device) the entry point obtains the real address with
// cudaGetSymbolAddress and remembers it; that first call should come before
// any stream capture.  Every call shares the array and it keeps the last
// call's contents, so calls whose kernels overlap on the GPU race; the
// queue counter is cleared at the start of every call and the metadata is
// rewritten by every call.
#include <cstdint>
#include <mutex>

#include "engine_state.h"

namespace {

constexpr size_t kNoallocScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kMaxDevices] = {};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Single-species batch metadata: identity work order, species 0, instance i
// at columns [i n, (i+1) n) and rows [i m, (i+1) m); plus the layout record.
__global__ void fill_uniform_batch(int count, int n, int m, int32_t* order, int32_t* species,
                                   int64_t* col_off, int64_t* row_off, fbalp::Layout layout,
                                   fbalp::Layout* layout_out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        order[i] = i;
        species[i] = 0;
        col_off[i] = static_cast<int64_t>(i) * n;
        row_off[i] = static_cast<int64_t>(i) * m;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *layout_out = layout;
}

// Device address of the scratch array on the current device (set-up on the
// first call per device).  The current device must be `want`, the engine's:
// its species data, stream and kernels live there.
int scratch_address(int want, unsigned char** out) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return fail(FBALP_ERR_CUDA, cudaGetErrorString(err));
    if (dev != want) return fail(FBALP_ERR_INVALID, "current device is not the engine's device");
    if (dev < 0 || dev >= kMaxDevices) return fail(FBALP_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err != cudaSuccess || !p)
            return fail(FBALP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(err));
        g_noalloc_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_noalloc_addr[dev]);
    return FBALP_OK;
}

}  // namespace

extern "C" int fbalp_engine_solve_noalloc(fbalp_engine* e, int64_t count, const double* lower,
                                          const double* upper, const double* cost, const double* rhs,
                                          const double* warm_x, const double* warm_y,
                                          const double* warm_omega, const fbalp_solve_params* params,
                                          int32_t* out_status, double* out_objective, double* out_x,
                                          double* out_y, int32_t* out_iterations, double* out_metrics,
                                          double* out_omega) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (e->species.size() != 1) return fail(FBALP_ERR_INVALID, "the no-allocation solve needs a one-species engine");
    if (e->dev_species_host[0].npatch > 0)
        return fail(FBALP_ERR_INVALID, "the no-allocation solve has no per-instance patched entries");
    if (count < 1 || count > INT32_MAX || !lower || !upper || !cost)
        return fail(FBALP_ERR_INVALID, "count >= 1 and lower/upper/cost are required");
    if (!out_status || !out_objective || !out_x || !out_y || !out_iterations || !out_metrics)
        return fail(FBALP_ERR_INVALID, "output arrays are required");
    fbalp_solve_params q;
    fbalp_default_solve_params(&q);
    if (params) q = *params;
    std::string err;
    if (!valid_params(q, &err)) return fail(FBALP_ERR_INVALID, err);
    if (q.precision != FBALP_PRECISION_FP64)
        return fail(FBALP_ERR_INVALID, "the no-allocation solve runs the FP64 kernel only (precision FP64)");

    unsigned char* scratch = nullptr;
    if (int rc = scratch_address(e->device, &scratch)) return rc;
    // the per-phase queries (times, iterations) cover fbalp_engine_solve
    // only: this call leaves them reporting no phase
    e->ran[0] = e->ran[1] = false;

    const SpeciesHost& sh = e->species[0];
    const int threads = e->opt.warps_per_block * 32;
    const size_t static_smem = sizeof(double) * (threads / 32 * fbalp::kRed + fbalp::kRed) + 64;
    int64_t cap = e->smem_optin > static_cast<int>(static_smem) + 1024
                      ? e->smem_optin - static_cast<int64_t>(static_smem) - 1024 : 0;
    if (e->opt.max_dynamic_smem > 0) cap = std::min<int64_t>(cap, e->opt.max_dynamic_smem);
    if (e->opt.fp64_max_dynamic_smem > 0) cap = std::min<int64_t>(cap, e->opt.fp64_max_dynamic_smem);
    fbalp::LayoutPlan P{};
    bool staged = false;
    if (e->opt.stage_matrix != 0) {
        P = fbalp::plan_layout_unscaled(sh.n, sh.m, e->opt.warps_per_block, sh.A.nslices, sh.AT.nslices,
                                        sh.A.off.back(), sh.AT.off.back(), cap);
        staged = P.layout.unscaled != 0;
    }
    if (!staged)
        P = fbalp::plan_layout(sh.n, sh.m, e->opt.warps_per_block, sh.A.nslices, sh.AT.nslices, sh.A.off.back(),
                               sh.AT.off.back(), sizeof(double), cap, false);
    if (P.smem_bytes > cap) return fail(FBALP_ERR_INVALID, "species schedule does not fit into shared memory");
    if (!fbalp::layout_aligned(P.layout)) return fail(FBALP_ERR_INVALID, "internal error: misaligned layout");
    const int64_t dyn = fbalp::align_up(std::max<int64_t>(P.smem_bytes, 16), 16);

    // scratch map: [queue counter | order | species | col_off | row_off | layout | spill slabs]
    const size_t n_inst = static_cast<size_t>(count);
    size_t off = 256;
    const size_t o_order = off;
    off += align256(4 * n_inst);
    const size_t o_species = off;
    off += align256(4 * n_inst);
    const size_t o_coloff = off;
    off += align256(8 * n_inst);
    const size_t o_rowoff = off;
    off += align256(8 * n_inst);
    const size_t o_layout = off;
    off += align256(sizeof(fbalp::Layout));
    const size_t o_spill = off;
    const size_t slab = static_cast<size_t>(P.slab_bytes);
    if (o_spill > kNoallocScratchBytes || (slab > 0 && o_spill + slab > kNoallocScratchBytes))
        return fail(FBALP_ERR_INVALID,
                    "batch too large for the no-allocation scratch (" + std::to_string(kNoallocScratchBytes) +
                        " bytes): needs " + std::to_string(o_spill + slab) + " bytes for one CTA");

    try {
        const void* k = fbalp::kernel_symbol(true, threads, staged);
        // the kernel's dynamic shared-memory limit is shared with every
        // engine in the process: raise it if needed, never lower it
        cudaFuncAttributes fa{};
        check(cudaFuncGetAttributes(&fa, k), "cudaFuncGetAttributes");
        if (fa.maxDynamicSharedSizeBytes < dyn)
            check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dyn)),
                  "cudaFuncSetAttribute");
        int per_sm = 0;
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, dyn), "occupancy");
        if (e->opt.blocks_per_sm > 0) per_sm = std::min(per_sm, e->opt.blocks_per_sm);
        if (per_sm < 1) return fail(FBALP_ERR_INVALID, "kernel does not fit on an SM with this configuration");
        int64_t grid = std::min<int64_t>(count, static_cast<int64_t>(per_sm) * e->sm_count);
        if (slab > 0) grid = std::min<int64_t>(grid, static_cast<int64_t>((kNoallocScratchBytes - o_spill) / slab));

        fbalp::KernelParams p{};
        p.species = e->dev_species;
        p.layouts = reinterpret_cast<const fbalp::Layout*>(scratch + o_layout);
        p.count = static_cast<int32_t>(count);
        p.order = reinterpret_cast<const int32_t*>(scratch + o_order);
        p.inst_species = reinterpret_cast<const int32_t*>(scratch + o_species);
        p.col_off = reinterpret_cast<const int64_t*>(scratch + o_coloff);
        p.row_off = reinterpret_cast<const int64_t*>(scratch + o_rowoff);
        p.lower = lower;
        p.upper = upper;
        p.cost = cost;
        p.rhs = rhs;
        p.warm_x = warm_x;
        p.warm_y = warm_y;
        p.warm_omega = warm_omega;
        p.prior_iters = nullptr;
        p.out_x = out_x;
        p.out_y = out_y;
        p.out_obj = out_objective;
        p.out_metrics = out_metrics;
        p.out_omega = out_omega;
        p.out_status = out_status;
        p.out_iters = out_iterations;
        p.queue = reinterpret_cast<int32_t*>(scratch);
        p.spill = slab > 0 ? scratch + o_spill : nullptr;
        p.spill_stride = static_cast<int64_t>(slab);
        p.max_iters = q.max_iterations;
        p.check_every = q.check_every;
        p.tol_p = q.tol_primal;
        p.tol_d = q.tol_dual;
        p.tol_g = q.tol_gap;
        p.rho = q.reflection;
        p.restarts = q.restarts;
        p.final_status = fbalp::kStatusOptimal;
        p.clip_output = 1;
        p.stall_checks = q.fp64_stall_checks;
        p.floor_tol = q.floor_tol;
        p.gate_p = q.gate_primal;
        p.gate_d = q.gate_dual;
        p.gate_g = q.gate_gap;
        p.omega_smoothing = q.primal_weight_smoothing;
        p.passthrough_tol = 0.0;
        p.fallback_iters = q.fallback_iterations;

        check(cudaMemsetAsync(scratch, 0, sizeof(int32_t), e->stream), "clear queue counter");
        const int fill_grid = static_cast<int>(std::min<int64_t>((count + 255) / 256, 1024));
        fill_uniform_batch<<<fill_grid, 256, 0, e->stream>>>(
            static_cast<int>(count), sh.n, sh.m, reinterpret_cast<int32_t*>(scratch + o_order),
            reinterpret_cast<int32_t*>(scratch + o_species), reinterpret_cast<int64_t*>(scratch + o_coloff),
            reinterpret_cast<int64_t*>(scratch + o_rowoff), P.layout,
            reinterpret_cast<fbalp::Layout*>(scratch + o_layout));
        check(cudaGetLastError(), "metadata kernel launch");
        check(fbalp::launch_pdhg(true, staged, static_cast<int>(grid), threads, dyn, e->stream, p),
              "pdhg kernel launch");
    } catch (const CudaError& ex) {
        return fail(FBALP_ERR_CUDA, ex.what());
    }
    return FBALP_OK;
}
