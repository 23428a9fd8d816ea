// Host engine and C ABI (include/fbalp.h).
//
// The engine owns the per-species preprocessed matrices (device, SELL-32
// slices of A and A^T in FP32 and FP64, scalings, permutations, warp
// schedules) and a small workspace (work queue counter, FP32->FP64 hand-off
// iterates, spill slabs).  Instance data and outputs stay caller-owned.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/fbalp.h"
#include "fbalp_internal.h"
#include "prepare.h"

#include "engine_state.h"

static_assert(fbalp::kMaxPatches == FBALP_MAX_PATCHES, "patch capacity of the kernel and the C ABI differ");

namespace {

// FP32 "hi" copy of unscaled SELL values plus, per (new-numbered) row, the
// list of FP64 "lo" remainders of the entries FP32 cannot represent exactly.
struct HiLo {
    std::vector<float> hi;
    std::vector<int32_t> lo_ptr, lo_idx;
    std::vector<double> lo_val;
};

static HiLo split_hi_lo(const fbalp::Sell& raw, int32_t rows) {
    HiLo h;
    h.hi.resize(raw.val.size());
    h.lo_ptr.assign(rows + 1, 0);
    std::vector<std::vector<std::pair<int32_t, double>>> per(rows);
    for (int32_t sl = 0; sl < raw.nslices; ++sl) {
        const int32_t len = raw.length[sl];
        for (int32_t k = 0; k < len; ++k)
            for (int32_t lane = 0; lane < 32; ++lane) {
                const int32_t e = raw.off[sl] + k * 32 + lane;
                const float f = static_cast<float>(raw.val[e]);
                h.hi[e] = f;
                const double lo = raw.val[e] - static_cast<double>(f);
                const int32_t r = sl * 32 + lane;
                if (lo != 0.0 && r < rows) per[r].emplace_back(raw.idx[e], lo);
            }
    }
    for (int32_t r = 0; r < rows; ++r) {
        for (auto& pr : per[r]) {
            h.lo_idx.push_back(pr.first);
            h.lo_val.push_back(pr.second);
        }
        h.lo_ptr[r + 1] = static_cast<int32_t>(h.lo_idx.size());
    }
    return h;
}

// Packed matrix words of the re-centred phase: index in the low 16 bits,
// the FP32 value rounded to nearest-even BF16 in the high 16 bits.
static std::vector<uint32_t> pack_bf16(const std::vector<int32_t>& idx, const std::vector<float>& val) {
    std::vector<uint32_t> out(idx.size());
    for (size_t e = 0; e < idx.size(); ++e) {
        uint32_t bits;
        std::memcpy(&bits, &val[e], sizeof(bits));
        const uint32_t rounded = (bits + 0x7fffu + ((bits >> 16) & 1u)) & 0xffff0000u;
        out[e] = rounded | static_cast<uint32_t>(idx[e] & 0xffff);
    }
    return out;
}

// Device copy of one re-centred operand (slices without the long lines in
// warp-schedule order, the long lines, masks, packed words, FP64 values);
// the uploaded slice list is kept on the host for the patched-slice flags.
fbalp::DevLines upload_lines(const fbalp::Sell& S, const std::vector<int32_t>& sched_off,
                             const std::vector<int32_t>& sched, const std::vector<int32_t>& lsched_off,
                             const std::vector<int32_t>& lsched, bool packable, std::vector<int4>* host_list,
                             int4** dev_list, std::vector<void*>& owned) {
    fbalp::DevLines d{};
    d.nslices = S.nslices;
    d.nlong = static_cast<int32_t>(S.long_line.size());
    d.elems = S.off.back();
    d.long_elems = S.long_off.back();
    host_list->clear();
    for (int32_t sl : sched) host_list->push_back(make_int4(sl, S.off[sl], S.length[sl], 0));
    std::vector<int4> llist;
    for (int32_t q : lsched) llist.push_back(make_int4(S.long_line[q], S.long_off[q], S.long_off[q + 1] - S.long_off[q], 0));
    d.list = *dev_list = dev_upload(*host_list, owned);
    d.sched_off = dev_upload(sched_off, owned);
    d.lmask = dev_upload(S.lmask, owned);
    d.long_list = dev_upload(llist, owned);
    d.long_sched_off = dev_upload(lsched_off, owned);
    const std::vector<float> v32(S.val.begin(), S.val.end()), l32(S.long_val.begin(), S.long_val.end());
    if (packable) {
        d.pk = dev_upload(pack_bf16(S.idx, v32), owned);
        d.long_pk = dev_upload(pack_bf16(S.long_idx, l32), owned);
    }
    d.idx = dev_upload(S.idx, owned);
    d.v64 = dev_upload(S.val, owned);
    d.v32 = dev_upload(v32, owned);
    d.long_idx = dev_upload(S.long_idx, owned);
    d.long_v64 = dev_upload(S.long_val, owned);
    d.long_v32 = dev_upload(l32, owned);
    return d;
}

}  // namespace

extern "C" {

void fbalp_default_options(fbalp_options* o) {
    if (!o) return;
    o->ruiz_iterations = 10;
    o->power_iterations = 256;
    o->step_safety = 0.99;
    o->warps_per_block = 16;
    o->blocks_per_sm = 0;
    o->max_dynamic_smem = 0;
    o->stage_matrix = 1;
    o->fp64_max_dynamic_smem = 0;
    o->pair_instances = 1;
    o->spread_banks = 1;
}

void fbalp_default_solve_params(fbalp_solve_params* p) {
    if (!p) return;
    p->precision = FBALP_PRECISION_MIXED;
    p->max_iterations = 20000;
    p->fp32_max_iterations = 20000;
    p->check_every = 64;
    p->tol_primal = 1e-9;
    p->tol_dual = 1e-9;
    p->tol_gap = 1e-7;
    p->fp32_tol_primal = 1e-6;
    p->fp32_tol_dual = 1e-6;
    p->fp32_tol_gap = 1e-4;
    p->reflection = 1.0;
    p->restarts = 1;
    p->fp32_stall_checks = 6;
    p->fp64_stall_checks = 8;
    p->floor_tol = 1e-7;
    p->fp32_passthrough_tol = 1e-3;
    p->fallback_iterations = 4096;
    p->fp32_recentre = 1;
    p->fp32_values_phase = 1;
    p->gate_primal = 1e-5;
    p->gate_dual = 1e-7;
    p->gate_gap = 1e-7;
    p->primal_weight_smoothing = 0.5;
}

const char* fbalp_last_error(void) { return g_last_error.c_str(); }

static bool valid_options(const fbalp_options& o, std::string* err) {
    if (o.ruiz_iterations < 0 || o.ruiz_iterations > 100) return *err = "ruiz_iterations out of [0,100]", false;
    if (o.power_iterations < 1 || o.power_iterations > 100000) return *err = "power_iterations out of range", false;
    if (!(o.step_safety > 0.0 && o.step_safety < 1.0)) return *err = "step_safety must be in (0,1)", false;
    if (o.warps_per_block < 1 || o.warps_per_block * 32 > fbalp::kMaxThreads)
        return *err = "warps_per_block must be in [1,32]", false;
    if (o.blocks_per_sm < 0 || o.blocks_per_sm > 32) return *err = "blocks_per_sm out of range", false;
    if (o.max_dynamic_smem < 0) return *err = "max_dynamic_smem must be non-negative", false;
    if (o.stage_matrix != 0 && o.stage_matrix != 1) return *err = "stage_matrix must be 0 or 1", false;
    if (o.fp64_max_dynamic_smem < 0) return *err = "fp64_max_dynamic_smem must be non-negative", false;
    if (o.pair_instances != 0 && o.pair_instances != 1) return *err = "pair_instances must be 0 or 1", false;
    if (o.spread_banks != 0 && o.spread_banks != 1) return *err = "spread_banks must be 0 or 1", false;
    return true;
}

int fbalp_prepare_matrix(int32_t rows, int32_t cols, const int64_t* indptr, const int32_t* indices,
                         const double* values, const fbalp_options* options, double* dr, double* dc,
                         double* sigma_max, double* eta) {
    try {
        fbalp_options o;
        fbalp_default_options(&o);
        if (options) o = *options;
        std::string err;
        if (!valid_options(o, &err)) return fail(FBALP_ERR_INVALID, err);
        fbalp::Csr a;
        if (!fbalp::canonical_csr(rows, cols, indptr, indices, values, &a, &err))
            return fail(FBALP_ERR_INVALID, err);
        fbalp::Scaling s = fbalp::scale_matrix(a, o.ruiz_iterations, o.power_iterations, o.step_safety);
        if (dr) std::copy(s.dr.begin(), s.dr.end(), dr);
        if (dc) std::copy(s.dc.begin(), s.dc.end(), dc);
        if (sigma_max) *sigma_max = s.sigma_max;
        if (eta) *eta = s.eta;
        return FBALP_OK;
    } catch (const std::exception& e) {
        return fail(FBALP_ERR_ALLOC, e.what());
    }
}

int fbalp_engine_create(int32_t num_species, const int32_t* rows, const int32_t* cols,
                        const int32_t* neq, const int64_t* const* indptr,
                        const int32_t* const* indices, const double* const* values,
                        const fbalp_options* options, void* stream, fbalp_engine** out) {
    if (!out) return fail(FBALP_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (num_species < 1 || !rows || !cols || !neq || !indptr || !indices || !values)
        return fail(FBALP_ERR_INVALID, "num_species >= 1 and non-NULL matrix arrays are required");
    fbalp_options o;
    fbalp_default_options(&o);
    if (options) o = *options;
    std::string err;
    if (!valid_options(o, &err)) return fail(FBALP_ERR_INVALID, err);
    std::unique_ptr<fbalp_engine> E(new fbalp_engine());
    E->opt = o;
    E->stream = static_cast<cudaStream_t>(stream);
    try {
        // --- host preprocessing (validates every matrix before any device work) ---
        for (int s = 0; s < num_species; ++s) {
            SpeciesHost sh;
            if (neq[s] < 0 || neq[s] > rows[s])
                return fail(FBALP_ERR_INVALID, "neq must identify an initial block of equality rows");
            fbalp::Csr a;
            if (!fbalp::canonical_csr(rows[s], cols[s], indptr[s], indices[s], values[s], &a, &err))
                return fail(FBALP_ERR_INVALID, "species " + std::to_string(s) + ": " + err);
            sh.m = a.rows;
            sh.n = a.cols;
            sh.neq = neq[s];
            sh.scaling = fbalp::scale_matrix(a, o.ruiz_iterations, o.power_iterations, o.step_safety);
            fbalp::Csr at = fbalp::transpose(a);
            // rows: equalities then inequalities, each by decreasing length
            sh.row_perm.resize(sh.m);
            std::iota(sh.row_perm.begin(), sh.row_perm.end(), 0);
            auto rlen = [&](int32_t i) { return a.ptr[i + 1] - a.ptr[i]; };
            std::stable_sort(sh.row_perm.begin(), sh.row_perm.begin() + sh.neq,
                             [&](int32_t x, int32_t y) { return rlen(x) > rlen(y); });
            std::stable_sort(sh.row_perm.begin() + sh.neq, sh.row_perm.end(),
                             [&](int32_t x, int32_t y) { return rlen(x) > rlen(y); });
            sh.col_perm.resize(sh.n);
            std::iota(sh.col_perm.begin(), sh.col_perm.end(), 0);
            auto clen = [&](int32_t j) { return at.ptr[j + 1] - at.ptr[j]; };
            std::stable_sort(sh.col_perm.begin(), sh.col_perm.end(),
                             [&](int32_t x, int32_t y) { return clen(x) > clen(y); });
            std::vector<int32_t> row_new(sh.m), col_new(sh.n);
            for (int32_t i = 0; i < sh.m; ++i) row_new[sh.row_perm[i]] = i;
            for (int32_t j = 0; j < sh.n; ++j) col_new[sh.col_perm[j]] = j;
            sh.A = fbalp::build_sell(a, sh.row_perm, col_new, sh.scaling.dr, sh.scaling.dc, sh.n);
            sh.AT = fbalp::build_sell(at, sh.col_perm, row_new, sh.scaling.dc, sh.scaling.dr, sh.m);
            const std::vector<double> ones_m(sh.m, 1.0), ones_n(sh.n, 1.0);
            sh.Araw = fbalp::build_sell(a, sh.row_perm, col_new, ones_m, ones_n, sh.n);
            sh.ATraw = fbalp::build_sell(at, sh.col_perm, row_new, ones_n, ones_m, sh.m);
            fbalp::warp_schedule(sh.A, o.warps_per_block, &sh.a_sched_off, &sh.a_sched);
            fbalp::warp_schedule(sh.AT, o.warps_per_block, &sh.at_sched_off, &sh.at_sched);
            sh.Ar = fbalp::build_sell(a, sh.row_perm, col_new, sh.scaling.dr, sh.scaling.dc, sh.n, fbalp::kLongCut);
            sh.ATr = fbalp::build_sell(at, sh.col_perm, row_new, sh.scaling.dc, sh.scaling.dr, sh.m, fbalp::kLongCut);
            if (o.spread_banks) {
                fbalp::spread_banks(&sh.Ar, sh.n);
                fbalp::spread_banks(&sh.ATr, sh.m);
            }
            fbalp::warp_schedule_split(sh.Ar, o.warps_per_block, &sh.ra_sched_off, &sh.ra_sched, &sh.ra_lsched_off,
                                       &sh.ra_lsched);
            fbalp::warp_schedule_split(sh.ATr, o.warps_per_block, &sh.rat_sched_off, &sh.rat_sched,
                                       &sh.rat_lsched_off, &sh.rat_lsched);
            E->species.push_back(std::move(sh));
        }
        // --- device ---
        check(cudaGetDevice(&E->device), "cudaGetDevice");
        check(cudaDeviceGetAttribute(&E->sm_count, cudaDevAttrMultiProcessorCount, E->device), "attr");
        check(cudaDeviceGetAttribute(&E->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, E->device),
              "attr");
        for (SpeciesHost& sh : E->species) {
            fbalp::DevSpecies d{};
            d.m = sh.m;
            d.n = sh.n;
            d.neq = sh.neq;
            d.a_nslices = sh.A.nslices;
            d.at_nslices = sh.AT.nslices;
            std::vector<float> a32(sh.A.val.begin(), sh.A.val.end()), at32(sh.AT.val.begin(), sh.AT.val.end());
            d.a_elems = sh.A.off.back();
            d.at_elems = sh.AT.off.back();
            std::vector<int4>& alist = sh.alist;
            std::vector<int4>& atlist = sh.atlist;
            for (int32_t sl : sh.a_sched)
                alist.push_back(make_int4(sl, sh.A.off[sl], sh.A.length[sl], 0));
            for (int32_t sl : sh.at_sched)
                atlist.push_back(make_int4(sl, sh.AT.off[sl], sh.AT.length[sl], 0));
            d.a_list = sh.d_alist = dev_upload(alist, E->owned);
            d.at_list = sh.d_atlist = dev_upload(atlist, E->owned);
            d.a_idx = dev_upload(sh.A.idx, E->owned);
            d.a_v32 = dev_upload(a32, E->owned);
            d.a_v64 = dev_upload(sh.A.val, E->owned);
            const bool packable = sh.n + 1 < 65536 && sh.m + 1 < 65536;
            d.ra = upload_lines(sh.Ar, sh.ra_sched_off, sh.ra_sched, sh.ra_lsched_off, sh.ra_lsched, packable,
                                &sh.ralist, &sh.d_ralist, E->owned);
            d.rat = upload_lines(sh.ATr, sh.rat_sched_off, sh.rat_sched, sh.rat_lsched_off, sh.rat_lsched, packable,
                                 &sh.ratlist, &sh.d_ratlist, E->owned);
            d.at_idx = dev_upload(sh.AT.idx, E->owned);
            d.at_v32 = dev_upload(at32, E->owned);
            d.at_v64 = dev_upload(sh.AT.val, E->owned);
            d.a_sched_off = dev_upload(sh.a_sched_off, E->owned);
            d.at_sched_off = dev_upload(sh.at_sched_off, E->owned);
            d.row_perm = dev_upload(sh.row_perm, E->owned);
            d.col_perm = dev_upload(sh.col_perm, E->owned);
            std::vector<double> drn(sh.m), dcn(sh.n);
            for (int32_t i = 0; i < sh.m; ++i) drn[i] = sh.scaling.dr[sh.row_perm[i]];
            for (int32_t j = 0; j < sh.n; ++j) dcn[j] = sh.scaling.dc[sh.col_perm[j]];
            d.dr = dev_upload(drn, E->owned);
            HiLo ha = split_hi_lo(sh.Araw, sh.m), ht = split_hi_lo(sh.ATraw, sh.n);
            d.a_hi = dev_upload(ha.hi, E->owned);
            d.at_hi = dev_upload(ht.hi, E->owned);
            d.lo_a_ptr = dev_upload(ha.lo_ptr, E->owned);
            d.lo_a_idx = dev_upload(ha.lo_idx, E->owned);
            d.lo_a_val = dev_upload(ha.lo_val, E->owned);
            d.lo_at_ptr = dev_upload(ht.lo_ptr, E->owned);
            d.lo_at_idx = dev_upload(ht.lo_idx, E->owned);
            d.lo_at_val = dev_upload(ht.lo_val, E->owned);
            d.dc = dev_upload(dcn, E->owned);
            std::vector<double> idr(sh.m), idc(sh.n);
            for (int32_t i = 0; i < sh.m; ++i) idr[i] = 1.0 / drn[i];
            for (int32_t j = 0; j < sh.n; ++j) idc[j] = 1.0 / dcn[j];
            d.inv_dr = dev_upload(idr, E->owned);
            d.inv_dc = dev_upload(idc, E->owned);
            d.eta = sh.scaling.eta;
            d.sigma_max = sh.scaling.sigma_max;
            E->dev_species_host.push_back(d);
        }
        E->dev_species = dev_upload(E->dev_species_host, E->owned);
        E->queue.ensure(16 * sizeof(int32_t));
        for (cudaEvent_t& v : E->ev) check(cudaEventCreate(&v), "cudaEventCreate");
    } catch (const CudaError& e) {
        return fail(FBALP_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(FBALP_ERR_ALLOC, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(FBALP_ERR_ALLOC, e.what());
    }
    *out = E.release();
    return FBALP_OK;
}

int fbalp_engine_destroy(fbalp_engine* e) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    delete e;
    return FBALP_OK;
}

int fbalp_engine_set_stream(fbalp_engine* e, void* stream) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    e->stream = static_cast<cudaStream_t>(stream);
    return FBALP_OK;
}

int fbalp_engine_set_instances(fbalp_engine* e, int64_t count, const int32_t* species_id,
                               const double* lower, const double* upper, const double* cost,
                               const double* rhs) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (count < 1 || count > INT32_MAX || !species_id || !lower || !upper || !cost)
        return fail(FBALP_ERR_INVALID, "count >= 1, species_id and lower/upper/cost are required");
    std::vector<int32_t> hs(species_id, species_id + count);
    std::vector<int64_t> co(count), ro(count);
    int64_t tc = 0, tr = 0;
    for (int64_t i = 0; i < count; ++i) {
        if (hs[i] < 0 || hs[i] >= static_cast<int32_t>(e->species.size()))
            return fail(FBALP_ERR_INVALID, "species id out of range");
        co[i] = tc;
        ro[i] = tr;
        tc += e->species[hs[i]].n;
        tr += e->species[hs[i]].m;
    }
    // longest instances first: better balance for the persistent queue
    std::vector<int32_t> ord(count);
    std::iota(ord.begin(), ord.end(), 0);
    // (species of equal size stay grouped: the paired kernel restages when
    // the species changes)
    std::stable_sort(ord.begin(), ord.end(), [&](int32_t x, int32_t y) {
        const SpeciesHost &a = e->species[hs[x]], &b = e->species[hs[y]];
        const int64_t sa = a.A.off.back() + a.AT.off.back(), sb = b.A.off.back() + b.AT.off.back();
        return sa != sb ? sa > sb : hs[x] < hs[y];
    });
    try {
        e->inst_species.ensure(count * sizeof(int32_t));
        e->col_off.ensure(count * sizeof(int64_t));
        e->row_off.ensure(count * sizeof(int64_t));
        e->order.ensure(count * sizeof(int32_t));
        check(cudaMemcpyAsync(e->inst_species.ptr, hs.data(), count * sizeof(int32_t), cudaMemcpyHostToDevice, e->stream), "copy");
        check(cudaMemcpyAsync(e->col_off.ptr, co.data(), count * sizeof(int64_t), cudaMemcpyHostToDevice, e->stream), "copy");
        check(cudaMemcpyAsync(e->row_off.ptr, ro.data(), count * sizeof(int64_t), cudaMemcpyHostToDevice, e->stream), "copy");
        check(cudaMemcpyAsync(e->order.ptr, ord.data(), count * sizeof(int32_t), cudaMemcpyHostToDevice, e->stream), "copy");
        // pageable sources: complete the copies before the host vectors die
        check(cudaStreamSynchronize(e->stream), "sync");
    } catch (const CudaError& ex) {
        e->bound = false;
        return fail(FBALP_ERR_CUDA, ex.what());
    }
    e->count = count;
    e->total_cols = tc;
    e->total_rows = tr;
    e->h_species = std::move(hs);
    e->h_coloff = std::move(co);
    e->h_rowoff = std::move(ro);
    e->lower = lower;
    e->upper = upper;
    e->cost = cost;
    e->rhs = rhs;
    e->hints = nullptr;
    e->patch_values = nullptr;
    e->patch_stride = 0;
    e->bound = true;
    return FBALP_OK;
}

int fbalp_engine_set_instance_data(fbalp_engine* e, const double* lower, const double* upper, const double* cost,
                                   const double* rhs) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (!e->bound) return fail(FBALP_ERR_STATE, "set_instances must be called first");
    if (!lower || !upper || !cost) return fail(FBALP_ERR_INVALID, "lower/upper/cost are required");
    e->lower = lower;
    e->upper = upper;
    e->cost = cost;
    e->rhs = rhs;
    return FBALP_OK;
}

int fbalp_engine_set_iteration_hints(fbalp_engine* e, const int32_t* hints) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (!e->bound) return fail(FBALP_ERR_STATE, "set_instances must be called first");
    e->hints = hints;
    return FBALP_OK;
}

int fbalp_engine_set_patches(fbalp_engine* e, int32_t species, int32_t count, const int32_t* rows,
                             const int32_t* cols) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (species < 0 || species >= static_cast<int32_t>(e->species.size()))
        return fail(FBALP_ERR_INVALID, "species id out of range");
    if (count < 0 || count > fbalp::kMaxPatches || (count > 0 && (!rows || !cols)))
        return fail(FBALP_ERR_INVALID, "between 0 and 8 patched entries with row and column indices");
    SpeciesHost& sh = e->species[species];
    std::vector<int32_t> row_new(sh.m), col_new(sh.n);
    for (int32_t i = 0; i < sh.m; ++i) row_new[sh.row_perm[i]] = i;
    for (int32_t j = 0; j < sh.n; ++j) col_new[sh.col_perm[j]] = j;
    for (int32_t q = 0; q < count; ++q) {
        if (rows[q] < 0 || rows[q] >= sh.m || cols[q] < 0 || cols[q] >= sh.n)
            return fail(FBALP_ERR_INVALID, "patched entry outside the species matrix");
        for (int32_t p = 0; p < q; ++p)
            if (rows[p] == rows[q] && cols[p] == cols[q])
                return fail(FBALP_ERR_INVALID, "a patched entry is declared twice");
    }
    fbalp::DevSpecies& d = e->dev_species_host[species];
    d.npatch = count;
    for (int q = 0; q < fbalp::kMaxPatches; ++q) {
        d.patch_row[q] = d.patch_col[q] = 0;
        d.patch_scale[q] = 0.0;
        d.patch_base[q] = 0.0;
    }
    d.patch_col_f2 = 0.0;
    for (auto* l : {&sh.alist, &sh.atlist, &sh.ralist, &sh.ratlist})
        for (auto& v : *l) v.w = 0;
    for (int32_t q = 0; q < count; ++q) {
        const int32_t r = row_new[rows[q]], c = col_new[cols[q]];
        d.patch_row[q] = r;
        d.patch_col[q] = c;
        d.patch_scale[q] = sh.scaling.dr[rows[q]] * sh.scaling.dc[cols[q]];
        for (auto* l : {&sh.alist, &sh.ralist})
            for (auto& v : *l)
                if (v.x == r / 32) v.w = 1;
        for (auto* l : {&sh.atlist, &sh.ratlist})
            for (auto& v : *l)
                if (v.x == c / 32) v.w = 1;
    }
    // scaled template values of the patched columns (row c of A~^T in the
    // SELL slices): each patched entry's base value, and the sum of squares
    // of the columns' other entries, for the per-instance step bound
    // ||A_i~||^2 <= ||A~||^2 + ||A_i~[:, patched columns]||_F^2
    std::vector<int32_t> cols_done;
    for (int32_t q = 0; q < count; ++q) {
        const int32_t c = d.patch_col[q];
        const bool first = std::find(cols_done.begin(), cols_done.end(), c) == cols_done.end();
        if (first) cols_done.push_back(c);
        const int32_t sl = c / 32, lane = c % 32;
        for (int32_t k = 0; k < sh.AT.length[sl]; ++k) {
            const int32_t e2 = sh.AT.off[sl] + k * 32 + lane;
            const int32_t r = sh.AT.idx[e2];
            const double v = sh.AT.val[e2];
            if (r >= sh.m || v == 0.0) continue;  // padding
            bool patched = false;
            for (int32_t p = 0; p < count; ++p)
                if (d.patch_col[p] == c && d.patch_row[p] == r) {
                    patched = true;
                    if (p == q) d.patch_base[q] = v;
                }
            if (first && !patched) d.patch_col_f2 += v * v;
        }
    }
    try {
        check(cudaMemcpy(sh.d_alist, sh.alist.data(), sh.alist.size() * sizeof(int4), cudaMemcpyHostToDevice),
              "copy schedule");
        check(cudaMemcpy(sh.d_atlist, sh.atlist.data(), sh.atlist.size() * sizeof(int4), cudaMemcpyHostToDevice),
              "copy schedule");
        if (!sh.ralist.empty())
            check(cudaMemcpy(sh.d_ralist, sh.ralist.data(), sh.ralist.size() * sizeof(int4), cudaMemcpyHostToDevice),
                  "copy schedule");
        if (!sh.ratlist.empty())
            check(cudaMemcpy(sh.d_ratlist, sh.ratlist.data(), sh.ratlist.size() * sizeof(int4),
                             cudaMemcpyHostToDevice),
                  "copy schedule");
        check(cudaMemcpy(e->dev_species + species, &d, sizeof(d), cudaMemcpyHostToDevice), "copy species");
    } catch (const CudaError& ex) {
        return fail(FBALP_ERR_CUDA, ex.what());
    }
    return FBALP_OK;
}

int fbalp_engine_set_patch_values(fbalp_engine* e, const double* values, int32_t stride) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (!e->bound) return fail(FBALP_ERR_STATE, "set_instances must be called first");
    if (values && (stride < 1 || stride > fbalp::kMaxPatches))
        return fail(FBALP_ERR_INVALID, "stride must be in [1, 8]");
    for (int32_t s : e->h_species)
        if (values && e->dev_species_host[s].npatch > stride)
            return fail(FBALP_ERR_INVALID, "stride is smaller than a species' number of patched entries");
    e->patch_values = values;
    e->patch_stride = values ? stride : 0;
    return FBALP_OK;
}

int fbalp_engine_layout(const fbalp_engine* e, int64_t* total_cols, int64_t* total_rows,
                        int64_t* col_offsets, int64_t* row_offsets) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (!e->bound) return fail(FBALP_ERR_STATE, "no instances are bound");
    if (total_cols) *total_cols = e->total_cols;
    if (total_rows) *total_rows = e->total_rows;
    if (col_offsets) std::copy(e->h_coloff.begin(), e->h_coloff.end(), col_offsets);
    if (row_offsets) std::copy(e->h_rowoff.begin(), e->h_rowoff.end(), row_offsets);
    return FBALP_OK;
}

}  // extern "C"

namespace {

// Static shared memory the dynamic allocation must leave room for: the
// largest actual static size (runtime attributes) among the kernels of a
// family at this engine's block size -- 0 the persistent kernels, 1 the
// re-centred ones, 2 the paired one -- and never below the reduction
// buffers' size.
int64_t static_smem_of(fbalp_engine* e, int family) {
    if (e->static_smem[family] >= 0) return e->static_smem[family];
    const int threads = e->opt.warps_per_block * 32;
    int64_t s = static_cast<int64_t>(sizeof(double) * (threads / 32 * fbalp::kRed + fbalp::kRed) + 64);
    std::vector<const void*> ks;
    if (family == 0) {
        for (int f = 0; f < 2; ++f)
            for (int fast = 0; fast < 2; ++fast) ks.push_back(fbalp::kernel_symbol(f != 0, threads, fast != 0));
    } else if (family == 1) {
        for (int st = 0; st < 2; ++st)
            for (int pa = 0; pa < 2; ++pa)
                for (int fv = 0; fv < 2; ++fv)
                    if (!(pa && fv)) ks.push_back(fbalp::recentred_symbol(threads, st != 0, pa != 0, fv != 0));
    } else {
        ks.push_back(fbalp::pair_symbol(threads));
    }
    for (const void* k : ks) {
        cudaFuncAttributes fa{};
        if (k && cudaFuncGetAttributes(&fa, k) == cudaSuccess)
            s = std::max<int64_t>(s, static_cast<int64_t>(fa.sharedSizeBytes));
        else
            cudaGetLastError();
    }
    e->static_smem[family] = s;
    return s;
}

// Re-centred FP32 layout of the bound batch: 1 when every species fits with
// its matrix staged in shared memory, 2 when every species' vectors fit
// with the matrix streamed from L2 (one variant per launch), 0 otherwise.
int recentred_mode(fbalp_engine* e) {
    const int threads = e->opt.warps_per_block * 32;
    const size_t static_smem = static_cast<size_t>(static_smem_of(e, 1));
    int64_t cap = e->smem_optin > static_cast<int>(static_smem) + 1024
                      ? e->smem_optin - static_cast<int64_t>(static_smem) - 1024 : 0;
    if (e->opt.max_dynamic_smem > 0) cap = std::min<int64_t>(cap, e->opt.max_dynamic_smem);
    std::vector<char> used(e->species.size(), 0);
    for (int32_t s : e->h_species) used[s] = 1;
    bool staged = e->opt.stage_matrix != 0, streamed = true;
    for (size_t s = 0; s < e->species.size(); ++s) {
        if (!used[s]) continue;
        const SpeciesHost& sh = e->species[s];
        for (int st = 0; st < 2; ++st) {
            bool& ok = st ? staged : streamed;
            if (ok && !fbalp::plan_layout_recentred(sh.n, sh.m, e->opt.warps_per_block, sh.shape_a(), sh.shape_at(),
                                                    cap, st != 0)
                           .layout.recentred)
                ok = false;
        }
    }
    return staged ? 1 : (streamed ? 2 : 0);
}

// The paired re-centred kernel (mode 3) instead of the staged one: enabled,
// reflection 1, no patched entries, every species of the batch fits the
// paired layout, and at least two instances per CTA of a full grid (below
// that, one instance per CTA keeps more SMs busy).
bool pair_mode(fbalp_engine* e, double reflection, bool patched) {
    if (!e->opt.pair_instances || reflection != 1.0 || patched) return false;
    if (e->count < 2 * static_cast<int64_t>(e->sm_count)) return false;
    const int threads = e->opt.warps_per_block * 32;
    const size_t static_smem = static_cast<size_t>(static_smem_of(e, 2));
    int64_t cap = e->smem_optin > static_cast<int>(static_smem) + 1024
                      ? e->smem_optin - static_cast<int64_t>(static_smem) - 1024 : 0;
    if (e->opt.max_dynamic_smem > 0) cap = std::min<int64_t>(cap, e->opt.max_dynamic_smem);
    std::vector<char> used(e->species.size(), 0);
    for (int32_t s : e->h_species) used[s] = 1;
    for (size_t s = 0; s < e->species.size(); ++s) {
        if (!used[s]) continue;
        const SpeciesHost& sh = e->species[s];
        if (!fbalp::plan_layout_pair(sh.n, sh.m, sh.neq, e->opt.warps_per_block, sh.shape_a(), sh.shape_at(), cap)
                 .layout.recentred)
            return false;
    }
    return true;
}

// The FP32-valued re-centred phase that continues the instances the BF16
// re-centred phase hands off: mode 4 when every species of the batch fits
// it with the matrix (16-bit indices and FP32 values) in shared memory, 5
// when only the vectors fit (matrix streamed), 0 when neither.
int f32_mode(fbalp_engine* e) {
    const int threads = e->opt.warps_per_block * 32;
    const size_t static_smem = static_cast<size_t>(static_smem_of(e, 1));
    int64_t cap = e->smem_optin > static_cast<int>(static_smem) + 1024
                      ? e->smem_optin - static_cast<int64_t>(static_smem) - 1024 : 0;
    if (e->opt.max_dynamic_smem > 0) cap = std::min<int64_t>(cap, e->opt.max_dynamic_smem);
    std::vector<char> used(e->species.size(), 0);
    for (int32_t s : e->h_species) used[s] = 1;
    bool staged = e->opt.stage_matrix != 0, streamed = true;
    for (size_t s = 0; s < e->species.size(); ++s) {
        if (!used[s]) continue;
        const SpeciesHost& sh = e->species[s];
        for (int st = 0; st < 2; ++st) {
            bool& ok = st ? staged : streamed;
            if (ok && !fbalp::plan_layout_recentred(sh.n, sh.m, e->opt.warps_per_block, sh.shape_a(), sh.shape_at(),
                                                    cap, st != 0, true)
                           .layout.recentred)
                ok = false;
        }
    }
    return staged ? 4 : (streamed ? 5 : 0);
}

// Launch one precision phase over the bound batch (`recentred`: the
// re-centred FP32 kernel in mode 1 (staged matrix), 2 (streamed), 3
// (staged, two instances per CTA), 4 / 5 (FP32 matrix values, staged /
// streamed)).  `book` is the phase's slot in the engine's per-phase records
// (0 first phase, 1 FP64 phase, 2 FP32-valued middle phase); the middle and
// FP64 phases share the second timing pair (`rec_start` / `rec_stop` say
// which ends of it this launch records).
void run_phase(fbalp_engine* e, bool fp64, fbalp::KernelParams p, int recentred = 0, int book = -1,
               bool rec_start = true, bool rec_stop = true) {
    if (book < 0) book = fp64 ? 1 : 0;
    const bool f32v = recentred >= 4;
    const int esz = fp64 ? static_cast<int>(sizeof(double)) : static_cast<int>(sizeof(float));
    const int threads = e->opt.warps_per_block * 32;
    const size_t static_smem = static_cast<size_t>(
        static_smem_of(e, recentred == 3 ? 2 : recentred ? 1 : 0));
    int64_t cap = e->smem_optin > static_cast<int>(static_smem) + 1024
                      ? e->smem_optin - static_cast<int64_t>(static_smem) - 1024 : 0;
    if (e->opt.max_dynamic_smem > 0) cap = std::min<int64_t>(cap, e->opt.max_dynamic_smem);
    if (fp64 && e->opt.fp64_max_dynamic_smem > 0) cap = std::min<int64_t>(cap, e->opt.fp64_max_dynamic_smem);
    std::vector<char> used(e->species.size(), 0);
    for (int32_t s : e->h_species) used[s] = 1;
    std::vector<fbalp::Layout>& layouts = fp64 ? e->layouts64 : e->layouts32;
    layouts.assign(e->species.size(), fbalp::Layout{});
    int64_t dyn = 0, slab = 0;
    bool all_fast = true;
    // FP64: the unscaled staged layout is used only when every species of
    // the batch fits it (one kernel variant per launch)
    bool unscaled = fp64 && e->opt.stage_matrix != 0;
    if (unscaled)
        for (size_t s = 0; s < e->species.size(); ++s) {
            if (!used[s]) continue;
            const SpeciesHost& sh = e->species[s];
            if (!fbalp::plan_layout_unscaled(sh.n, sh.m, e->opt.warps_per_block, sh.A.nslices, sh.AT.nslices,
                                             sh.A.off.back(), sh.AT.off.back(), cap).layout.unscaled)
                unscaled = false;
        }
    for (size_t s = 0; s < e->species.size(); ++s) {
        if (!used[s]) continue;
        const SpeciesHost& sh = e->species[s];
        fbalp::LayoutPlan P = recentred == 3
            ? fbalp::plan_layout_pair(sh.n, sh.m, sh.neq, e->opt.warps_per_block, sh.shape_a(), sh.shape_at(), cap)
            : recentred
            ? fbalp::plan_layout_recentred(sh.n, sh.m, e->opt.warps_per_block, sh.shape_a(), sh.shape_at(), cap,
                                           recentred == 1 || recentred == 4, f32v)
            : unscaled
            ? fbalp::plan_layout_unscaled(sh.n, sh.m, e->opt.warps_per_block, sh.A.nslices, sh.AT.nslices,
                                          sh.A.off.back(), sh.AT.off.back(), cap)
            : fbalp::plan_layout(sh.n, sh.m, e->opt.warps_per_block, sh.A.nslices, sh.AT.nslices,
                                 sh.A.off.back(), sh.AT.off.back(), esz, cap, !fp64 && e->opt.stage_matrix != 0);
        if (recentred && !P.layout.recentred) throw CudaError("species does not fit the re-centred layout");
        if (P.smem_bytes > cap) throw CudaError("species schedule does not fit into shared memory");
        if (!fbalp::layout_aligned(P.layout)) throw CudaError("internal error: misaligned shared-memory layout");
        layouts[s] = P.layout;
        all_fast = all_fast && (recentred || (fp64 ? unscaled
                                                   : (P.layout.mat_smem && (P.layout.smem_mask & 0x1ff) == 0x1ff)));
        dyn = std::max(dyn, P.smem_bytes);
        slab = std::max(slab, P.slab_bytes);
    }
    dyn = fbalp::align_up(std::max<int64_t>(dyn, 16), 16);
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    check(cudaStreamIsCapturing(e->stream, &capture), "cudaStreamIsCapturing");
    const bool capturing = capture != cudaStreamCaptureStatusNone;
    const int kind = recentred ? 1 + recentred : (fp64 ? 1 : 0);
    Buffer& dl = e->layout_dev[kind];
    std::vector<fbalp::Layout>& cached = e->layout_host[kind];
    const size_t lbytes = layouts.size() * sizeof(fbalp::Layout);
    if (cached.size() != layouts.size() || std::memcmp(cached.data(), layouts.data(), lbytes) != 0) {
        if (capturing) throw CudaError("launch layouts changed during stream capture; solve once before capturing");
        dl.ensure(lbytes);
        check(cudaMemcpy(dl.ptr, layouts.data(), lbytes, cudaMemcpyHostToDevice), "copy layouts");
        cached = layouts;
    }
    const bool patched = recentred && p.patch_values != nullptr;
    const bool pair = recentred == 3;
    const bool staged = recentred == 1 || recentred == 4;
    const void* k = pair ? fbalp::pair_symbol(threads)
                         : recentred ? fbalp::recentred_symbol(threads, staged, patched, f32v)
                                     : fbalp::kernel_symbol(fp64, threads, all_fast);
    // the dynamic shared-memory limit is a property of the kernel in this
    // process (shared by every engine): raise it when this launch needs
    // more, never lower it
    cudaFuncAttributes fa{};
    check(cudaFuncGetAttributes(&fa, k), "cudaFuncGetAttributes");
    if (fa.maxDynamicSharedSizeBytes < dyn)
        check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dyn)),
              "cudaFuncSetAttribute");
    int per_sm = 0;
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, dyn), "occupancy");
    if (e->opt.blocks_per_sm > 0) per_sm = std::min(per_sm, e->opt.blocks_per_sm);
    if (per_sm < 1)
        throw CudaError("kernel does not fit on an SM with this configuration (threads " + std::to_string(threads) +
                        ", dynamic shared memory " + std::to_string(dyn) + " B, static " +
                        std::to_string(fa.sharedSizeBytes) + " B, registers " + std::to_string(fa.numRegs) +
                        ", opt-in limit " + std::to_string(e->smem_optin) + " B)");
    // the paired kernel holds two instances (and two slabs) per CTA
    const int64_t per_cta = pair ? 2 : 1;
    const int grid = static_cast<int>(std::min<int64_t>((e->count + per_cta - 1) / per_cta,
                                                        static_cast<int64_t>(per_sm) * e->sm_count));
    p.layouts = static_cast<const fbalp::Layout*>(dl.ptr);
    if (slab > 0) {
        const size_t want = static_cast<size_t>(slab) * per_cta * grid;
        if (capturing && e->spill.bytes < want)
            throw CudaError("workspace would grow during stream capture; solve once before capturing");
        e->spill.ensure(want);
        p.spill = static_cast<unsigned char*>(e->spill.ptr);
        p.spill_stride = slab;
    } else {
        p.spill = nullptr;
        p.spill_stride = 0;
    }
    p.queue = static_cast<int32_t*>(e->queue.ptr) + book;
    check(cudaMemsetAsync(p.queue, 0, sizeof(int32_t), e->stream), "memset queue");
    const int ph = (fp64 || f32v) ? 1 : 0;
    // phase timing events only outside a capture (a graph replay has no
    // per-phase timing)
    if (!capturing && rec_start) check(cudaEventRecord(e->ev[2 * ph], e->stream), "cudaEventRecord");
    // a selected timing slot records around the launch in either case (an
    // external event node under capture)
    cudaEvent_t* sev = e->slot >= 0 ? &e->slot_ev[4 * static_cast<size_t>(e->slot)] : nullptr;
    const unsigned rec_flags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    if (sev && rec_start) check(cudaEventRecordWithFlags(sev[2 * ph], e->stream, rec_flags), "timing slot record");
    if (pair)
        check(fbalp::launch_pair(grid, threads, dyn, e->stream, p), "paired re-centred pdhg kernel launch");
    else if (recentred)
        check(fbalp::launch_recentred(staged, patched, grid, threads, dyn, e->stream, p, f32v),
              "re-centred pdhg kernel launch");
    else
        check(fbalp::launch_pdhg(fp64, all_fast, grid, threads, dyn, e->stream, p), "pdhg kernel launch");
    if (sev && rec_stop) {
        check(cudaEventRecordWithFlags(sev[2 * ph + 1], e->stream, rec_flags), "timing slot record");
        e->slot_ran[2 * static_cast<size_t>(e->slot) + ph] = 1;
    }
    if (!capturing && rec_stop) check(cudaEventRecord(e->ev[2 * ph + 1], e->stream), "cudaEventRecord");
    if (rec_stop) e->ran[ph] = !capturing;
    e->last_grid[book] = grid;
    e->last_kind[book] = kind;
    e->last_smem[book] = dyn;
}


}  // namespace

extern "C" int fbalp_engine_solve(fbalp_engine* e, const double* warm_x, const double* warm_y,
                                  const double* warm_omega, const fbalp_solve_params* params,
                                  int32_t* out_status, double* out_objective, double* out_x,
                                  double* out_y, int32_t* out_iterations, double* out_metrics,
                                  double* out_omega) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (!e->bound) return fail(FBALP_ERR_STATE, "set_instances must be called before solve");
    if (!out_status || !out_objective || !out_x || !out_y || !out_iterations || !out_metrics)
        return fail(FBALP_ERR_INVALID, "output arrays are required");
    fbalp_solve_params q;
    fbalp_default_solve_params(&q);
    if (params) q = *params;
    std::string err;
    if (!valid_params(q, &err)) return fail(FBALP_ERR_INVALID, err);
    try {
        e->ran[0] = e->ran[1] = false;
        e->last_kind[0] = e->last_kind[1] = e->last_kind[2] = -1;
        fbalp::KernelParams p{};
        p.species = e->dev_species;
        p.count = static_cast<int32_t>(e->count);
        p.order = static_cast<const int32_t*>(e->order.ptr);
        p.inst_species = static_cast<const int32_t*>(e->inst_species.ptr);
        p.col_off = static_cast<const int64_t*>(e->col_off.ptr);
        p.row_off = static_cast<const int64_t*>(e->row_off.ptr);
        p.lower = e->lower;
        p.upper = e->upper;
        p.cost = e->cost;
        p.rhs = e->rhs;
        p.check_every = q.check_every;
        p.rho = q.reflection;
        p.restarts = q.restarts;
        p.gate_p = q.gate_primal;
        p.gate_d = q.gate_dual;
        p.gate_g = q.gate_gap;
        p.omega_smoothing = q.primal_weight_smoothing;
        bool patched = false;
        if (e->patch_values)
            for (int32_t sp_id : e->h_species) patched = patched || e->dev_species_host[sp_id].npatch > 0;
        if (patched && !(q.precision == FBALP_PRECISION_MIXED && q.fp32_recentre && recentred_mode(e) != 0))
            return fail(FBALP_ERR_INVALID, "patched entries need the re-centred mixed schedule");
        if (q.precision == FBALP_PRECISION_FP64 || q.precision == FBALP_PRECISION_FP32) {
            const bool fp64 = q.precision == FBALP_PRECISION_FP64;
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
            p.max_iters = fp64 ? q.max_iterations : q.fp32_max_iterations;
            p.tol_p = fp64 ? q.tol_primal : q.fp32_tol_primal;
            p.tol_d = fp64 ? q.tol_dual : q.fp32_tol_dual;
            p.tol_g = fp64 ? q.tol_gap : q.fp32_tol_gap;
            p.final_status = fp64 ? fbalp::kStatusOptimal : fbalp::kStatusHandoff;
            p.clip_output = 1;
            p.stall_checks = fp64 ? q.fp64_stall_checks : q.fp32_stall_checks;
            p.floor_tol = q.floor_tol;
            p.passthrough_tol = 0.0;
            p.fallback_iters = q.fallback_iterations;
            run_phase(e, fp64, p);
        } else if (q.fp32_recentre && q.fp32_values_phase == 2 && !patched && recentred_mode(e) != 0 &&
                   f32_mode(e) != 0) {
            // continuation: every instance runs in the FP32-valued re-centred
            // phase directly, from the caller's point (iterates that an
            // earlier call left in that phase would only be set back by the
            // BF16-matrix phase and its cold fallback)
            fbalp::KernelParams pn = p;
            pn.warm_x = warm_x;
            pn.warm_y = warm_y;
            pn.warm_omega = warm_omega;
            pn.prior_iters = nullptr;
            pn.out_x = out_x;
            pn.out_y = out_y;
            pn.out_obj = out_objective;
            pn.out_metrics = out_metrics;
            pn.out_omega = out_omega;
            pn.out_status = out_status;
            pn.out_iters = out_iterations;
            pn.max_iters = q.max_iterations;
            pn.tol_p = q.tol_primal;
            pn.tol_d = q.tol_dual;
            pn.tol_g = q.tol_gap;
            pn.final_status = fbalp::kStatusOptimal;
            pn.clip_output = 1;
            pn.stall_checks = q.fp64_stall_checks;
            pn.floor_tol = q.floor_tol;
            pn.passthrough_tol = 0.0;
            pn.fallback_iters = 0;
            pn.handoff_on_stall = 0;
            run_phase(e, false, pn, f32_mode(e), 2, true, true);
        } else if (q.fp32_recentre && recentred_mode(e) != 0) {
            // re-centred FP32 phase to the FP64 tolerances; what it does not
            // certify (stalled instances) continues in the FP64 phase
            e->mid_x.ensure(e->total_cols * sizeof(double));
            e->mid_y.ensure(std::max<int64_t>(1, e->total_rows) * sizeof(double));
            e->mid_omega.ensure(e->count * sizeof(double));
            e->mid_iters.ensure(e->count * sizeof(int32_t));
            e->hand_list.ensure(e->count * sizeof(int32_t));
            e->hand_count.ensure(sizeof(int32_t));
            check(cudaMemsetAsync(e->hand_count.ptr, 0, sizeof(int32_t), e->stream), "memset handoff count");
            fbalp::KernelParams pr = p;
            pr.warm_x = warm_x;
            pr.warm_y = warm_y;
            pr.warm_omega = warm_omega;
            pr.prior_iters = nullptr;
            pr.out_x = out_x;
            pr.out_y = out_y;
            pr.out_obj = out_objective;
            pr.out_metrics = out_metrics;
            pr.out_omega = out_omega;
            pr.out_status = out_status;
            pr.out_iters = out_iterations;
            pr.max_iters = q.max_iterations;
            pr.tol_p = q.tol_primal;
            pr.tol_d = q.tol_dual;
            pr.tol_g = q.tol_gap;
            pr.final_status = fbalp::kStatusOptimal;
            pr.clip_output = 1;
            pr.stall_checks = q.fp64_stall_checks;
            pr.floor_tol = q.floor_tol;
            pr.passthrough_tol = 0.0;
            pr.fallback_iters = q.fallback_iterations;
            pr.handoff_list = static_cast<int32_t*>(e->hand_list.ptr);
            pr.handoff_count = static_cast<int32_t*>(e->hand_count.ptr);
            pr.hand_x = static_cast<double*>(e->mid_x.ptr);
            pr.hand_y = static_cast<double*>(e->mid_y.ptr);
            pr.hand_omega = static_cast<double*>(e->mid_omega.ptr);
            pr.hand_iters = static_cast<int32_t*>(e->mid_iters.ptr);
            pr.handoff_on_stall = 4 * q.fp64_stall_checks;
            pr.hint_iters = e->hints;
            pr.patch_values = patched ? e->patch_values : nullptr;
            pr.patch_stride = e->patch_stride;
            if (patched) pr.handoff_on_stall = 0;  // the FP64 phase has no patched entries
            const int mode = recentred_mode(e);
            run_phase(e, false, pr, mode == 1 && pair_mode(e, q.reflection, patched) ? 3 : mode);
            // instances the BF16-matrix phase hands off (a stall: on badly
            // scaled models the BF16-rounded matrix limits the correction
            // LPs) continue from their own point with FP32 matrix values;
            // what that phase hands off in turn finishes in FP64
            const int fmode = (q.fp32_values_phase && !patched) ? f32_mode(e) : 0;
            // the handed-off instances continue from their own point
            fbalp::KernelParams pn = p;
            pn.order = static_cast<const int32_t*>(e->hand_list.ptr);
            pn.count_dev = static_cast<const int32_t*>(e->hand_count.ptr);
            pn.warm_x = static_cast<const double*>(e->mid_x.ptr);
            pn.warm_y = static_cast<const double*>(e->mid_y.ptr);
            pn.warm_omega = static_cast<const double*>(e->mid_omega.ptr);
            pn.prior_iters = static_cast<const int32_t*>(e->mid_iters.ptr);
            pn.out_x = out_x;
            pn.out_y = out_y;
            pn.out_obj = out_objective;
            pn.out_metrics = out_metrics;
            pn.out_omega = out_omega;
            pn.out_status = out_status;
            pn.out_iters = out_iterations;
            pn.max_iters = q.max_iterations;
            pn.tol_p = q.tol_primal;
            pn.tol_d = q.tol_dual;
            pn.tol_g = q.tol_gap;
            pn.final_status = fbalp::kStatusOptimal;
            pn.clip_output = 1;
            pn.floor_tol = q.floor_tol;
            pn.passthrough_tol = 0.0;
            if (fmode) {
                // with FP32 matrix values (the BF16-rounded matrix of the
                // first phase is what stalls on badly scaled models); no
                // stall rule and no further hand-off: on real models slow
                // phases outlast any stall window (measured plateaus beyond
                // 512 tests) and converge at this phase's rate, which the
                // FP64 phase would only repeat at ~20x the cost per
                // iteration; an instance that exhausts the budget reports
                // the iteration limit with its iterate (a caller's next pass
                // continues from it)
                pn.stall_checks = q.fp64_stall_checks;
                pn.fallback_iters = 0;  // a stalled point restarting cold would lose its progress
                pn.handoff_on_stall = 0;
                run_phase(e, false, pn, fmode, 2, true, true);
            } else {
                pn.stall_checks = q.fp64_stall_checks;
                pn.fallback_iters = q.fallback_iterations;
                run_phase(e, true, pn, 0, 1, true, true);
            }
        } else {
            e->mid_x.ensure(e->total_cols * sizeof(double));
            e->mid_y.ensure(std::max<int64_t>(1, e->total_rows) * sizeof(double));
            e->mid_omega.ensure(e->count * sizeof(double));
            e->mid_iters.ensure(e->count * sizeof(int32_t));
            e->mid_status.ensure(e->count * sizeof(int32_t));
            e->mid_obj.ensure(e->count * sizeof(double));
            e->mid_metrics.ensure(e->count * fbalp::kMetrics * sizeof(double));
            fbalp::KernelParams p32 = p;
            p32.warm_x = warm_x;
            p32.warm_y = warm_y;
            p32.warm_omega = warm_omega;
            p32.prior_iters = nullptr;
            p32.out_x = static_cast<double*>(e->mid_x.ptr);
            p32.out_y = static_cast<double*>(e->mid_y.ptr);
            p32.out_obj = static_cast<double*>(e->mid_obj.ptr);
            p32.out_metrics = static_cast<double*>(e->mid_metrics.ptr);
            p32.out_omega = static_cast<double*>(e->mid_omega.ptr);
            p32.out_status = static_cast<int32_t*>(e->mid_status.ptr);
            p32.out_iters = static_cast<int32_t*>(e->mid_iters.ptr);
            p32.max_iters = q.fp32_max_iterations;
            p32.tol_p = q.fp32_tol_primal;
            p32.tol_d = q.fp32_tol_dual;
            p32.tol_g = q.fp32_tol_gap;
            p32.final_status = fbalp::kStatusHandoff;
            p32.clip_output = 0;
            p32.stall_checks = q.fp32_stall_checks;
            p32.floor_tol = q.floor_tol;
            p32.passthrough_tol = q.fp32_passthrough_tol;
            p32.fallback_iters = 0;  // the FP32 phase hands off on a stall instead
            run_phase(e, false, p32);
            fbalp::KernelParams p64 = p;
            p64.warm_x = static_cast<const double*>(e->mid_x.ptr);
            p64.warm_y = static_cast<const double*>(e->mid_y.ptr);
            p64.warm_omega = static_cast<const double*>(e->mid_omega.ptr);
            p64.prior_iters = static_cast<const int32_t*>(e->mid_iters.ptr);
            p64.out_x = out_x;
            p64.out_y = out_y;
            p64.out_obj = out_objective;
            p64.out_metrics = out_metrics;
            p64.out_omega = out_omega;
            p64.out_status = out_status;
            p64.out_iters = out_iterations;
            p64.max_iters = q.max_iterations;
            p64.tol_p = q.tol_primal;
            p64.tol_d = q.tol_dual;
            p64.tol_g = q.tol_gap;
            p64.final_status = fbalp::kStatusOptimal;
            p64.clip_output = 1;
            p64.stall_checks = q.fp64_stall_checks;
            p64.floor_tol = q.floor_tol;
            p64.passthrough_tol = 0.0;
            p64.fallback_iters = q.fallback_iterations;
            run_phase(e, true, p64);
        }
    } catch (const CudaError& ex) {
        return fail(FBALP_ERR_CUDA, ex.what());
    } catch (const std::exception& ex) {
        return fail(FBALP_ERR_ALLOC, ex.what());
    }
    return FBALP_OK;
}

extern "C" int fbalp_engine_phase_times(fbalp_engine* e, float* ms_fp32, float* ms_fp64) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    float* outs[2] = {ms_fp32, ms_fp64};
    for (int ph = 0; ph < 2; ++ph) {
        if (!outs[ph]) continue;
        *outs[ph] = 0.0f;
        if (!e->ran[ph]) continue;
        cudaError_t err = cudaEventSynchronize(e->ev[2 * ph + 1]);
        if (err == cudaSuccess) err = cudaEventElapsedTime(outs[ph], e->ev[2 * ph], e->ev[2 * ph + 1]);
        if (err != cudaSuccess) return fail(FBALP_ERR_CUDA, cudaGetErrorString(err));
    }
    return FBALP_OK;
}

extern "C" int fbalp_engine_phase_kernels(fbalp_engine* e, int32_t* fp32_kind, int32_t* fp64_kind) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (fp32_kind) *fp32_kind = e->last_kind[0];
    if (fp64_kind) *fp64_kind = e->last_kind[2] >= 0 ? e->last_kind[2] : e->last_kind[1];
    return FBALP_OK;
}

extern "C" int fbalp_engine_timing_slots(fbalp_engine* e, int32_t slots) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (slots < 0 || slots > 64) return fail(FBALP_ERR_INVALID, "slots must be in [0, 64]");
    for (cudaEvent_t& v : e->slot_ev)
        if (v) cudaEventDestroy(v);
    e->slot_ev.assign(4 * static_cast<size_t>(slots), nullptr);
    e->slot_ran.assign(2 * static_cast<size_t>(slots), 0);
    e->slot = -1;
    for (cudaEvent_t& v : e->slot_ev) {
        cudaError_t err = cudaEventCreate(&v);
        if (err != cudaSuccess) return fail(FBALP_ERR_CUDA, cudaGetErrorString(err));
    }
    return FBALP_OK;
}

extern "C" int fbalp_engine_use_timing_slot(fbalp_engine* e, int32_t slot) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (slot < -1 || slot >= static_cast<int32_t>(e->slot_ran.size() / 2))
        return fail(FBALP_ERR_INVALID, "timing slot out of range");
    e->slot = slot;
    return FBALP_OK;
}

extern "C" int fbalp_engine_slot_times(fbalp_engine* e, int32_t slot, float* ms_fp32, float* ms_fp64) {
    if (!e) return fail(FBALP_ERR_INVALID, "engine is NULL");
    if (slot < 0 || slot >= static_cast<int32_t>(e->slot_ran.size() / 2))
        return fail(FBALP_ERR_INVALID, "timing slot out of range");
    float* outs[2] = {ms_fp32, ms_fp64};
    for (int ph = 0; ph < 2; ++ph) {
        if (!outs[ph]) continue;
        *outs[ph] = 0.0f;
        if (!e->slot_ran[2 * static_cast<size_t>(slot) + ph]) continue;
        const cudaEvent_t* sev = &e->slot_ev[4 * static_cast<size_t>(slot)];
        cudaError_t err = cudaEventSynchronize(sev[2 * ph + 1]);
        if (err == cudaSuccess) err = cudaEventElapsedTime(outs[ph], sev[2 * ph], sev[2 * ph + 1]);
        if (err != cudaSuccess) return fail(FBALP_ERR_CUDA, cudaGetErrorString(err));
    }
    return FBALP_OK;
}

extern "C" int fbalp_engine_phase_iterations(fbalp_engine* e, int32_t* out_fp32_iterations) {
    if (!e || !out_fp32_iterations) return fail(FBALP_ERR_INVALID, "engine and output are required");
    if (!e->bound) return fail(FBALP_ERR_STATE, "no instances are bound");
    if (!e->ran[0] || !e->ran[1]) return fail(FBALP_ERR_STATE, "the last solve was not a mixed-precision solve");
    cudaError_t err = cudaMemcpyAsync(out_fp32_iterations, e->mid_iters.ptr, e->count * sizeof(int32_t),
                                      cudaMemcpyDeviceToDevice, e->stream);
    if (err != cudaSuccess) return fail(FBALP_ERR_CUDA, cudaGetErrorString(err));
    return FBALP_OK;
}
