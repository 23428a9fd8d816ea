// Persistent instance-resident restarted Halpern PDHG kernel (sm_100a).
// See pdhg_kernel.cuh for the design and oracle/pdhg.py for the restatement.
#include "pdhg_kernel.cuh"
#include "fbalp_internal.h"

#include <cmath>

namespace fbalp {

template <typename T> struct Vals;
template <> struct Vals<float> {
    __device__ static const float* a(const DevSpecies* s) { return s->a_v32; }
    __device__ static const float* at(const DevSpecies* s) { return s->at_v32; }
};
template <> struct Vals<double> {
    __device__ static const double* a(const DevSpecies* s) { return s->a_v64; }
    __device__ static const double* at(const DevSpecies* s) { return s->at_v64; }
};

template <typename T> __device__ __forceinline__ T clampT(T v, T l, T u) {
    // NaN-preserving projection: a NaN compares false and passes through.
    return v < l ? l : (v > u ? u : v);
}

// One SELL-32 slice row product: lane `lane` owns row (slice*32 + lane) and
// element k of that row sits at base + 32*k + lane, so every step is one
// coalesced load of 32 indices and 32 values.  Loads are issued in batches
// of U before any is used (one memory round trip per batch).
template <typename T, typename V, typename I, bool GLOBAL>
__device__ __forceinline__ T slice_dot(const I* __restrict__ idx, const V* __restrict__ val,
                                       int base, int len, int lane, const T* g) {
    constexpr int U = GLOBAL ? (sizeof(V) == 4 ? 8 : 4) : 4;
    const I* ip = idx + base + lane;
    const V* vp = val + base + lane;
    T acc = T(0);
    for (int k0 = 0; k0 < len; k0 += U) {
        int ii[U];
        V vv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + u;
            if (k < len) {
                if (GLOBAL) {
                    ii[u] = __ldg(reinterpret_cast<const int32_t*>(ip) + (k << 5));
                    vv[u] = __ldg(vp + (k << 5));
                } else {
                    ii[u] = ip[k << 5];
                    vv[u] = vp[k << 5];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k0 + u < len) acc = fma(static_cast<T>(vv[u]), g[ii[u]], acc);
    }
    return acc;
}

// FP64 product for the convergence test, whatever the iterate precision
// (always the global FP64 slices).
template <typename T>
__device__ __forceinline__ double slice_dot64(const int32_t* __restrict__ idx,
                                              const double* __restrict__ val, int base, int len,
                                              int lane, const T* g) {
    constexpr int U = 4;
    const int32_t* ip = idx + base + lane;
    const double* vp = val + base + lane;
    double acc = 0.0;
    for (int k0 = 0; k0 < len; k0 += U) {
        int ii[U];
        double vv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + u;
            if (k < len) {
                ii[u] = __ldg(ip + (k << 5));
                vv[u] = __ldg(vp + (k << 5));
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k0 + u < len) acc = fma(vv[u], static_cast<double>(g[ii[u]]), acc);
    }
    return acc;
}

template <typename T> struct Arrays {
    T *xbar, *y, *x, *xa, *ya, *cs, *ls, *us, *bs, *xs, *ys, *w;
};

// Sums for q < kRedSums, maxima above.  Deterministic order.
__device__ __forceinline__ void block_reduce_body(double* v, double (*s_red)[kRed], double* s_tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < kRed; ++q) {
        double x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = (q < kRedSums) ? x + y : fmax(x, y);
        }
        v[q] = x;
    }
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < kRed; ++q) s_red[warp][q] = v[q];
    }
    __syncthreads();
    if (threadIdx.x < kRed) {
        const int q = threadIdx.x;
        double x = s_red[0][q];
        for (int w = 1; w < nw; ++w) x = (q < kRedSums) ? x + s_red[w][q] : fmax(x, s_red[w][q]);
        s_tot[q] = x;
    }
    __syncthreads();
}

// Out-of-line copy for the kernels that reduce rarely.
__device__ __noinline__ void block_reduce(double* v, double (*s_red)[kRed], double* s_tot) {
    block_reduce_body(v, s_red, s_tot);
}

// FP64 KKT quantities at the candidate (xs, ys), in ORIGINAL units and with
// the caller's exact FP64 bounds, objective and right-hand side (the scaled
// copies in shared memory may be FP32).  Partial sums / maxima of this thread
// are added to v.  Index map of v (oracle/pdhg.py kkt_metrics is the twin):
//  0 c.x   1 b.y   2 sum bound-dual terms   3 bound complementarity
//  4 row complementarity   5 |xn-x|^2  6 |yn-y|^2  7 |xn-xa|^2  8 |yn-ya|^2
//  10 max primal row residual  11 max dual violation  12 max bound violation
//  13 |x|_inf  14 |c|_inf  15 NaN flag
template <typename T>
__device__ __noinline__ void kkt_partials(const DevSpecies* sp, const int4* alist, const int4* atlist,
                                          int a0, int a1, int t0, int t1, const T* xs, const T* ys,
                                          const double* lower, const double* upper,
                                          const double* cost, const double* rhs, int lane,
                                          double* v) {
    const int n = sp->n, m = sp->m, neq = sp->neq;
    for (int t = t0; t < t1; ++t) {
        const int4 sl = atlist[t];
        const double g = slice_dot64<T>(sp->at_idx, sp->at_v64, sl.y, sl.z, lane, ys);
        const int j = (sl.x << 5) + lane;
        if (j < n) {
            const int jo = sp->col_perm[j];
            const double dcj = sp->dc[j];
            const double c = cost[jo], l = lower[jo], u = upper[jo];
            const double xv = static_cast<double>(xs[j]) * dcj;
            const double r = c - g / dcj;  // c - A^T y in original units
            v[0] += c * xv;
            if (r > 0.0) {
                if (isfinite(l)) v[2] += r * l;
                else v[11] = fmax(v[11], r);
            } else if (r < 0.0) {
                if (isfinite(u)) v[2] += r * u;
                else v[11] = fmax(v[11], -r);
            }
            const double tg = (r >= 0.0) ? l : u;
            if (isfinite(tg)) v[3] += fabs(r * (xv - tg));
            v[12] = fmax(v[12], fmax(l - xv, xv - u));
            v[13] = fmax(v[13], fabs(xv));
            v[14] = fmax(v[14], fabs(c));
            if (isnan(g) || isnan(xv)) v[15] = 1.0;
        }
    }
    for (int t = a0; t < a1; ++t) {
        const int4 sl = alist[t];
        const double h = slice_dot64<T>(sp->a_idx, sp->a_v64, sl.y, sl.z, lane, xs);
        const int i = (sl.x << 5) + lane;
        if (i < m) {
            const double dri = sp->dr[i];
            const double b = rhs ? rhs[sp->row_perm[i]] : 0.0;
            const double yv = static_cast<double>(ys[i]) * dri;
            const double ro = h / dri - b;  // A x - b in original units
            if (i < neq) {
                v[10] = fmax(v[10], fabs(ro));
            } else {
                v[10] = fmax(v[10], ro);
                v[4] += fabs(yv * ro);
                v[11] = fmax(v[11], yv);
            }
            v[1] += b * yv;
            if (isnan(h) || isnan(yv)) v[15] = 1.0;
        }
    }
}

struct Metrics {
    double primal, dual, kgap, pobj, dobj, rgap, xinf, cinf, r;
    bool nan, conv;
};

__device__ Metrics evaluate(const double* s_tot, double omega, double tol_p, double tol_d,
                            double tol_g) {
    Metrics M;
    M.pobj = s_tot[0];
    M.dobj = s_tot[1] + s_tot[2];
    M.primal = fmax(fmax(s_tot[10], s_tot[12]), 0.0);
    M.dual = fmax(s_tot[11], 0.0);
    M.kgap = (s_tot[3] + s_tot[4]) / fmax(1.0, fabs(M.pobj));
    M.rgap = fabs(M.pobj - M.dobj) / (1.0 + fabs(M.pobj) + fabs(M.dobj));
    M.xinf = s_tot[13];
    M.cinf = s_tot[14];
    M.r = sqrt(__fma_rn(omega, s_tot[5], s_tot[6] / omega));  // explicit: both re-centred kernels round alike
    M.nan = s_tot[15] > 0.0 || !isfinite(M.pobj) || !isfinite(M.dobj) || !isfinite(M.kgap) ||
            !isfinite(M.primal);
    M.conv = !M.nan && M.primal <= tol_p * (1.0 + M.xinf) && M.dual <= tol_d * (1.0 + M.cinf) &&
             M.rgap <= tol_g && M.kgap <= tol_g;
    return M;
}

// The stall-floor rule accepts a point that meets floor_tol relative to the
// iterate's and the cost's magnitudes AND the original-LP certificate gate
// in absolute terms (with open 1000 bounds the relative test alone admits
// primal residuals of 1e-4).
__device__ __forceinline__ bool floor_accepts(const Metrics& M, const KernelParams& p) {
    return M.primal <= p.floor_tol * (1.0 + M.xinf) && M.dual <= p.floor_tol * (1.0 + M.cinf) &&
           M.primal <= p.gate_p && M.dual <= p.gate_d && M.kgap <= p.gate_g;
}

// Stage one species' warp schedule (and, when the layout says so, its matrix
// slices with 16-bit indices) into shared memory.
template <typename T>
__device__ __forceinline__ bool layout_is_fast(const Layout& L) {
    return L.mat_smem && (L.smem_mask & 0x1ff) == 0x1ff;
}

// For fast layouts the staged 16-bit indices are ELEMENT offsets from the
// start of dynamic shared memory (the gather target's base already added),
// so a gather is one shared load of S[idx].
// Stage the re-centred kernels' operands (A and A^T with their long lines
// split off): slice and long-line schedules, lists and per-slice long-lane
// masks, and -- when the layout stages the matrix -- the packed words with
// their indices pre-offset to the gather targets (dxbar for A, dy for A^T)
// in units of `unit` bytes from the start of shared memory (4: FP32
// targets, 8: the paired kernel's float2 targets).
__device__ void stage_recentred_ops(const DevSpecies* sp, const Layout& L, unsigned char* sm, int warps, int unit) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const DevLines& a = sp->ra;
    const DevLines& t = sp->rat;
    int32_t* soa = reinterpret_cast<int32_t*>(sm + L.sched_a_off);
    int32_t* sot = reinterpret_cast<int32_t*>(sm + L.sched_at_off);
    int32_t* loa = reinterpret_cast<int32_t*>(sm + L.lsched_a_off);
    int32_t* lot = reinterpret_cast<int32_t*>(sm + L.lsched_at_off);
    for (int w = tid; w <= warps; w += nt) {
        soa[w] = a.sched_off[w];
        sot[w] = t.sched_off[w];
        loa[w] = a.long_sched_off[w];
        lot[w] = t.long_sched_off[w];
    }
    int4* la = reinterpret_cast<int4*>(sm + L.list_a);
    int4* lt = reinterpret_cast<int4*>(sm + L.list_at);
    int4* lla = reinterpret_cast<int4*>(sm + L.llist_a);
    int4* llt = reinterpret_cast<int4*>(sm + L.llist_at);
    uint32_t* ma = reinterpret_cast<uint32_t*>(sm + L.lmask_a);
    uint32_t* mt = reinterpret_cast<uint32_t*>(sm + L.lmask_at);
    for (int q = tid; q < a.nslices; q += nt) {
        la[q] = a.list[q];
        ma[q] = a.lmask[q];
    }
    for (int q = tid; q < t.nslices; q += nt) {
        lt[q] = t.list[q];
        mt[q] = t.lmask[q];
    }
    for (int q = tid; q < a.nlong; q += nt) lla[q] = a.long_list[q];
    for (int q = tid; q < t.nlong; q += nt) llt[q] = t.long_list[q];
    if (!L.mat_smem) return;
    const uint32_t a_add = static_cast<uint32_t>(L.arr[kXbar] / unit), t_add = static_cast<uint32_t>(L.arr[kY] / unit);
    if (L.f32_values) {  // 16-bit indices (pre-offset) and FP32 values
        auto put16 = [&](int64_t off_idx, int64_t off_val, const int32_t* idx, const float* val, int64_t count,
                         uint32_t add) {
            uint16_t* di = reinterpret_cast<uint16_t*>(sm + off_idx);
            float* dv = reinterpret_cast<float*>(sm + off_val);
            for (int64_t e = tid; e < count; e += nt) {
                di[e] = static_cast<uint16_t>(static_cast<uint32_t>(idx[e]) + add);
                dv[e] = val[e];
            }
        };
        put16(L.mat_a_idx, L.mat_a_val, a.idx, a.v32, a.elems, a_add);
        put16(L.mat_at_idx, L.mat_at_val, t.idx, t.v32, t.elems, t_add);
        put16(L.mat_a_long, L.mat_a_lval, a.long_idx, a.long_v32, a.long_elems, a_add);
        put16(L.mat_at_long, L.mat_at_lval, t.long_idx, t.long_v32, t.long_elems, t_add);
        return;
    }
    auto put = [&](uint32_t* dst, const uint32_t* src, int64_t count, uint32_t add) {
        for (int64_t e = tid; e < count; e += nt) {
            const uint32_t w = src[e];
            dst[e] = (w & 0xffff0000u) | ((w & 0xffffu) + add);
        }
    };
    put(reinterpret_cast<uint32_t*>(sm + L.mat_a_idx), a.pk, a.elems, a_add);
    put(reinterpret_cast<uint32_t*>(sm + L.mat_at_idx), t.pk, t.elems, t_add);
    put(reinterpret_cast<uint32_t*>(sm + L.mat_a_long), a.long_pk, a.long_elems, a_add);
    put(reinterpret_cast<uint32_t*>(sm + L.mat_at_long), t.long_pk, t.long_elems, t_add);
}

// Stage one species' warp schedule (and, when the layout says so, its matrix
// slices with 16-bit indices) into shared memory.
template <typename T>
__device__ void stage_species(const DevSpecies* sp, const Layout& L, unsigned char* sm, int warps) {
    if (L.recentred) {
        stage_recentred_ops(sp, L, sm, warps, 4);
        return;
    }
    const int tid = threadIdx.x, nt = blockDim.x;
    int32_t* soa = reinterpret_cast<int32_t*>(sm + L.sched_a_off);
    int32_t* sot = reinterpret_cast<int32_t*>(sm + L.sched_at_off);
    for (int w = tid; w <= warps; w += nt) {
        soa[w] = sp->a_sched_off[w];
        sot[w] = sp->at_sched_off[w];
    }
    int4* la = reinterpret_cast<int4*>(sm + L.list_a);
    int4* lt = reinterpret_cast<int4*>(sm + L.list_at);
    for (int t = tid; t < sp->a_nslices; t += nt) la[t] = sp->a_list[t];
    for (int t = tid; t < sp->at_nslices; t += nt) lt[t] = sp->at_list[t];
    if (L.unscaled) {
        // unscaled FP32 values; indices pre-offset to the FP64 gather targets
        // z (A pass) and w (A^T pass)
        uint16_t* ai = reinterpret_cast<uint16_t*>(sm + L.mat_a_idx);
        uint16_t* ti = reinterpret_cast<uint16_t*>(sm + L.mat_at_idx);
        float* av = reinterpret_cast<float*>(sm + L.mat_a_val);
        float* tv = reinterpret_cast<float*>(sm + L.mat_at_val);
        const int a_add = static_cast<int>(L.arr[kXbar] / 8), t_add = static_cast<int>(L.arr[kW] / 8);
        for (int64_t e = tid; e < sp->a_elems; e += nt) {
            ai[e] = static_cast<uint16_t>(sp->a_idx[e] + a_add);
            av[e] = sp->a_hi[e];
        }
        for (int64_t e = tid; e < sp->at_elems; e += nt) {
            ti[e] = static_cast<uint16_t>(sp->at_idx[e] + t_add);
            tv[e] = sp->at_hi[e];
        }
    } else if (L.mat_smem) {
        uint16_t* ai = reinterpret_cast<uint16_t*>(sm + L.mat_a_idx);
        uint16_t* ti = reinterpret_cast<uint16_t*>(sm + L.mat_at_idx);
        T* av = reinterpret_cast<T*>(sm + L.mat_a_val);
        T* tv = reinterpret_cast<T*>(sm + L.mat_at_val);
        const T* ga = Vals<T>::a(sp);
        const T* gt = Vals<T>::at(sp);
        const bool fast = layout_is_fast<T>(L);
        const int a_add = fast ? static_cast<int>(L.arr[kXbar] / sizeof(T)) : 0;
        const int t_add = fast ? static_cast<int>(L.arr[kY] / sizeof(T)) : 0;
        for (int64_t e = tid; e < sp->a_elems; e += nt) {
            ai[e] = static_cast<uint16_t>(sp->a_idx[e] + a_add);
            av[e] = ga[e];
        }
        for (int64_t e = tid; e < sp->at_elems; e += nt) {
            ti[e] = static_cast<uint16_t>(sp->at_idx[e] + t_add);
            tv[e] = gt[e];
        }
    }
}

// Element offsets (in units of T, or of uint16 for indices) of one species'
// working set when EVERYTHING lives in shared memory; the fast passes index
// the dynamic shared array directly, so the compiler keeps 32-bit shared
// addresses and the per-element instruction count low.
struct FastOffsets {
    int xbar, y, x, xa, ya, c, l, u, b;
    int a_idx, at_idx, a_val, at_val;  // matrix slices
};

template <typename T>
__device__ __forceinline__ FastOffsets fast_offsets(const Layout& L) {
    FastOffsets o;
    const int e = sizeof(T);
    o.xbar = L.arr[kXbar] / e;
    o.y = L.arr[kY] / e;
    o.x = L.arr[kX] / e;
    o.xa = L.arr[kXa] / e;
    o.ya = L.arr[kYa] / e;
    o.c = L.arr[kC] / e;
    o.l = L.arr[kL] / e;
    o.u = L.arr[kU] / e;
    o.b = L.arr[kB] / e;
    o.a_idx = L.mat_a_idx / 2;
    o.at_idx = L.mat_at_idx / 2;
    o.a_val = L.mat_a_val / e;
    o.at_val = L.mat_at_val / e;
    return o;
}

// Slice product from shared memory: four coalesced index/value loads and
// four gathers per step with no bounds guards, then the tail; the
// accumulation order (k ascending, one accumulator) is the generic path's.
template <typename T>
__device__ __forceinline__ T slice_dot_fast(const uint16_t* ip, const T* vp, const T* g, int len) {
    T acc = T(0);
    int k = 0;
    for (; k + 4 <= len; k += 4, ip += 128, vp += 128) {
        const int i0 = ip[0], i1 = ip[32], i2 = ip[64], i3 = ip[96];
        const T v0 = vp[0], v1 = vp[32], v2 = vp[64], v3 = vp[96];
        acc = fma(v0, g[i0], acc);
        acc = fma(v1, g[i1], acc);
        acc = fma(v2, g[i2], acc);
        acc = fma(v3, g[i3], acc);
    }
    for (; k < len; ++k, ip += 32, vp += 32) acc = fma(vp[0], g[ip[0]], acc);
    return acc;
}

// xs / ys (written only on convergence-test iterations) may live in the
// global slab, so they come in as generic pointers.
template <typename T>
__device__ __forceinline__ void primal_pass_fast(const FastOffsets& o, T* xs, const int4* atlist, int t0,
                                                 int t1, int n, int lane, T tau, T w, T w1, T rho,
                                                 bool check, double& pdx2, double& pdxa2) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    T* const S = reinterpret_cast<T*>(dyn_smem);
    const uint16_t* const SI = reinterpret_cast<const uint16_t*>(dyn_smem);
    for (int t = t0; t < t1; ++t) {
        const int4 sl = atlist[t];
        const T g = slice_dot_fast<T>(SI + o.at_idx + sl.y + lane, S + o.at_val + sl.y + lane, S, sl.z);
        const int j = (sl.x << 5) + lane;
        if (j < n) {
            const T xo = S[o.x + j];
            const T xn = clampT(xo - tau * (S[o.c + j] - g), S[o.l + j], S[o.u + j]);
            const T xb = xn + xn - xo;
            S[o.xbar + j] = xb;
            const T xh = (rho == T(1)) ? xb : (T(1) + rho) * xn - rho * xo;
            const T xav = S[o.xa + j];
            S[o.x + j] = w * xh + w1 * xav;
            if (check) {
                xs[j] = xn;
                const double d = static_cast<double>(xn) - static_cast<double>(xo);
                const double da = static_cast<double>(xn) - static_cast<double>(xav);
                pdx2 += d * d;
                pdxa2 += da * da;
            }
        }
    }
}

template <typename T>
__device__ __forceinline__ void dual_pass_fast(const FastOffsets& o, T* ys, const int4* alist, int t0,
                                               int t1, int m, int neq, int lane, T sigma, T w, T w1,
                                               T rho, bool check, double& pdy2, double& pdya2) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    T* const S = reinterpret_cast<T*>(dyn_smem);
    const uint16_t* const SI = reinterpret_cast<const uint16_t*>(dyn_smem);
    for (int t = t0; t < t1; ++t) {
        const int4 sl = alist[t];
        const T h = slice_dot_fast<T>(SI + o.a_idx + sl.y + lane, S + o.a_val + sl.y + lane, S, sl.z);
        const int i = (sl.x << 5) + lane;
        if (i < m) {
            const T yo = S[o.y + i];
            T yn = yo + sigma * (S[o.b + i] - h);
            if (i >= neq && yn > T(0)) yn = T(0);
            const T yh = (rho == T(1)) ? yn + yn - yo : (T(1) + rho) * yn - rho * yo;
            const T yav = S[o.ya + i];
            S[o.y + i] = w * yh + w1 * yav;
            if (check) {
                ys[i] = yn;
                const double d = static_cast<double>(yn) - static_cast<double>(yo);
                const double da = static_cast<double>(yn) - static_cast<double>(yav);
                pdy2 += d * d;
                pdya2 += da * da;
            }
        }
    }
}

// ---- unscaled FP64 passes (matrix staged as FP32 + FP64 remainders) ----
// The A^T pass computes (A~^T y)_j = dc_j * sum_i A_ij w_i with w = dr * y,
// the A pass (A~ xbar)_i = dr_i * sum_j A_ij z_j with z = dc * xbar; the
// staged A_ij are the FP32 parts and the per-row remainder lists restore
// the FP64 products.  Owned data (c, l, u, y, ...) may live in the global
// slab; it is loaded before the slice's dot product so that its latency
// overlaps the shared-memory work.
__device__ __forceinline__ double slice_dot_hi(const uint16_t* ip, const float* vp, const double* S, int len) {
    double acc = 0.0;
    int k = 0;
    for (; k + 4 <= len; k += 4, ip += 128, vp += 128) {
        const int i0 = ip[0], i1 = ip[32], i2 = ip[64], i3 = ip[96];
        const float v0 = vp[0], v1 = vp[32], v2 = vp[64], v3 = vp[96];
        acc = fma(static_cast<double>(v0), S[i0], acc);
        acc = fma(static_cast<double>(v1), S[i1], acc);
        acc = fma(static_cast<double>(v2), S[i2], acc);
        acc = fma(static_cast<double>(v3), S[i3], acc);
    }
    for (; k < len; ++k, ip += 32, vp += 32) acc = fma(static_cast<double>(vp[0]), S[ip[0]], acc);
    return acc;
}

__device__ __forceinline__ void primal_pass_unscaled(const DevSpecies* sp, const Layout& L, Arrays<double>& A,
                                                     const int4* atlist, int t0, int t1, int n, int lane,
                                                     double tau, double w, double w1, double rho, bool check,
                                                     double& pdx2, double& pdxa2) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const double* const S = reinterpret_cast<const double*>(dyn_smem);
    const uint16_t* const TI = reinterpret_cast<const uint16_t*>(dyn_smem + L.mat_at_idx);
    const float* const TV = reinterpret_cast<const float*>(dyn_smem + L.mat_at_val);
    for (int t = t0; t < t1; ++t) {
        const int4 sl = atlist[t];
        const int j = (sl.x << 5) + lane;
        const bool own = j < n;
        double cj = 0, lj = 0, uj = 0, xo = 0, xav = 0, dcj = 0;
        int lb = 0, le = 0;
        if (own) {
            cj = A.cs[j];
            lj = A.ls[j];
            uj = A.us[j];
            xo = A.x[j];
            xav = A.xa[j];
            dcj = sp->dc[j];
            lb = sp->lo_at_ptr[j];
            le = sp->lo_at_ptr[j + 1];
        }
        double acc = slice_dot_hi(TI + sl.y + lane, TV + sl.y + lane, S, sl.z);
        if (own) {
            for (int k = lb; k < le; ++k) acc = fma(sp->lo_at_val[k], A.w[sp->lo_at_idx[k]], acc);
            const double g = dcj * acc;
            const double xn = clampT(xo - tau * (cj - g), lj, uj);
            const double xb = xn + xn - xo;
            A.xbar[j] = dcj * xb;  // z
            const double xh = (rho == 1.0) ? xb : (1.0 + rho) * xn - rho * xo;
            A.x[j] = w * xh + w1 * xav;
            if (check) {
                A.xs[j] = xn;
                const double d = xn - xo, da = xn - xav;
                pdx2 += d * d;
                pdxa2 += da * da;
            }
        }
    }
}

__device__ __forceinline__ void dual_pass_unscaled(const DevSpecies* sp, const Layout& L, Arrays<double>& A,
                                                   const int4* alist, int t0, int t1, int m, int neq, int lane,
                                                   double sigma, double w, double w1, double rho, bool check,
                                                   double& pdy2, double& pdya2) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const double* const S = reinterpret_cast<const double*>(dyn_smem);
    const uint16_t* const AI = reinterpret_cast<const uint16_t*>(dyn_smem + L.mat_a_idx);
    const float* const AV = reinterpret_cast<const float*>(dyn_smem + L.mat_a_val);
    for (int t = t0; t < t1; ++t) {
        const int4 sl = alist[t];
        const int i = (sl.x << 5) + lane;
        const bool own = i < m;
        double yo = 0, yav = 0, bi = 0, dri = 0;
        int lb = 0, le = 0;
        if (own) {
            yo = A.y[i];
            yav = A.ya[i];
            bi = A.bs[i];
            dri = sp->dr[i];
            lb = sp->lo_a_ptr[i];
            le = sp->lo_a_ptr[i + 1];
        }
        double acc = slice_dot_hi(AI + sl.y + lane, AV + sl.y + lane, S, sl.z);
        if (own) {
            for (int k = lb; k < le; ++k) acc = fma(sp->lo_a_val[k], A.xbar[sp->lo_a_idx[k]], acc);
            const double h = dri * acc;
            double yn = yo + sigma * (bi - h);
            if (i >= neq && yn > 0.0) yn = 0.0;
            const double yh = (rho == 1.0) ? yn + yn - yo : (1.0 + rho) * yn - rho * yo;
            const double ynew = w * yh + w1 * yav;
            A.y[i] = ynew;
            A.w[i] = dri * ynew;
            if (check) {
                A.ys[i] = yn;
                const double d = yn - yo, da = yn - yav;
                pdy2 += d * d;
                pdya2 += da * da;
            }
        }
    }
}

// FAST = every species of the launch has a fast layout (matrix and all
// per-iteration arrays in shared memory); that variant carries no code for
// the generic path, which keeps its register budget small.
// MODE 0: generic; 1 (FAST): matrix and every per-iteration array in shared
// memory, scaled values; 2 (UNSCALED, FP64 only): unscaled FP32 matrix with
// FP64 remainders staged, FP64 gather targets in shared memory.
template <typename T, int MAXT, int MODE>
__global__ void __launch_bounds__(MAXT, 1) pdhg_persistent(const __grid_constant__ KernelParams p) {
    constexpr bool FAST = MODE == 1;
    constexpr bool UNS = MODE == 2;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ double s_red[MAXT / 32][kRed];
    __shared__ double s_tot[kRed];
    __shared__ int s_inst;
    __shared__ int s_loaded;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nthreads = blockDim.x;
    const int warps = nthreads >> 5;
    unsigned char* slab = p.spill ? p.spill + static_cast<int64_t>(blockIdx.x) * p.spill_stride : nullptr;
    const T rho = static_cast<T>(p.rho);
    const int count = p.count_dev ? *p.count_dev : p.count;
    if (tid == 0) s_loaded = -1;

    for (;;) {
        if (tid == 0) s_inst = atomicAdd(p.queue, 1);
        __syncthreads();
        const int q = s_inst;
        if (q >= count) break;
        const int inst = p.order[q];
        const int species = p.inst_species[inst];
        const DevSpecies* __restrict__ sp = p.species + species;
        const Layout& L = p.layouts[species];
        const int n = sp->n, m = sp->m, neq = sp->neq;
        const int64_t coff = p.col_off[inst], roff = p.row_off[inst];
        if (s_loaded != species) {  // block-uniform
            stage_species<T>(sp, L, dyn_smem, warps);
            __syncthreads();
            if (tid == 0) s_loaded = species;
        }
        Arrays<T> A;
        {
            T** ptrs[kArrayCount] = {&A.xbar, &A.y, &A.x, &A.xa, &A.ya, &A.cs, &A.ls, &A.us, &A.bs, &A.xs, &A.ys, &A.w};
            const int mask = L.smem_mask;
#pragma unroll
            for (int a = 0; a < kArrayCount; ++a)
                *ptrs[a] = reinterpret_cast<T*>(((mask >> a) & 1) ? dyn_smem + L.arr[a] : slab + L.arr[a]);
        }
        const int4* alist = reinterpret_cast<const int4*>(dyn_smem + L.list_a);
        const int4* atlist = reinterpret_cast<const int4*>(dyn_smem + L.list_at);
        const int32_t* soa = reinterpret_cast<const int32_t*>(dyn_smem + L.sched_a_off);
        const int32_t* sot = reinterpret_cast<const int32_t*>(dyn_smem + L.sched_at_off);
        const int aw0 = soa[warp], aw1 = soa[warp + 1];
        const int tw0 = sot[warp], tw1 = sot[warp + 1];
        const bool mat_smem = L.mat_smem != 0;
        const uint16_t* s_aidx = reinterpret_cast<const uint16_t*>(dyn_smem + L.mat_a_idx);
        const uint16_t* s_tidx = reinterpret_cast<const uint16_t*>(dyn_smem + L.mat_at_idx);
        const T* s_aval = reinterpret_cast<const T*>(dyn_smem + L.mat_a_val);
        const T* s_tval = reinterpret_cast<const T*>(dyn_smem + L.mat_at_val);
        const T* __restrict__ g_aval = Vals<T>::a(sp);
        const T* __restrict__ g_tval = Vals<T>::at(sp);
        // fast path: matrix and every per-iteration array in shared memory
        const bool fast = FAST || (!UNS && layout_is_fast<T>(L));
        const FastOffsets fo = fast_offsets<T>(L);

        // ---- load the instance (scaled, in the species' permuted order) ----
        int bad = 0;
        for (int j = tid; j < n; j += nthreads) {
            const int jo = sp->col_perm[j];
            const double dcj = sp->dc[j];
            const double lv = p.lower[coff + jo], uv = p.upper[coff + jo], cv = p.cost[coff + jo];
            if (isnan(lv) || isnan(uv) || lv > uv || !isfinite(cv) || lv == INFINITY || uv == -INFINITY)
                bad = 1;
            const T l = static_cast<T>(lv / dcj), u = static_cast<T>(uv / dcj);
            A.ls[j] = l;
            A.us[j] = u;
            A.cs[j] = static_cast<T>(cv * dcj);
            double x0 = p.warm_x ? p.warm_x[coff + jo] / dcj : 0.0;
            if (!isfinite(x0)) x0 = 0.0;
            const T xv = clampT(static_cast<T>(x0), l, u);
            A.x[j] = xv;
            A.xa[j] = xv;
            A.xs[j] = xv;
        }
        for (int i = tid; i < m; i += nthreads) {
            const int io = sp->row_perm[i];
            const double dri = sp->dr[i];
            const double bv = p.rhs ? p.rhs[roff + io] : 0.0;
            if (!isfinite(bv)) bad = 1;
            A.bs[i] = static_cast<T>(bv * dri);
            double y0 = p.warm_y ? p.warm_y[roff + io] / dri : 0.0;
            if (!isfinite(y0)) y0 = 0.0;
            if (i >= neq && y0 > 0.0) y0 = 0.0;
            A.y[i] = static_cast<T>(y0);
            A.ya[i] = static_cast<T>(y0);
            A.ys[i] = static_cast<T>(y0);
            if (UNS) A.w[i] = static_cast<T>(dri * static_cast<T>(y0));
        }
        if (tid == 0) {
            A.xbar[n] = T(0);
            A.xs[n] = T(0);
            A.y[m] = T(0);
            A.ys[m] = T(0);
            if (UNS) A.w[m] = T(0);
        }
        bad = __syncthreads_or(bad);
        double omega = 1.0;
        if (p.warm_omega) {
            const double w0 = p.warm_omega[inst];
            if (isfinite(w0) && w0 > 0.0) omega = w0;
        }
        const int prior = p.prior_iters ? p.prior_iters[inst] : 0;
        if (bad) {
            for (int j = tid; j < n; j += nthreads) p.out_x[coff + sp->col_perm[j]] = NAN;
            for (int i = tid; i < m; i += nthreads) p.out_y[roff + sp->row_perm[i]] = NAN;
            if (tid == 0) {
                p.out_status[inst] = kStatusInvalid;
                p.out_iters[inst] = prior;
                p.out_obj[inst] = NAN;
                for (int k = 0; k < kMetrics; ++k) p.out_metrics[static_cast<int64_t>(inst) * kMetrics + k] = NAN;
                if (p.out_omega) p.out_omega[inst] = omega;
            }
            continue;
        }

        const double eta = sp->eta;
        const double* lo_i = p.lower + coff;
        const double* up_i = p.upper + coff;
        const double* c_i = p.cost + coff;
        const double* b_i = p.rhs ? p.rhs + roff : nullptr;
        int status = -1;
        Metrics M;
        // ---- iteration-0 test of the (projected) starting point ----
        {
            double v[kRed];
#pragma unroll
            for (int qq = 0; qq < kRed; ++qq) v[qq] = 0.0;
            kkt_partials<T>(sp, alist, atlist, aw0, aw1, tw0, tw1, A.xs, A.ys, lo_i, up_i, c_i, b_i,
                            lane, v);
            block_reduce(v, s_red, s_tot);
            M = evaluate(s_tot, omega, p.tol_p, p.tol_d, p.tol_g);
            if (M.conv) status = p.final_status;
            else if (p.max_iters <= 0) status = M.nan ? kStatusNumerical : kStatusIterationLimit;
            // FP32 phase: a warm start already at FP32-floor accuracy gains
            // nothing from FP32 iterations (their rounding would only lose
            // digits), so it is handed to the FP64 phase unchanged.
            if (status < 0 && p.passthrough_tol > 0.0 && p.warm_x && !M.nan &&
                fmax(fmax(M.primal / (1.0 + M.xinf), M.dual / (1.0 + M.cinf)), fmax(M.rgap, M.kgap)) <=
                    p.passthrough_tol)
                status = p.final_status;
        }

        int k = 0, it = 0, stall = 0;
        bool fell_back = false;
        double r_restart = INFINITY, r_prev = INFINITY, best_err = INFINITY;
        while (status < 0) {
            ++it;
            // full tests (restart rule, stall rule) every check_every iterations;
            // cheap termination-only tests at 8, 16, 32, ... below that
            const bool full = (it % p.check_every == 0) || (it >= p.max_iters);
            const bool check = full || (it >= 8 && it < p.check_every && (it & (it - 1)) == 0);
            const T tau = static_cast<T>(eta / omega), sigma = static_cast<T>(eta * omega);
            const T w = static_cast<T>((k + 1.0) / (k + 2.0));
            const T w1 = T(1) - w;
            double pdx2 = 0.0, pdy2 = 0.0, pdxa2 = 0.0, pdya2 = 0.0;
            // primal pass: g = A^T y, projected step, extrapolation, Halpern
            if constexpr (UNS) {
                primal_pass_unscaled(sp, L, A, atlist, tw0, tw1, n, lane, tau, w, w1, rho, check, pdx2, pdxa2);
            } else if (FAST || fast) {
                primal_pass_fast<T>(fo, A.xs, atlist, tw0, tw1, n, lane, tau, w, w1, rho, check, pdx2, pdxa2);
            } else if (!FAST) {
                for (int t = tw0; t < tw1; ++t) {
                    const int4 sl = atlist[t];
                    const T g = mat_smem ? slice_dot<T, T, uint16_t, false>(s_tidx, s_tval, sl.y, sl.z, lane, A.y)
                                         : slice_dot<T, T, int32_t, true>(sp->at_idx, g_tval, sl.y, sl.z, lane, A.y);
                    const int j = (sl.x << 5) + lane;
                    if (j < n) {
                        const T xo = A.x[j];
                        const T xn = clampT(xo - tau * (A.cs[j] - g), A.ls[j], A.us[j]);
                        const T xb = xn + xn - xo;
                        A.xbar[j] = xb;
                        const T xh = (rho == T(1)) ? xb : (T(1) + rho) * xn - rho * xo;
                        const T xav = A.xa[j];
                        A.x[j] = w * xh + w1 * xav;
                        if (check) {
                            A.xs[j] = xn;
                            const double d = static_cast<double>(xn) - static_cast<double>(xo);
                            const double da = static_cast<double>(xn) - static_cast<double>(xav);
                            pdx2 += d * d;
                            pdxa2 += da * da;
                        }
                    }
                }
            }
            __syncthreads();
            // dual pass: h = A xbar, projected dual step, Halpern
            if constexpr (UNS) {
                dual_pass_unscaled(sp, L, A, alist, aw0, aw1, m, neq, lane, sigma, w, w1, rho, check, pdy2, pdya2);
            } else if (FAST || fast) {
                dual_pass_fast<T>(fo, A.ys, alist, aw0, aw1, m, neq, lane, sigma, w, w1, rho, check, pdy2, pdya2);
            } else if (!FAST) {
                for (int t = aw0; t < aw1; ++t) {
                    const int4 sl = alist[t];
                    const T h = mat_smem ? slice_dot<T, T, uint16_t, false>(s_aidx, s_aval, sl.y, sl.z, lane, A.xbar)
                                         : slice_dot<T, T, int32_t, true>(sp->a_idx, g_aval, sl.y, sl.z, lane, A.xbar);
                    const int i = (sl.x << 5) + lane;
                    if (i < m) {
                        const T yo = A.y[i];
                        T yn = yo + sigma * (A.bs[i] - h);
                        if (i >= neq && yn > T(0)) yn = T(0);
                        const T yh = (rho == T(1)) ? yn + yn - yo : (T(1) + rho) * yn - rho * yo;
                        const T yav = A.ya[i];
                        A.y[i] = w * yh + w1 * yav;
                        if (check) {
                            A.ys[i] = yn;
                            const double d = static_cast<double>(yn) - static_cast<double>(yo);
                            const double da = static_cast<double>(yn) - static_cast<double>(yav);
                            pdy2 += d * d;
                            pdya2 += da * da;
                        }
                    }
                }
            }
            __syncthreads();
            ++k;
            if (!check) continue;

            double v[kRed];
#pragma unroll
            for (int qq = 0; qq < kRed; ++qq) v[qq] = 0.0;
            v[5] = pdx2;
            v[6] = pdy2;
            v[7] = pdxa2;
            v[8] = pdya2;
            kkt_partials<T>(sp, alist, atlist, aw0, aw1, tw0, tw1, A.xs, A.ys, lo_i, up_i, c_i, b_i,
                            lane, v);
            block_reduce(v, s_red, s_tot);
            M = evaluate(s_tot, omega, p.tol_p, p.tol_d, p.tol_g);
            if (M.nan || !isfinite(M.r)) {
                status = kStatusNumerical;
                break;
            }
            if (M.conv) {
                status = p.final_status;
                break;
            }
            if (it >= p.max_iters) {
                status = kStatusIterationLimit;
                break;
            }
            if (!full) continue;
            // precision floor: once the KKT error has stopped halving for
            // `stall_checks` consecutive tests, the FP32 phase hands off, and
            // the FP64 phase accepts the point if it meets the floor
            // tolerance (otherwise it keeps iterating to its budget).
            {
                const double e = fmax(fmax(M.primal / (1.0 + M.xinf), M.dual / (1.0 + M.cinf)),
                                      fmax(M.rgap, M.kgap));
                if (e < 0.5 * best_err) {
                    best_err = e;
                    stall = 0;
                } else {
                    ++stall;
                }
                if (p.stall_checks > 0 && stall >= p.stall_checks) {
                    if (p.final_status == kStatusHandoff && best_err <= kStallFloor) {
                        status = p.final_status;
                        break;
                    }
                    if (p.final_status == kStatusOptimal && e <= p.floor_tol && floor_accepts(M, p)) {
                        status = p.final_status;
                        break;
                    }
                }
            }
            // cold fallback: a warm-started instance that has not converged
            // after `fallback_iters` iterations restarts once from the cold
            // point (x = projection of 0, y = 0, omega = 1)
            if (p.fallback_iters > 0 && !fell_back && it >= p.fallback_iters &&
                (p.warm_x != nullptr || p.warm_y != nullptr)) {
                fell_back = true;
                omega = 1.0;
                for (int j = tid; j < n; j += nthreads) {
                    const T xv = clampT(T(0), A.ls[j], A.us[j]);
                    A.x[j] = xv;
                    A.xa[j] = xv;
                }
                for (int i = tid; i < m; i += nthreads) {
                    A.y[i] = T(0);
                    A.ya[i] = T(0);
                    if (UNS) A.w[i] = T(0);
                }
                k = 0;
                r_restart = INFINITY;
                r_prev = INFINITY;
                best_err = INFINITY;
                stall = 0;
                __syncthreads();
                continue;
            }
            if (p.restarts && (M.r <= kBetaSufficient * r_restart ||
                               (M.r <= kBetaNecessary * r_restart && M.r > r_prev) ||
                               k >= kBetaArtificial * it)) {
                const double nx = sqrt(s_tot[7]), ny = sqrt(s_tot[8]);
                if (nx > 1e-10 && ny > 1e-10)
                    omega = exp(__fma_rn(p.omega_smoothing, log(ny / nx), (1.0 - p.omega_smoothing) * log(omega)));
                for (int j = tid; j < n; j += nthreads) {
                    const T xv = A.xs[j];
                    A.x[j] = xv;
                    A.xa[j] = xv;
                }
                for (int i = tid; i < m; i += nthreads) {
                    const T yv = A.ys[i];
                    A.y[i] = yv;
                    A.ya[i] = yv;
                    if (UNS) A.w[i] = static_cast<T>(sp->dr[i] * yv);
                }
                k = 0;
                r_restart = M.r;
                r_prev = INFINITY;
                __syncthreads();
            } else {
                r_prev = M.r;
            }
        }

        // ---- results in original units and original order ----
        // (an FP32 phase that stopped at its iteration-0 test passes the FP64
        // warm start through untouched)
        const bool pass = p.passthrough_tol > 0.0 && it == 0 && p.warm_x != nullptr;
        for (int j = tid; j < n; j += nthreads) {
            const int jo = sp->col_perm[j];
            double xv = pass ? p.warm_x[coff + jo] : static_cast<double>(A.xs[j]) * sp->dc[j];
            if (p.clip_output) {
                const double lv = p.lower[coff + jo], uv = p.upper[coff + jo];
                xv = xv < lv ? lv : (xv > uv ? uv : xv);
            }
            p.out_x[coff + jo] = xv;
        }
        for (int i = tid; i < m; i += nthreads) {
            const int io = sp->row_perm[i];
            p.out_y[roff + io] = (pass && p.warm_y) ? p.warm_y[roff + io] : static_cast<double>(A.ys[i]) * sp->dr[i];
        }
        if (tid == 0) {
            double* mo = p.out_metrics + static_cast<int64_t>(inst) * kMetrics;
            mo[0] = M.primal;
            mo[1] = M.dual;
            mo[2] = M.kgap;
            mo[3] = M.pobj;
            mo[4] = M.dobj;
            mo[5] = M.rgap;
            mo[6] = M.xinf;
            mo[7] = omega;
            p.out_obj[inst] = M.pobj;
            p.out_status[inst] = status;
            p.out_iters[inst] = prior + it;
            if (p.out_omega) p.out_omega[inst] = omega;
        }
    }
}

// ---------------------------------------------------------------------------
// Re-centred FP32 PDHG (the default first phase of the mixed schedule).
//
// The iterates are kept as FP32 differences from an FP64 base point
// (x^, y^) held in the CTA's global slab:  x = x^ + dx,  y = y^ + dy.  The
// base moves to the current candidate at every restart (where the Halpern
// anchor is reset to that candidate anyway), so the anchor is always the
// base and dx, dy restart from zero.  Per base the FP32 problem is the
// correction LP
//     min d.dx  s.t.  A dx = r,  l - x^ <= dx <= u - x^   (y^ + dy <= 0 on
//     inequality rows)
// with d = c - A^T y^ and r = b - A x^ evaluated in FP64 and rounded once.
// In exact arithmetic the sequence equals plain PDHG from the same start;
// in FP32 the rounding error scales with |dx|, |dy|, d and r, which shrink
// as the solve converges, so FP32 iterations reach the FP64 tolerances
// (plain FP32 iterates floor near a 1e-4 relative gap).  Every convergence
// test evaluates the FP64 candidate x^ + dx_n, y^ + dy_n with the FP64
// matrix, exactly like the FP64 phase.
// Shared memory holds dxbar, dy (gather targets), the FP32 matrix slices,
// dx, d, l - x^, u - x^, r and the inequality-row bound -y^ (in the slots of
// xbar, y, x, c, l, u, b, ya).  The slab also keeps the instance's scaled
// FP64 objective and bounds (new column order) and right-hand side, so the
// convergence test reads them without permutation or division.
// ---------------------------------------------------------------------------

// Slice product over packed matrix words (16-bit index | BF16 value): one
// 32-bit shared-memory load per element, two accumulators (even / odd k).
// The BF16 value is the word with its index bits cleared.
__device__ __forceinline__ float slice_dot_pk(const uint32_t* wp, const float* g, int len) {
    float a0 = 0.0f, a1 = 0.0f;
    int k = 0;
    for (; k + 4 <= len; k += 4, wp += 128) {
        const uint32_t w0 = wp[0], w1 = wp[32], w2 = wp[64], w3 = wp[96];
        a0 = fmaf(__uint_as_float(w0 & 0xffff0000u), g[w0 & 0xffffu], a0);
        a1 = fmaf(__uint_as_float(w1 & 0xffff0000u), g[w1 & 0xffffu], a1);
        a0 = fmaf(__uint_as_float(w2 & 0xffff0000u), g[w2 & 0xffffu], a0);
        a1 = fmaf(__uint_as_float(w3 & 0xffff0000u), g[w3 & 0xffffu], a1);
    }
    if (k + 2 <= len) {
        const uint32_t w0 = wp[0], w1 = wp[32];
        a0 = fmaf(__uint_as_float(w0 & 0xffff0000u), g[w0 & 0xffffu], a0);
        a1 = fmaf(__uint_as_float(w1 & 0xffff0000u), g[w1 & 0xffffu], a1);
        k += 2;
        wp += 64;
    }
    if (k < len) {
        const uint32_t w0 = wp[0];
        a0 = fmaf(__uint_as_float(w0 & 0xffff0000u), g[w0 & 0xffffu], a0);
    }
    return a0 + a1;
}

// The same product with the packed words streamed from global memory (raw
// indices relative to the gather target `g`); identical accumulation order.
__device__ __forceinline__ float slice_dot_pk_global(const uint32_t* __restrict__ wp, const float* g, int len) {
    constexpr int U = 8;
    float a0 = 0.0f, a1 = 0.0f;
    for (int k0 = 0; k0 < len; k0 += U) {
        uint32_t ww[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k0 + u < len) ww[u] = __ldg(wp + ((k0 + u) << 5));
#pragma unroll
        for (int u = 0; u < U; u += 2) {
            if (k0 + u < len) a0 = fmaf(__uint_as_float(ww[u] & 0xffff0000u), g[ww[u] & 0xffffu], a0);
            if (k0 + u + 1 < len) a1 = fmaf(__uint_as_float(ww[u + 1] & 0xffff0000u), g[ww[u + 1] & 0xffffu], a1);
        }
    }
    return a0 + a1;
}

// Per-instance patched entries held by the CTA for the current instance.
struct Patches {
    int n;
    const int* row;
    const int* col;
    const float* v32;
    const double* v64;
};

// One operand of the re-centred kernels as the calling warp sees it: its
// slices and long lines, the per-slice long-lane masks and, when the matrix
// is staged, the packed words in shared memory (indices pre-offset to the
// gather target); otherwise the words are streamed from global memory.
struct OpsView {
    uint32_t list, llist, lmask;  // byte offsets into dynamic shared memory
    uint32_t words, lwords;       // staged slice / long-line words, or 16-bit indices with FP32 values
    uint32_t vals, lvals;         // staged FP32 values (FP32-valued layouts)
    int t0, t1;                   // this warp's slices
    int l0, l1;                   // this warp's long lines
};

// Shared-memory pointers from byte offsets (the extern array keeps the
// accesses in the shared window).
__device__ __forceinline__ const int4* sm_int4(uint32_t off) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    return reinterpret_cast<const int4*>(dyn_smem + off);
}
__device__ __forceinline__ const uint32_t* sm_u32(uint32_t off) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    return reinterpret_cast<const uint32_t*>(dyn_smem + off);
}

// The calling warp's views of A (the dual pass) and A^T (the primal pass)
// from a re-centred layout staged in shared memory.
__device__ __forceinline__ void ops_views(const Layout& L, const unsigned char* sm, int warp, OpsView* A, OpsView* T) {
    const int32_t* soa = reinterpret_cast<const int32_t*>(sm + L.sched_a_off);
    const int32_t* sot = reinterpret_cast<const int32_t*>(sm + L.sched_at_off);
    const int32_t* loa = reinterpret_cast<const int32_t*>(sm + L.lsched_a_off);
    const int32_t* lot = reinterpret_cast<const int32_t*>(sm + L.lsched_at_off);
    A->list = static_cast<uint32_t>(L.list_a);
    T->list = static_cast<uint32_t>(L.list_at);
    A->llist = static_cast<uint32_t>(L.llist_a);
    T->llist = static_cast<uint32_t>(L.llist_at);
    A->lmask = static_cast<uint32_t>(L.lmask_a);
    T->lmask = static_cast<uint32_t>(L.lmask_at);
    A->t0 = soa[warp];
    A->t1 = soa[warp + 1];
    T->t0 = sot[warp];
    T->t1 = sot[warp + 1];
    A->l0 = loa[warp];
    A->l1 = loa[warp + 1];
    T->l0 = lot[warp];
    T->l1 = lot[warp + 1];
    A->words = static_cast<uint32_t>(L.mat_a_idx);
    T->words = static_cast<uint32_t>(L.mat_at_idx);
    A->lwords = static_cast<uint32_t>(L.mat_a_long);
    T->lwords = static_cast<uint32_t>(L.mat_at_long);
    A->vals = static_cast<uint32_t>(L.mat_a_val);
    T->vals = static_cast<uint32_t>(L.mat_at_val);
    A->lvals = static_cast<uint32_t>(L.mat_a_lval);
    T->lvals = static_cast<uint32_t>(L.mat_at_lval);
}

__device__ __forceinline__ const uint16_t* sm_u16(uint32_t off) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    return reinterpret_cast<const uint16_t*>(dyn_smem + off);
}
__device__ __forceinline__ const float* sm_f32(uint32_t off) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    return reinterpret_cast<const float*>(dyn_smem + off);
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Product of one long line's packed words with the gather target g, the
// whole warp together: lane l takes entries l, l + 32, ... in order, then a
// fixed xor-shuffle tree; every lane returns the sum.  GLOBAL: words from
// global memory (raw indices relative to g).
template <bool GLOBAL>
__device__ __forceinline__ float long_dot_pk(const uint32_t* wp, const float* g, int len, int lane) {
    float acc = 0.0f;
    for (int k = lane; k < len; k += 32) {
        const uint32_t w = GLOBAL ? __ldg(wp + k) : wp[k];
        acc = fmaf(__uint_as_float(w & 0xffff0000u), g[w & 0xffffu], acc);
    }
    return warp_sum_f(acc);
}

// Slice product over separate 16-bit indices (pre-offset to the gather
// target) and FP32 values in shared memory -- the FP32-valued layout of
// solves the BF16-rounded matrix stalls -- in the order of slice_dot_pk.
__device__ __forceinline__ float slice_dot_sv(const uint16_t* ip, const float* vp, const float* g, int len) {
    float a0 = 0.0f, a1 = 0.0f;
    int k = 0;
    for (; k + 4 <= len; k += 4, ip += 128, vp += 128) {
        const int i0 = ip[0], i1 = ip[32], i2 = ip[64], i3 = ip[96];
        const float v0 = vp[0], v1 = vp[32], v2 = vp[64], v3 = vp[96];
        a0 = fmaf(v0, g[i0], a0);
        a1 = fmaf(v1, g[i1], a1);
        a0 = fmaf(v2, g[i2], a0);
        a1 = fmaf(v3, g[i3], a1);
    }
    if (k + 2 <= len) {
        a0 = fmaf(vp[0], g[ip[0]], a0);
        a1 = fmaf(vp[32], g[ip[32]], a1);
        k += 2;
        ip += 64;
        vp += 64;
    }
    if (k < len) a0 = fmaf(vp[0], g[ip[0]], a0);
    return a0 + a1;
}

// The same with the raw int32 indices and FP32 values streamed from global
// memory (indices relative to `g`); identical accumulation order.
__device__ __forceinline__ float slice_dot_sv_global(const int32_t* __restrict__ ip, const float* __restrict__ vp,
                                                     const float* g, int len) {
    constexpr int U = 8;
    float a0 = 0.0f, a1 = 0.0f;
    for (int k0 = 0; k0 < len; k0 += U) {
        int ii[U];
        float vv[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k0 + u < len) {
                ii[u] = __ldg(ip + ((k0 + u) << 5));
                vv[u] = __ldg(vp + ((k0 + u) << 5));
            }
#pragma unroll
        for (int u = 0; u < U; u += 2) {
            if (k0 + u < len) a0 = fmaf(vv[u], g[ii[u]], a0);
            if (k0 + u + 1 < len) a1 = fmaf(vv[u + 1], g[ii[u + 1]], a1);
        }
    }
    return a0 + a1;
}

// A long line with separate indices and FP32 values (staged 16-bit or
// streamed int32), the warp together in long_dot_pk's order.
template <bool GLOBAL>
__device__ __forceinline__ float long_dot_sv(const uint16_t* ip16, const int32_t* ip32, const float* vp, const float* g,
                                             int len, int lane) {
    float acc = 0.0f;
    for (int k = lane; k < len; k += 32) {
        const int i = GLOBAL ? __ldg(ip32 + k) : static_cast<int>(ip16[k]);
        const float v = GLOBAL ? __ldg(vp + k) : vp[k];
        acc = fmaf(v, g[i], acc);
    }
    return warp_sum_f(acc);
}

// The FP64 product of one long line for the convergence test (the same
// order): indices from the staged words (minus the gather-target offset
// `sub`) or from global memory, FP64 values from global memory.
template <bool STAGED, bool F32V = false>
__device__ __forceinline__ double long_dot64(const void* wp, int sub, const int32_t* __restrict__ ip,
                                             const double* __restrict__ vp, const double* g, int len, int lane) {
    double acc = 0.0;
    for (int k = lane; k < len; k += 32) {
        const int i = !STAGED ? __ldg(ip + k)
                              : (F32V ? static_cast<int>(static_cast<const uint16_t*>(wp)[k])
                                      : static_cast<int>(static_cast<const uint32_t*>(wp)[k] & 0xffffu)) - sub;
        acc = fma(__ldg(vp + k), g[i], acc);
    }
    return warp_sum_d(acc);
}

// The primal update of column j (shared by the slice lanes and the long
// columns' lane 0).
__device__ __forceinline__ void primal_update(const FastOffsets& o, int j, float xo, float dj, float lj, float uj,
                                              float g, float tau, float w, float rho, bool check, const double* bx,
                                              double* cx, double& pdx2, double& pdxa2) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float* const S = reinterpret_cast<float*>(dyn_smem);
    // explicit roundings (no contraction choice left to the compiler): the
    // paired kernel repeats them bit for bit
    const float xn = clampT(__fmaf_rn(-tau, __fsub_rn(dj, g), xo), lj, uj);
    const float xb = __fsub_rn(__fadd_rn(xn, xn), xo);
    S[o.xbar + j] = xb;
    const float xh = (rho == 1.0f) ? xb : (1.0f + rho) * xn - rho * xo;
    S[o.x + j] = __fmul_rn(w, xh);  // the anchor is the base: dx_anchor = 0
    if (check) {
        cx[j] = bx[j] + static_cast<double>(xn);
        const double d = static_cast<double>(xn) - static_cast<double>(xo);
        pdx2 = __fma_rn(d, d, pdx2);
        pdxa2 = __fma_rn(static_cast<double>(xn), static_cast<double>(xn), pdxa2);
    }
}

__device__ __forceinline__ void dual_update(const FastOffsets& o, int i, int neq, float yo, float ri, float yl,
                                            float h, float sigma, float w, float rho, bool check, const double* by,
                                            double* cy, double& pdy2, double& pdya2) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float* const S = reinterpret_cast<float*>(dyn_smem);
    float yn = __fmaf_rn(sigma, __fsub_rn(ri, h), yo);
    if (i >= neq && yn > yl) yn = yl;  // y^ + dy <= 0
    const float yh = (rho == 1.0f) ? __fsub_rn(__fadd_rn(yn, yn), yo) : (1.0f + rho) * yn - rho * yo;
    S[o.y + i] = __fmul_rn(w, yh);
    if (check) {
        cy[i] = by[i] + static_cast<double>(yn);
        const double d = static_cast<double>(yn) - static_cast<double>(yo);
        pdy2 = __fma_rn(d, d, pdy2);
        pdya2 = __fma_rn(static_cast<double>(yn), static_cast<double>(yn), pdya2);
    }
}

// STAGED: the species' packed matrix words are in shared memory (indices
// pre-offset to the gather target); otherwise they are streamed from L2.
template <bool STAGED, bool PATCHED, bool F32V>
__device__ __forceinline__ void primal_pass_recentred(const DevSpecies* sp, const FastOffsets& o, const OpsView& T,
                                                      int n, int lane, float tau, float w, float rho, bool check,
                                                      const double* bx, double* cx, double& pdx2, double& pdxa2,
                                                      const Patches& pt) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float* const S = reinterpret_cast<float*>(dyn_smem);
    for (int t = T.t0; t < T.t1; ++t) {
        const int4 sl = sm_int4(T.list)[t];
        const int j = (sl.x << 5) + lane;
        const bool own = j < n && !((sm_u32(T.lmask)[sl.x] >> lane) & 1u);
        const int jj = j < n ? j : 0;
        // the column's operands first: their latency overlaps the product
        const float xo = S[o.x + jj], dj = S[o.c + jj], lj = S[o.l + jj], uj = S[o.u + jj];
        float g;
        if (F32V)
            g = STAGED ? slice_dot_sv(sm_u16(T.words) + sl.y + lane, sm_f32(T.vals) + sl.y + lane, S, sl.z)
                       : slice_dot_sv_global(sp->rat.idx + sl.y + lane, sp->rat.v32 + sl.y + lane, S + o.y, sl.z);
        else
            g = STAGED ? slice_dot_pk(sm_u32(T.words) + sl.y + lane, S, sl.z)
                       : slice_dot_pk_global(sp->rat.pk + sl.y + lane, S + o.y, sl.z);
        if (PATCHED && sl.w && pt.n)  // a slice holding a patched column
            for (int q = 0; q < pt.n; ++q)
                if (pt.col[q] == j) g = fmaf(pt.v32[q], S[o.y + pt.row[q]], g);
        if (own) primal_update(o, j, xo, dj, lj, uj, g, tau, w, rho, check, bx, cx, pdx2, pdxa2);
    }
    for (int t = T.l0; t < T.l1; ++t) {  // long columns: the warp together, lane 0 updates
        const int4 ll = sm_int4(T.llist)[t];
        const int j = ll.x;
        float g;
        if (F32V)
            g = STAGED ? long_dot_sv<false>(sm_u16(T.lwords) + ll.y, nullptr, sm_f32(T.lvals) + ll.y, S, ll.z, lane)
                       : long_dot_sv<true>(nullptr, sp->rat.long_idx + ll.y, sp->rat.long_v32 + ll.y, S + o.y, ll.z,
                                           lane);
        else
            g = STAGED ? long_dot_pk<false>(sm_u32(T.lwords) + ll.y, S, ll.z, lane)
                       : long_dot_pk<true>(sp->rat.long_pk + ll.y, S + o.y, ll.z, lane);
        if (PATCHED && pt.n)
            for (int q = 0; q < pt.n; ++q)
                if (pt.col[q] == j) g = fmaf(pt.v32[q], S[o.y + pt.row[q]], g);
        if (lane == 0)
            primal_update(o, j, S[o.x + j], S[o.c + j], S[o.l + j], S[o.u + j], g, tau, w, rho, check, bx, cx, pdx2,
                          pdxa2);
    }
}

template <bool STAGED, bool PATCHED, bool F32V>
__device__ __forceinline__ void dual_pass_recentred(const DevSpecies* sp, const FastOffsets& o, const OpsView& A,
                                                    int m, int neq, int lane, float sigma, float w, float rho,
                                                    bool check, const double* by, double* cy, double& pdy2,
                                                    double& pdya2, const Patches& pt) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float* const S = reinterpret_cast<float*>(dyn_smem);
    for (int t = A.t0; t < A.t1; ++t) {
        const int4 sl = sm_int4(A.list)[t];
        const int i = (sl.x << 5) + lane;
        const bool own = i < m && !((sm_u32(A.lmask)[sl.x] >> lane) & 1u);
        const int ii = i < m ? i : 0;
        const float yo = S[o.y + ii], ri = S[o.b + ii], yl = S[o.ya + ii];
        float h;
        if (F32V)
            h = STAGED ? slice_dot_sv(sm_u16(A.words) + sl.y + lane, sm_f32(A.vals) + sl.y + lane, S, sl.z)
                       : slice_dot_sv_global(sp->ra.idx + sl.y + lane, sp->ra.v32 + sl.y + lane, S + o.xbar, sl.z);
        else
            h = STAGED ? slice_dot_pk(sm_u32(A.words) + sl.y + lane, S, sl.z)
                       : slice_dot_pk_global(sp->ra.pk + sl.y + lane, S + o.xbar, sl.z);
        if (PATCHED && sl.w && pt.n)  // a slice holding a patched row
            for (int q = 0; q < pt.n; ++q)
                if (pt.row[q] == i) h = fmaf(pt.v32[q], S[o.xbar + pt.col[q]], h);
        if (own) dual_update(o, i, neq, yo, ri, yl, h, sigma, w, rho, check, by, cy, pdy2, pdya2);
    }
    for (int t = A.l0; t < A.l1; ++t) {  // long rows
        const int4 ll = sm_int4(A.llist)[t];
        const int i = ll.x;
        float h;
        if (F32V)
            h = STAGED ? long_dot_sv<false>(sm_u16(A.lwords) + ll.y, nullptr, sm_f32(A.lvals) + ll.y, S, ll.z, lane)
                       : long_dot_sv<true>(nullptr, sp->ra.long_idx + ll.y, sp->ra.long_v32 + ll.y, S + o.xbar, ll.z,
                                           lane);
        else
            h = STAGED ? long_dot_pk<false>(sm_u32(A.lwords) + ll.y, S, ll.z, lane)
                       : long_dot_pk<true>(sp->ra.long_pk + ll.y, S + o.xbar, ll.z, lane);
        if (PATCHED && pt.n)
            for (int q = 0; q < pt.n; ++q)
                if (pt.row[q] == i) h = fmaf(pt.v32[q], S[o.xbar + pt.col[q]], h);
        if (lane == 0)
            dual_update(o, i, neq, S[o.y + i], S[o.b + i], S[o.ya + i], h, sigma, w, rho, check, by, cy, pdy2, pdya2);
    }
}

// FP64 slice product for the convergence test: the 16-bit column indices
// come from the staged packed words in shared memory (minus the
// gather-target offset `sub`), the FP64 values from global memory, the FP64 gather
// target from the slab.  The value loads do not depend on the indices, so
// one memory round trip serves each batch.
__device__ __forceinline__ double slice_dot64_staged(const uint32_t* wp, int sub, const double* __restrict__ vp,
                                                     const double* g, int len) {
    constexpr int U = 4;
    double acc0 = 0.0, acc1 = 0.0;
    for (int k0 = 0; k0 < len; k0 += U) {
        double vv[U], gg[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + u;
            if (k < len) {
                vv[u] = __ldg(vp + (k << 5));
                gg[u] = g[static_cast<int>(wp[k << 5] & 0xffffu) - sub];
            } else {
                vv[u] = 0.0;
                gg[u] = 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < U; u += 2) {
            acc0 = fma(vv[u], gg[u], acc0);
            acc1 = fma(vv[u + 1], gg[u + 1], acc1);
        }
    }
    return acc0 + acc1;
}

// slice_dot64_staged over staged 16-bit indices (the FP32-valued layout).
__device__ __forceinline__ double slice_dot64_staged16(const uint16_t* ip, int sub, const double* __restrict__ vp,
                                                       const double* g, int len) {
    constexpr int U = 4;
    double acc0 = 0.0, acc1 = 0.0;
    for (int k0 = 0; k0 < len; k0 += U) {
        double vv[U], gg[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + u;
            if (k < len) {
                vv[u] = __ldg(vp + (k << 5));
                gg[u] = g[static_cast<int>(ip[k << 5]) - sub];
            } else {
                vv[u] = 0.0;
                gg[u] = 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < U; u += 2) {
            acc0 = fma(vv[u], gg[u], acc0);
            acc1 = fma(vv[u + 1], gg[u + 1], acc1);
        }
    }
    return acc0 + acc1;
}

// The same product with the indices streamed from global memory; the
// accumulation order equals slice_dot64_staged's, so both variants produce
// identical results.
__device__ __forceinline__ double slice_dot64_global2(const int32_t* __restrict__ ip, const double* __restrict__ vp,
                                                      const double* g, int len) {
    constexpr int U = 4;
    double acc0 = 0.0, acc1 = 0.0;
    for (int k0 = 0; k0 < len; k0 += U) {
        double vv[U], gg[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + u;
            if (k < len) {
                vv[u] = __ldg(vp + (k << 5));
                gg[u] = g[__ldg(ip + (k << 5))];
            } else {
                vv[u] = 0.0;
                gg[u] = 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < U; u += 2) {
            acc0 = fma(vv[u], gg[u], acc0);
            acc1 = fma(vv[u + 1], gg[u + 1], acc1);
        }
    }
    return acc0 + acc1;
}

// One column's contribution to the FP64 KKT partials (see
// kkt_partials_recentred).
__device__ __forceinline__ void kkt_column(const DevSpecies* sp, int j, double g, double* xc, const double* cs,
                                           const double* ls, const double* us, float* dcand, bool cinf, double* v) {
    const double cj = cs[j], lj = ls[j], uj = us[j], dcj = __ldg(sp->dc + j);
    double xsc = xc[j];
    if (xsc < lj || xsc > uj) {
        xsc = xsc < lj ? lj : uj;
        xc[j] = xsc;
    }
    const double rs = cj - g;
    dcand[j] = static_cast<float>(rs);
    v[0] = __fma_rn(cj, xsc, v[0]);
    if (rs > 0.0) {
        if (isfinite(lj)) v[2] = __fma_rn(rs, lj, v[2]);
        else v[11] = fmax(v[11], rs * __ldg(sp->inv_dc + j));
    } else if (rs < 0.0) {
        if (isfinite(uj)) v[2] = __fma_rn(rs, uj, v[2]);
        else v[11] = fmax(v[11], -rs * __ldg(sp->inv_dc + j));
    }
    const double tg = (rs >= 0.0) ? lj : uj;
    if (isfinite(tg)) v[3] += fabs(rs * (xsc - tg));
    v[12] = fmax(v[12], dcj * fmax(lj - xsc, xsc - uj));
    v[13] = fmax(v[13], fabs(xsc * dcj));
    if (cinf) v[14] = fmax(v[14], fabs(cj * __ldg(sp->inv_dc + j)));
    if (isnan(g) || isnan(xsc)) v[15] = 1.0;
}

__device__ __forceinline__ void kkt_row(const DevSpecies* sp, int i, double h, const double* yc, const double* bs,
                                        float* rcand, double* v) {
    const double bi = bs[i], ysc = yc[i];
    const double rr = bi - h;                        // scaled b - A x
    const double ro = -rr * __ldg(sp->inv_dr + i);   // A x - b in original units
    rcand[i] = static_cast<float>(rr);
    if (i < sp->neq) {
        v[10] = fmax(v[10], fabs(ro));
    } else {
        v[10] = fmax(v[10], ro);
        v[4] += fabs(ysc * rr);
        v[11] = fmax(v[11], ysc * __ldg(sp->dr + i));
    }
    v[1] = __fma_rn(bi, ysc, v[1]);
    if (isnan(h) || isnan(ysc)) v[15] = 1.0;
}

// FP64 KKT partials at the candidate (xc, yc) (scaled, FP64) in the index
// map of kkt_partials, computed in scaled space with the slab's scaled
// objective cs, bounds ls/us and right-hand side bs (c.x = cs.xs,
// r_j l_j = rs_j ls_j with rs = cs - A~^T y the scaled reduced cost, ...).
// The candidate x is projected onto the exact FP64 bounds (written back: the
// FP32 bounds l - x^ are rounded), and rs and the scaled primal residual
// bs - A~ xc are stored in FP32 for a re-centring at this candidate.
// |c|_inf (v[14]) is accumulated only when `cinf` is set.  Long lines are
// walked by the whole warp and counted by its lane 0.  All threads call it
// (it synchronises between the column and the row loops).
template <bool STAGED, bool PATCHED, bool F32V>
__device__ __forceinline__ void kkt_partials_body(const DevSpecies* sp, const OpsView& A, const OpsView& T, int a_sub,
                                                    int t_sub, double* xc, const double* yc, const double* cs,
                                                    const double* ls, const double* us, const double* bs,
                                                    float* dcand, float* rcand, bool cinf, int lane, double* v,
                                                    const Patches& pt) {
    const int n = sp->n, m = sp->m;
    for (int t = T.t0; t < T.t1; ++t) {
        const int4 sl = sm_int4(T.list)[t];
        const int j = (sl.x << 5) + lane;
        double g = !STAGED ? slice_dot64_global2(sp->rat.idx + sl.y + lane, sp->rat.v64 + sl.y + lane, yc, sl.z)
                   : F32V  ? slice_dot64_staged16(sm_u16(T.words) + sl.y + lane, t_sub, sp->rat.v64 + sl.y + lane,
                                                  yc, sl.z)
                           : slice_dot64_staged(sm_u32(T.words) + sl.y + lane, t_sub, sp->rat.v64 + sl.y + lane, yc,
                                                sl.z);
        if (PATCHED && sl.w && pt.n)
            for (int q = 0; q < pt.n; ++q)
                if (pt.col[q] == j) g = fma(pt.v64[q], yc[pt.row[q]], g);
        if (j < n && !((sm_u32(T.lmask)[sl.x] >> lane) & 1u)) kkt_column(sp, j, g, xc, cs, ls, us, dcand, cinf, v);
    }
    for (int t = T.l0; t < T.l1; ++t) {
        const int4 ll = sm_int4(T.llist)[t];
        const int j = ll.x;
        const void* lw = F32V ? static_cast<const void*>(sm_u16(T.lwords) + ll.y)
                              : static_cast<const void*>(sm_u32(T.lwords) + ll.y);
        double g = long_dot64<STAGED, F32V>(STAGED ? lw : nullptr, t_sub, sp->rat.long_idx + ll.y,
                                            sp->rat.long_v64 + ll.y, yc, ll.z, lane);
        if (PATCHED && pt.n)
            for (int q = 0; q < pt.n; ++q)
                if (pt.col[q] == j) g = fma(pt.v64[q], yc[pt.row[q]], g);
        if (lane == 0) kkt_column(sp, j, g, xc, cs, ls, us, dcand, cinf, v);
    }
    __syncthreads();  // the projected xc is the gather target below
    for (int t = A.t0; t < A.t1; ++t) {
        const int4 sl = sm_int4(A.list)[t];
        const int i = (sl.x << 5) + lane;
        double h = !STAGED ? slice_dot64_global2(sp->ra.idx + sl.y + lane, sp->ra.v64 + sl.y + lane, xc, sl.z)
                   : F32V  ? slice_dot64_staged16(sm_u16(A.words) + sl.y + lane, a_sub, sp->ra.v64 + sl.y + lane,
                                                  xc, sl.z)
                           : slice_dot64_staged(sm_u32(A.words) + sl.y + lane, a_sub, sp->ra.v64 + sl.y + lane, xc,
                                                sl.z);
        if (PATCHED && sl.w && pt.n)
            for (int q = 0; q < pt.n; ++q)
                if (pt.row[q] == i) h = fma(pt.v64[q], xc[pt.col[q]], h);
        if (i < m && !((sm_u32(A.lmask)[sl.x] >> lane) & 1u)) kkt_row(sp, i, h, yc, bs, rcand, v);
    }
    for (int t = A.l0; t < A.l1; ++t) {
        const int4 ll = sm_int4(A.llist)[t];
        const int i = ll.x;
        const void* lw = F32V ? static_cast<const void*>(sm_u16(A.lwords) + ll.y)
                              : static_cast<const void*>(sm_u32(A.lwords) + ll.y);
        double h = long_dot64<STAGED, F32V>(STAGED ? lw : nullptr, a_sub, sp->ra.long_idx + ll.y,
                                            sp->ra.long_v64 + ll.y, xc, ll.z, lane);
        if (PATCHED && pt.n)
            for (int q = 0; q < pt.n; ++q)
                if (pt.row[q] == i) h = fma(pt.v64[q], xc[pt.col[q]], h);
        if (lane == 0) kkt_row(sp, i, h, yc, bs, rcand, v);
    }
}

// Out-of-line copy for the single-instance kernel; the paired kernel's slot
// start and test routines (themselves out of line) inline the body: one
// call boundary per test instead of three.  Measured: each call boundary
// saved and restored ~100 registers per thread through local memory, and
// the paired kernel's FP64 test cost fell from ~12 to ~7.6 iterations.
template <bool STAGED, bool PATCHED, bool F32V>
__device__ __noinline__ void kkt_partials_recentred(const DevSpecies* sp, const OpsView& A, const OpsView& T, int a_sub,
                                                    int t_sub, double* xc, const double* yc, const double* cs,
                                                    const double* ls, const double* us, const double* bs,
                                                    float* dcand, float* rcand, bool cinf, int lane, double* v,
                                                    const Patches& pt) {
    kkt_partials_body<STAGED, PATCHED, F32V>(sp, A, T, a_sub, t_sub, xc, yc, cs, ls, us, bs, dcand, rcand, cinf, lane,
                                             v, pt);
}

// Move the base to (bx, by) (the candidate the last kkt_partials_recentred
// call evaluated): load its reduced cost and residual, shift the bounds and
// zero the differences.  Callers synchronise afterwards.
__device__ __forceinline__ void recentre(const DevSpecies* sp, const FastOffsets& o, const double* bx,
                                         const double* by, const float* dcand, const float* rcand,
                                         const double* ls, const double* us) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float* const S = reinterpret_cast<float*>(dyn_smem);
    const int n = sp->n, m = sp->m, neq = sp->neq;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double xb = bx[j];
        S[o.c + j] = dcand[j];
        S[o.l + j] = static_cast<float>(ls[j] - xb);
        S[o.u + j] = static_cast<float>(us[j] - xb);
        S[o.x + j] = 0.0f;
    }
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        S[o.b + i] = rcand[i];
        S[o.ya + i] = i >= neq ? static_cast<float>(-by[i]) : 0.0f;
        S[o.y + i] = 0.0f;
    }
}

template <int MAXT, bool STAGED, bool PATCHED, bool F32V>
__global__ void __launch_bounds__(MAXT, 1) pdhg_recentred(const __grid_constant__ KernelParams p) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ double s_red[MAXT / 32][kRed];
    __shared__ double s_tot[kRed];
    __shared__ int s_inst;
    __shared__ int s_loaded;
    __shared__ int s_prow[kMaxPatches], s_pcol[kMaxPatches];
    __shared__ float s_pv32[kMaxPatches];
    __shared__ double s_pv64[kMaxPatches];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nthreads = blockDim.x;
    const int warps = nthreads >> 5;
    unsigned char* const slab = p.spill + static_cast<int64_t>(blockIdx.x) * p.spill_stride;
    const float rho = static_cast<float>(p.rho);
    const int count = p.count_dev ? *p.count_dev : p.count;
    if (tid == 0) s_loaded = -1;

    for (;;) {
        if (tid == 0) s_inst = atomicAdd(p.queue, 1);
        __syncthreads();
        const int q = s_inst;
        if (q >= count) break;
        const int inst = p.order[q];
        const int species = p.inst_species[inst];
        const DevSpecies* __restrict__ sp = p.species + species;
        const Layout& L = p.layouts[species];
        const int n = sp->n, m = sp->m, neq = sp->neq;
        const int64_t coff = p.col_off[inst], roff = p.row_off[inst];
        if (s_loaded != species) {  // block-uniform
            stage_species<float>(sp, L, dyn_smem, warps);
            __syncthreads();
            if (tid == 0) s_loaded = species;
        }
        float* const S = reinterpret_cast<float*>(dyn_smem);
        const FastOffsets o = fast_offsets<float>(L);
        // the staged packed words' indices carry the gather-target offsets
        const int a_sub = static_cast<int>(L.arr[kXbar] / 4), t_sub = static_cast<int>(L.arr[kY] / 4);
        OpsView OA, OT;
        ops_views(L, dyn_smem, warp, &OA, &OT);
        // the two point buffers; selected by value (no local-memory array)
        double* const px0 = reinterpret_cast<double*>(slab + L.pt_x[0]);
        double* const px1 = reinterpret_cast<double*>(slab + L.pt_x[1]);
        double* const py0 = reinterpret_cast<double*>(slab + L.pt_y[0]);
        double* const py1 = reinterpret_cast<double*>(slab + L.pt_y[1]);
        auto PX = [&](int b) { return b ? px1 : px0; };
        auto PY = [&](int b) { return b ? py1 : py0; };
        float* const dcand = reinterpret_cast<float*>(slab + L.dcand);
        float* const rcand = reinterpret_cast<float*>(slab + L.rcand);
        double* const cs = reinterpret_cast<double*>(slab + L.sc_c);
        double* const ls = reinterpret_cast<double*>(slab + L.sc_l);
        double* const us = reinterpret_cast<double*>(slab + L.sc_u);
        double* const bs = reinterpret_cast<double*>(slab + L.sc_b);
        const double* lo_i = p.lower + coff;
        const double* up_i = p.upper + coff;
        const double* c_i = p.cost + coff;
        const double* b_i = p.rhs ? p.rhs + roff : nullptr;

        // ---- this instance's patched entries (scaled deltas) ----
        // (compiled out of the variant for batches without patched entries)
        const int npatch = (PATCHED && p.patch_values != nullptr) ? sp->npatch : 0;
        int bad = 0;
        if (tid < npatch) {
            const double dv = p.patch_values[static_cast<int64_t>(inst) * p.patch_stride + tid];
            if (!isfinite(dv)) bad = 1;
            const double sv = dv * sp->patch_scale[tid];
            s_prow[tid] = sp->patch_row[tid];
            s_pcol[tid] = sp->patch_col[tid];
            s_pv64[tid] = sv;
            s_pv32[tid] = static_cast<float>(sv);
        }
        const Patches pt{npatch, s_prow, s_pcol, s_pv32, s_pv64};

        // ---- scaled instance data and the start point (FP64, projected) ----
        for (int j = tid; j < n; j += nthreads) {
            const int jo = sp->col_perm[j];
            const double dcj = sp->dc[j];
            const double lv = lo_i[jo], uv = up_i[jo], cv = c_i[jo];
            if (isnan(lv) || isnan(uv) || lv > uv || !isfinite(cv) || lv == INFINITY || uv == -INFINITY)
                bad = 1;
            const double lsj = lv / dcj, usj = uv / dcj;
            cs[j] = cv * dcj;
            ls[j] = lsj;
            us[j] = usj;
            double x0 = p.warm_x ? p.warm_x[coff + jo] / dcj : 0.0;
            if (!isfinite(x0)) x0 = 0.0;
            PX(0)[j] = x0 < lsj ? lsj : (x0 > usj ? usj : x0);
        }
        for (int i = tid; i < m; i += nthreads) {
            const int io = sp->row_perm[i];
            const double dri = sp->dr[i];
            const double bv = b_i ? b_i[io] : 0.0;
            if (!isfinite(bv)) bad = 1;
            bs[i] = bv * dri;
            double y0 = p.warm_y ? p.warm_y[roff + io] / dri : 0.0;
            if (!isfinite(y0)) y0 = 0.0;
            if (i >= neq && y0 > 0.0) y0 = 0.0;
            PY(0)[i] = y0;
        }
        if (tid == 0) {
            PX(0)[n] = 0.0;
            PX(1)[n] = 0.0;
            PY(0)[m] = 0.0;
            PY(1)[m] = 0.0;
            S[o.xbar + n] = 0.0f;
            S[o.y + m] = 0.0f;
        }
        bad = __syncthreads_or(bad);
        double omega = 1.0;
        if (p.warm_omega) {
            const double w0 = p.warm_omega[inst];
            if (isfinite(w0) && w0 > 0.0) omega = w0;
        }
        if (bad) {
            for (int j = tid; j < n; j += nthreads) p.out_x[coff + sp->col_perm[j]] = NAN;
            for (int i = tid; i < m; i += nthreads) p.out_y[roff + sp->row_perm[i]] = NAN;
            if (tid == 0) {
                p.out_status[inst] = kStatusInvalid;
                p.out_iters[inst] = p.prior_iters ? p.prior_iters[inst] : 0;
                if (p.hand_iters) p.hand_iters[inst] = 0;
                p.out_obj[inst] = NAN;
                for (int k = 0; k < kMetrics; ++k) p.out_metrics[static_cast<int64_t>(inst) * kMetrics + k] = NAN;
                if (p.out_omega) p.out_omega[inst] = omega;
            }
            continue;
        }

        // step size: the shared matrix's, shrunk so that it stays below
        // 1/||A~ + patches||, bounded by the smaller of ||A~|| + ||deltas||_F
        // and sqrt(||A~||^2 + ||patched columns of this instance||_F^2)
        double eta = sp->eta;
        if (PATCHED && npatch) {
            double f2 = 0.0, c2 = sp->patch_col_f2;
            for (int q = 0; q < npatch; ++q) {
                f2 += s_pv64[q] * s_pv64[q];
                const double v = sp->patch_base[q] + s_pv64[q];
                c2 += v * v;
            }
            const double s = sp->sigma_max;
            eta *= s / fmin(s + sqrt(f2), sqrt(s * s + c2));
        }
        int status = -1;
        int cur = 0;   // buffer holding the base
        int ev = 0;    // buffer holding the last evaluated point
        double cinf = 0.0;
        Metrics M;
        {
            double v[kRed];
#pragma unroll
            for (int qq = 0; qq < kRed; ++qq) v[qq] = 0.0;
            kkt_partials_recentred<STAGED, PATCHED, F32V>(sp, OA, OT, a_sub, t_sub, PX(0), PY(0), cs, ls,
                                   us, bs, dcand, rcand, true, lane, v, pt);
            block_reduce(v, s_red, s_tot);
            cinf = s_tot[14];
            M = evaluate(s_tot, omega, p.tol_p, p.tol_d, p.tol_g);
            if (M.conv) status = p.final_status;
            else if (p.max_iters <= 0) status = M.nan ? kStatusNumerical : kStatusIterationLimit;
            if (status < 0) {
                recentre(sp, o, PX(0), PY(0), dcand, rcand, ls, us);
                __syncthreads();
            }
        }

        int k = 0, it = 0, stall = 0;
        bool fell_back = false;
        // early termination tests only for instances expected to finish early
        const bool early = p.hint_iters == nullptr || p.hint_iters[inst] < p.check_every;
        double r_restart = INFINITY, r_prev = INFINITY, best_err = INFINITY;
        while (status < 0) {
            ++it;
            const bool full = (it % p.check_every == 0) || (it >= p.max_iters);
            const bool check = full || (early && it >= 8 && it < p.check_every && (it & (it - 1)) == 0);
            const float tau = static_cast<float>(eta / omega), sigma = static_cast<float>(eta * omega);
            const float w = static_cast<float>((k + 1.0) / (k + 2.0));
            double pdx2 = 0.0, pdy2 = 0.0, pdxa2 = 0.0, pdya2 = 0.0;
            primal_pass_recentred<STAGED, PATCHED, F32V>(sp, o, OT, n, lane, tau, w, rho, check, PX(cur), PX(cur ^ 1),
                                          pdx2, pdxa2, pt);
            __syncthreads();
            dual_pass_recentred<STAGED, PATCHED, F32V>(sp, o, OA, m, neq, lane, sigma, w, rho, check, PY(cur),
                                        PY(cur ^ 1), pdy2, pdya2, pt);
            __syncthreads();
            ++k;
            if (!check) continue;

            double v[kRed];
#pragma unroll
            for (int qq = 0; qq < kRed; ++qq) v[qq] = 0.0;
            v[5] = pdx2;
            v[6] = pdy2;
            v[7] = pdxa2;
            v[8] = pdya2;
            kkt_partials_recentred<STAGED, PATCHED, F32V>(sp, OA, OT, a_sub, t_sub, PX(cur ^ 1), PY(cur ^ 1),
                                   cs, ls, us, bs, dcand, rcand, false, lane, v, pt);
            block_reduce(v, s_red, s_tot);
            if (threadIdx.x == 0) s_tot[14] = cinf;
            __syncthreads();
            M = evaluate(s_tot, omega, p.tol_p, p.tol_d, p.tol_g);
            ev = cur ^ 1;
            if (M.nan || !isfinite(M.r)) {
                status = kStatusNumerical;
                break;
            }
            if (M.conv) {
                status = p.final_status;
                break;
            }
            if (it >= p.max_iters) {
                status = kStatusIterationLimit;
                break;
            }
            if (!full) continue;
            {
                const double e = fmax(fmax(M.primal / (1.0 + M.xinf), M.dual / (1.0 + M.cinf)),
                                      fmax(M.rgap, M.kgap));
                if (e < 0.5 * best_err) {
                    best_err = e;
                    stall = 0;
                } else {
                    ++stall;
                }
                if (p.stall_checks > 0 && stall >= p.stall_checks && e <= p.floor_tol && floor_accepts(M, p)) {
                    status = p.final_status;
                    break;
                }
                // a long stall (slow phases of PDHG last a few tests; an FP32
                // rounding floor does not end) continues in FP64
                if (p.handoff_on_stall > 0 && stall >= p.handoff_on_stall) {
                    status = kStatusHandoff;
                    break;
                }
            }
            if (p.fallback_iters > 0 && !fell_back && it >= p.fallback_iters &&
                (p.warm_x != nullptr || p.warm_y != nullptr)) {
                // cold fallback: evaluate the cold point in the candidate
                // buffer and re-centre there
                fell_back = true;
                omega = 1.0;
                double* cx = PX(cur ^ 1);
                double* cyv = PY(cur ^ 1);
                for (int j = tid; j < n; j += nthreads) cx[j] = 0.0 < ls[j] ? ls[j] : (0.0 > us[j] ? us[j] : 0.0);
                for (int i = tid; i < m; i += nthreads) cyv[i] = 0.0;
                __syncthreads();
                double vv[kRed];
#pragma unroll
                for (int qq = 0; qq < kRed; ++qq) vv[qq] = 0.0;
                kkt_partials_recentred<STAGED, PATCHED, F32V>(sp, OA, OT, a_sub, t_sub, cx, cyv, cs, ls, us,
                                       bs, dcand, rcand, false, lane, vv, pt);
                block_reduce(vv, s_red, s_tot);
                cur ^= 1;
                ev = cur;
                recentre(sp, o, PX(cur), PY(cur), dcand, rcand, ls, us);
                k = 0;
                r_restart = INFINITY;
                r_prev = INFINITY;
                best_err = INFINITY;
                stall = 0;
                __syncthreads();
                continue;
            }
            if (p.restarts && (M.r <= kBetaSufficient * r_restart ||
                               (M.r <= kBetaNecessary * r_restart && M.r > r_prev) ||
                               k >= kBetaArtificial * it)) {
                const double nx = sqrt(s_tot[7]), ny = sqrt(s_tot[8]);
                if (nx > 1e-10 && ny > 1e-10)
                    omega = exp(__fma_rn(p.omega_smoothing, log(ny / nx), (1.0 - p.omega_smoothing) * log(omega)));
                cur ^= 1;  // the candidate becomes the base
                recentre(sp, o, PX(cur), PY(cur), dcand, rcand, ls, us);
                k = 0;
                r_restart = M.r;
                r_prev = INFINITY;
                __syncthreads();
            } else {
                r_prev = M.r;
            }
        }

        // ---- results (original units and order) from the last evaluated point ----
        const bool hand = p.handoff_list != nullptr && status == kStatusHandoff;
        const double* fx = PX(ev);
        const double* fy = PY(ev);
        double* ox = hand ? p.hand_x : p.out_x;
        double* oy = hand ? p.hand_y : p.out_y;
        for (int j = tid; j < n; j += nthreads) {
            const int jo = sp->col_perm[j];
            double xv = fx[j] * sp->dc[j];
            if (p.clip_output && !hand) {
                const double lv = lo_i[jo], uv = up_i[jo];
                xv = xv < lv ? lv : (xv > uv ? uv : xv);
            }
            ox[coff + jo] = xv;
        }
        for (int i = tid; i < m; i += nthreads) oy[roff + sp->row_perm[i]] = fy[i] * sp->dr[i];
        if (tid == 0) {
            if (p.hand_iters) p.hand_iters[inst] = (p.prior_iters ? p.prior_iters[inst] : 0) + it;
            if (hand) {
                p.hand_omega[inst] = omega;
                p.handoff_list[atomicAdd(p.handoff_count, 1)] = inst;
            } else {
                double* mo = p.out_metrics + static_cast<int64_t>(inst) * kMetrics;
                mo[0] = M.primal;
                mo[1] = M.dual;
                mo[2] = M.kgap;
                mo[3] = M.pobj;
                mo[4] = M.dobj;
                mo[5] = M.rgap;
                mo[6] = M.xinf;
                mo[7] = omega;
                p.out_obj[inst] = M.pobj;
                p.out_status[inst] = status;
                p.out_iters[inst] = (p.prior_iters ? p.prior_iters[inst] : 0) + it;
                if (p.out_omega) p.out_omega[inst] = omega;
            }
        }
        // the next instance reuses the slab and shared memory
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Paired re-centred FP32 PDHG: two instances of one species per CTA.
//
// The arithmetic of pdhg_recentred (reflection 1, staged matrix, no patched
// entries) applied to two instances at once.  Their FP32 vectors are
// interleaved as float2 in shared memory (component s belongs to instance
// slot s), so every packed matrix word read from shared memory serves both
// instances and one 64-bit shared load gathers both instances' operands:
// the species' matrix multiplies a block of two vectors (a sparse matrix
// times a dense n x 2 block) instead of one.  Each slot runs its own solve
// -- iteration count, Halpern weight, step sizes, restarts, convergence
// tests, FP64 slab and work-queue instance -- with the operations of
// pdhg_recentred in the same order, so a slot's iterates equal the
// single-instance kernel's bit for bit.  The Halpern iterate x is not
// stored: with reflection 1 it is w xbar (w the previous iteration's
// Halpern weight), which is how pdhg_recentred computes it.  A slot whose
// instance finishes takes the next queued instance of the staged species;
// an instance of another species waits until both slots are free, then the
// CTA restages.  A free slot's vectors are zero (step sizes and weights
// zero), so it computes zeros beside the busy one.
// ---------------------------------------------------------------------------

struct PairOffsets {
    int xbar, y, c, l, u, b, ya;  // float2 element offsets from the start of shared memory
};

__device__ __forceinline__ PairOffsets pair_offsets(const Layout& L) {
    PairOffsets o;
    o.xbar = static_cast<int>(L.arr[kXbar] / 8);
    o.y = static_cast<int>(L.arr[kY] / 8);
    o.c = static_cast<int>(L.arr[kC] / 8);
    o.l = static_cast<int>(L.arr[kL] / 8);
    o.u = static_cast<int>(L.arr[kU] / 8);
    o.b = static_cast<int>(L.arr[kB] / 8);
    o.ya = static_cast<int>(L.arr[kYa] / 8);
    return o;
}

// Stage a species for the paired kernel: schedule lists, packed words with
// the indices pre-offset to the float2 gather targets, and every vector
// region zeroed (both slots free).
__device__ void stage_species_pair(const DevSpecies* sp, const Layout& L, unsigned char* sm, int warps) {
    const int tid = threadIdx.x, nt = blockDim.x;
    stage_recentred_ops(sp, L, sm, warps, 8);
    float2* const S2 = reinterpret_cast<float2*>(sm);
    const PairOffsets o = pair_offsets(L);
    const int n = sp->n, m = sp->m, mi = sp->m - sp->neq;
    const float2 z = make_float2(0.0f, 0.0f);
    for (int j = tid; j <= n; j += nt) S2[o.xbar + j] = z;  // [n]: the padding target
    for (int i = tid; i <= m; i += nt) S2[o.y + i] = z;     // [m]: the padding target
    for (int j = tid; j < n; j += nt) {
        S2[o.c + j] = z;
        S2[o.l + j] = z;
        S2[o.u + j] = z;
    }
    for (int i = tid; i < m; i += nt) S2[o.b + i] = z;
    for (int i = tid; i < mi; i += nt) S2[o.ya + i] = z;
}

// Slice product of the packed words against both slots' gather targets:
// per slot the accumulation of slice_dot_pk (even k into a0, odd k into a1,
// then a0 + a1).
__device__ __forceinline__ float2 slice_dot_pk2(const uint32_t* wp, const float2* g, int len) {
    float a0x = 0.0f, a0y = 0.0f, a1x = 0.0f, a1y = 0.0f;
    int k = 0;
    for (; k + 4 <= len; k += 4, wp += 128) {
        const uint32_t w0 = wp[0], w1 = wp[32], w2 = wp[64], w3 = wp[96];
        const float2 g0 = g[w0 & 0xffffu], g1 = g[w1 & 0xffffu], g2 = g[w2 & 0xffffu], g3 = g[w3 & 0xffffu];
        const float v0 = __uint_as_float(w0 & 0xffff0000u), v1 = __uint_as_float(w1 & 0xffff0000u);
        const float v2 = __uint_as_float(w2 & 0xffff0000u), v3 = __uint_as_float(w3 & 0xffff0000u);
        a0x = fmaf(v0, g0.x, a0x);
        a0y = fmaf(v0, g0.y, a0y);
        a1x = fmaf(v1, g1.x, a1x);
        a1y = fmaf(v1, g1.y, a1y);
        a0x = fmaf(v2, g2.x, a0x);
        a0y = fmaf(v2, g2.y, a0y);
        a1x = fmaf(v3, g3.x, a1x);
        a1y = fmaf(v3, g3.y, a1y);
    }
    if (k + 2 <= len) {
        const uint32_t w0 = wp[0], w1 = wp[32];
        const float2 g0 = g[w0 & 0xffffu], g1 = g[w1 & 0xffffu];
        const float v0 = __uint_as_float(w0 & 0xffff0000u), v1 = __uint_as_float(w1 & 0xffff0000u);
        a0x = fmaf(v0, g0.x, a0x);
        a0y = fmaf(v0, g0.y, a0y);
        a1x = fmaf(v1, g1.x, a1x);
        a1y = fmaf(v1, g1.y, a1y);
        k += 2;
        wp += 64;
    }
    if (k < len) {
        const uint32_t w0 = wp[0];
        const float2 g0 = g[w0 & 0xffffu];
        const float v0 = __uint_as_float(w0 & 0xffff0000u);
        a0x = fmaf(v0, g0.x, a0x);
        a0y = fmaf(v0, g0.y, a0y);
    }
    return make_float2(a0x + a1x, a0y + a1y);
}

// One long line's product against both slots' gather targets, the whole
// warp together (per slot the order of long_dot_pk).
__device__ __forceinline__ float2 long_dot_pk2(const uint32_t* wp, const float2* g, int len, int lane) {
    float ax = 0.0f, ay = 0.0f;
    for (int k = lane; k < len; k += 32) {
        const uint32_t w = wp[k];
        const float2 gg = g[w & 0xffffu];
        const float v = __uint_as_float(w & 0xffff0000u);
        ax = fmaf(v, gg.x, ax);
        ay = fmaf(v, gg.y, ay);
    }
    return make_float2(warp_sum_f(ax), warp_sum_f(ay));
}

// One slot's FP64 slab: the re-centred slab of pdhg_recentred.
struct PairSlab {
    double *px0, *px1, *py0, *py1;
    float *dcand, *rcand;
    double *cs, *ls, *us, *bs;
    __device__ double* X(int b) const { return b ? px1 : px0; }
    __device__ double* Y(int b) const { return b ? py1 : py0; }
};

__device__ __forceinline__ PairSlab pair_slab(const KernelParams& p, const Layout& L, int slot) {
    unsigned char* const base = p.spill + (2 * static_cast<int64_t>(blockIdx.x) + slot) * p.spill_stride;
    PairSlab b;
    b.px0 = reinterpret_cast<double*>(base + L.pt_x[0]);
    b.px1 = reinterpret_cast<double*>(base + L.pt_x[1]);
    b.py0 = reinterpret_cast<double*>(base + L.pt_y[0]);
    b.py1 = reinterpret_cast<double*>(base + L.pt_y[1]);
    b.dcand = reinterpret_cast<float*>(base + L.dcand);
    b.rcand = reinterpret_cast<float*>(base + L.rcand);
    b.cs = reinterpret_cast<double*>(base + L.sc_c);
    b.ls = reinterpret_cast<double*>(base + L.sc_l);
    b.us = reinterpret_cast<double*>(base + L.sc_u);
    b.bs = reinterpret_cast<double*>(base + L.sc_b);
    return b;
}

// Per-slot solve state (block-uniform: one copy in shared memory, written by
// thread 0 between barriers).
struct PairSlot {
    int inst;  // -1: free
    int cur, ev, k, it, stall;
    bool fell_back, early;
    bool full, chk;           // the next iteration's tests (slot_next)
    float tau, sig, w, wp;    // the next iteration's steps and weights
    int64_t coff, roff;
    double omega, eta, cinf, r_restart, r_prev, best_err;
};

// The next iteration's tests and FP32 steps of a slot (the formulas of
// pdhg_recentred: steps eta / omega and eta omega, Halpern weights
// (k + 1) / (k + 2) and k / (k + 1) in FP64, rounded once), computed once
// where the slot's state changes instead of by every thread every iteration.
__device__ __forceinline__ void slot_next(PairSlot& st, const KernelParams& p) {
    const int it = st.it + 1;
    st.full = (it % p.check_every == 0) || (it >= p.max_iters);
    st.chk = st.full || (st.early && it >= 8 && it < p.check_every && (it & (it - 1)) == 0);
    st.tau = static_cast<float>(st.eta / st.omega);
    st.sig = static_cast<float>(st.eta * st.omega);
    st.w = static_cast<float>((st.k + 1.0) / (st.k + 2.0));
    st.wp = static_cast<float>(st.k / (st.k + 1.0));
}

__device__ __forceinline__ float& comp(float2* a, int slot) { return reinterpret_cast<float*>(a)[slot]; }

__device__ __forceinline__ int lane_id() { return static_cast<int>(threadIdx.x & 31); }

// Move slot `slot`'s base to (bx, by) (the candidate last evaluated): its
// components of d, l - x^, u - x^, r, -y^ and zero differences.
__device__ __forceinline__ void recentre_pair(const DevSpecies* sp, const PairOffsets& o, int slot, const double* bx,
                                              const double* by, const float* dcand, const float* rcand,
                                              const double* ls, const double* us) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float2* const S2 = reinterpret_cast<float2*>(dyn_smem);
    const int n = sp->n, m = sp->m, neq = sp->neq;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double xb = bx[j];
        comp(S2 + o.c + j, slot) = dcand[j];
        comp(S2 + o.l + j, slot) = static_cast<float>(ls[j] - xb);
        comp(S2 + o.u + j, slot) = static_cast<float>(us[j] - xb);
        comp(S2 + o.xbar + j, slot) = 0.0f;
    }
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        comp(S2 + o.b + i, slot) = rcand[i];
        if (i >= neq) comp(S2 + o.ya + (i - neq), slot) = static_cast<float>(-by[i]);
        comp(S2 + o.y + i, slot) = 0.0f;
    }
}

// Free slot `slot`: zero its vector components (it then computes zeros).
__device__ __forceinline__ void clear_slot(const DevSpecies* sp, const PairOffsets& o, int slot) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float2* const S2 = reinterpret_cast<float2*>(dyn_smem);
    const int n = sp->n, m = sp->m, neq = sp->neq;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        comp(S2 + o.c + j, slot) = 0.0f;
        comp(S2 + o.l + j, slot) = 0.0f;
        comp(S2 + o.u + j, slot) = 0.0f;
        comp(S2 + o.xbar + j, slot) = 0.0f;
    }
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        comp(S2 + o.b + i, slot) = 0.0f;
        if (i >= neq) comp(S2 + o.ya + (i - neq), slot) = 0.0f;
        comp(S2 + o.y + i, slot) = 0.0f;
    }
}

// Primal update of column j in both slots (shared by the slice lanes and the
// long columns' lane 0).  CHECK: some slot tests this iteration (c0 / c1
// say which); it then writes its candidate and accumulates pd[4 s + 0..1]
// (|xn - x|^2 and |xn|^2).  xo = wp xbar (reflection 1).
template <bool CHECK>
__device__ __forceinline__ void primal_update_pair(const PairOffsets& o, int j, float2 xbo, float2 dj, float2 lj,
                                                   float2 uj, float2 g, float2 tau, float2 wp, bool c0, bool c1,
                                                   const double* bx0, double* cx0, const double* bx1, double* cx1,
                                                   double* pd) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float2* const S2 = reinterpret_cast<float2*>(dyn_smem);
    const float xo0 = __fmul_rn(wp.x, xbo.x), xo1 = __fmul_rn(wp.y, xbo.y);
    const float xn0 = clampT(__fmaf_rn(-tau.x, __fsub_rn(dj.x, g.x), xo0), lj.x, uj.x);
    const float xn1 = clampT(__fmaf_rn(-tau.y, __fsub_rn(dj.y, g.y), xo1), lj.y, uj.y);
    S2[o.xbar + j] = make_float2(__fsub_rn(__fadd_rn(xn0, xn0), xo0), __fsub_rn(__fadd_rn(xn1, xn1), xo1));
    if (CHECK) {
        if (c0) {
            cx0[j] = bx0[j] + static_cast<double>(xn0);
            const double d = static_cast<double>(xn0) - static_cast<double>(xo0);
            pd[0] = __fma_rn(d, d, pd[0]);
            pd[1] = __fma_rn(static_cast<double>(xn0), static_cast<double>(xn0), pd[1]);
        }
        if (c1) {
            cx1[j] = bx1[j] + static_cast<double>(xn1);
            const double d = static_cast<double>(xn1) - static_cast<double>(xo1);
            pd[4] = __fma_rn(d, d, pd[4]);
            pd[5] = __fma_rn(static_cast<double>(xn1), static_cast<double>(xn1), pd[5]);
        }
    }
}

template <bool CHECK>
__device__ __forceinline__ void dual_update_pair(const PairOffsets& o, int i, int neq, float2 yo, float2 ri,
                                                 float2 yl, float2 h, float2 sigma, float2 w, bool c0, bool c1,
                                                 const double* by0, double* cy0, const double* by1, double* cy1,
                                                 double* pd) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float2* const S2 = reinterpret_cast<float2*>(dyn_smem);
    float yn0 = __fmaf_rn(sigma.x, __fsub_rn(ri.x, h.x), yo.x);
    float yn1 = __fmaf_rn(sigma.y, __fsub_rn(ri.y, h.y), yo.y);
    if (i >= neq) {  // y^ + dy <= 0
        if (yn0 > yl.x) yn0 = yl.x;
        if (yn1 > yl.y) yn1 = yl.y;
    }
    S2[o.y + i] = make_float2(__fmul_rn(w.x, __fsub_rn(__fadd_rn(yn0, yn0), yo.x)),
                              __fmul_rn(w.y, __fsub_rn(__fadd_rn(yn1, yn1), yo.y)));
    if (CHECK) {
        if (c0) {
            cy0[i] = by0[i] + static_cast<double>(yn0);
            const double d = static_cast<double>(yn0) - static_cast<double>(yo.x);
            pd[2] = __fma_rn(d, d, pd[2]);
            pd[3] = __fma_rn(static_cast<double>(yn0), static_cast<double>(yn0), pd[3]);
        }
        if (c1) {
            cy1[i] = by1[i] + static_cast<double>(yn1);
            const double d = static_cast<double>(yn1) - static_cast<double>(yo.y);
            pd[6] = __fma_rn(d, d, pd[6]);
            pd[7] = __fma_rn(static_cast<double>(yn1), static_cast<double>(yn1), pd[7]);
        }
    }
}

// Primal pass of both slots over this warp's A^T slices and long columns.
template <bool CHECK>
__device__ __forceinline__ void primal_pass_pair(const PairOffsets& o, const OpsView& T, int n, float2 tau, float2 wp,
                                                 bool c0, bool c1, const double* bx0, double* cx0, const double* bx1,
                                                 double* cx1, double* pd) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float2* const S2 = reinterpret_cast<float2*>(dyn_smem);
    const int lane = threadIdx.x & 31;
    for (int t = T.t0; t < T.t1; ++t) {
        const int4 sl = sm_int4(T.list)[t];
        const int j = (sl.x << 5) + lane;
        const bool own = j < n && !((sm_u32(T.lmask)[sl.x] >> lane) & 1u);
        const int jj = j < n ? j : 0;
        const float2 xbo = S2[o.xbar + jj], dj = S2[o.c + jj], lj = S2[o.l + jj], uj = S2[o.u + jj];
        const float2 g = slice_dot_pk2(sm_u32(T.words) + sl.y + lane, S2, sl.z);
        if (own) primal_update_pair<CHECK>(o, j, xbo, dj, lj, uj, g, tau, wp, c0, c1, bx0, cx0, bx1, cx1, pd);
    }
    for (int t = T.l0; t < T.l1; ++t) {
        const int4 ll = sm_int4(T.llist)[t];
        const int j = ll.x;
        const float2 g = long_dot_pk2(sm_u32(T.lwords) + ll.y, S2, ll.z, lane);
        if (lane == 0)
            primal_update_pair<CHECK>(o, j, S2[o.xbar + j], S2[o.c + j], S2[o.l + j], S2[o.u + j], g, tau, wp, c0, c1,
                                      bx0, cx0, bx1, cx1, pd);
    }
}

// Dual pass of both slots over this warp's A slices and long rows.
template <bool CHECK>
__device__ __forceinline__ void dual_pass_pair(const PairOffsets& o, const OpsView& A, int m, int neq, float2 sigma,
                                               float2 w, bool c0, bool c1, const double* by0, double* cy0,
                                               const double* by1, double* cy1, double* pd) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float2* const S2 = reinterpret_cast<float2*>(dyn_smem);
    const int lane = threadIdx.x & 31;
    const float2 z = make_float2(0.0f, 0.0f);
    for (int t = A.t0; t < A.t1; ++t) {
        const int4 sl = sm_int4(A.list)[t];
        const int i = (sl.x << 5) + lane;
        const bool own = i < m && !((sm_u32(A.lmask)[sl.x] >> lane) & 1u);
        const int ii = i < m ? i : 0;
        const float2 yo = S2[o.y + ii], ri = S2[o.b + ii];
        const float2 yl = (i < m && i >= neq) ? S2[o.ya + (i - neq)] : z;
        const float2 h = slice_dot_pk2(sm_u32(A.words) + sl.y + lane, S2, sl.z);
        if (own) dual_update_pair<CHECK>(o, i, neq, yo, ri, yl, h, sigma, w, c0, c1, by0, cy0, by1, cy1, pd);
    }
    for (int t = A.l0; t < A.l1; ++t) {
        const int4 ll = sm_int4(A.llist)[t];
        const int i = ll.x;
        const float2 h = long_dot_pk2(sm_u32(A.lwords) + ll.y, S2, ll.z, lane);
        if (lane == 0)
            dual_update_pair<CHECK>(o, i, neq, S2[o.y + i], S2[o.b + i], i >= neq ? S2[o.ya + (i - neq)] : z, h,
                                    sigma, w, c0, c1, by0, cy0, by1, cy1, pd);
    }
}

// The staged species' context (in shared memory: one copy per CTA).
struct PairStage {
    Layout L;                 // the species' layout record
    const DevSpecies* sp;
    int n, m, neq;            // its dimensions
};

// This warp's views of the staged operands, and the gather-target offsets of
// the staged indices (float2 units).
__device__ __forceinline__ void pair_views(const PairStage& g, OpsView* A, OpsView* T) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    ops_views(g.L, dyn_smem, threadIdx.x >> 5, A, T);
}

// The slot's results (original units and order) from its last evaluated
// point; the slot's vector components are zeroed.  All threads call it.
__device__ __noinline__ void finish_pair_slot(const KernelParams& p, const PairStage& g, int slot, int inst,
                                              int64_t coff, int64_t roff, int ev, int it, double omega, int status,
                                              const Metrics& M) {
    const DevSpecies* sp = g.sp;
    const int n = sp->n, m = sp->m, tid = threadIdx.x, nthreads = blockDim.x;
    const PairSlab b = pair_slab(p, g.L, slot);
    const bool hand = p.handoff_list != nullptr && status == kStatusHandoff;
    const double* fx = b.X(ev);
    const double* fy = b.Y(ev);
    double* ox = hand ? p.hand_x : p.out_x;
    double* oy = hand ? p.hand_y : p.out_y;
    const double* lo_i = p.lower + coff;
    const double* up_i = p.upper + coff;
    for (int j = tid; j < n; j += nthreads) {
        const int jo = sp->col_perm[j];
        double xv = fx[j] * sp->dc[j];
        if (p.clip_output && !hand) {
            const double lv = lo_i[jo], uv = up_i[jo];
            xv = xv < lv ? lv : (xv > uv ? uv : xv);
        }
        ox[coff + jo] = xv;
    }
    for (int i = tid; i < m; i += nthreads) oy[roff + sp->row_perm[i]] = fy[i] * sp->dr[i];
    if (tid == 0) {
        if (p.hand_iters) p.hand_iters[inst] = it;
        if (hand) {
            p.hand_omega[inst] = omega;
            p.handoff_list[atomicAdd(p.handoff_count, 1)] = inst;
        } else {
            double* mo = p.out_metrics + static_cast<int64_t>(inst) * kMetrics;
            mo[0] = M.primal;
            mo[1] = M.dual;
            mo[2] = M.kgap;
            mo[3] = M.pobj;
            mo[4] = M.dobj;
            mo[5] = M.rgap;
            mo[6] = M.xinf;
            mo[7] = omega;
            p.out_obj[inst] = M.pobj;
            p.out_status[inst] = status;
            p.out_iters[inst] = it;
            if (p.out_omega) p.out_omega[inst] = omega;
        }
    }
    clear_slot(sp, pair_offsets(g.L), slot);
}

// Publish a slot's state computed (identically) by every thread.
__device__ __forceinline__ void store_slot(PairSlot* s_st, int slot, const PairSlot& st) {
    __syncthreads();
    if (threadIdx.x == 0) s_st[slot] = st;
    __syncthreads();
}

// Load instance `inst` into slot `slot`: scaled data, start point and its
// test; a start point that already passes finishes the slot at once.  All
// threads call it.
__device__ __noinline__ void start_pair_slot(const KernelParams& p, const PairStage& g, PairSlot* s_st, int slot,
                                             int inst, double (*s_red)[kRed], double* s_tot) {
    const DevSpecies* sp = g.sp;
    const int n = sp->n, m = sp->m, neq = sp->neq, tid = threadIdx.x, nthreads = blockDim.x;
    const PairSlab b = pair_slab(p, g.L, slot);
    const Patches nopatch{0, nullptr, nullptr, nullptr, nullptr};
    PairSlot st{};
    st.inst = inst;
    st.coff = p.col_off[inst];
    st.roff = p.row_off[inst];
    const double* lo_i = p.lower + st.coff;
    const double* up_i = p.upper + st.coff;
    const double* c_i = p.cost + st.coff;
    const double* b_i = p.rhs ? p.rhs + st.roff : nullptr;
    int bad = 0;
    for (int j = tid; j < n; j += nthreads) {
        const int jo = sp->col_perm[j];
        const double dcj = sp->dc[j];
        const double lv = lo_i[jo], uv = up_i[jo], cv = c_i[jo];
        if (isnan(lv) || isnan(uv) || lv > uv || !isfinite(cv) || lv == INFINITY || uv == -INFINITY) bad = 1;
        const double lsj = lv / dcj, usj = uv / dcj;
        b.cs[j] = cv * dcj;
        b.ls[j] = lsj;
        b.us[j] = usj;
        double x0 = p.warm_x ? p.warm_x[st.coff + jo] / dcj : 0.0;
        if (!isfinite(x0)) x0 = 0.0;
        b.px0[j] = x0 < lsj ? lsj : (x0 > usj ? usj : x0);
    }
    for (int i = tid; i < m; i += nthreads) {
        const int io = sp->row_perm[i];
        const double dri = sp->dr[i];
        const double bv = b_i ? b_i[io] : 0.0;
        if (!isfinite(bv)) bad = 1;
        b.bs[i] = bv * dri;
        double y0 = p.warm_y ? p.warm_y[st.roff + io] / dri : 0.0;
        if (!isfinite(y0)) y0 = 0.0;
        if (i >= neq && y0 > 0.0) y0 = 0.0;
        b.py0[i] = y0;
    }
    if (tid == 0) {
        b.px0[n] = 0.0;
        b.px1[n] = 0.0;
        b.py0[m] = 0.0;
        b.py1[m] = 0.0;
    }
    bad = __syncthreads_or(bad);
    st.omega = 1.0;
    if (p.warm_omega) {
        const double w0 = p.warm_omega[inst];
        if (isfinite(w0) && w0 > 0.0) st.omega = w0;
    }
    if (bad) {
        for (int j = tid; j < n; j += nthreads) p.out_x[st.coff + sp->col_perm[j]] = NAN;
        for (int i = tid; i < m; i += nthreads) p.out_y[st.roff + sp->row_perm[i]] = NAN;
        if (tid == 0) {
            p.out_status[inst] = kStatusInvalid;
            p.out_iters[inst] = 0;
            if (p.hand_iters) p.hand_iters[inst] = 0;
            p.out_obj[inst] = NAN;
            for (int k = 0; k < kMetrics; ++k) p.out_metrics[static_cast<int64_t>(inst) * kMetrics + k] = NAN;
            if (p.out_omega) p.out_omega[inst] = st.omega;
        }
        st.inst = -1;
        store_slot(s_st, slot, st);
        return;
    }
    st.eta = sp->eta;
    OpsView A, T;
    pair_views(g, &A, &T);
    const PairOffsets o = pair_offsets(g.L);
    double v[kRed];
#pragma unroll
    for (int qq = 0; qq < kRed; ++qq) v[qq] = 0.0;
    kkt_partials_body<true, false, false>(sp, A, T, o.xbar, o.y, b.px0, b.py0, b.cs, b.ls, b.us, b.bs, b.dcand,
                                        b.rcand, true, lane_id(), v, nopatch);
    block_reduce_body(v, s_red, s_tot);
    st.cinf = s_tot[14];
    const Metrics M = evaluate(s_tot, st.omega, p.tol_p, p.tol_d, p.tol_g);
    int status = -1;
    if (M.conv) status = p.final_status;
    else if (p.max_iters <= 0) status = M.nan ? kStatusNumerical : kStatusIterationLimit;
    if (status >= 0) {
        finish_pair_slot(p, g, slot, inst, st.coff, st.roff, 0, 0, st.omega, status, M);
        st.inst = -1;
        store_slot(s_st, slot, st);
        return;
    }
    recentre_pair(sp, o, slot, b.px0, b.py0, b.dcand, b.rcand, b.ls, b.us);
    st.early = p.hint_iters == nullptr || p.hint_iters[inst] < p.check_every;
    st.r_restart = INFINITY;
    st.r_prev = INFINITY;
    st.best_err = INFINITY;
    slot_next(st, p);
    store_slot(s_st, slot, st);
}

// The convergence test of slot `slot` after a check iteration (its
// candidate is in the buffer cur ^ 1): termination, stall, hand-off, cold
// fallback and restart rules of pdhg_recentred.  All threads call it.
__device__ __noinline__ void check_pair_slot(const KernelParams& p, const PairStage& g, PairSlot* s_st, int slot,
                                             bool full, double pdx2, double pdxa2, double pdy2, double pdya2,
                                             double (*s_red)[kRed], double* s_tot) {
    const DevSpecies* sp = g.sp;
    const int n = sp->n, m = sp->m, tid = threadIdx.x, nthreads = blockDim.x;
    const PairSlab b = pair_slab(p, g.L, slot);
    const Patches nopatch{0, nullptr, nullptr, nullptr, nullptr};
    PairSlot st = s_st[slot];
    OpsView A, T;
    pair_views(g, &A, &T);
    const PairOffsets o = pair_offsets(g.L);
    double v[kRed];
#pragma unroll
    for (int qq = 0; qq < kRed; ++qq) v[qq] = 0.0;
    v[5] = pdx2;
    v[6] = pdy2;
    v[7] = pdxa2;
    v[8] = pdya2;
    kkt_partials_body<true, false, false>(sp, A, T, o.xbar, o.y, b.X(st.cur ^ 1), b.Y(st.cur ^ 1), b.cs, b.ls, b.us,
                                        b.bs, b.dcand, b.rcand, false, lane_id(), v, nopatch);
    block_reduce_body(v, s_red, s_tot);
    if (tid == 0) s_tot[14] = st.cinf;
    __syncthreads();
    const Metrics M = evaluate(s_tot, st.omega, p.tol_p, p.tol_d, p.tol_g);
    const double nx = sqrt(s_tot[7]), ny = sqrt(s_tot[8]);
    __syncthreads();  // s_tot is rewritten by the other slot's test
    st.ev = st.cur ^ 1;
    int status = -1;
    if (M.nan || !isfinite(M.r)) status = kStatusNumerical;
    else if (M.conv) status = p.final_status;
    else if (st.it >= p.max_iters) status = kStatusIterationLimit;
    if (status < 0 && full) {
        const double e = fmax(fmax(M.primal / (1.0 + M.xinf), M.dual / (1.0 + M.cinf)), fmax(M.rgap, M.kgap));
        if (e < 0.5 * st.best_err) {
            st.best_err = e;
            st.stall = 0;
        } else {
            ++st.stall;
        }
        if (p.stall_checks > 0 && st.stall >= p.stall_checks && e <= p.floor_tol && floor_accepts(M, p))
            status = p.final_status;
        else if (p.handoff_on_stall > 0 && st.stall >= p.handoff_on_stall)
            status = kStatusHandoff;
    }
    if (status >= 0) {
        finish_pair_slot(p, g, slot, st.inst, st.coff, st.roff, st.ev, st.it, st.omega, status, M);
        st.inst = -1;
    } else if (full && p.fallback_iters > 0 && !st.fell_back && st.it >= p.fallback_iters &&
               (p.warm_x != nullptr || p.warm_y != nullptr)) {
        // cold fallback: evaluate the cold point in the candidate buffer
        // and re-centre there
        st.fell_back = true;
        st.omega = 1.0;
        double* cx = b.X(st.cur ^ 1);
        double* cyv = b.Y(st.cur ^ 1);
        for (int j = tid; j < n; j += nthreads) cx[j] = 0.0 < b.ls[j] ? b.ls[j] : (0.0 > b.us[j] ? b.us[j] : 0.0);
        for (int i = tid; i < m; i += nthreads) cyv[i] = 0.0;
        __syncthreads();
        double vv[kRed];
#pragma unroll
        for (int qq = 0; qq < kRed; ++qq) vv[qq] = 0.0;
        kkt_partials_body<true, false, false>(sp, A, T, o.xbar, o.y, cx, cyv, b.cs, b.ls, b.us, b.bs, b.dcand,
                                            b.rcand, false, lane_id(), vv, nopatch);
        block_reduce_body(vv, s_red, s_tot);
        st.cur ^= 1;
        st.ev = st.cur;
        recentre_pair(sp, o, slot, b.X(st.cur), b.Y(st.cur), b.dcand, b.rcand, b.ls, b.us);
        st.k = 0;
        st.r_restart = INFINITY;
        st.r_prev = INFINITY;
        st.best_err = INFINITY;
        st.stall = 0;
    } else if (full && p.restarts &&
               (M.r <= kBetaSufficient * st.r_restart || (M.r <= kBetaNecessary * st.r_restart && M.r > st.r_prev) ||
                st.k >= kBetaArtificial * st.it)) {
        if (nx > 1e-10 && ny > 1e-10)
            st.omega = exp(__fma_rn(p.omega_smoothing, log(ny / nx), (1.0 - p.omega_smoothing) * log(st.omega)));
        st.cur ^= 1;  // the candidate becomes the base
        recentre_pair(sp, o, slot, b.X(st.cur), b.Y(st.cur), b.dcand, b.rcand, b.ls, b.us);
        st.k = 0;
        st.r_restart = M.r;
        st.r_prev = INFINITY;
    } else if (full) {
        st.r_prev = M.r;
    }
    if (st.inst >= 0) slot_next(st, p);
    store_slot(s_st, slot, st);
}

template <int MAXT>
__global__ void __launch_bounds__(MAXT, 1) pdhg_recentred_pair(const __grid_constant__ KernelParams p) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ double s_red[MAXT / 32][kRed];
    __shared__ double s_tot[kRed];
    __shared__ int s_q;
    __shared__ PairSlot s_st[2];
    __shared__ PairStage s_g;
    const int tid = threadIdx.x;
    const int warps = blockDim.x >> 5;
    const int count = p.count_dev ? *p.count_dev : p.count;
    if (tid < 2) s_st[tid].inst = -1;
    __syncthreads();
    int staged = -1, pending = -1;
    bool drained = false;

    for (;;) {
        // ---- fill the free slots from the work queue ----
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            while (s_st[s].inst < 0 && !drained) {
                int q = pending;
                if (q < 0) {
                    if (tid == 0) s_q = atomicAdd(p.queue, 1);
                    __syncthreads();
                    q = s_q;
                    __syncthreads();  // s_q is rewritten by the next fetch
                }
                if (q >= count) {
                    drained = true;
                    break;
                }
                const int inst = p.order[q];
                const int species = p.inst_species[inst];
                if (species != staged) {
                    if (s_st[s ^ 1].inst >= 0) {  // the other slot still runs the staged species
                        pending = q;
                        break;
                    }
                    // the species' layout record and context into shared memory
                    constexpr int words = static_cast<int>(sizeof(Layout) / sizeof(int64_t));
                    if (tid < words)
                        reinterpret_cast<int64_t*>(&s_g.L)[tid] =
                            reinterpret_cast<const int64_t*>(p.layouts + species)[tid];
                    if (tid == 0) {
                        const DevSpecies* sp = p.species + species;
                        s_g.sp = sp;
                        s_g.n = sp->n;
                        s_g.m = sp->m;
                        s_g.neq = sp->neq;
                    }
                    __syncthreads();
                    stage_species_pair(p.species + species, s_g.L, dyn_smem, warps);
                    __syncthreads();
                    staged = species;
                }
                pending = -1;
                start_pair_slot(p, s_g, s_st, s, inst, s_red, s_tot);
            }
        }
        const bool a0 = s_st[0].inst >= 0, a1 = s_st[1].inst >= 0;
        if (!a0 && !a1) {
            if (pending >= 0) continue;
            break;
        }

        // ---- one iteration of every busy slot ----
        bool chk[2], full[2];
        int cur[2];
        float tau[2], sig[2], w[2], wp[2];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const bool busy = s ? a1 : a0;
            if (busy) {
                cur[s] = s_st[s].cur;
                full[s] = s_st[s].full;
                chk[s] = s_st[s].chk;
                tau[s] = s_st[s].tau;
                sig[s] = s_st[s].sig;
                w[s] = s_st[s].w;
                wp[s] = s_st[s].wp;
            } else {
                cur[s] = 0;
                full[s] = chk[s] = false;
                tau[s] = sig[s] = w[s] = wp[s] = 0.0f;
            }
        }
        const float2 tau2 = make_float2(tau[0], tau[1]), sig2 = make_float2(sig[0], sig[1]);
        const float2 w2 = make_float2(w[0], w[1]), wp2 = make_float2(wp[0], wp[1]);
        const int n = s_g.n, m = s_g.m, neq = s_g.neq;
        const PairOffsets o = pair_offsets(s_g.L);
        OpsView A, T;
        pair_views(s_g, &A, &T);
        double pd[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) pd[q] = 0.0;
        if (chk[0] || chk[1]) {
            const PairSlab b0 = pair_slab(p, s_g.L, 0), b1 = pair_slab(p, s_g.L, 1);
            primal_pass_pair<true>(o, T, n, tau2, wp2, chk[0], chk[1], b0.X(cur[0]), b0.X(cur[0] ^ 1), b1.X(cur[1]),
                                   b1.X(cur[1] ^ 1), pd);
            __syncthreads();
            dual_pass_pair<true>(o, A, m, neq, sig2, w2, chk[0], chk[1], b0.Y(cur[0]), b0.Y(cur[0] ^ 1),
                                 b1.Y(cur[1]), b1.Y(cur[1] ^ 1), pd);
        } else {
            primal_pass_pair<false>(o, T, n, tau2, wp2, false, false, nullptr, nullptr, nullptr, nullptr, nullptr);
            __syncthreads();
            dual_pass_pair<false>(o, A, m, neq, sig2, w2, false, false, nullptr, nullptr, nullptr, nullptr, nullptr);
        }
        // every thread read this iteration's state before the barrier above
        if (tid == 0) {
            if (a0) {
                s_st[0].it += 1;
                s_st[0].k += 1;
                slot_next(s_st[0], p);
            }
            if (a1) {
                s_st[1].it += 1;
                s_st[1].k += 1;
                slot_next(s_st[1], p);
            }
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < 2; ++s)
            if (chk[s]) check_pair_slot(p, s_g, s_st, s, full[s], pd[4 * s], pd[4 * s + 1], pd[4 * s + 2], pd[4 * s + 3],
                                        s_red, s_tot);
    }
}

#define FBALP_INSTANTIATE_RECENTRED(MAXT)                                            \
    template __global__ void pdhg_recentred<MAXT, true, false, false>(const __grid_constant__ KernelParams);  \
    template __global__ void pdhg_recentred<MAXT, false, false, false>(const __grid_constant__ KernelParams); \
    template __global__ void pdhg_recentred<MAXT, true, true, false>(const __grid_constant__ KernelParams);   \
    template __global__ void pdhg_recentred<MAXT, false, true, false>(const __grid_constant__ KernelParams);  \
    template __global__ void pdhg_recentred<MAXT, true, false, true>(const __grid_constant__ KernelParams);   \
    template __global__ void pdhg_recentred<MAXT, false, false, true>(const __grid_constant__ KernelParams);
#define FBALP_INSTANTIATE(MAXT)                                               \
    template __global__ void pdhg_persistent<float, MAXT, 0>(const __grid_constant__ KernelParams);   \
    template __global__ void pdhg_persistent<float, MAXT, 1>(const __grid_constant__ KernelParams);   \
    template __global__ void pdhg_persistent<double, MAXT, 0>(const __grid_constant__ KernelParams);  \
    template __global__ void pdhg_persistent<double, MAXT, 1>(const __grid_constant__ KernelParams);  \
    template __global__ void pdhg_persistent<double, MAXT, 2>(const __grid_constant__ KernelParams);  \
    FBALP_INSTANTIATE_RECENTRED(MAXT)
FBALP_INSTANTIATE(512)
FBALP_INSTANTIATE(1024)
// the re-centred kernel also at 768 threads (an 85-register budget: more
// warps per scheduler to hide shared-memory latency)
FBALP_INSTANTIATE_RECENTRED(768)
template __global__ void pdhg_recentred_pair<512>(const __grid_constant__ KernelParams);
template __global__ void pdhg_recentred_pair<640>(const __grid_constant__ KernelParams);
template __global__ void pdhg_recentred_pair<768>(const __grid_constant__ KernelParams);
template __global__ void pdhg_recentred_pair<1024>(const __grid_constant__ KernelParams);
#undef FBALP_INSTANTIATE
#undef FBALP_INSTANTIATE_RECENTRED

// Blocks of up to 512 threads use the variant with a 128-register budget,
// larger blocks the 64-register one.  `fast`: FP32 launches take the
// shared-memory-only variant, FP64 launches the unscaled staged one.
template <int MAXT>
static const void* symbol_for(bool fp64, bool fast) {
    if (fp64)
        return fast ? reinterpret_cast<const void*>(&pdhg_persistent<double, MAXT, 2>)
                    : reinterpret_cast<const void*>(&pdhg_persistent<double, MAXT, 0>);
    return fast ? reinterpret_cast<const void*>(&pdhg_persistent<float, MAXT, 1>)
                : reinterpret_cast<const void*>(&pdhg_persistent<float, MAXT, 0>);
}

const void* kernel_symbol(bool fp64, int threads, bool fast) {
    return threads <= 512 ? symbol_for<512>(fp64, fast) : symbol_for<1024>(fp64, fast);
}

template <int MAXT>
static void launch_for(bool fp64, bool fast, int grid, int threads, size_t smem, cudaStream_t stream,
                       const KernelParams& p) {
    if (fp64) {
        if (fast) pdhg_persistent<double, MAXT, 2><<<grid, threads, smem, stream>>>(p);
        else pdhg_persistent<double, MAXT, 0><<<grid, threads, smem, stream>>>(p);
    } else {
        if (fast) pdhg_persistent<float, MAXT, 1><<<grid, threads, smem, stream>>>(p);
        else pdhg_persistent<float, MAXT, 0><<<grid, threads, smem, stream>>>(p);
    }
}

cudaError_t launch_pdhg(bool fp64, bool fast, int grid, int threads, size_t smem, cudaStream_t stream,
                        const KernelParams& p) {
    if (threads <= 512) launch_for<512>(fp64, fast, grid, threads, smem, stream, p);
    else launch_for<1024>(fp64, fast, grid, threads, smem, stream, p);
    return cudaGetLastError();
}

// `patched`: the variant that applies per-instance patched entries (launched
// only for batches that bind patch values; the other variant has none of
// that code); `f32`: FP32 matrix values (unpatched batches only).
template <int MAXT>
static const void* recentred_for(bool staged, bool patched, bool f32) {
    if (f32)
        return staged ? reinterpret_cast<const void*>(&pdhg_recentred<MAXT, true, false, true>)
                      : reinterpret_cast<const void*>(&pdhg_recentred<MAXT, false, false, true>);
    if (patched)
        return staged ? reinterpret_cast<const void*>(&pdhg_recentred<MAXT, true, true, false>)
                      : reinterpret_cast<const void*>(&pdhg_recentred<MAXT, false, true, false>);
    return staged ? reinterpret_cast<const void*>(&pdhg_recentred<MAXT, true, false, false>)
                  : reinterpret_cast<const void*>(&pdhg_recentred<MAXT, false, false, false>);
}

const void* recentred_symbol(int threads, bool staged, bool patched, bool f32) {
    if (threads <= 512) return recentred_for<512>(staged, patched, f32);
    if (threads <= 768) return recentred_for<768>(staged, patched, f32);
    return recentred_for<1024>(staged, patched, f32);
}

template <int MAXT>
static void launch_recentred_for(bool staged, bool patched, bool f32, int grid, int threads, size_t smem,
                                 cudaStream_t stream, const KernelParams& p) {
    if (f32) {
        if (staged) pdhg_recentred<MAXT, true, false, true><<<grid, threads, smem, stream>>>(p);
        else pdhg_recentred<MAXT, false, false, true><<<grid, threads, smem, stream>>>(p);
    } else if (patched) {
        if (staged) pdhg_recentred<MAXT, true, true, false><<<grid, threads, smem, stream>>>(p);
        else pdhg_recentred<MAXT, false, true, false><<<grid, threads, smem, stream>>>(p);
    } else {
        if (staged) pdhg_recentred<MAXT, true, false, false><<<grid, threads, smem, stream>>>(p);
        else pdhg_recentred<MAXT, false, false, false><<<grid, threads, smem, stream>>>(p);
    }
}

cudaError_t launch_recentred(bool staged, bool patched, int grid, int threads, size_t smem, cudaStream_t stream,
                             const KernelParams& p, bool f32) {
    if (threads <= 512) launch_recentred_for<512>(staged, patched, f32, grid, threads, smem, stream, p);
    else if (threads <= 768) launch_recentred_for<768>(staged, patched, f32, grid, threads, smem, stream, p);
    else launch_recentred_for<1024>(staged, patched, f32, grid, threads, smem, stream, p);
    return cudaGetLastError();
}

const void* pair_symbol(int threads) {
    if (threads <= 512) return reinterpret_cast<const void*>(&pdhg_recentred_pair<512>);
    if (threads <= 640) return reinterpret_cast<const void*>(&pdhg_recentred_pair<640>);
    if (threads <= 768) return reinterpret_cast<const void*>(&pdhg_recentred_pair<768>);
    return reinterpret_cast<const void*>(&pdhg_recentred_pair<1024>);
}

cudaError_t launch_pair(int grid, int threads, size_t smem, cudaStream_t stream, const KernelParams& p) {
    if (threads <= 512) pdhg_recentred_pair<512><<<grid, threads, smem, stream>>>(p);
    else if (threads <= 640) pdhg_recentred_pair<640><<<grid, threads, smem, stream>>>(p);
    else if (threads <= 768) pdhg_recentred_pair<768><<<grid, threads, smem, stream>>>(p);
    else pdhg_recentred_pair<1024><<<grid, threads, smem, stream>>>(p);
    return cudaGetLastError();
}

}  // namespace fbalp
