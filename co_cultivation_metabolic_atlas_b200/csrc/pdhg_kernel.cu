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

// One SELL-32 slice row product: lane `lane` of the warp owns row
// (slice*32 + lane); element k of that row sits at base + 32*k + lane, so
// every step of the loop is one coalesced load of 32 indices and 32 values.
template <typename T, typename V>
__device__ __forceinline__ T slice_dot(const int32_t* __restrict__ idx, const V* __restrict__ val,
                                       int base, int len, int lane, const T* g) {
    const int32_t* ip = idx + base + lane;
    const V* vp = val + base + lane;
    T acc0 = T(0), acc1 = T(0);
    int k = 0;
    for (; k + 1 < len; k += 2) {
        const int i0 = __ldg(ip + (k << 5));
        const int i1 = __ldg(ip + ((k + 1) << 5));
        const V v0 = __ldg(vp + (k << 5));
        const V v1 = __ldg(vp + ((k + 1) << 5));
        acc0 = fma(static_cast<T>(v0), g[i0], acc0);
        acc1 = fma(static_cast<T>(v1), g[i1], acc1);
    }
    if (k < len) acc0 = fma(static_cast<T>(__ldg(vp + (k << 5))), g[__ldg(ip + (k << 5))], acc0);
    return acc0 + acc1;
}

// FP64 product for the convergence test, whatever the iterate precision.
template <typename T>
__device__ __forceinline__ double slice_dot64(const int32_t* __restrict__ idx,
                                              const double* __restrict__ val, int base, int len,
                                              int lane, const T* g) {
    const int32_t* ip = idx + base + lane;
    const double* vp = val + base + lane;
    double acc = 0.0;
    for (int k = 0; k < len; ++k)
        acc = fma(__ldg(vp + (k << 5)), static_cast<double>(g[__ldg(ip + (k << 5))]), acc);
    return acc;
}

template <typename T> struct Arrays {
    T *xbar, *y, *x, *xa, *ya, *cs, *ls, *us, *bs, *xs, *ys;
};

template <typename T>
__device__ void place_arrays(Arrays<T>& A, T* smem, int64_t smem_elems, T* slab, int n, int m) {
    int64_t sizes[kArrayCount];
    array_sizes(n, m, sizes);
    T** ptrs[kArrayCount] = {&A.xbar, &A.y, &A.x, &A.xa, &A.ya, &A.cs, &A.ls, &A.us, &A.bs, &A.xs, &A.ys};
    int64_t so = 0, go = 0;
#pragma unroll
    for (int a = 0; a < kArrayCount; ++a) {
        const int64_t sz = sizes[a];
        if (so + sz <= smem_elems) {
            *ptrs[a] = smem + so;
            so += sz;
        } else {
            *ptrs[a] = slab + go;
            go += sz;
        }
    }
}

// Sums for q < kRedSums, maxima above.  Deterministic order.
__device__ void block_reduce(double* v, double (*s_red)[kRed], double* s_tot) {
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

// FP64 KKT quantities at the candidate (xs, ys); partial sums / maxima of
// this thread are added to v.  Index map of v (see also oracle/pdhg.py
// kkt_metrics):
//  0 c.x   1 b.y   2 sum bound-dual terms   3 bound complementarity
//  4 row complementarity   5 |xn-x|^2  6 |yn-y|^2  7 |xn-xa|^2  8 |yn-ya|^2
//  10 max primal row residual  11 max dual violation  12 max bound violation
//  13 |x|_inf  14 |c|_inf  15 NaN flag
template <typename T>
__device__ void kkt_partials(const DevSpecies* sp, const Arrays<T>& A, int warp, int lane,
                             double* v) {
    const int n = sp->n, m = sp->m, neq = sp->neq;
    for (int t = sp->at_sched_off[warp]; t < sp->at_sched_off[warp + 1]; ++t) {
        const int s = sp->at_sched[t];
        const int base = sp->at_off[s];
        const int len = (sp->at_off[s + 1] - base) >> 5;
        const double g = slice_dot64<T>(sp->at_idx, sp->at_v64, base, len, lane, A.ys);
        const int j = (s << 5) + lane;
        if (j < n) {
            const double dcj = sp->dc[j];
            const double c = A.cs[j], l = A.ls[j], u = A.us[j], xv = A.xs[j];
            const double r = c - g;
            v[0] += c * xv;
            if (r > 0.0) {
                if (isfinite(l)) v[2] += r * l;
                else v[11] = fmax(v[11], r / dcj);
            } else if (r < 0.0) {
                if (isfinite(u)) v[2] += r * u;
                else v[11] = fmax(v[11], -r / dcj);
            }
            const double tg = (r >= 0.0) ? l : u;
            if (isfinite(tg)) v[3] += fabs(r * (xv - tg));
            v[12] = fmax(v[12], fmax((l - xv) * dcj, (xv - u) * dcj));
            v[13] = fmax(v[13], fabs(xv * dcj));
            v[14] = fmax(v[14], fabs(c / dcj));
            if (isnan(g) || isnan(xv)) v[15] = 1.0;
        }
    }
    for (int t = sp->a_sched_off[warp]; t < sp->a_sched_off[warp + 1]; ++t) {
        const int s = sp->a_sched[t];
        const int base = sp->a_off[s];
        const int len = (sp->a_off[s + 1] - base) >> 5;
        const double h = slice_dot64<T>(sp->a_idx, sp->a_v64, base, len, lane, A.xs);
        const int i = (s << 5) + lane;
        if (i < m) {
            const double dri = sp->dr[i];
            const double b = A.bs[i], yv = A.ys[i];
            const double rt = h - b;
            const double ro = rt / dri;
            if (i < neq) {
                v[10] = fmax(v[10], fabs(ro));
            } else {
                v[10] = fmax(v[10], ro);
                v[4] += fabs(yv * rt);
                v[11] = fmax(v[11], yv * dri);
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
    M.r = sqrt(omega * s_tot[5] + s_tot[6] / omega);
    M.nan = s_tot[15] > 0.0 || !isfinite(M.pobj) || !isfinite(M.dobj) || !isfinite(M.kgap) ||
            !isfinite(M.primal);
    M.conv = !M.nan && M.primal <= tol_p * (1.0 + M.xinf) && M.dual <= tol_d * (1.0 + M.cinf) &&
             M.rgap <= tol_g && M.kgap <= tol_g;
    return M;
}

template <typename T>
__global__ void __launch_bounds__(kMaxWarps * 32, 2) pdhg_persistent(KernelParams p) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ double s_red[kMaxWarps][kRed];
    __shared__ double s_tot[kRed];
    __shared__ int s_inst;
    T* smem = reinterpret_cast<T*>(dyn_smem);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nthreads = blockDim.x;
    T* slab = p.spill ? reinterpret_cast<T*>(p.spill) + static_cast<int64_t>(blockIdx.x) * p.spill_stride
                      : nullptr;
    const T rho = static_cast<T>(p.rho);

    for (;;) {
        if (tid == 0) s_inst = atomicAdd(p.queue, 1);
        __syncthreads();
        const int q = s_inst;
        if (q >= p.count) break;
        const int inst = p.order[q];
        const DevSpecies* __restrict__ sp = p.species + p.inst_species[inst];
        const int n = sp->n, m = sp->m, neq = sp->neq;
        const int64_t coff = p.col_off[inst], roff = p.row_off[inst];
        Arrays<T> A;
        place_arrays<T>(A, smem, p.smem_elems, slab, n, m);

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
        }
        if (tid == 0) {
            A.xbar[n] = T(0);
            A.xs[n] = T(0);
            A.y[m] = T(0);
            A.ys[m] = T(0);
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

        // ---- iteration-0 test of the (projected) starting point ----
        const double eta = sp->eta;
        int status = -1;
        Metrics M;
        {
            double v[kRed];
#pragma unroll
            for (int qq = 0; qq < kRed; ++qq) v[qq] = 0.0;
            kkt_partials<T>(sp, A, warp, lane, v);
            block_reduce(v, s_red, s_tot);
            M = evaluate(s_tot, omega, p.tol_p, p.tol_d, p.tol_g);
            if (M.conv) status = p.final_status;
            else if (p.max_iters <= 0) status = M.nan ? kStatusNumerical : kStatusIterationLimit;
        }

        int k = 0, it = 0;
        double r_restart = INFINITY, r_prev = INFINITY;
        const int aw0 = sp->a_sched_off[warp], aw1 = sp->a_sched_off[warp + 1];
        const int tw0 = sp->at_sched_off[warp], tw1 = sp->at_sched_off[warp + 1];
        const T* __restrict__ atv = Vals<T>::at(sp);
        const T* __restrict__ av = Vals<T>::a(sp);
        while (status < 0) {
            ++it;
            const bool check = (it % p.check_every == 0) || (it >= p.max_iters);
            const T tau = static_cast<T>(eta / omega), sigma = static_cast<T>(eta * omega);
            const T w = static_cast<T>((k + 1.0) / (k + 2.0));
            const T w1 = T(1) - w;
            double pdx2 = 0.0, pdy2 = 0.0, pdxa2 = 0.0, pdya2 = 0.0;
            // primal pass: g = A^T y, projected step, extrapolation, Halpern
            for (int t = tw0; t < tw1; ++t) {
                const int s = sp->at_sched[t];
                const int base = sp->at_off[s];
                const int len = (sp->at_off[s + 1] - base) >> 5;
                const T g = slice_dot<T>(sp->at_idx, atv, base, len, lane, A.y);
                const int j = (s << 5) + lane;
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
            __syncthreads();
            // dual pass: h = A xbar, projected dual step, Halpern
            for (int t = aw0; t < aw1; ++t) {
                const int s = sp->a_sched[t];
                const int base = sp->a_off[s];
                const int len = (sp->a_off[s + 1] - base) >> 5;
                const T h = slice_dot<T>(sp->a_idx, av, base, len, lane, A.xbar);
                const int i = (s << 5) + lane;
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
            kkt_partials<T>(sp, A, warp, lane, v);
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
            if (p.restarts && (M.r <= kBetaSufficient * r_restart ||
                               (M.r <= kBetaNecessary * r_restart && M.r > r_prev) ||
                               k >= kBetaArtificial * it)) {
                const double nx = sqrt(s_tot[7]), ny = sqrt(s_tot[8]);
                if (nx > 1e-10 && ny > 1e-10)
                    omega = exp(kOmegaSmoothing * log(ny / nx) + (1.0 - kOmegaSmoothing) * log(omega));
                for (int j = tid; j < n; j += nthreads) {
                    const T xv = A.xs[j];
                    A.x[j] = xv;
                    A.xa[j] = xv;
                }
                for (int i = tid; i < m; i += nthreads) {
                    const T yv = A.ys[i];
                    A.y[i] = yv;
                    A.ya[i] = yv;
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
        for (int j = tid; j < n; j += nthreads) {
            const int jo = sp->col_perm[j];
            double xv = static_cast<double>(A.xs[j]) * sp->dc[j];
            if (p.clip_output) {
                const double lv = p.lower[coff + jo], uv = p.upper[coff + jo];
                xv = xv < lv ? lv : (xv > uv ? uv : xv);
            }
            p.out_x[coff + jo] = xv;
        }
        for (int i = tid; i < m; i += nthreads)
            p.out_y[roff + sp->row_perm[i]] = static_cast<double>(A.ys[i]) * sp->dr[i];
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

template __global__ void pdhg_persistent<float>(KernelParams);
template __global__ void pdhg_persistent<double>(KernelParams);

const void* kernel_symbol(bool fp64) {
    return fp64 ? reinterpret_cast<const void*>(&pdhg_persistent<double>)
                : reinterpret_cast<const void*>(&pdhg_persistent<float>);
}

cudaError_t launch_pdhg(bool fp64, int grid, int threads, size_t smem, cudaStream_t stream,
                        const KernelParams& p) {
    if (fp64) pdhg_persistent<double><<<grid, threads, smem, stream>>>(p);
    else pdhg_persistent<float><<<grid, threads, smem, stream>>>(p);
    return cudaGetLastError();
}

}  // namespace fbalp
