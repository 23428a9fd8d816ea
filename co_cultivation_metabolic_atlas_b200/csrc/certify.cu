// Original-LP certificate of solutions of diagonally scaled LPs, one launch
// for a whole batch (C ABI: fbalp_scaled_certificate in include/fbalp.h).
//
// Every instance solved the LP  A_i w (=,<=) b_i,  l_i <= w <= u_i,  min c_i.w
// whose matrix is a shared template plus per-instance patched entries,
// A_i = A + sum_q delta_iq e_{r_q} e_{c_q}^T, and which is the original LP
// under positive diagonal scalings: A_i = R A_orig D^{-1}, b_i = R b_orig,
// w = D v, c_i = D^{-1} c_orig.  R and D are given per row / column by a
// group index into a per-instance scale table.  The certificate is the
// original LP's, evaluated from the scaled quantities:
//   primal = max( |A w - b|_eq / R, (A w - b)_ub^+ / R, bound violation / D )
//   dual   = max( (R y)_ub^+, (D d)^+ where l = -inf, (-D d)^+ where u = +inf )
//   gap    = ( sum |d (w - active bound)| + sum_ub |y (b - A w)| ) / max(1, |c.w|)
// (complementarity terms and the objective are invariant under the
// scalings), with d = c - A^T y.  NaN anywhere makes all three NaN.
//
// One CTA per instance (grid-stride over instances); the template's CSR and
// its transpose are read from L2, each instance's vectors once.
#include <cmath>
#include <cstdint>

#include "../../include/fbalp.h"
#include "engine_state.h"

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct CertArgs {
    int count, rows, cols, neq, npatch, groups;
    const int32_t *a_ptr, *a_idx, *at_ptr, *at_idx;
    const double *a_val, *at_val;
    const int32_t *prow, *pcol;
    const double* deltas;
    const double *x, *y, *c, *l, *u, *b;
    const int32_t *row_group, *col_group;
    const double* table;
    double *primal, *dual, *gap;
};

__global__ void __launch_bounds__(kThreads) scaled_certificate_kernel(CertArgs a) {
    __shared__ double s_red[4][kThreads / 32];
    __shared__ int s_prow[FBALP_MAX_PATCHES], s_pcol[FBALP_MAX_PATCHES];
    __shared__ double s_dv[FBALP_MAX_PATCHES];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int inst = blockIdx.x; inst < a.count; inst += gridDim.x) {
        const int64_t xo = static_cast<int64_t>(inst) * a.cols;
        const int64_t yo = static_cast<int64_t>(inst) * a.rows;
        const double* x = a.x + xo;
        const double* y = a.y + yo;
        const double* tab = a.table + static_cast<int64_t>(inst) * a.groups;
        if (tid < a.npatch) {
            s_prow[tid] = a.prow[tid];
            s_pcol[tid] = a.pcol[tid];
            s_dv[tid] = a.deltas ? a.deltas[static_cast<int64_t>(inst) * a.npatch + tid] : 0.0;
        }
        __syncthreads();
        double pmax = 0.0, dmax = 0.0, comp = 0.0, cx = 0.0;
        bool bad = false;
        // rows: activity, residual, inequality duals
        for (int i = tid; i < a.rows; i += kThreads) {
            double act = 0.0;
            for (int k = a.a_ptr[i]; k < a.a_ptr[i + 1]; ++k) act = fma(a.a_val[k], x[a.a_idx[k]], act);
            for (int q = 0; q < a.npatch; ++q)
                if (s_prow[q] == i) act = fma(s_dv[q], x[s_pcol[q]], act);
            const double R = tab[a.row_group[i]];
            const double res = act - a.b[yo + i];
            const double yi = y[i];
            bad |= isnan(res) || isnan(yi);
            if (i < a.neq) {
                pmax = fmax(pmax, fabs(res) / R);
            } else {
                pmax = fmax(pmax, fmax(res, 0.0) / R);
                dmax = fmax(dmax, fmax(yi * R, 0.0));
                comp += fabs(yi * res);
            }
        }
        // columns: reduced costs, bounds, complementarity, objective
        for (int j = tid; j < a.cols; j += kThreads) {
            double aty = 0.0;
            for (int k = a.at_ptr[j]; k < a.at_ptr[j + 1]; ++k) aty = fma(a.at_val[k], y[a.at_idx[k]], aty);
            for (int q = 0; q < a.npatch; ++q)
                if (s_pcol[q] == j) aty = fma(s_dv[q], y[s_prow[q]], aty);
            const double D = tab[a.col_group[j]];
            const double xj = x[j], cj = a.c[xo + j], lj = a.l[xo + j], uj = a.u[xo + j];
            const double d = cj - aty;
            bad |= isnan(d) || isnan(xj);
            const double viol = fmax(fmax(lj - xj, xj - uj), 0.0);
            if (isfinite(viol)) pmax = fmax(pmax, viol / D);
            const double dv = d * D;
            if (isinf(lj)) dmax = fmax(dmax, fmax(dv, 0.0));
            if (isinf(uj)) dmax = fmax(dmax, fmax(-dv, 0.0));
            const double t = d >= 0.0 ? lj : uj;
            if (isfinite(t)) comp += fabs(d * (xj - t));
            cx = fma(cj, xj, cx);
        }
        // block reductions
        const double v0 = warp_max(pmax), v1 = warp_max(dmax), v2 = warp_sum(comp), v3 = warp_sum(cx);
        const unsigned nan_any = __ballot_sync(0xffffffffu, bad);
        if (lane == 0) {
            s_red[0][warp] = v0;
            s_red[1][warp] = v1;
            s_red[2][warp] = v2;
            s_red[3][warp] = nan_any ? NAN : v3;
        }
        __syncthreads();
        if (tid == 0) {
            double p = 0.0, dd = 0.0, cs = 0.0, o = 0.0;
            bool nanf = false;
            for (int w = 0; w < kThreads / 32; ++w) {
                p = fmax(p, s_red[0][w]);
                dd = fmax(dd, s_red[1][w]);
                cs += s_red[2][w];
                if (isnan(s_red[3][w])) nanf = true;
                else o += s_red[3][w];
            }
            if (nanf) {
                a.primal[inst] = a.dual[inst] = a.gap[inst] = NAN;
            } else {
                a.primal[inst] = p;
                a.dual[inst] = dd;
                a.gap[inst] = cs / fmax(1.0, fabs(o));
            }
        }
        __syncthreads();
    }
}

}  // namespace

extern "C" int fbalp_scaled_certificate(int32_t count, int32_t rows, int32_t cols, int32_t neq,
                                        const int32_t* a_ptr, const int32_t* a_idx, const double* a_val,
                                        const int32_t* at_ptr, const int32_t* at_idx, const double* at_val,
                                        int32_t npatch, const int32_t* patch_rows, const int32_t* patch_cols,
                                        const double* deltas, const double* x, const double* y, const double* cost,
                                        const double* lower, const double* upper, const double* rhs,
                                        const int32_t* row_group, const int32_t* col_group, int32_t groups,
                                        const double* scale_table, double* out_primal, double* out_dual,
                                        double* out_gap, void* stream) {
    if (count < 0 || rows < 0 || cols < 1 || neq < 0 || neq > rows || groups < 1)
        return fail(FBALP_ERR_INVALID, "invalid certificate dimensions");
    if (npatch < 0 || npatch > FBALP_MAX_PATCHES || (npatch > 0 && (!patch_rows || !patch_cols)))
        return fail(FBALP_ERR_INVALID, "npatch must be in [0, FBALP_MAX_PATCHES] with its row/column arrays");
    if (!a_ptr || !at_ptr || (rows > 0 && (!y || !rhs || !row_group)) || !x || !cost || !lower || !upper ||
        !col_group || !scale_table || !out_primal || !out_dual || !out_gap)
        return fail(FBALP_ERR_INVALID, "a required array is NULL");
    if (count == 0) return FBALP_OK;
    CertArgs a{count, rows, cols, neq, npatch, groups, a_ptr, a_idx, at_ptr, at_idx, a_val, at_val,
               patch_rows, patch_cols, deltas, x, y, cost, lower, upper, rhs, row_group, col_group,
               scale_table, out_primal, out_dual, out_gap};
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                  cudaSuccess)
        return fail(FBALP_ERR_CUDA, "cannot query the device");
    const int grid = count < 8 * sms ? count : 8 * sms;
    scaled_certificate_kernel<<<grid, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(a);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return fail(FBALP_ERR_CUDA, cudaGetErrorString(err));
    return FBALP_OK;
}
