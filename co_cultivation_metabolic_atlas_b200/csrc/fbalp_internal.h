// Constants and helpers shared by the host engine and the kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pdhg_kernel.cuh"

namespace fbalp {

constexpr int kMetrics = 8;
constexpr int kRedSums = 10;
constexpr int kArrayCount = 11;
constexpr int kMaxThreads = 512;

constexpr int kStatusOptimal = 0;
constexpr int kStatusIterationLimit = 1;
constexpr int kStatusNumerical = 2;
constexpr int kStatusInvalid = 3;
constexpr int kStatusNotRun = 4;
constexpr int kStatusHandoff = 5;

// Restart rule of the Halpern scheme (Lu & Yang; cuPDLPx) and the PDLP
// primal-weight smoothing.
constexpr double kBetaSufficient = 0.2;
constexpr double kBetaNecessary = 0.8;
constexpr double kBetaArtificial = 0.36;
constexpr double kOmegaSmoothing = 0.5;

// Per-instance arrays in placement priority order:
// xbar, y, x, xa, ya, c, l, u, b, xs, ys  (gather targets carry a zero slot).
__host__ __device__ inline void array_sizes(int n, int m, int64_t* s) {
    const int64_t cols[kArrayCount] = {n + 1, 0, n, n, 0, n, n, n, 0, n + 1, 0};
    const int64_t rows[kArrayCount] = {0, m + 1, 0, 0, m, 0, 0, 0, m, 0, m + 1};
    for (int a = 0; a < kArrayCount; ++a) s[a] = ((cols[a] + rows[a]) + 3) & ~int64_t(3);
}

// Elements that do not fit into `smem_elems` (first-fit in priority order).
__host__ __device__ inline int64_t spill_elems(int n, int m, int64_t smem_elems) {
    int64_t s[kArrayCount];
    array_sizes(n, m, s);
    int64_t so = 0, go = 0;
    for (int a = 0; a < kArrayCount; ++a) {
        if (so + s[a] <= smem_elems) so += s[a];
        else go += s[a];
    }
    return go;
}

__host__ __device__ inline int64_t total_elems(int n, int m) {
    int64_t s[kArrayCount];
    array_sizes(n, m, s);
    int64_t t = 0;
    for (int a = 0; a < kArrayCount; ++a) t += s[a];
    return t;
}

const void* kernel_symbol(bool fp64);
cudaError_t launch_pdhg(bool fp64, int grid, int threads, size_t smem, cudaStream_t stream,
                        const KernelParams& p);

}  // namespace fbalp
