/*
 * fbalp_mlp.h -- C ABI of the BF16 tensor-core kernels behind the learned
 * warm start (an MLP from medium state to primal-dual LP solutions).
 *
 * The reference's warm-start model is a PyTorch MLP/GRU (`src/temporal_lp_model.py:58-142`,
 * TemporalLPModel; trained by `scripts/train_temporal_lp.py:23-88` with Adam on an MSE
 * loss).  These entry points are the hand-written sm_100a replacements of its
 * `torch.nn.Linear` forward/backward, GELU, MSE gradient and Adam update.
 *
 * All pointers are DEVICE pointers; `stream` is a cudaStream_t (NULL = legacy
 * default stream); calls are asynchronous.  BF16 tensors are raw 16-bit arrays.
 */
#ifndef FBALP_MLP_H
#define FBALP_MLP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FBALP_MLP_OK 0
#define FBALP_MLP_ERR_INVALID 1
#define FBALP_MLP_ERR_CUDA 2

#define FBALP_EPI_NONE 0
#define FBALP_EPI_BIAS 1
#define FBALP_EPI_BIAS_GELU 2

/* C[M,N] = alpha * op(A) op(B)^T  (+ bias[N])  (GELU, storing the
 * pre-activation into Z when Z != NULL).  op(A) is M x K: A[m*lda + k]
 * (transA = 0) or A[k*lda + m] (transA = 1); op(B) is N x K: B[n*ldb + k]
 * (transB = 0) or B[k*ldb + n] (transB = 1).  A, B are BF16; the FP32
 * accumulator lives in tensor memory (tcgen05.mma kind::f16).  Results go to
 * C32 (FP32; added to its contents when accumulate_c = 1) and/or C16 (BF16),
 * row stride ldc.  Operands that start on a 16-byte boundary with a row
 * stride (lda, ldb) of a multiple of 8 elements are read by TMA; any other
 * operand is staged by ordinary loads (same results, slower).  Replaces torch.nn.Linear forward/backward in
 * `src/temporal_lp_model.py:58-142`. */
int fbalp_gemm_bf16(int M, int N, int K, const void* A, int lda, int transA, const void* B, int ldb,
                    int transB, const float* bias, int epilogue, float alpha, float* C32, void* C16,
                    int ldc, float* Z, int ldz, int accumulate_c, void* stream);

/* Reads (and optionally clears) the device flag raised when a GEMM's bounded
 * mbarrier wait timed out (synchronous). */
int fbalp_mlp_error_flag(int* out, int clear);

/* dZ = dH * GELU'(Z) elementwise (FP32 and/or BF16 output). */
int fbalp_gelu_backward(int64_t count, const float* dH, const float* Z, float* dZ32, void* dZ16,
                        void* stream);

/* dY = scale * (Y - T); *loss += sum (Y - T)^2 (FP64 accumulation). */
int fbalp_mse_grad(int rows, int cols, const float* Y, const float* T, float scale, float* dY32,
                   void* dY16, double* loss, void* stream);

/* out[c] = sum_r X[r, c]  (bias gradients). */
int fbalp_column_sum(int rows, int cols, const float* X, float* out, void* stream);

/* Adam on FP32 master weights (bias-corrected, decoupled weight decay);
 * refreshes the BF16 copy w16 when non-NULL.  Replaces torch.optim.Adam in
 * `scripts/train_temporal_lp.py:23-88`. */
int fbalp_adam_step(int64_t count, float* w, const float* g, float* m, float* v, void* w16, float lr,
                    float beta1, float beta2, float eps, int step, float weight_decay, void* stream);

/* y = bf16(x). */
int fbalp_to_bf16(int64_t count, const float* x, void* y, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FBALP_MLP_H */
