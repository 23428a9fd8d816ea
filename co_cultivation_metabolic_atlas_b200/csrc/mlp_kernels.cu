// BF16 tensor-core kernels of the learned warm start (sm_100a).
//
// gemm_tcgen05: C = alpha * op(A) op(B)^T (+ bias, + GELU), BF16 operands,
// FP32 accumulation in tensor memory.  One CTA of 128 threads computes a
// 128 x 128 tile: every thread stages its share of the 128 x 64 A and B
// K-slices into shared memory in the canonical K-major, no-swizzle UMMA
// layout (8-row x 16-byte core matrices), one elected thread issues four
// `tcgen05.mma.cta_group::1.kind::f16` (K = 16 each) per slice, and
// `tcgen05.commit` signals an mbarrier; the epilogue reads the accumulator
// with `tcgen05.ld.32x32b` (warp w owns TMEM lanes 32w..32w+31).  The
// loaders accept row-major or transposed operands, so the backward pass
// (dW = dY^T H, dH = dY W) needs no explicit transposes.  Two shared-memory
// stages let the loads of slice k+1 overlap the MMAs of slice k.
//
// gemm_tcgen05_tma is the same tile with its operands brought in by TMA
// (`cp.async.bulk.tensor.2d`, 128-byte swizzle, no multicast) through a
// three-stage mbarrier pipeline: one thread issues the loads and the MMAs,
// K-major operands as 128 x 64 boxes, transposed (MN-major) ones as two
// 64 x 64 boxes described to the MMA as MN-major, so the tensor core reads
// either storage directly.  It serves every call whose operands start on a
// 16-byte boundary with a row stride of a multiple of 8 elements (all calls
// of the warm-start network); gemm_tcgen05 serves the rest.  Epilogues store
// 16-byte vectors where the output allows it.
//
// Every mbarrier wait is bounded; on timeout the kernel raises an error flag
// (read by the host), skips the rest of the tile, waits (bounded) for its
// copies and MMAs in flight, frees its TMEM and returns.
#include <cuda.h>  // CUtensorMap and its enums; the encoder is looked up at run time
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/fbalp_mlp.h"

namespace fbalp_mlp {

constexpr int BM = 128, BN = 128, BK = 64;
constexpr int kThreads = 128;
constexpr int kStageBytes = (BM + BN) * BK * 2;  // A and B slices, 32 KB
constexpr int kStages = 2;
constexpr uint32_t kTmemCols = 128;
constexpr long long kWaitLimit = 1ll << 26;
constexpr int kTmaStages = 3;  // 96 KB of operand stages: two CTAs per SM
// an MN-major operand tile is two 64 (MN) x 64 (K) boxes of 8 KB
constexpr int kMnBoxBytes = 64 * BK * 2;
static_assert(2 * kMnBoxBytes == BM * BK * 2, "two MN-major boxes fill one operand tile");
constexpr int kTmaSmem = kTmaStages * kStageBytes + 1024;

__device__ int g_error = 0;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Canonical K-major interleaved offset (bytes) of element (row, k) of a
// 128 x 64 BF16 tile: core matrix (row/8, k/8) at (row/8)*1024 + (k/8)*128,
// row r%8 at +16*(r%8), element k%8 at +2*(k%8).  LBO = 128 B (next 8 K
// elements), SBO = 1024 B (next 8 rows).
__device__ __forceinline__ int tile_off(int row, int k) {
    return ((row >> 3) << 10) + ((k >> 3) << 7) + ((row & 7) << 4) + ((k & 7) << 1);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    const uint64_t lbo = 128 >> 4, sbo = 1024 >> 4;
    return (static_cast<uint64_t>((addr >> 4) & 0x3FFF)) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D = F32, A = B = BF16, both K-major.
__host__ __device__ constexpr uint32_t instr_desc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void mma_issue(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.u32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// tcgen05 shared-memory descriptor of a 128-byte-swizzled operand tile
// (layout type 2 in bits 61-63; LBO / SBO in bytes).
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Rows [r0, r0+128) x K-slice [k0, k0+64) of op(X) into a 16 KB tile: a
// K-major operand as one 64 x 128 box (row r at 128 r bytes, 8-row atoms of
// 1 KB), an MN-major one as two 64 x 64 boxes (K row k at 128 k bytes inside
// each; the second box holds rows r0+64..r0+127).  Both are 1 KB aligned.
__device__ __forceinline__ void tma_operand(unsigned char* dst, const CUtensorMap* map, int mn_major, int r0, int k0,
                                            uint64_t* bar) {
    if (!mn_major) {
        tma_load_2d(dst, map, k0, r0, bar);
    } else {
        tma_load_2d(dst, map, r0, k0, bar);
        tma_load_2d(dst + kMnBoxBytes, map, r0 + 64, k0, bar);
    }
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z) {
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

// Stage rows [r0, r0+128) x k-slice [k0, k0+64) of op(X) (op(X) is R x K;
// trans = 0: X[r*ld + k], trans = 1: X[k*ld + r]) into the canonical layout.
__device__ __forceinline__ void load_tile(unsigned char* dst, const __nv_bfloat16* X, int ld, int trans,
                                          int R, int K, int r0, int k0, bool vec_ok) {
    const int tid = threadIdx.x;
    if (!trans && vec_ok) {
        // 16-byte chunks: 128 rows x 8 chunks = 1024 chunks, 8 per thread
        for (int c = tid; c < BM * (BK / 8); c += kThreads) {
            const int row = c >> 3, kc = c & 7;
            const int r = r0 + row, k = k0 + kc * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (r < R && k + 8 <= K) {
                v = *reinterpret_cast<const uint4*>(X + static_cast<int64_t>(r) * ld + k);
            } else if (r < R) {
                __nv_bfloat16 tmp[8];
                for (int e = 0; e < 8; ++e)
                    tmp[e] = (k + e < K) ? X[static_cast<int64_t>(r) * ld + k + e] : __float2bfloat16(0.0f);
                v = *reinterpret_cast<uint4*>(tmp);
            }
            *reinterpret_cast<uint4*>(dst + tile_off(row, kc * 8)) = v;
        }
    } else if (trans) {
        // X[k*ld + r]: consecutive threads walk r (coalesced along r)
        for (int e = tid; e < BM * BK; e += kThreads) {
            const int row = e % BM, kk = e / BM;
            const int r = r0 + row, k = k0 + kk;
            __nv_bfloat16 v = __float2bfloat16(0.0f);
            if (r < R && k < K) v = X[static_cast<int64_t>(k) * ld + r];
            *reinterpret_cast<__nv_bfloat16*>(dst + tile_off(row, kk)) = v;
        }
    } else {
        for (int e = tid; e < BM * BK; e += kThreads) {
            const int row = e / BK, kk = e % BK;
            const int r = r0 + row, k = k0 + kk;
            __nv_bfloat16 v = __float2bfloat16(0.0f);
            if (r < R && k < K) v = X[static_cast<int64_t>(r) * ld + k];
            *reinterpret_cast<__nv_bfloat16*>(dst + tile_off(row, kk)) = v;
        }
    }
}

// 32 consecutive FP32 outputs of one row (n of them inside the matrix):
// eight 16-byte stores when the row segment is whole and aligned.
__device__ __forceinline__ void store_f32x32(float* p, const float* v, int n, bool vec, int accumulate) {
    if (n >= 32 && vec) {
#pragma unroll
        for (int j = 0; j < 32; j += 4) {
            float4 w = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
            if (accumulate) {
                const float4 o = *reinterpret_cast<const float4*>(p + j);
                w.x += o.x;
                w.y += o.y;
                w.z += o.z;
                w.w += o.w;
            }
            *reinterpret_cast<float4*>(p + j) = w;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 32; ++j)
            if (j < n) p[j] = accumulate ? p[j] + v[j] : v[j];
    }
}

__device__ __forceinline__ void store_bf16x32(__nv_bfloat16* p, const float* v, int n, bool vec) {
    if (n >= 32 && vec) {
#pragma unroll
        for (int j = 0; j < 32; j += 8) {
            __align__(16) __nv_bfloat16 t[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) t[e] = __float2bfloat16(v[j + e]);
            *reinterpret_cast<uint4*>(p + j) = *reinterpret_cast<const uint4*>(t);
        }
    } else {
#pragma unroll
        for (int j = 0; j < 32; ++j)
            if (j < n) p[j] = __float2bfloat16(v[j]);
    }
}

// Epilogue of a 128 x 128 tile: warp w reads TMEM lanes 32w..32w+31 (one
// output row per thread) in four 32-column chunks and writes alpha * acc
// (+ bias, GELU with the pre-activation kept in Z) to C32 / C16.
__device__ __forceinline__ void epilogue_tile(uint32_t tmem, int m0, int n0, int M, int N, const float* bias,
                                              int epilogue, float alpha, float* C32, __nv_bfloat16* C16, int ldc,
                                              float* Z, int ldz, int accumulate_c) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = m0 + warp * 32 + lane;
    const bool vec32 = C32 && (ldc & 3) == 0 && (reinterpret_cast<uintptr_t>(C32) & 15) == 0;
    const bool vec16 = C16 && (ldc & 7) == 0 && (reinterpret_cast<uintptr_t>(C16) & 15) == 0;
    const bool vecz = Z && (ldz & 3) == 0 && (reinterpret_cast<uintptr_t>(Z) & 15) == 0;
    for (int c0 = 0; c0 < BN; c0 += 32) {
        uint32_t r[32];
        const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0;
        __syncwarp();
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
            "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
              "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
              "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int col0 = n0 + c0;
        if (row < M && col0 < N) {
            const int n = N - col0;
            float v[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                v[j] = alpha * __uint_as_float(r[j]);
                if (epilogue >= FBALP_EPI_BIAS && bias && j < n) v[j] += bias[col0 + j];
            }
            if (epilogue == FBALP_EPI_BIAS_GELU) {
                if (Z) store_f32x32(Z + static_cast<int64_t>(row) * ldz + col0, v, n, vecz, 0);
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = gelu(v[j]);
            }
            const int64_t o = static_cast<int64_t>(row) * ldc + col0;
            if (C32) store_f32x32(C32 + o, v, n, vec32, accumulate_c);
            if (C16) store_bf16x32(C16 + o, v, n, vec16);
        }
    }
}

__global__ void __launch_bounds__(kThreads, 1)
gemm_tcgen05(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda, int transA,
             const __nv_bfloat16* __restrict__ B, int ldb, int transB, const float* __restrict__ bias,
             int epilogue, float alpha, float* __restrict__ C32, __nv_bfloat16* __restrict__ C16, int ldc,
             float* __restrict__ Z, int ldz, int accumulate_c) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[kStages];
    __shared__ uint32_t tmem_base_s;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    // 1024-byte aligned stage buffers
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem) + 1023) & ~uintptr_t(1023));

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_s)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_s;

    const bool vecA = ((lda & 7) == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0);
    const bool vecB = ((ldb & 7) == 0) && ((reinterpret_cast<uintptr_t>(B) & 15) == 0);
    const uint32_t idesc = instr_desc(BM, BN);
    const int ktiles = (K + BK - 1) / BK;
    uint32_t phase[kStages] = {0, 0};
    int ok = 1;
    int issued = 0;  // slices whose MMAs were committed
    for (int kt = 0; kt < ktiles; ++kt) {
        const int s = kt % kStages;
        unsigned char* sa = base + s * kStageBytes;
        unsigned char* sb = sa + BM * BK * 2;
        // the MMAs that last read this stage (slice kt - kStages) must be done
        if (kt >= kStages) {
            if (!mbar_wait(&bars[s], phase[s])) ok = 0;
            phase[s] ^= 1;
        }
        ok = __syncthreads_and(ok);
        if (!ok) break;
        load_tile(sa, A, lda, transA, M, K, m0, kt * BK, vecA);
        load_tile(sb, B, ldb, transB, N, K, n0, kt * BK, vecB);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
#pragma unroll
            for (int ks = 0; ks < BK / 16; ++ks) {
                // K = 16 step = two 8-element core-matrix columns = 256 bytes
                mma_issue(tmem, smem_desc(a0 + ks * 256), smem_desc(b0 + ks * 256), idesc,
                          (kt > 0 || ks > 0) ? 1u : 0u);
            }
            mma_commit(&bars[s]);
        }
        issued = kt + 1;
    }
    // drain: wait (bounded) for the commits not yet waited on, also after a
    // timeout, so that no MMA is in flight when the TMEM is released
    for (int kt = (issued > kStages ? issued - kStages : 0); kt < issued; ++kt) {
        const int s = kt % kStages;
        if (!mbar_wait(&bars[s], phase[s])) ok = 0;
        phase[s] ^= 1;
    }
    ok = __syncthreads_and(ok);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (ok && ktiles > 0)
        epilogue_tile(tmem, m0, n0, M, N, bias, epilogue, alpha, C32, C16, ldc, Z, ldz, accumulate_c);
    if (!ok && tid == 0) atomicExch(&g_error, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// One elected thread runs the whole main loop: k-tile kt waits for its
// stage's loads (full), issues its four MMAs and commits them to the stage's
// `empty` barrier; then the stage of k-tile kt-1 is refilled with k-tile
// kt-1+S as soon as kt-1's MMAs have read it, so the tensor pipe always has
// the next k-tile's MMAs queued while a load is in flight.  The other
// threads wait at the block barrier and join for the epilogue.
__global__ void __launch_bounds__(kThreads, 2)
gemm_tcgen05_tma(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int M, int N,
                 int K, int transA, int transB, const float* __restrict__ bias, int epilogue, float alpha,
                 float* __restrict__ C32, __nv_bfloat16* __restrict__ C16, int ldc, float* __restrict__ Z, int ldz,
                 int accumulate_c) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[kTmaStages];
    __shared__ __align__(8) uint64_t empty[kTmaStages];
    __shared__ __align__(8) uint64_t done;
    __shared__ uint32_t tmem_base_s;
    __shared__ int ok_s;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem) + 1023) & ~uintptr_t(1023));

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_s)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < kTmaStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        ok_s = 1;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_s;
    const int ktiles = (K + BK - 1) / BK;

    if (tid == 0) {
        // K-major tiles: 8-row x 128-byte atoms at SBO = 1 KB, K = 16 is 32
        // bytes into the atom; MN-major tiles: 8 K-row atoms at SBO = 1 KB,
        // the second 64 rows at LBO = 8 KB, K = 16 is two atoms (2 KB)
        const uint32_t idesc = instr_desc(BM, BN) | (static_cast<uint32_t>(transA != 0) << 15) |
                               (static_cast<uint32_t>(transB != 0) << 16);
        const uint32_t stepA = transA ? 2048u : 32u, stepB = transB ? 2048u : 32u;
        const uint32_t lboA = transA ? kMnBoxBytes : 16u, lboB = transB ? kMnBoxBytes : 16u;
        auto issue = [&](int t) {
            const int s = t % kTmaStages;
            unsigned char* sa = base + s * kStageBytes;
            mbar_expect_tx(&full[s], kStageBytes);
            tma_operand(sa, &mapA, transA, m0, t * BK, &full[s]);
            tma_operand(sa + BM * BK * 2, &mapB, transB, n0, t * BK, &full[s]);
        };
        int loaded = 0;    // k-tiles whose loads were issued
        int arrived = 0;   // k-tiles whose loads were waited for
        bool good = true;
        for (; loaded < ktiles && loaded < kTmaStages; ++loaded) issue(loaded);
        for (int kt = 0; kt < ktiles; ++kt) {
            const int s = kt % kTmaStages;
            if (!mbar_wait(&full[s], (kt / kTmaStages) & 1)) {
                good = false;
                break;
            }
            arrived = kt + 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(base + s * kStageBytes), b0 = a0 + BM * BK * 2;
#pragma unroll
            for (int ks = 0; ks < BK / 16; ++ks)
                mma_issue(tmem, smem_desc_sw128(a0 + ks * stepA, lboA, 1024), smem_desc_sw128(b0 + ks * stepB, lboB, 1024),
                          idesc, (kt > 0 || ks > 0) ? 1u : 0u);
            mma_commit(&empty[s]);
            if (kt >= 1 && loaded < ktiles) {
                // loaded == kt - 1 + kTmaStages: the stage k-tile kt-1 used
                if (!mbar_wait(&empty[(kt - 1) % kTmaStages], ((kt - 1) / kTmaStages) & 1)) {
                    good = false;
                    break;
                }
                issue(loaded++);
            }
        }
        // every MMA issued above completes before `done`
        mma_commit(&done);
        if (!good) {
            // let the copies still in flight land before the block exits
            for (int t = arrived; t < loaded; ++t) mbar_wait(&full[t % kTmaStages], (t / kTmaStages) & 1);
        }
        if (!mbar_wait(&done, 0)) good = false;
        ok_s = good ? 1 : 0;
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok_s) epilogue_tile(tmem, m0, n0, M, N, bias, epilogue, alpha, C32, C16, ldc, Z, ldz, accumulate_c);
    else if (tid == 0) atomicExch(&g_error, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// ---------------------------------------------------------------- elementwise
__global__ void gelu_backward(int64_t count, const float* __restrict__ dH, const float* __restrict__ Z,
                              float* __restrict__ dZ32, __nv_bfloat16* __restrict__ dZ16) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float g = dH[i] * gelu_grad(Z[i]);
        if (dZ32) dZ32[i] = g;
        if (dZ16) dZ16[i] = __float2bfloat16(g);
    }
}

// dY = scale * (Y - T) (masked rows have weight 0); loss partial sums.
__global__ void mse_grad(int rows, int cols, const float* __restrict__ Y, const float* __restrict__ T,
                         float scale, float* __restrict__ dY32, __nv_bfloat16* __restrict__ dY16,
                         double* __restrict__ loss) {
    double acc = 0.0;
    const int64_t count = static_cast<int64_t>(rows) * cols;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float d = Y[i] - T[i];
        acc += static_cast<double>(d) * d;
        const float g = scale * d;
        if (dY32) dY32[i] = g;
        if (dY16) dY16[i] = __float2bfloat16(g);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, acc);
}

// column sums (bias gradients): out[c] = sum_r X[r*cols + c].  A block of
// 32 x 32 threads owns 32 columns: thread (ty, tx) sums rows ty, ty+32, ...
// of column tx (coalesced along the row), then a fixed-order tree over the
// 32 partial sums (deterministic).
__global__ void __launch_bounds__(1024) column_sum(int rows, int cols, const float* __restrict__ X,
                                                   float* __restrict__ out) {
    __shared__ float part[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int c = blockIdx.x * 32 + tx;
    float acc = 0.0f;
    if (c < cols)
        for (int r = ty; r < rows; r += 32) acc += X[static_cast<int64_t>(r) * cols + c];
    part[ty][tx] = acc;
    __syncthreads();
    for (int h = 16; h > 0; h >>= 1) {
        if (ty < h) part[ty][tx] += part[ty + h][tx];
        __syncthreads();
    }
    if (ty == 0 && c < cols) out[c] = part[0][tx];
}

// Adam step on FP32 master weights; refreshes the BF16 copy.
__global__ void adam_step(int64_t count, float* __restrict__ w, const float* __restrict__ g,
                          float* __restrict__ m, float* __restrict__ v, __nv_bfloat16* __restrict__ w16,
                          float lr, float beta1, float beta2, float eps, float bc1, float bc2, float wd) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float gi = g[i] + wd * w[i];
        const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
        const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        w[i] = wi;
        if (w16) w16[i] = __float2bfloat16(wi);
    }
}

__global__ void to_bf16(int64_t count, const float* __restrict__ x, __nv_bfloat16* __restrict__ y) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

static int grid_for(int64_t count) {
    int64_t g = (count + 255) / 256;
    return static_cast<int>(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

}  // namespace fbalp_mlp

using namespace fbalp_mlp;

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encoder() {
    static EncodeTiledFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return static_cast<EncodeTiledFn>(nullptr);
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    return fn;
}

// Tensor map of op(X) (R x K) for gemm_tcgen05_tma, 128-byte swizzle, zero
// fill outside the matrix: X[r*ld + k] (K-major) as {K, R} with 64 x 128
// boxes, X[k*ld + r] (MN-major) as {R, K} with 64 x 64 boxes.  False when
// TMA cannot address the operand (start not on 16 bytes, row stride not a
// multiple of 8 elements, or rows overlapping).
bool encode_operand(CUtensorMap* map, const void* X, int ld, int trans, int R, int K) {
    const EncodeTiledFn fn = encoder();
    if (!fn || (reinterpret_cast<uintptr_t>(X) & 15) || (ld & 7) || ld < (trans ? R : K)) return false;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(trans ? R : K), static_cast<cuuint64_t>(trans ? K : R)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * 2};
    const cuuint32_t box[2] = {64, static_cast<cuuint32_t>(trans ? 64 : BM)};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(X), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The dynamic shared-memory limit of a kernel is an attribute of the
// current device's context: query it on every call (a host-side read) and
// raise it when this launch needs more, never lower it.
bool allow_dynamic_smem(const void* kernel, int bytes) {
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return false;
    if (fa.maxDynamicSharedSizeBytes >= bytes) return true;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess;
}

}  // namespace

extern "C" int fbalp_gemm_bf16(int M, int N, int K, const void* A, int lda, int transA, const void* B,
                               int ldb, int transB, const float* bias, int epilogue, float alpha,
                               float* C32, void* C16, int ldc, float* Z, int ldz, int accumulate_c,
                               void* stream) {
    if (M < 0 || N < 0 || K < 1 || !A || !B || (!C32 && !C16) || ldc < N || epilogue < 0 || epilogue > 2)
        return FBALP_MLP_ERR_INVALID;
    if (lda < 1 || ldb < 1) return FBALP_MLP_ERR_INVALID;
    if (M == 0 || N == 0) return FBALP_MLP_OK;
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    CUtensorMap mapA, mapB;
    if (encode_operand(&mapA, A, lda, transA, M, K) && encode_operand(&mapB, B, ldb, transB, N, K)) {
        if (!allow_dynamic_smem(reinterpret_cast<const void*>(gemm_tcgen05_tma), kTmaSmem)) return FBALP_MLP_ERR_CUDA;
        gemm_tcgen05_tma<<<grid, kThreads, kTmaSmem, static_cast<cudaStream_t>(stream)>>>(
            mapA, mapB, M, N, K, transA, transB, bias, epilogue, alpha, C32, static_cast<__nv_bfloat16*>(C16), ldc,
            Z, ldz > 0 ? ldz : ldc, accumulate_c);
        return cudaGetLastError() == cudaSuccess ? FBALP_MLP_OK : FBALP_MLP_ERR_CUDA;
    }
    const int smem = kStages * kStageBytes + 1024;
    if (!allow_dynamic_smem(reinterpret_cast<const void*>(gemm_tcgen05), smem)) return FBALP_MLP_ERR_CUDA;
    gemm_tcgen05<<<grid, kThreads, smem, static_cast<cudaStream_t>(stream)>>>(
        M, N, K, static_cast<const __nv_bfloat16*>(A), lda, transA, static_cast<const __nv_bfloat16*>(B), ldb,
        transB, bias, epilogue, alpha, C32, static_cast<__nv_bfloat16*>(C16), ldc, Z, ldz > 0 ? ldz : ldc,
        accumulate_c);
    return cudaGetLastError() == cudaSuccess ? FBALP_MLP_OK : FBALP_MLP_ERR_CUDA;
}

extern "C" int fbalp_mlp_error_flag(int* out, int clear) {
    if (!out) return FBALP_MLP_ERR_INVALID;
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_error, sizeof(int)) != cudaSuccess) return FBALP_MLP_ERR_CUDA;
    *out = v;
    if (clear) {
        int z = 0;
        if (cudaMemcpyToSymbol(g_error, &z, sizeof(int)) != cudaSuccess) return FBALP_MLP_ERR_CUDA;
    }
    return FBALP_MLP_OK;
}

extern "C" int fbalp_gelu_backward(int64_t count, const float* dH, const float* Z, float* dZ32, void* dZ16,
                                   void* stream) {
    if (count < 0 || !dH || !Z || (!dZ32 && !dZ16)) return FBALP_MLP_ERR_INVALID;
    if (count == 0) return FBALP_MLP_OK;
    gelu_backward<<<grid_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        count, dH, Z, dZ32, static_cast<__nv_bfloat16*>(dZ16));
    return cudaGetLastError() == cudaSuccess ? FBALP_MLP_OK : FBALP_MLP_ERR_CUDA;
}

extern "C" int fbalp_mse_grad(int rows, int cols, const float* Y, const float* T, float scale, float* dY32,
                              void* dY16, double* loss, void* stream) {
    if (rows < 0 || cols < 0 || !Y || !T) return FBALP_MLP_ERR_INVALID;
    const int64_t count = static_cast<int64_t>(rows) * cols;
    if (count == 0) return FBALP_MLP_OK;
    mse_grad<<<grid_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        rows, cols, Y, T, scale, dY32, static_cast<__nv_bfloat16*>(dY16), loss);
    return cudaGetLastError() == cudaSuccess ? FBALP_MLP_OK : FBALP_MLP_ERR_CUDA;
}

extern "C" int fbalp_column_sum(int rows, int cols, const float* X, float* out, void* stream) {
    if (rows < 0 || cols < 0 || !X || !out) return FBALP_MLP_ERR_INVALID;
    if (cols == 0) return FBALP_MLP_OK;
    column_sum<<<(cols + 31) / 32, 1024, 0, static_cast<cudaStream_t>(stream)>>>(rows, cols, X, out);
    return cudaGetLastError() == cudaSuccess ? FBALP_MLP_OK : FBALP_MLP_ERR_CUDA;
}

extern "C" int fbalp_adam_step(int64_t count, float* w, const float* g, float* m, float* v, void* w16, float lr,
                               float beta1, float beta2, float eps, int step, float weight_decay, void* stream) {
    if (count < 0 || !w || !g || !m || !v || step < 1) return FBALP_MLP_ERR_INVALID;
    if (count == 0) return FBALP_MLP_OK;
    const float bc1 = 1.0f - powf(beta1, static_cast<float>(step));
    const float bc2 = 1.0f - powf(beta2, static_cast<float>(step));
    adam_step<<<grid_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        count, w, g, m, v, static_cast<__nv_bfloat16*>(w16), lr, beta1, beta2, eps, bc1, bc2, weight_decay);
    return cudaGetLastError() == cudaSuccess ? FBALP_MLP_OK : FBALP_MLP_ERR_CUDA;
}

extern "C" int fbalp_to_bf16(int64_t count, const float* x, void* y, void* stream) {
    if (count < 0 || !x || !y) return FBALP_MLP_ERR_INVALID;
    if (count == 0) return FBALP_MLP_OK;
    to_bf16<<<grid_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(count, x,
                                                                              static_cast<__nv_bfloat16*>(y));
    return cudaGetLastError() == cudaSuccess ? FBALP_MLP_OK : FBALP_MLP_ERR_CUDA;
}
