/*
 * mlp_umma.cuh — the surrogate network's matrix products on the sm_100a tensor cores.
 *
 * One CTA of eight warps computes a 128-row tile of D = A B^T, A [M x K] and B [N x K] both
 * BF16 with K contiguous (K-major), N-tile BN (64 or 256 columns):
 *   * TMA (cp.async.bulk.tensor.2d) brings 64-column K blocks of A and B into shared memory
 *     in the 128-byte swizzled layout, through a ring of stages guarded by mbarriers (full:
 *     the copy landed; empty: the products reading it completed);
 *   * one thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32, M 128, N BN, K 16;
 *     four per K block) into a BN-column accumulator in tensor memory, and tcgen05.commit
 *     releases each stage to the copy thread;
 *   * after the last product all eight warps read the accumulators back (tcgen05.ld: warp w
 *     reads tensor-memory lanes 32 (w % 4) .. + 31, i.e. one row of the tile per thread, and
 *     the column half w / 4, 16 columns at a time) and run the layer's elementwise work on
 *     them before anything leaves the SM:
 *       EPI_HIDDEN  z = acc + b, h = SiLU(z): z (FP32, for the backward pass), h as BF16 rows
 *                   and, for the weight gradients, as BF16 columns (h transposed);
 *       EPI_HEAD    the last hidden map with the 1-wide output map folded in (the tile spans
 *                   every column): logit = b_out + sum_n SiLU(acc + b)_n w_out[n]; inference
 *                   writes sigmoid(logit); training writes the row's sigmoid cross-entropy,
 *                   dlogit = (sigmoid - y) / rows, SiLU(z) transposed, and the gradient of
 *                   the hidden map's pre-activation dz = dlogit w_out SiLU'(z) as BF16 rows
 *                   and columns;
 *       EPI_BACK    dz_prev = acc * SiLU'(z_prev) (acc = dz W, the gradient reaching the
 *                   previous map's output) as BF16 rows and columns;
 *       EPI_F32     the FP32 accumulators themselves, column-major so that a warp's stores
 *                   are contiguous (weight gradients, computed transposed: the column-major
 *                   D = dW^T is dW row-major; a K split writes its own slice, summed in a
 *                   fixed order afterwards).
 * Rows and columns past M and N read as zeros (TMA fills them) and are not stored.
 *
 * Every wait is bounded by the global timer: past kWaitNs a thread raises MIND_ETIMEOUT in
 * `err` (atomic max), stops issuing work, and the CTA still frees its tensor memory before
 * it returns.
 */
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/mindgpu.h"

namespace mlp {

constexpr int kTileM = 128;           // rows per CTA (= tensor-memory lanes)
constexpr int kBlockK = 64;           // K columns per stage: 128 bytes of BF16, one swizzle row
constexpr int kThreads = 256;            // eight warps
constexpr uint64_t kWaitNs = 2000000000ull;   // 2 s

enum Epilogue { EPI_HIDDEN = 0, EPI_HEAD = 1, EPI_BACK = 2, EPI_F32 = 3 };

struct EpiParams {
    int32_t M, N;                 // valid rows and columns of D
    int32_t ld_out;               // row stride of the row-major outputs (elements)
    int32_t ld_t;                 // row stride of the transposed outputs (elements)
    const float *bias;            // [N]
    float *z;                     // EPI_HIDDEN: pre-activations [M x ld_out] (may be null)
    __nv_bfloat16 *rows;          // BF16 rows [M x ld_out]: h (HIDDEN) or dz (HEAD, BACK)
    __nv_bfloat16 *cols;          // BF16 columns [N x ld_t]: h^T (HIDDEN) or dz^T (HEAD, BACK)
    const float *z_prev;          // EPI_BACK: pre-activations of the previous map [M x ld_out]
    const float *w_out;           // EPI_HEAD: output map weights [N] and bias [1]
    const float *b_out;
    float *prob;                  // EPI_HEAD inference: sigmoid(logit) [M]
    const float *y;               // EPI_HEAD training: targets [M]
    float *dlogit;                // EPI_HEAD training: (sigmoid - y) / rows_total [M]
    float *row_loss;              // EPI_HEAD training: per-row cross-entropy [M]
    __nv_bfloat16 *h_cols;        // EPI_HEAD training: SiLU(z) transposed [N x ld_t]
    float rows_total;             // EPI_HEAD training: the mean's denominator
    float *out;                   // EPI_F32: D column-major, [splits][N][ld_out] (ld_out >= M)
    int32_t *err;
};

// ---------------------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

/* Wait for the phase of `parity` to complete; false after kWaitNs. */
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try(bar, parity)) {
        if (global_ns() - t0 > kWaitNs) return false;
        __nanosleep(32);
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int32_t x, int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap *map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/* D[tmem] (+)= A[smem] B[smem]^T, one 128 x N x 16 product. */
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

/* Arrive on `bar` once the products issued so far by this thread have completed. */
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

/* This thread's tensor-memory lane, 16 consecutive 32-bit columns from `taddr`. */
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

/* Shared-memory matrix descriptor of a K-major tile in the 128-byte swizzled layout: rows of
 * 128 bytes, 8-row groups 1024 bytes apart (stride byte offset), descriptor version 1
 * (sm_100), layout type 2 (128-byte swizzle).  The leading byte offset is unused for this
 * layout and set to 16 bytes. */
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

/* Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both K-major, N, M. */
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

/* Logistic function with the fast exponential and an approximate reciprocal (relative
 * error ~1e-7, far below the BF16 rounding of the products' operands). */
__device__ __forceinline__ float sigmoid_f(float x) { return __fdividef(1.0f, 1.0f + __expf(-x)); }

template <int BN>
struct Shape {
    // K blocks in flight: the products here have 4 to 11 K blocks, so a short ring suffices
    // and leaves room for 2 (BN 256) or 3 (BN 64) CTAs per SM, whose epilogues overlap
    static constexpr int kStages = BN == 256 ? 2 : 3;
    static constexpr int kBytesA = kTileM * kBlockK * 2;
    static constexpr int kBytesB = BN * kBlockK * 2;
    static constexpr int kStageBytes = kBytesA + kBytesB;
    // stages (1024-aligned), then 2 * kStages + 1 mbarriers and the tensor-memory slot
    static constexpr int kSmemBytes = 1024 + kStages * kStageBytes + (2 * kStages + 2) * 8;
    static constexpr uint32_t kTmemCols = BN < 32 ? 32 : BN;
    static constexpr int kCols = BN / 2;   // columns per epilogue warp (two warps per lane quarter)
};

// ---------------------------------------------------------------------------------------
// the epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (one row per thread) and
// the column half w / 4 of the tile
// ---------------------------------------------------------------------------------------

__device__ __forceinline__ float silu_grad(float z) {
    const float s = sigmoid_f(z);
    return s * (1.0f + z * (1.0f - s));
}

/* 16 consecutive floats from 16-byte-aligned memory. */
__device__ __forceinline__ void load16(const float *p, float (&v)[16]) {
    const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float4 t = __ldg(q + k);
        v[4 * k] = t.x;
        v[4 * k + 1] = t.y;
        v[4 * k + 2] = t.z;
        v[4 * k + 3] = t.w;
    }
}

__device__ __forceinline__ void store16(float *p, const float (&v)[16]) {
    float4 *q = reinterpret_cast<float4 *>(p);
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}

/* 16 BF16 values as two 16-byte stores. */
__device__ __forceinline__ void store16_bf16(__nv_bfloat16 *p, const float (&v)[16]) {
    uint32_t w[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
        w[j] = (uint32_t)__bfloat16_as_ushort(h.x) | ((uint32_t)__bfloat16_as_ushort(h.y) << 16);
    }
    uint4 *q = reinterpret_cast<uint4 *>(p);
    q[0] = make_uint4(w[0], w[1], w[2], w[3]);
    q[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

/* Row-major BF16 rows (vector stores for whole chunks) and, if wanted, the transposed copy. */
__device__ __forceinline__ void store_rows_cols(const EpiParams &E, int32_t row, int32_t nc, const float (&v)[16]) {
    if (nc + 16 <= E.N) {
        store16_bf16(E.rows + (int64_t)row * E.ld_out + nc, v);
    } else {
        for (int j = 0; j < 16 && nc + j < E.N; ++j) E.rows[(int64_t)row * E.ld_out + nc + j] = __float2bfloat16(v[j]);
    }
    if (E.cols)
#pragma unroll
        for (int j = 0; j < 16; ++j)
            if (nc + j < E.N) E.cols[(int64_t)(nc + j) * E.ld_t + row] = __float2bfloat16(v[j]);
}

/* 16 per-column parameters, zero past N (N and the tile are multiples of 16: whole chunks). */
__device__ __forceinline__ void column_params(const float *p, int32_t nc, int32_t N, float (&v)[16]) {
    if (nc + 16 <= N) {
        load16(p + nc, v);
    } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = nc + j < N ? p[nc + j] : 0.0f;
    }
}

template <int EPI, int BN>
__device__ __forceinline__ void epilogue(const EpiParams &E, uint32_t tacc, int32_t row, int32_t c0, int32_t half,
                                         int32_t split, float *s_logit, const float *pre) {
    constexpr int C = Shape<BN>::kCols;
    const bool live = row < E.M;
    const int32_t r = threadIdx.x & 127;   // row within the tile (quarter * 32 + lane)
    if constexpr (EPI == EPI_HEAD) {
        // pass 1: this half's share of the logit, SiLU(z) transposed (training)
        float part = 0.0f;
#pragma unroll 1
        for (int c = 0; c < C; c += 16) {
            float v[16], b[16], w[16];
            tmem_ld16(tacc + c, v);
            const int32_t nc = c0 + c;
            column_params(E.bias, nc, E.N, b);
            column_params(E.w_out, nc, E.N, w);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const float z = v[j] + b[j];
                v[j] = z * sigmoid_f(z);
                part = fmaf(v[j], w[j], part);
            }
            if (live && E.h_cols)
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if (nc + j < E.N) E.h_cols[(int64_t)(nc + j) * E.ld_t + row] = __float2bfloat16(v[j]);
        }
        s_logit[half * kTileM + r] = part;
        __syncthreads();
        const float logit = s_logit[r] + s_logit[kTileM + r] + E.b_out[0];
        if (!E.y) {
            if (live && half == 0) E.prob[row] = sigmoid_f(logit);
            return;
        }
        float g = 0.0f;
        if (live) {
            const float t = E.y[row];
            g = (sigmoid_f(logit) - t) / E.rows_total;
            if (half == 0) {
                E.row_loss[row] = fmaxf(logit, 0.0f) - logit * t + log1pf(__expf(-fabsf(logit)));
                E.dlogit[row] = g;
            }
        }
        // pass 2: the last hidden map's dz = dlogit w_out SiLU'(z)
#pragma unroll 1
        for (int c = 0; c < C; c += 16) {
            float v[16], b[16], w[16];
            tmem_ld16(tacc + c, v);
            if (!live) continue;
            const int32_t nc = c0 + c;
            column_params(E.bias, nc, E.N, b);
            column_params(E.w_out, nc, E.N, w);
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = g * w[j] * silu_grad(v[j] + b[j]);
            store_rows_cols(E, row, nc, v);
        }
    } else {
#pragma unroll
        for (int c = 0; c < C; c += 16) {   // C = 32: two chunks, unrolled (pre[] stays in registers)
            float v[16];
            tmem_ld16(tacc + c, v);
            if (!live) continue;
            const int32_t nc = c0 + c;
            if (nc >= E.N) continue;
            if constexpr (EPI == EPI_F32) {
                // column-major: a column's 32 rows of this warp are 128 contiguous bytes
                float *o = E.out + ((int64_t)split * E.N + nc) * E.ld_out + row;
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if (nc + j < E.N) o[(int64_t)j * E.ld_out] = v[j];
            } else if constexpr (EPI == EPI_HIDDEN) {
                float b[16];
                column_params(E.bias, nc, E.N, b);
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] += b[j];
                if (E.z) store16(E.z + (int64_t)row * E.ld_out + nc, v);
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = v[j] * sigmoid_f(v[j]);
                store_rows_cols(E, row, nc, v);
            } else {   // EPI_BACK: z_prev was loaded while the products ran
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] *= silu_grad(pre[c + j]);
                store_rows_cols(E, row, nc, v);
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------------------

/* grid (ceil(M/128), ceil(N/BN), splits); K blocks [split * kb_per_split, ...) up to kb_total.
 * Eight warps: warp 0 lane 0 issues the copies, warp 1 lane 0 the products, and all eight run
 * the epilogue (two per tensor-memory lane quarter, one column half each). */
template <int EPI, int BN>
__global__ void __launch_bounds__(kThreads, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                     int32_t kb_total, int32_t kb_per_split, const EpiParams E) {
    using S = Shape<BN>;
    extern __shared__ unsigned char smem_raw[];
    __shared__ float s_logit[2 * kTileM];
    __shared__ int failed;
    unsigned char *base = reinterpret_cast<unsigned char *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + S::kStages * S::kStageBytes);
    uint64_t *empty = full + S::kStages;
    uint64_t *done = empty + S::kStages;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int32_t m0 = blockIdx.x * kTileM, n0 = blockIdx.y * BN, split = blockIdx.z;
    const int32_t kb0 = split * kb_per_split;
    const int32_t nkb = min(kb_total - kb0, kb_per_split);

    if (threadIdx.x == 0) {
        failed = 0;
        tma_prefetch_map(&map_a);
        tma_prefetch_map(&map_b);
        for (int s = 0; s < S::kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        mbar_fence_init();
    }
    if (warp == 0) {
        tmem_alloc(tmem_slot, S::kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (nkb > 0 && warp == 0 && lane == 0) {
        // copies: stage s is free again once the products that read it committed
        for (int32_t i = 0; i < nkb; ++i) {
            const int s = i % S::kStages;
            if (i >= S::kStages && !mbar_wait(&empty[s], ((i / S::kStages) - 1) & 1)) {
                atomicExch(&failed, 1);
                break;
            }
            unsigned char *sa = base + s * S::kStageBytes;
            mbar_expect_tx(&full[s], S::kStageBytes);
            tma_load_2d(sa, &map_a, &full[s], (kb0 + i) * kBlockK, m0);
            tma_load_2d(sa + S::kBytesA, &map_b, &full[s], (kb0 + i) * kBlockK, n0);
        }
    } else if (nkb > 0 && warp == 1 && lane == 0) {
        constexpr uint32_t idesc = idesc_bf16(kTileM, BN);
        for (int32_t i = 0; i < nkb; ++i) {
            const int s = i % S::kStages;
            if (!mbar_wait(&full[s], (i / S::kStages) & 1)) {
                atomicExch(&failed, 1);
                break;
            }
            tc_fence_after();
            const uint32_t sa = smem_u32(base + s * S::kStageBytes);
            const uint64_t da = smem_desc_sw128(sa), db = smem_desc_sw128(sa + S::kBytesA);
#pragma unroll
            for (int kk = 0; kk < kBlockK / 16; ++kk)   // 16 BF16 = 32 bytes = 2 descriptor units
                mma_bf16(tmem, da + 2 * kk, db + 2 * kk, idesc, (i | kk) != 0);
            mma_commit(&empty[s]);
        }
        mma_commit(done);   // also after a failed wait: the epilogue's wait then ends
    }
    __syncwarp();

    const int quarter = warp & 3, half = warp >> 2;
    const int32_t row = m0 + quarter * 32 + lane, c0 = n0 + half * S::kCols;
    // operands of the epilogue that do not depend on the products, loaded while they run
    float pre[EPI == EPI_BACK ? S::kCols : 1];
    if constexpr (EPI == EPI_BACK) {
#pragma unroll
        for (int c = 0; c < S::kCols; c += 16) {
            float z[16];
            if (row < E.M && c0 + c + 16 <= E.N) {
                load16(E.z_prev + (int64_t)row * E.ld_out + c0 + c, z);
            } else {
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    z[j] = (row < E.M && c0 + c + j < E.N) ? E.z_prev[(int64_t)row * E.ld_out + c0 + c + j] : 0.0f;
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) pre[c + j] = z[j];
        }
    }
    if (nkb <= 0 || !mbar_wait(done, 0)) atomicExch(&failed, 1);
    __syncthreads();
    if (failed) {
        if (threadIdx.x == 0) atomicMax(E.err, (int32_t)MIND_ETIMEOUT);
    } else {
        tc_fence_after();
        const uint32_t tacc = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(half * S::kCols);
        epilogue<EPI, BN>(E, tacc, row, c0, half, split, s_logit, pre);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, S::kTmemCols);
}

}  // namespace mlp
