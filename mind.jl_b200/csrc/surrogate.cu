/*
 * surrogate.cu — the spike-output surrogate: a multilayer perceptron trained on
 * windows the cable solver produced (no counterpart in the reference).
 *
 * Network: n_in -> hidden (SiLU) x layers -> 1 logit; the spike probability of the
 * next 1 ms bin is sigmoid(logit).  Parameters are FP32 masters; every matrix product
 * runs in BF16 with FP32 accumulation on the tensor cores, in this library's own
 * tcgen05 kernels (mlp_umma.cuh) whose epilogues carry the elementwise work:
 *
 *   forward   map l < last hidden:  z_l = h_l W_l^T + b_l, h_{l+1} = SiLU(z_l)      EPI_HIDDEN
 *             last hidden map + output map: logit, sigmoid (inference), or the
 *             cross-entropy, dlogit and dz of the last hidden map (training)          EPI_HEAD
 *   backward  dW_l = dz_l^T h_l (rows split into K slices, summed in a fixed order)   EPI_F32
 *             dz_{l-1} = (dz_l W_l) * SiLU'(z_{l-1})                                  EPI_BACK
 *
 * and small kernels here for the rest: BF16 staging and transposes of the inputs, the
 * output map's gradients and the bias gradients (row sums in a fixed order), and Adam with
 * the BF16 weight copies (row-major for the forward products, transposed for the backward
 * ones).  The products' operands are K-major everywhere, so every activation and gradient
 * that a weight gradient needs is also written transposed (rows of the batch contiguous).
 * Parameter layout: for each linear map l, W_l [out x in] row-major, then b_l [out], maps in
 * order.  hidden must be a multiple of 16 and at most 256 (one tile spans a hidden layer).
 */
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mindgpu.h"
#include "mlp_umma.cuh"

struct MindMlp {
    std::vector<int32_t> dims;       // n_in, hidden..., 1
    int32_t hidden = 0;
    int32_t maps = 0;                // linear maps: layers hidden ones, then the output map
    int32_t ld0 = 0;                 // n_in rounded up to 8: row stride of the BF16 inputs and of w0
    std::vector<int64_t> w_off, b_off;
    int64_t n_params = 0;
    float *master = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
    __nv_bfloat16 *wbf = nullptr;    // BF16 copy of the parameters (forward operands of maps >= 1)
    __nv_bfloat16 *w0 = nullptr;     // BF16 first-map weights [hidden x ld0], zero past n_in
    __nv_bfloat16 *wt = nullptr;     // BF16 W_l^T of the hidden maps 1..layers-1 [hidden x hidden] each
    float *loss = nullptr;           // the last batch's mean loss
    float *loss_hist = nullptr;      // per-step batch losses of a training call
    int32_t loss_cap = 0;
    int64_t adam_t = 0;
    uint64_t *step_dev = nullptr;    // Adam steps taken, on the device (read by a captured step)
    cudaStream_t stream = nullptr;
    cudaEvent_t ready = nullptr, done = nullptr;
    int32_t *err = nullptr;          // device status word of the products (MIND_ETIMEOUT)
    // activations, rows of the batch: cap rows; transposed copies: rows of capT elements
    int64_t cap = 0, capT = 0;
    __nv_bfloat16 *x = nullptr;      // inputs [cap x ld0]
    __nv_bfloat16 *xt = nullptr;     // inputs transposed [ld0 x capT]
    std::vector<float *> z;          // pre-activations of hidden maps 0..layers-2 [cap x hidden]
    std::vector<__nv_bfloat16 *> h, ht;   // outputs of hidden maps 0..layers-2, rows and transposed
    __nv_bfloat16 *ht_last = nullptr;     // SiLU of the last hidden map, transposed
    __nv_bfloat16 *dzr[2] = {nullptr, nullptr}, *dzc[2] = {nullptr, nullptr};   // dz rows / transposed
    float *y = nullptr, *prob = nullptr, *dlogit = nullptr, *row_loss = nullptr;
    float *part = nullptr;           // weight-gradient K slices [kMaxSplits x hidden x max(n_in, hidden)]
    float *xin = nullptr;            // FP32 rows uploaded by predict / gradients [cap x n_in]
    float last_ms = 0.0f;            // device time of the last call's network work
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    float *data_x = nullptr, *data_y = nullptr;  // training set (FP32 on the device)
    int64_t data_n = 0, data_cap = 0;
    std::string error;
};

namespace {

constexpr int kT = 256;
constexpr int kMaxSplits = 32;

int fail(MindMlp *m, int code, const std::string &why) {
    if (m) m->error = why;
    return code;
}

#define MLP_CUDA(m, call)                                                                         \
    do {                                                                                          \
        cudaError_t _e = (call);                                                                  \
        if (_e != cudaSuccess) return fail((m), MIND_ECUDA, std::string(#call ": ") + cudaGetErrorString(_e)); \
    } while (0)
#define MLP_TRY(call)         \
    do {                      \
        int _s = (call);      \
        if (_s) return _s;    \
    } while (0)

int grid(int64_t n) { return (int)std::min<int64_t>((n + kT - 1) / kT, 148 * 16); }

// ---------------------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------------------

/* The BF16 copies of parameter k (value v): the flat copy, w0 (first map, rows of stride
 * ld0), and W_l^T for the hidden maps l = 1..layers-1. */
struct CopyLayout {
    __nv_bfloat16 *wbf, *w0, *wt;
    int64_t w0_off, n0, hid_off, hid_stride;
    int32_t d, ld0, hidden, n_hidden_maps;
};

__device__ __forceinline__ void store_copies(const CopyLayout &C, int64_t k, float v) {
    const __nv_bfloat16 b = __float2bfloat16(v);
    C.wbf[k] = b;
    const int64_t j = k - C.w0_off;
    if (j >= 0 && j < C.n0) C.w0[(j / C.d) * C.ld0 + j % C.d] = b;
    const int64_t q = k - C.hid_off;
    if (q >= 0 && C.n_hidden_maps > 0) {
        const int64_t map = q / C.hid_stride, r = q - map * C.hid_stride;
        const int64_t hh = (int64_t)C.hidden * C.hidden;
        if (map < C.n_hidden_maps && r < hh) {
            const int64_t o = r / C.hidden, i = r - o * C.hidden;
            C.wt[map * hh + i * C.hidden + o] = b;
        }
    }
}

__global__ void copies_kernel(const float *w, int64_t n, CopyLayout C) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        store_copies(C, k, w[k]);
}

/* Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the FP32 masters, then the BF16 copies; the
 * bias corrections use t = *step + 1. */
__global__ void adam_kernel(float *w, const float *g, float *m1, float *m2, int64_t n, float lr, const uint64_t *step,
                            CopyLayout C) {
    const float t = (float)(*step + 1);
    const float c1 = 1.0f - powf(0.9f, t), c2 = 1.0f - powf(0.999f, t);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const float gk = g[k];
        const float a = 0.9f * m1[k] + 0.1f * gk, b = 0.999f * m2[k] + 0.001f * gk * gk;
        m1[k] = a;
        m2[k] = b;
        const float v = w[k] - lr * (a / c1) / (sqrtf(b / c2) + 1e-8f);
        w[k] = v;
        store_copies(C, k, v);
    }
}

/* Row kernels: blockIdx.y strides over rows, the threads of blockIdx.x over a row's
 * columns (consecutive threads, consecutive columns: coalesced, no index division). */
dim3 row_grid(int64_t rows, int32_t cols) {
    return dim3((unsigned)((cols + kT - 1) / kT), (unsigned)std::max<int64_t>(1, std::min<int64_t>(rows, 16384)));
}

/* FP32 rows [n x d] -> BF16 rows of stride ld, zero past d. */
__global__ void to_bf16_rows_kernel(const float *x, __nv_bfloat16 *out, int64_t n, int32_t d, int32_t ld) {
    for (int64_t row = blockIdx.y; row < n; row += gridDim.y)
        for (int32_t col = blockIdx.x * blockDim.x + threadIdx.x; col < ld; col += gridDim.x * blockDim.x)
            out[row * ld + col] = __float2bfloat16(col < d ? x[row * d + col] : 0.0f);
}

/* Rows of the training set drawn for Adam step *step + 1 (a 64-bit mix of step and slot), as
 * BF16 rows of stride ld (zero past d), and their targets. */
__global__ void gather_kernel(const float *x, const float *y, __nv_bfloat16 *hx, float *hy, int64_t n, int32_t d,
                              int32_t ld, int32_t batch, const uint64_t *step_dev) {
    const uint64_t step = *step_dev + 1;
    for (int64_t row = blockIdx.y; row < batch; row += gridDim.y) {
        uint64_t s = step * 0x9E3779B97F4A7C15ull + (uint64_t)row * 0xBF58476D1CE4E5B9ull + 0x94D049BB133111EBull;
        s ^= s >> 31;
        s *= 0xD6E8FEB86659FD93ull;
        s ^= s >> 32;
        const int64_t src = (int64_t)(s % (uint64_t)n);
        for (int32_t col = blockIdx.x * blockDim.x + threadIdx.x; col < ld; col += gridDim.x * blockDim.x) {
            hx[row * ld + col] = __float2bfloat16(col < d ? x[src * d + col] : 0.0f);
            if (col == 0) hy[row] = y[src];
        }
    }
}

/* dst [cols x ld_dst] = src [rows x ld_src]^T for the first `cols` columns (BF16), through
 * 32 x 32 shared-memory tiles so that both sides are read and written along rows. */
__global__ void transpose_kernel(const __nv_bfloat16 *src, int64_t rows, int32_t cols, int32_t ld_src,
                                 __nv_bfloat16 *dst, int64_t ld_dst) {
    __shared__ __nv_bfloat16 tile[32][34];
    const int64_t r0 = (int64_t)blockIdx.x * 32;
    const int32_t c0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int64_t r = r0 + k;
        const int32_t c = c0 + threadIdx.x;
        tile[k][threadIdx.x] = (r < rows && c < cols) ? src[r * ld_src + c] : __float2bfloat16(0.0f);
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int32_t c = c0 + k;
        const int64_t r = r0 + threadIdx.x;
        if (c < cols && r < rows) dst[(int64_t)c * ld_dst + r] = tile[threadIdx.x][k];
    }
}

/* Fixed-order block sum of per-thread partials (blockDim.x == kT). */
__device__ __forceinline__ float block_sum(float v, float *scratch) {
    scratch[threadIdx.x] = v;
    __syncthreads();
    for (int s = kT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) scratch[threadIdx.x] += scratch[threadIdx.x + s];
        __syncthreads();
    }
    return scratch[0];
}

/* out[o] = sum over r < R of w[r] * src[o][r] (w null: 1), one block per o, in a fixed order. */
__global__ void rowsum_kernel(const __nv_bfloat16 *src, int64_t ld, int64_t R, const float *w, float *out) {
    __shared__ float scratch[kT];
    const int64_t o = blockIdx.x;
    float s = 0.0f;
    for (int64_t r = threadIdx.x; r < R; r += kT) {
        const float v = __bfloat162float(src[o * ld + r]);
        s += w ? w[r] * v : v;
    }
    const float t = block_sum(s, scratch);
    if (threadIdx.x == 0) out[o] = t;
}

/* The output map's bias gradient (sum of dlogit) and the batch's mean loss. */
__global__ void head_scalars_kernel(const float *dlogit, const float *row_loss, int64_t R, float *db, float *loss) {
    __shared__ float scratch[kT];
    float a = 0.0f, b = 0.0f;
    for (int64_t r = threadIdx.x; r < R; r += kT) {
        a += dlogit[r];
        b += row_loss[r];
    }
    const float sa = block_sum(a, scratch);
    __syncthreads();
    const float sb = block_sum(b, scratch);
    if (threadIdx.x == 0) {
        *db = sa;
        *loss = sb / (float)R;
    }
}

/* The end of an Adam step: its loss into the call's history, the step counter advanced. */
__global__ void step_end_kernel(uint64_t *step, const float *loss, float *hist, uint64_t first) {
    hist[*step - first] = *loss;
    *step += 1;
}

/* grad[k] = sum over the K slices s (in order) of part[s][k], k < n. */
__global__ void split_sum_kernel(const float *part, int32_t splits, int64_t n, float *grad) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        float t = 0.0f;
        for (int32_t s = 0; s < splits; ++s) t += part[(int64_t)s * n + k];
        grad[k] = t;
    }
}

// ---------------------------------------------------------------------------------------
// tensor maps and product launches
// ---------------------------------------------------------------------------------------

PFN_cuTensorMapEncodeTiled encoder() {
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
    });
    return fn;
}

/* A K-major BF16 operand: `outer` rows of `inner` elements, rows `ld` elements apart; boxes
 * of 64 elements (128 bytes, the swizzle span) by box_rows rows. */
int operand_map(MindMlp *m, CUtensorMap *map, const __nv_bfloat16 *ptr, int64_t inner, int64_t outer, int64_t ld,
                int32_t box_rows) {
    PFN_cuTensorMapEncodeTiled encode = encoder();
    if (!encode) return fail(m, MIND_ECUDA, "cuTensorMapEncodeTiled unavailable");
    if (((uintptr_t)ptr & 15) || (ld * 2) % 16) return fail(m, MIND_ECUDA, "operand not 16-byte aligned");
    const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
    const cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
    const cuuint32_t box[2] = {(cuuint32_t)mlp::kBlockK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(ptr), dims, strides,
                              box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(m, MIND_ECUDA, "cuTensorMapEncodeTiled failed");
    return MIND_OK;
}

/* D [M x N] = A [M x K] B [N x K]^T with epilogue EPI on N tiles of BN columns and `splits`
 * K slices (EPI_F32 only). */
template <int EPI, int BN>
int product(MindMlp *m, const __nv_bfloat16 *A, int64_t lda, const __nv_bfloat16 *B, int64_t ldb, int32_t M, int32_t N,
            int32_t K, int32_t splits, mlp::EpiParams E, cudaStream_t s, int32_t *splits_used = nullptr) {
    using S = mlp::Shape<BN>;
    if (M < 1 || N < 1 || K < 1) return fail(m, MIND_EARG, "empty product");
    CUtensorMap ma, mb;
    MLP_TRY(operand_map(m, &ma, A, K, M, lda, mlp::kTileM));
    // B's rows: the tensor map spans the rows the operand holds (at least N)
    MLP_TRY(operand_map(m, &mb, B, K, N, ldb, BN));
    const int32_t kb_total = (K + mlp::kBlockK - 1) / mlp::kBlockK;
    splits = std::max(1, std::min(splits, kb_total));
    const int32_t per = (kb_total + splits - 1) / splits;
    splits = (kb_total + per - 1) / per;   // no empty slice
    if (splits_used) *splits_used = splits;
    E.M = M;
    E.N = N;
    E.err = m->err;
    const dim3 g((M + mlp::kTileM - 1) / mlp::kTileM, (N + BN - 1) / BN, splits);
    mlp::umma_gemm_kernel<EPI, BN><<<g, mlp::kThreads, S::kSmemBytes, s>>>(ma, mb, kb_total, per, E);
    MLP_CUDA(m, cudaGetLastError());
    return MIND_OK;
}

/* Shared-memory opt-in of the product kernels (once per network, on its device). */
int prepare_products(MindMlp *m) {
    MLP_CUDA(m, cudaFuncSetAttribute(mlp::umma_gemm_kernel<mlp::EPI_HIDDEN, 64>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::Shape<64>::kSmemBytes));
    MLP_CUDA(m, cudaFuncSetAttribute(mlp::umma_gemm_kernel<mlp::EPI_BACK, 64>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::Shape<64>::kSmemBytes));
    MLP_CUDA(m, cudaFuncSetAttribute(mlp::umma_gemm_kernel<mlp::EPI_F32, 64>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::Shape<64>::kSmemBytes));
    MLP_CUDA(m, cudaFuncSetAttribute(mlp::umma_gemm_kernel<mlp::EPI_HEAD, 256>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::Shape<256>::kSmemBytes));
    return MIND_OK;
}

/* K slices for a weight gradient: about two CTAs per SM, at least 4 K blocks per slice. */
int32_t grad_splits(int32_t tiles, int64_t rows) {
    const int32_t kb = (int32_t)((rows + mlp::kBlockK - 1) / mlp::kBlockK);
    int32_t s = (2 * 148 + tiles - 1) / tiles;
    s = std::min(s, std::max(1, kb / 4));
    return std::max(1, std::min(s, kMaxSplits));
}

void free_activations(MindMlp *m) {
    for (float *p : m->z) cudaFree(p);
    for (__nv_bfloat16 *p : m->h) cudaFree(p);
    for (__nv_bfloat16 *p : m->ht) cudaFree(p);
    m->z.clear();
    m->h.clear();
    m->ht.clear();
    for (void *p : {(void *)m->x, (void *)m->xt, (void *)m->ht_last, (void *)m->dzr[0], (void *)m->dzr[1],
                    (void *)m->dzc[0], (void *)m->dzc[1], (void *)m->y, (void *)m->prob, (void *)m->dlogit,
                    (void *)m->row_loss, (void *)m->part, (void *)m->xin})
        cudaFree(p);
    m->xin = nullptr;
    m->x = m->xt = m->ht_last = m->dzr[0] = m->dzr[1] = m->dzc[0] = m->dzc[1] = nullptr;
    m->y = m->prob = m->dlogit = m->row_loss = m->part = nullptr;
    m->cap = m->capT = 0;
}

int reserve(MindMlp *m, int64_t rows) {
    if (rows <= m->cap) return MIND_OK;
    const int64_t cap = std::max<int64_t>(rows, 2 * m->cap);
    const int64_t capT = (cap + 7) / 8 * 8;
    free_activations(m);
    const int64_t H = m->hidden;
    const int32_t inner = m->maps - 2;   // hidden maps whose outputs feed another hidden map
    m->z.assign(inner, nullptr);
    m->h.assign(inner, nullptr);
    m->ht.assign(inner, nullptr);
    for (int32_t l = 0; l < inner; ++l) {
        MLP_CUDA(m, cudaMalloc(&m->z[l], cap * H * sizeof(float)));
        MLP_CUDA(m, cudaMalloc(&m->h[l], cap * H * sizeof(__nv_bfloat16)));
        MLP_CUDA(m, cudaMalloc(&m->ht[l], H * capT * sizeof(__nv_bfloat16)));
    }
    MLP_CUDA(m, cudaMalloc(&m->x, cap * m->ld0 * sizeof(__nv_bfloat16)));
    MLP_CUDA(m, cudaMalloc(&m->xin, cap * m->dims[0] * sizeof(float)));
    MLP_CUDA(m, cudaMalloc(&m->xt, (int64_t)m->ld0 * capT * sizeof(__nv_bfloat16)));
    MLP_CUDA(m, cudaMalloc(&m->ht_last, H * capT * sizeof(__nv_bfloat16)));
    for (int k = 0; k < 2; ++k) {
        MLP_CUDA(m, cudaMalloc(&m->dzr[k], cap * H * sizeof(__nv_bfloat16)));
        MLP_CUDA(m, cudaMalloc(&m->dzc[k], H * capT * sizeof(__nv_bfloat16)));
    }
    for (float **p : {&m->y, &m->prob, &m->dlogit, &m->row_loss}) MLP_CUDA(m, cudaMalloc(p, cap * sizeof(float)));
    MLP_CUDA(m, cudaMalloc(&m->part, (size_t)kMaxSplits * H * std::max<int64_t>(m->dims[0], H) * sizeof(float)));
    m->cap = cap;
    m->capT = capT;
    return MIND_OK;
}

CopyLayout copy_layout(const MindMlp *m) {
    CopyLayout C{};
    C.wbf = m->wbf;
    C.w0 = m->w0;
    C.wt = m->wt;
    C.w0_off = m->w_off[0];
    C.n0 = (int64_t)m->dims[0] * m->hidden;
    C.d = m->dims[0];
    C.ld0 = m->ld0;
    C.hidden = m->hidden;
    C.n_hidden_maps = m->maps - 2;   // hidden maps 1..layers-1
    C.hid_off = m->maps > 2 ? m->w_off[1] : 0;
    C.hid_stride = (int64_t)m->hidden * m->hidden + m->hidden;
    return C;
}

/* Forward over `rows` rows whose BF16 inputs are in m->x; `train` keeps what the backward
 * pass needs and computes the loss against m->y, otherwise m->prob receives the
 * probabilities. */
int forward(MindMlp *m, int64_t rows, bool train, cudaStream_t s, float *prob = nullptr) {
    const int32_t R = (int32_t)rows, H = m->hidden, last = m->maps - 2;   // last hidden map
    for (int32_t l = 0; l <= last; ++l) {
        const __nv_bfloat16 *A = l == 0 ? m->x : m->h[l - 1];
        const int64_t lda = l == 0 ? m->ld0 : H;
        const int32_t K = l == 0 ? m->ld0 : H;
        const __nv_bfloat16 *W = l == 0 ? m->w0 : m->wbf + m->w_off[l];
        mlp::EpiParams E{};
        E.bias = m->master + m->b_off[l];
        E.ld_out = H;
        E.ld_t = (int32_t)m->capT;
        if (l < last) {
            E.z = train ? m->z[l] : nullptr;
            E.rows = m->h[l];
            E.cols = train ? m->ht[l] : nullptr;
            MLP_TRY((product<mlp::EPI_HIDDEN, 64>(m, A, lda, W, K, R, H, K, 1, E, s)));
        } else {
            E.w_out = m->master + m->w_off[m->maps - 1];
            E.b_out = m->master + m->b_off[m->maps - 1];
            if (train) {
                E.y = m->y;
                E.dlogit = m->dlogit;
                E.row_loss = m->row_loss;
                E.h_cols = m->ht_last;
                E.rows = m->dzr[0];
                E.cols = m->dzc[0];
                E.rows_total = (float)rows;
            } else {
                E.prob = prob ? prob : m->prob;
            }
            MLP_TRY((product<mlp::EPI_HEAD, 256>(m, A, lda, W, K, R, H, K, 1, E, s)));
        }
    }
    return MIND_OK;
}

/* Gradients of the mean loss into m->grad after forward(train); m->xt must hold the inputs
 * transposed. */
int backward(MindMlp *m, int64_t rows, cudaStream_t s) {
    const int32_t R = (int32_t)rows, H = m->hidden, last = m->maps - 2;
    const int64_t T = m->capT;
    // output map: dW[n] = sum_r dlogit[r] SiLU(z)[r][n], db = sum_r dlogit[r], and the loss
    rowsum_kernel<<<H, kT, 0, s>>>(m->ht_last, T, rows, m->dlogit, m->grad + m->w_off[m->maps - 1]);
    head_scalars_kernel<<<1, kT, 0, s>>>(m->dlogit, m->row_loss, rows, m->grad + m->b_off[m->maps - 1], m->loss);
    int cur = 0;
    for (int32_t l = last; l >= 0; --l) {
        const int32_t in = l == 0 ? m->dims[0] : H;
        // dW_l^T [in x H] = h_l^T dz_l: A = h_l transposed [in x R], B = dz_l transposed [H x R];
        // stored column-major, which is dW_l [H x in] row-major, the parameters' layout
        const __nv_bfloat16 *At = l == 0 ? m->xt : m->ht[l - 1];
        const int32_t tiles = ((in + 127) / 128) * ((H + 63) / 64);
        const int32_t splits = grad_splits(tiles, rows);
        mlp::EpiParams E{};
        E.ld_out = in;
        E.out = m->part;
        int32_t used = 1;
        MLP_TRY((product<mlp::EPI_F32, 64>(m, At, T, m->dzc[cur], T, in, H, R, splits, E, s, &used)));
        split_sum_kernel<<<grid((int64_t)H * in), kT, 0, s>>>(m->part, used, (int64_t)H * in, m->grad + m->w_off[l]);
        rowsum_kernel<<<H, kT, 0, s>>>(m->dzc[cur], T, rows, nullptr, m->grad + m->b_off[l]);
        if (l == 0) break;
        // dz_{l-1} = (dz_l W_l) * SiLU'(z_{l-1}): A = dz_l rows [R x H], B = W_l^T [H x H]
        mlp::EpiParams B{};
        B.ld_out = H;
        B.ld_t = (int32_t)T;
        B.z_prev = m->z[l - 1];
        B.rows = m->dzr[cur ^ 1];
        B.cols = m->dzc[cur ^ 1];
        const __nv_bfloat16 *Wt = m->wt + (int64_t)(l - 1) * H * H;
        MLP_TRY((product<mlp::EPI_BACK, 64>(m, m->dzr[cur], H, Wt, H, R, H, H, 1, B, s)));
        cur ^= 1;
    }
    MLP_CUDA(m, cudaGetLastError());
    return MIND_OK;
}

void transpose_inputs(MindMlp *m, int64_t rows, cudaStream_t s) {
    const dim3 g((unsigned)((rows + 31) / 32), (unsigned)((m->ld0 + 31) / 32));
    transpose_kernel<<<g, dim3(32, 8), 0, s>>>(m->x, rows, m->ld0, m->ld0, m->xt, m->capT);
}

/* Host FP32 rows into m->xin; the timed region of the call starts after the copy.  The
 * runtime's per-thread last-error slot is cleared first: the products check their launches
 * with cudaGetLastError, which must not report the host's other CUDA code. */
int upload_rows(MindMlp *m, const float *x, int64_t n) {
    (void)cudaGetLastError();
    MLP_TRY(reserve(m, n));
    MLP_CUDA(m, cudaMemcpyAsync(m->xin, x, n * m->dims[0] * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    MLP_CUDA(m, cudaEventRecord(m->t0, m->stream));
    to_bf16_rows_kernel<<<row_grid(n, m->ld0), kT, 0, m->stream>>>(m->xin, m->x, n, m->dims[0], m->ld0);
    return MIND_OK;
}

/* Ends the timed region of a call (after its network work, before its copies back). */
int stop_clock(MindMlp *m) {
    MLP_CUDA(m, cudaEventRecord(m->t1, m->stream));
    return MIND_OK;
}

/* The products' status word: MIND_ETIMEOUT when a wait inside a product ran out. */
int check(MindMlp *m) {
    int32_t code = 0;
    MLP_CUDA(m, cudaMemcpyAsync(&code, m->err, sizeof code, cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(m, cudaStreamSynchronize(m->stream));
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, m->t0, m->t1) == cudaSuccess) m->last_ms = ms;
    if (code) {
        cudaMemsetAsync(m->err, 0, sizeof(int32_t), m->stream);
        return fail(m, code, "a tensor-core product's wait ran out of time");
    }
    return MIND_OK;
}

}  // namespace

/* For the library's own runs (surrogate cells): probabilities of n rows of FP32 inputs that
 * are already on the device, ordered after `stream`'s work and before its later work.  The
 * rows must fit the buffers reserved by mind_mlp_reserve_device; a product whose wait runs
 * out raises MIND_ETIMEOUT in `err` (the run's status word). */
int mind_mlp_forward_device(MindMlp *m, const float *x, int64_t n, float *prob, cudaStream_t stream, int32_t *err) {
    if (n > m->cap) return fail(m, MIND_ECAPACITY, "more rows than reserved");
    if (n == 0) return MIND_OK;
    MLP_CUDA(m, cudaEventRecord(m->ready, stream));
    MLP_CUDA(m, cudaStreamWaitEvent(m->stream, m->ready, 0));
    to_bf16_rows_kernel<<<row_grid(n, m->ld0), kT, 0, m->stream>>>(x, m->x, n, m->dims[0], m->ld0);
    int32_t *own = m->err;
    m->err = err;
    const int s = forward(m, n, false, m->stream, prob);
    m->err = own;
    if (s) return s;
    MLP_CUDA(m, cudaEventRecord(m->done, m->stream));
    MLP_CUDA(m, cudaStreamWaitEvent(stream, m->done, 0));
    return MIND_OK;
}

int mind_mlp_reserve_device(MindMlp *m, int64_t rows) { return reserve(m, rows); }
int32_t mind_mlp_inputs(const MindMlp *m) { return m->dims[0]; }

extern "C" {

int mind_mlp_create(const MindMlpConfig *config, MindMlp **out) {
    if (!config || !out) return MIND_EARG;
    *out = nullptr;
    if (config->n_in < 1 || config->layers < 1 || config->hidden < 16 || config->hidden > 256 ||
        config->hidden % 16)
        return MIND_EARG;
    MindMlp *m = new MindMlp();
    m->hidden = config->hidden;
    m->dims.push_back(config->n_in);
    for (int32_t l = 0; l < config->layers; ++l) m->dims.push_back(config->hidden);
    m->dims.push_back(1);
    m->maps = (int32_t)m->dims.size() - 1;
    m->ld0 = (config->n_in + 7) / 8 * 8;
    for (size_t l = 0; l + 1 < m->dims.size(); ++l) {
        m->w_off.push_back(m->n_params);
        m->n_params += (int64_t)m->dims[l] * m->dims[l + 1];
        m->b_off.push_back(m->n_params);
        m->n_params += m->dims[l + 1];
    }
    // uniform(-1/sqrt(in), 1/sqrt(in)) weights, zero biases, from a 64-bit mix of the seed
    std::vector<float> init(m->n_params, 0.0f);
    uint64_t state = config->seed * 0x9E3779B97F4A7C15ull + 1;
    for (size_t l = 0; l + 1 < m->dims.size(); ++l) {
        const float bound = 1.0f / std::sqrt((float)m->dims[l]);
        for (int64_t k = 0; k < (int64_t)m->dims[l] * m->dims[l + 1]; ++k) {
            state += 0x9E3779B97F4A7C15ull;
            uint64_t z = state;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            const float u = (float)((z >> 11) * (1.0 / 9007199254740992.0));
            init[m->w_off[l] + k] = (2.0f * u - 1.0f) * bound;
        }
    }
    *out = m;
    int s = mind_mlp_set_params(m, init.data(), m->n_params);
    if (s) return s;
    if (cudaMalloc(&m->grad, m->n_params * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&m->m1, m->n_params * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&m->m2, m->n_params * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess)
        return fail(m, MIND_ECUDA, "device allocation failed");
    cudaMemset(m->m1, 0, m->n_params * sizeof(float));
    cudaMemset(m->m2, 0, m->n_params * sizeof(float));
    return MIND_OK;
}

int mind_mlp_destroy(MindMlp *m) {
    if (!m) return MIND_OK;
    if (m->stream) cudaStreamSynchronize(m->stream);
    free_activations(m);
    for (void *p : {(void *)m->master, (void *)m->grad, (void *)m->m1, (void *)m->m2, (void *)m->wbf, (void *)m->w0,
                    (void *)m->wt, (void *)m->loss, (void *)m->loss_hist, (void *)m->data_x, (void *)m->data_y,
                    (void *)m->err, (void *)m->step_dev})
        cudaFree(p);
    if (m->ready) cudaEventDestroy(m->ready);
    if (m->done) cudaEventDestroy(m->done);
    if (m->t0) cudaEventDestroy(m->t0);
    if (m->t1) cudaEventDestroy(m->t1);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return MIND_OK;
}

const char *mind_mlp_last_error(const MindMlp *m) { return m ? m->error.c_str() : "no network"; }

int mind_mlp_last_ms(const MindMlp *m, float *ms) {
    if (!m || !ms) return MIND_EARG;
    *ms = m->last_ms;
    return MIND_OK;
}

int mind_mlp_param_count(const MindMlp *m, int64_t *n) {
    if (!m || !n) return MIND_EARG;
    *n = m->n_params;
    return MIND_OK;
}

int mind_mlp_set_params(MindMlp *m, const float *params, int64_t n) {
    if (!m || !params || n != m->n_params) return MIND_EARG;
    if (!m->stream) {
        MLP_CUDA(m, cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
        MLP_CUDA(m, cudaEventCreateWithFlags(&m->ready, cudaEventDisableTiming));
        MLP_CUDA(m, cudaEventCreateWithFlags(&m->done, cudaEventDisableTiming));
        MLP_CUDA(m, cudaEventCreate(&m->t0));
        MLP_CUDA(m, cudaEventCreate(&m->t1));
        MLP_CUDA(m, cudaMalloc(&m->err, sizeof(int32_t)));
        MLP_CUDA(m, cudaMemsetAsync(m->err, 0, sizeof(int32_t), m->stream));
        MLP_CUDA(m, cudaMalloc(&m->step_dev, sizeof(uint64_t)));
        MLP_TRY(prepare_products(m));
    }
    if (!m->master) {
        const int64_t H = m->hidden;
        MLP_CUDA(m, cudaMalloc(&m->master, n * sizeof(float)));
        MLP_CUDA(m, cudaMalloc(&m->wbf, n * sizeof(__nv_bfloat16)));
        MLP_CUDA(m, cudaMalloc(&m->w0, H * m->ld0 * sizeof(__nv_bfloat16)));
        MLP_CUDA(m, cudaMemsetAsync(m->w0, 0, H * m->ld0 * sizeof(__nv_bfloat16), m->stream));
        MLP_CUDA(m, cudaMalloc(&m->wt, std::max<int64_t>(1, (int64_t)(m->maps - 2) * H * H) * sizeof(__nv_bfloat16)));
    }
    MLP_CUDA(m, cudaMemcpyAsync(m->master, params, n * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    copies_kernel<<<grid(n), kT, 0, m->stream>>>(m->master, n, copy_layout(m));
    MLP_CUDA(m, cudaStreamSynchronize(m->stream));
    return MIND_OK;
}

int mind_mlp_get_params(const MindMlp *m, float *params, int64_t n) {
    if (!m || !params || n != m->n_params) return MIND_EARG;
    if (cudaMemcpy(params, m->master, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) return MIND_ECUDA;
    return MIND_OK;
}

int mind_mlp_predict(MindMlp *m, const float *x, int64_t n, float *prob) {
    if (!m || n < 0 || (n > 0 && (!x || !prob))) return MIND_EARG;
    if (n == 0) return MIND_OK;
    MLP_TRY(upload_rows(m, x, n));
    MLP_TRY(forward(m, n, false, m->stream));
    MLP_TRY(stop_clock(m));
    MLP_CUDA(m, cudaMemcpyAsync(prob, m->prob, n * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    return check(m);
}

int mind_mlp_gradients(MindMlp *m, const float *x, const float *y, int64_t n, float *grad, float *loss) {
    if (!m || n < 1 || !x || !y || !grad || !loss) return MIND_EARG;
    MLP_TRY(reserve(m, n));
    MLP_CUDA(m, cudaMemcpyAsync(m->y, y, n * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    MLP_TRY(upload_rows(m, x, n));
    transpose_inputs(m, n, m->stream);
    MLP_TRY(forward(m, n, true, m->stream));
    MLP_TRY(backward(m, n, m->stream));
    MLP_TRY(stop_clock(m));
    MLP_CUDA(m, cudaMemcpyAsync(grad, m->grad, m->n_params * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(m, cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    return check(m);
}

int mind_mlp_set_data(MindMlp *m, const float *x, const float *y, int64_t n) {
    if (!m || n < 1 || !x || !y) return MIND_EARG;
    if (n > m->data_cap) {
        cudaFree(m->data_x);
        cudaFree(m->data_y);
        m->data_x = m->data_y = nullptr;
        MLP_CUDA(m, cudaMalloc(&m->data_x, n * m->dims[0] * sizeof(float)));
        MLP_CUDA(m, cudaMalloc(&m->data_y, n * sizeof(float)));
        m->data_cap = n;
    }
    MLP_CUDA(m, cudaMemcpyAsync(m->data_x, x, n * m->dims[0] * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    MLP_CUDA(m, cudaMemcpyAsync(m->data_y, y, n * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    MLP_CUDA(m, cudaStreamSynchronize(m->stream));
    m->data_n = n;
    return MIND_OK;
}

int mind_mlp_train(MindMlp *m, int32_t steps, int32_t batch, float lr, float *losses, float *ms) {
    if (!m || steps < 0 || batch < 1 || m->data_n < 1) return MIND_EARG;
    MLP_TRY(reserve(m, batch));
    if (steps > m->loss_cap) {
        cudaFree(m->loss_hist);
        m->loss_hist = nullptr;
        MLP_CUDA(m, cudaMalloc(&m->loss_hist, (size_t)steps * sizeof(float)));
        m->loss_cap = steps;
    }
    const CopyLayout C = copy_layout(m);
    (void)cudaGetLastError();   // the products check their own launches only
    // One Adam step is captured as a graph and replayed `steps` times: the batch draw and the
    // bias corrections read the device step counter, which the step's last kernel advances.
    const uint64_t first = (uint64_t)m->adam_t;
    MLP_CUDA(m, cudaMemcpyAsync(m->step_dev, &first, sizeof first, cudaMemcpyHostToDevice, m->stream));
    MLP_CUDA(m, cudaStreamSynchronize(m->stream));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    MLP_CUDA(m, cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
    gather_kernel<<<row_grid(batch, m->ld0), kT, 0, m->stream>>>(m->data_x, m->data_y, m->x, m->y, m->data_n,
                                                                    m->dims[0], m->ld0, batch, m->step_dev);
    transpose_inputs(m, batch, m->stream);
    int status = forward(m, batch, true, m->stream);
    if (!status) status = backward(m, batch, m->stream);
    adam_kernel<<<grid(m->n_params), kT, 0, m->stream>>>(m->master, m->grad, m->m1, m->m2, m->n_params, lr,
                                                         m->step_dev, C);
    step_end_kernel<<<1, 1, 0, m->stream>>>(m->step_dev, m->loss, m->loss_hist, first);
    const cudaError_t captured = cudaStreamEndCapture(m->stream, &graph);
    if (status) {
        if (graph) cudaGraphDestroy(graph);
        return status;
    }
    MLP_CUDA(m, captured);
    const cudaError_t made = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    MLP_CUDA(m, made);
    MLP_CUDA(m, cudaEventRecord(m->t0, m->stream));
    cudaError_t launched = cudaSuccess;
    for (int32_t k = 0; k < steps && launched == cudaSuccess; ++k) launched = cudaGraphLaunch(exec, m->stream);
    cudaEventRecord(m->t1, m->stream);
    if (launched == cudaSuccess && losses && steps > 0)
        cudaMemcpyAsync(losses, m->loss_hist, (size_t)steps * sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    const cudaError_t sync = cudaStreamSynchronize(m->stream);
    cudaGraphExecDestroy(exec);
    MLP_CUDA(m, launched);
    MLP_CUDA(m, sync);
    m->adam_t += steps;
    const int s = check(m);
    if (ms) *ms = m->last_ms;
    return s;
}

}  // extern "C"
