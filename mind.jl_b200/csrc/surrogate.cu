/*
 * surrogate.cu — the spike-output surrogate: a multilayer perceptron trained on
 * windows the cable solver produced (no counterpart in the reference).
 *
 * Network: n_in -> hidden (SiLU) x layers -> 1 logit; the spike probability of the
 * next 1 ms bin is sigmoid(logit).  Parameters are FP32 masters; every matrix product
 * runs in BF16 with FP32 accumulation on the tensor cores (cuBLAS GEMMs, the plain
 * library case), and the parts around the products are this file's fused kernels:
 * bias + SiLU (keeping the pre-activation for the backward pass) with the BF16 cast
 * for the next product, the sigmoid cross-entropy loss and its gradient, SiLU's
 * derivative applied to the incoming gradient, bias sums, and Adam with the BF16
 * weight copy.  Parameter layout: for each linear map l, W_l [out x in] row-major, then
 * b_l [out], maps in order.
 */
#include <cublas_v2.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mindgpu.h"

struct MindMlp {
    std::vector<int32_t> dims;       // n_in, hidden..., 1
    int32_t ld0 = 0;                 // n_in rounded up to 8: row stride of the BF16 inputs and of w0
    std::vector<int64_t> w_off, b_off;
    int64_t n_params = 0;
    float *master = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
    __nv_bfloat16 *wbf = nullptr;    // BF16 copy of the parameters
    __nv_bfloat16 *w0 = nullptr;     // BF16 first-map weights [dims[1] x ld0], zero past n_in
    float *gw0 = nullptr;            // FP32 first-map weight gradient [dims[1] x ld0]
    float *part = nullptr;           // bias-gradient partial sums [chunks x widest]
    float *loss_hist = nullptr;      // per-step batch losses of a training call
    int32_t loss_cap = 0;
    int64_t adam_t = 0;
    cublasHandle_t blas = nullptr;
    cudaStream_t stream = nullptr;
    int64_t cap = 0;                 // rows the activation buffers hold
    std::vector<float *> z;          // pre-activations per map [cap x out]
    std::vector<__nv_bfloat16 *> h;  // inputs of each map [cap x in] (h[0] = X, rows of ld0)
    __nv_bfloat16 *dzb = nullptr;    // BF16 gradient of a map's output [cap x widest]
    float *dh = nullptr, *dz = nullptr, *y = nullptr, *loss = nullptr;
    float *data_x = nullptr, *data_y = nullptr;  // training set (FP32 on the device)
    int64_t data_n = 0, data_cap = 0;
    std::string error;
};

namespace {

constexpr int kT = 256;

int fail(MindMlp *m, int code, const std::string &why) {
    if (m) m->error = why;
    return code;
}

#define MLP_CUDA(m, call)                                                                         \
    do {                                                                                          \
        cudaError_t _e = (call);                                                                  \
        if (_e != cudaSuccess) return fail((m), MIND_ECUDA, std::string(#call ": ") + cudaGetErrorString(_e)); \
    } while (0)
#define MLP_BLAS(m, call)                                                        \
    do {                                                                         \
        cublasStatus_t _s = (call);                                              \
        if (_s != CUBLAS_STATUS_SUCCESS) return fail((m), MIND_ECUDA, #call);    \
    } while (0)

int grid(int64_t n) { return (int)std::min<int64_t>((n + kT - 1) / kT, 148 * 16); }

__device__ __forceinline__ float sigmoidf_(float x) { return 1.0f / (1.0f + __expf(-x)); }

/* z = acc + b (per column); h_next = BF16(SiLU(z)) unless last. */
__global__ void bias_act_kernel(float *z, const float *b, __nv_bfloat16 *h_next, int64_t rows, int32_t cols, int last) {
    const int64_t n = rows * cols;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const float v = z[k] + b[k % cols];
        z[k] = v;
        if (!last) h_next[k] = __float2bfloat16(v * sigmoidf_(v));
    }
}

/* Mean sigmoid cross-entropy of the logits and its gradient (1/rows) (p - y). */
__global__ void bce_kernel(const float *logit, const float *y, float *dz, float *loss, int64_t rows) {
    float local = 0.0f;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < rows; k += (int64_t)gridDim.x * blockDim.x) {
        const float z = logit[k], t = y[k];
        local += fmaxf(z, 0.0f) - z * t + log1pf(__expf(-fabsf(z)));
        dz[k] = (sigmoidf_(z) - t) / (float)rows;
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, local / (float)rows);
}

__global__ void sigmoid_kernel(const float *logit, float *p, int64_t rows) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < rows; k += (int64_t)gridDim.x * blockDim.x)
        p[k] = sigmoidf_(logit[k]);
}

/* dz = dh * SiLU'(z), and its BF16 copy for the next products. */
__global__ void silu_back_kernel(const float *dh, const float *z, float *dz, __nv_bfloat16 *dzb, int64_t n) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const float s = sigmoidf_(z[k]);
        const float g = dh[k] * (s * (1.0f + z[k] * (1.0f - s)));
        dz[k] = g;
        dzb[k] = __float2bfloat16(g);
    }
}

__global__ void to_bf16_kernel(const float *x, __nv_bfloat16 *out, int64_t n) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        out[k] = __float2bfloat16(x[k]);
}

/* Bias gradients db[c] = sum over rows of dz[r][c], in a fixed order: block (x, y) of
 * 32 x 8 threads sums columns 32x.. of the rows of chunk y (a warp reads 32 consecutive
 * columns of one row), the 8 row phases are added in order into part[y][c]; then
 * colsum_finish adds the chunks in order. */
constexpr int kColChunk = 128;
__global__ void colsum_kernel(const float *dz, float *part, int64_t rows, int32_t cols) {
    __shared__ float acc[8][33];
    const int32_t c = blockIdx.x * 32 + threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.y * kColChunk;
    float s = 0.0f;
    if (c < cols)
        for (int64_t r = r0 + threadIdx.y; r < rows && r < r0 + kColChunk; r += 8) s += dz[r * cols + c];
    acc[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < cols) {
        float t = acc[0][threadIdx.x];
        for (int k = 1; k < 8; ++k) t += acc[k][threadIdx.x];
        part[(int64_t)blockIdx.y * cols + c] = t;
    }
}

__global__ void colsum_finish(const float *part, float *db, int32_t chunks, int32_t cols) {
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
        float t = 0.0f;
        for (int32_t k = 0; k < chunks; ++k) t += part[(int64_t)k * cols + c];
        db[c] = t;
    }
}

/* FP32 rows [n x d] -> BF16 rows of stride ld, zero past d. */
__global__ void to_bf16_rows_kernel(const float *x, __nv_bfloat16 *out, int64_t n, int32_t d, int32_t ld) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n * ld; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = k / ld;
        const int32_t col = (int32_t)(k - row * ld);
        out[k] = __float2bfloat16(col < d ? x[row * d + col] : 0.0f);
    }
}

/* First-map weight gradient, [o x ld] -> the packed [o x d] of the parameter vector. */
__global__ void compact_rows_kernel(const float *in, float *out, int32_t o, int32_t d, int32_t ld) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)o * d;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = k / d;
        out[k] = in[row * ld + (k - row * d)];
    }
}

/* Rows of the training set drawn for one step (Philox-free: a 64-bit mix of step and slot),
 * as BF16 rows of stride ld (zero past d). */
__global__ void gather_kernel(const float *x, const float *y, __nv_bfloat16 *hx, float *hy, int64_t n, int32_t d,
                              int32_t ld, int32_t batch, uint64_t step) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)batch * ld;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = k / ld, col = k % ld;
        uint64_t s = step * 0x9E3779B97F4A7C15ull + (uint64_t)row * 0xBF58476D1CE4E5B9ull + 0x94D049BB133111EBull;
        s ^= s >> 31;
        s *= 0xD6E8FEB86659FD93ull;
        s ^= s >> 32;
        const int64_t src = (int64_t)(s % (uint64_t)n);
        hx[k] = __float2bfloat16(col < d ? x[src * d + col] : 0.0f);
        if (col == 0) hy[row] = y[src];
    }
}

/* Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the FP32 masters, then the BF16 copies (the
 * first map's weights, the first n0 = o*d parameters after w0_off, also into w0 rows of
 * stride ld). */
__global__ void adam_kernel(float *w, const float *g, float *m1, float *m2, __nv_bfloat16 *wbf, int64_t n, float lr,
                            float c1, float c2, __nv_bfloat16 *w0, int64_t w0_off, int64_t n0, int32_t d, int32_t ld) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const float gk = g[k];
        const float a = 0.9f * m1[k] + 0.1f * gk, b = 0.999f * m2[k] + 0.001f * gk * gk;
        m1[k] = a;
        m2[k] = b;
        const float v = w[k] - lr * (a / c1) / (sqrtf(b / c2) + 1e-8f);
        w[k] = v;
        wbf[k] = __float2bfloat16(v);
        const int64_t j = k - w0_off;
        if (j >= 0 && j < n0) w0[(j / d) * ld + j % d] = __float2bfloat16(v);
    }
}

/* w0 from the BF16 copy: rows of stride ld, zero past d. */
__global__ void pad_w0_kernel(const __nv_bfloat16 *wbf, __nv_bfloat16 *w0, int32_t o, int32_t d, int32_t ld) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)o * ld;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = k / ld;
        const int32_t col = (int32_t)(k - row * ld);
        w0[k] = col < d ? wbf[row * d + col] : __float2bfloat16(0.0f);
    }
}

int reserve(MindMlp *m, int64_t rows) {
    if (rows <= m->cap) return MIND_OK;
    const int64_t cap = std::max<int64_t>(rows, 2 * m->cap);
    for (float *p : m->z) cudaFree(p);
    for (__nv_bfloat16 *p : m->h) cudaFree(p);
    cudaFree(m->dzb);
    cudaFree(m->dh);
    cudaFree(m->dz);
    cudaFree(m->y);
    const size_t L = m->dims.size() - 1;
    int32_t widest = 0;
    for (int32_t d : m->dims) widest = std::max(widest, d);
    m->z.assign(L, nullptr);
    m->h.assign(L, nullptr);
    for (size_t l = 0; l < L; ++l) {
        MLP_CUDA(m, cudaMalloc(&m->z[l], cap * m->dims[l + 1] * sizeof(float)));
        MLP_CUDA(m, cudaMalloc(&m->h[l], cap * (l == 0 ? m->ld0 : m->dims[l]) * sizeof(__nv_bfloat16)));
    }
    cudaFree(m->part);
    MLP_CUDA(m, cudaMalloc(&m->part, ((cap + kColChunk - 1) / kColChunk) * widest * sizeof(float)));
    MLP_CUDA(m, cudaMalloc(&m->dzb, cap * widest * sizeof(__nv_bfloat16)));
    MLP_CUDA(m, cudaMalloc(&m->dh, cap * widest * sizeof(float)));
    MLP_CUDA(m, cudaMalloc(&m->dz, cap * widest * sizeof(float)));
    MLP_CUDA(m, cudaMalloc(&m->y, cap * sizeof(float)));
    m->cap = cap;
    return MIND_OK;
}

/* Row-major C[rows x o] = A[rows x i] * W[o x i]^T (BF16 in, FP32 out). */
int gemm_forward(MindMlp *m, const __nv_bfloat16 *A, const __nv_bfloat16 *W, float *C, int64_t rows, int32_t i, int32_t o) {
    const float one = 1.0f, zero = 0.0f;
    MLP_BLAS(m, cublasGemmEx(m->blas, CUBLAS_OP_T, CUBLAS_OP_N, o, (int)rows, i, &one, W, CUDA_R_16BF, i, A,
                             CUDA_R_16BF, i, &zero, C, CUDA_R_32F, o, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT));
    return MIND_OK;
}

/* Forward over `rows` rows whose BF16 inputs are in h[0]; logits end in z.back(). */
int forward(MindMlp *m, int64_t rows) {
    const size_t L = m->dims.size() - 1;
    for (size_t l = 0; l < L; ++l) {
        // the first map runs over ld0 columns (zero past n_in) so every leading dimension
        // is a multiple of 8 BF16 elements
        const int32_t i = l == 0 ? m->ld0 : m->dims[l], o = m->dims[l + 1];
        int s = gemm_forward(m, m->h[l], l == 0 ? m->w0 : m->wbf + m->w_off[l], m->z[l], rows, i, o);
        if (s) return s;
        bias_act_kernel<<<grid(rows * o), kT, 0, m->stream>>>(m->z[l], m->master + m->b_off[l],
                                                               l + 1 < L ? m->h[l + 1] : nullptr, rows, o, l + 1 == L);
    }
    return MIND_OK;
}

/* Gradients of the mean loss into m->grad (targets in m->y); loss into m->loss. */
int backward(MindMlp *m, int64_t rows) {
    const size_t L = m->dims.size() - 1;
    MLP_CUDA(m, cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream));
    bce_kernel<<<grid(rows), kT, 0, m->stream>>>(m->z[L - 1], m->y, m->dz, m->loss, rows);
    to_bf16_kernel<<<grid(rows), kT, 0, m->stream>>>(m->dz, m->dzb, rows);
    const float one = 1.0f, zero = 0.0f;
    const int32_t chunks = (int32_t)((rows + kColChunk - 1) / kColChunk);
    for (size_t l = L; l-- > 0;) {
        const int32_t i = l == 0 ? m->ld0 : m->dims[l], o = m->dims[l + 1];
        // dW[o x i] = dz^T h  (column-major: dWc[i x o] = hc[i x rows] * dzc[o x rows]^T)
        float *dw = l == 0 ? m->gw0 : m->grad + m->w_off[l];
        MLP_BLAS(m, cublasGemmEx(m->blas, CUBLAS_OP_N, CUBLAS_OP_T, i, o, (int)rows, &one, m->h[l], CUDA_R_16BF, i,
                                 m->dzb, CUDA_R_16BF, o, &zero, dw, CUDA_R_32F, i, CUBLAS_COMPUTE_32F,
                                 CUBLAS_GEMM_DEFAULT));
        if (l == 0)
            compact_rows_kernel<<<grid((int64_t)o * m->dims[0]), kT, 0, m->stream>>>(m->gw0, m->grad + m->w_off[0], o,
                                                                                  m->dims[0], m->ld0);
        colsum_kernel<<<dim3((o + 31) / 32, chunks), dim3(32, 8), 0, m->stream>>>(m->dz, m->part, rows, o);
        colsum_finish<<<(o + kT - 1) / kT, kT, 0, m->stream>>>(m->part, m->grad + m->b_off[l], chunks, o);
        if (l == 0) break;
        // dh[rows x i] = dz[rows x o] W[o x i]  (column-major: dhc[i x rows] = Wc[i x o] dzc[o x rows])
        MLP_BLAS(m, cublasGemmEx(m->blas, CUBLAS_OP_N, CUBLAS_OP_N, i, (int)rows, o, &one, m->wbf + m->w_off[l],
                                 CUDA_R_16BF, i, m->dzb, CUDA_R_16BF, o, &zero, m->dh, CUDA_R_32F, i, CUBLAS_COMPUTE_32F,
                                 CUBLAS_GEMM_DEFAULT));
        silu_back_kernel<<<grid(rows * i), kT, 0, m->stream>>>(m->dh, m->z[l - 1], m->dz, m->dzb, rows * i);
    }
    return MIND_OK;
}

int upload_rows(MindMlp *m, const float *x, int64_t n) {
    int s = reserve(m, n);
    if (s) return s;
    const int32_t d = m->dims[0], ld = m->ld0;
    std::vector<__nv_bfloat16> xb((size_t)n * ld, __float2bfloat16(0.0f));
    for (int64_t r = 0; r < n; ++r)
        for (int32_t c = 0; c < d; ++c) xb[(size_t)r * ld + c] = __float2bfloat16(x[(size_t)r * d + c]);
    MLP_CUDA(m, cudaMemcpyAsync(m->h[0], xb.data(), xb.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice, m->stream));
    MLP_CUDA(m, cudaStreamSynchronize(m->stream));
    return MIND_OK;
}

}  // namespace

/* For the library's own runs (surrogate cells): probabilities of n rows of FP32 inputs that
 * are already on the device, ordered after `stream`'s work and before its later work.
 * The rows must fit the buffers reserved by mind_mlp_reserve_device. */
int mind_mlp_forward_device(MindMlp *m, const float *x, int64_t n, float *prob, cudaStream_t stream) {
    if (n > m->cap) return fail(m, MIND_ECAPACITY, "more rows than reserved");
    cudaEvent_t ready, done;
    MLP_CUDA(m, cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    MLP_CUDA(m, cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    cudaEventRecord(ready, stream);
    cudaStreamWaitEvent(m->stream, ready, 0);
    to_bf16_rows_kernel<<<grid(n * m->ld0), kT, 0, m->stream>>>(x, m->h[0], n, m->dims[0], m->ld0);
    int s = forward(m, n);
    if (!s) sigmoid_kernel<<<grid(n), kT, 0, m->stream>>>(m->z.back(), prob, n);
    cudaEventRecord(done, m->stream);
    cudaStreamWaitEvent(stream, done, 0);
    cudaEventDestroy(ready);
    cudaEventDestroy(done);
    return s;
}

int mind_mlp_reserve_device(MindMlp *m, int64_t rows) { return reserve(m, rows); }
int32_t mind_mlp_inputs(const MindMlp *m) { return m->dims[0]; }

extern "C" {

int mind_mlp_create(const MindMlpConfig *config, MindMlp **out) {
    if (!config || !out) return MIND_EARG;
    *out = nullptr;
    if (config->n_in < 1 || config->hidden < 1 || config->layers < 1) return MIND_EARG;
    MindMlp *m = new MindMlp();
    m->dims.push_back(config->n_in);
    for (int32_t l = 0; l < config->layers; ++l) m->dims.push_back(config->hidden);
    m->dims.push_back(1);
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
        cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess ||
        cudaMalloc(&m->gw0, (size_t)m->dims[1] * m->ld0 * sizeof(float)) != cudaSuccess)
        return fail(m, MIND_ECUDA, "device allocation failed");
    cudaMemset(m->m1, 0, m->n_params * sizeof(float));
    cudaMemset(m->m2, 0, m->n_params * sizeof(float));
    return MIND_OK;
}

int mind_mlp_destroy(MindMlp *m) {
    if (!m) return MIND_OK;
    if (m->stream) cudaStreamSynchronize(m->stream);
    for (float *p : m->z) cudaFree(p);
    for (__nv_bfloat16 *p : m->h) cudaFree(p);
    for (void *p : {(void *)m->master, (void *)m->grad, (void *)m->m1, (void *)m->m2, (void *)m->wbf, (void *)m->dzb,
                    (void *)m->dh, (void *)m->dz, (void *)m->y, (void *)m->loss, (void *)m->data_x, (void *)m->data_y,
                    (void *)m->w0, (void *)m->gw0, (void *)m->part, (void *)m->loss_hist})
        cudaFree(p);
    if (m->blas) cublasDestroy(m->blas);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return MIND_OK;
}

const char *mind_mlp_last_error(const MindMlp *m) { return m ? m->error.c_str() : "no network"; }

int mind_mlp_param_count(const MindMlp *m, int64_t *n) {
    if (!m || !n) return MIND_EARG;
    *n = m->n_params;
    return MIND_OK;
}

int mind_mlp_set_params(MindMlp *m, const float *params, int64_t n) {
    if (!m || !params || n != m->n_params) return MIND_EARG;
    if (!m->stream) {
        MLP_CUDA(m, cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
        MLP_BLAS(m, cublasCreate(&m->blas));
        MLP_BLAS(m, cublasSetStream(m->blas, m->stream));
        MLP_BLAS(m, cublasSetMathMode(m->blas, CUBLAS_DEFAULT_MATH));
    }
    if (!m->master) {
        MLP_CUDA(m, cudaMalloc(&m->master, n * sizeof(float)));
        MLP_CUDA(m, cudaMalloc(&m->wbf, n * sizeof(__nv_bfloat16)));
        MLP_CUDA(m, cudaMalloc(&m->w0, (size_t)m->dims[1] * m->ld0 * sizeof(__nv_bfloat16)));
    }
    MLP_CUDA(m, cudaMemcpyAsync(m->master, params, n * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    to_bf16_kernel<<<grid(n), kT, 0, m->stream>>>(m->master, m->wbf, n);
    pad_w0_kernel<<<grid((int64_t)m->dims[1] * m->ld0), kT, 0, m->stream>>>(m->wbf + m->w_off[0], m->w0, m->dims[1],
                                                                           m->dims[0], m->ld0);
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
    int s = upload_rows(m, x, n);
    if (s) return s;
    s = forward(m, n);
    if (s) return s;
    sigmoid_kernel<<<grid(n), kT, 0, m->stream>>>(m->z.back(), m->dz, n);
    MLP_CUDA(m, cudaMemcpyAsync(prob, m->dz, n * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(m, cudaStreamSynchronize(m->stream));
    return MIND_OK;
}

int mind_mlp_gradients(MindMlp *m, const float *x, const float *y, int64_t n, float *grad, float *loss) {
    if (!m || n < 1 || !x || !y || !grad || !loss) return MIND_EARG;
    int s = upload_rows(m, x, n);
    if (s) return s;
    MLP_CUDA(m, cudaMemcpyAsync(m->y, y, n * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    s = forward(m, n);
    if (s) return s;
    s = backward(m, n);
    if (s) return s;
    MLP_CUDA(m, cudaMemcpyAsync(grad, m->grad, m->n_params * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(m, cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(m, cudaStreamSynchronize(m->stream));
    return MIND_OK;
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
    int s = reserve(m, batch);
    if (s) return s;
    if (steps > m->loss_cap) {
        cudaFree(m->loss_hist);
        m->loss_hist = nullptr;
        MLP_CUDA(m, cudaMalloc(&m->loss_hist, (size_t)steps * sizeof(float)));
        m->loss_cap = steps;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, m->stream);
    for (int32_t k = 0; k < steps; ++k) {
        gather_kernel<<<grid((int64_t)batch * m->ld0), kT, 0, m->stream>>>(m->data_x, m->data_y, m->h[0], m->y,
                                                                        m->data_n, m->dims[0], m->ld0, batch,
                                                                        (uint64_t)(m->adam_t + 1));
        s = forward(m, batch);
        if (s) return s;
        s = backward(m, batch);
        if (s) return s;
        m->adam_t += 1;
        const float c1 = 1.0f - std::pow(0.9f, (float)m->adam_t), c2 = 1.0f - std::pow(0.999f, (float)m->adam_t);
        adam_kernel<<<grid(m->n_params), kT, 0, m->stream>>>(m->master, m->grad, m->m1, m->m2, m->wbf, m->n_params,
                                                             lr, c1, c2, m->w0, m->w_off[0],
                                                             (int64_t)m->dims[0] * m->dims[1], m->dims[0], m->ld0);
        // the step's loss stays on the device: no host round trip inside the loop
        MLP_CUDA(m, cudaMemcpyAsync(m->loss_hist + k, m->loss, sizeof(float), cudaMemcpyDeviceToDevice, m->stream));
    }
    cudaEventRecord(e1, m->stream);
    if (losses && steps > 0)
        MLP_CUDA(m, cudaMemcpyAsync(losses, m->loss_hist, (size_t)steps * sizeof(float), cudaMemcpyDeviceToHost,
                                    m->stream));
    MLP_CUDA(m, cudaStreamSynchronize(m->stream));
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return MIND_OK;
}

}  // extern "C"
