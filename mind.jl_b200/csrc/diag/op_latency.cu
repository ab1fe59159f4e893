/*
 * op_latency.cu — dependent-chain latency of the operations on the Hines solve's critical
 * path, on one warp (diagnostic; not part of libmindgpu.so).
 *
 * Each loop runs 256 dependent instances of one operation between clock64() reads:
 *   dfma            x = fma(x, y, z)
 *   dadd            x = x + y
 *   rcp.approx.f64  x = rcp.approx.ftz.f64(x)
 *   ddiv            x = y / x                     (IEEE division, as the FP64 path uses)
 *   lds+use         shared-memory load whose value feeds the next address (with one DMUL)
 *   ffma+cvt        FP32 fma between f64->f32 and f32->f64 conversions
 * Build and run (one GPU):
 *   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o op_latency op_latency.cu && ./op_latency
 */
#include <cstdio>
#include <cuda_runtime.h>

__global__ void op_latency(double *io, long long *cycles) {
    double x = io[0];
    const double y = io[1], z = io[2];
    __shared__ double sh[32];
    long long t[8];
    t[0] = clock64();
#pragma unroll 1
    for (int k = 0; k < 256; ++k) x = fma(x, y, z);
    t[1] = clock64();
#pragma unroll 1
    for (int k = 0; k < 256; ++k) x = x + y;
    t[2] = clock64();
#pragma unroll 1
    for (int k = 0; k < 256; ++k) {
        double r;
        asm volatile("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
        x = r;
    }
    t[3] = clock64();
#pragma unroll 1
    for (int k = 0; k < 256; ++k) x = y / x;
    t[4] = clock64();
    sh[threadIdx.x] = x;
    __syncwarp();
    int idx = threadIdx.x;
    t[5] = clock64();
#pragma unroll 1
    for (int k = 0; k < 256; ++k) {
        const double v = sh[idx];
        idx = (int)(v * 0.0) + ((idx + 1) & 31);
    }
    t[6] = clock64();
#pragma unroll 1
    for (int k = 0; k < 256; ++k) {
        float f = (float)x;
        f = __fmaf_rn(f, 1.0001f, 0.5f);
        x = (double)f;
    }
    t[7] = clock64();
    if (threadIdx.x == 0)
        for (int k = 0; k < 6; ++k) cycles[k] = t[k + 1 + (k >= 4 ? 1 : 0)] - t[k + (k >= 4 ? 1 : 0)];
    io[3 + threadIdx.x] = x + idx;
}

int main() {
    double *io;
    long long *cycles;
    cudaMalloc(&io, 40 * sizeof(double));
    cudaMalloc(&cycles, 8 * sizeof(long long));
    const double init[3] = {1.0000001, 0.9999999, 1e-9};
    cudaMemcpy(io, init, sizeof init, cudaMemcpyHostToDevice);
    for (int rep = 0; rep < 2; ++rep) op_latency<<<1, 32>>>(io, cycles);
    long long host[6];
    cudaMemcpy(host, cycles, sizeof host, cudaMemcpyDeviceToHost);
    const char *names[6] = {"dfma", "dadd", "rcp.approx.f64", "ddiv", "lds+use", "ffma+cvt"};
    for (int k = 0; k < 6; ++k) printf("%-15s %6.1f cycles per dependent operation\n", names[k], host[k] / 256.0);
    const cudaError_t e = cudaDeviceSynchronize();
    printf("%s\n", cudaGetErrorString(e));
    return e == cudaSuccess ? 0 : 1;
}
