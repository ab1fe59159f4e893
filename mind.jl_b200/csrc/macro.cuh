/*
 * macro.cuh — neural-mass regions coupled to the micro network (advance_macro!,
 * src/runtime/step.jl:156-204; src/runtime/cuda/macro.jl).
 *
 * The equations, the input and output rules and the random streams are stated with
 * mind_attach_macro in include/mindgpu.h.  Device layout: region states [n][6] and
 * parameters [n][9] (FP64), an output history ring [hist_cap][n] indexed by macro step,
 * rate-bin spike counts [bin_ring][n], edges sorted by (destination, edge order) as a
 * CSR, inputs as parallel arrays.  Per window, before the micro steps:
 *   macro_advance_kernel  one CTA, a thread per region: RK4 over the window's macro
 *                         steps, a block barrier between steps (edges read other
 *                         regions' history);
 *   macro_input_kernel    a thread per input: Poisson events of the window's macro steps
 *                         through the input source's NetCons into the delivery ring.
 * After the window, route_kernel adds the cell spikes to their regions' rate bins.
 */
#pragma once

#include "kernels.cuh"

namespace mind {

struct MacroParams {
    int32_t n;                 // regions (0: no macro side)
    int32_t steps_per_macro;   // micro steps per macro step
    int32_t macro_per_bin;     // macro steps per rate bin
    int32_t hist_cap;          // output history ring length (> largest delay)
    int32_t bin_ring;
    double dt_s, dt_ms;        // macro step in s (right-hand side) and ms (event times)
    double bin_s;
    uint64_t seed;
    const double *par;         // [n][9]
    double *y;                 // [n][6]
    const double *micro_gain;  // [n]
    const double *cells;       // [n] detector sources per region (as double)
    double *hist;              // [hist_cap][n] out(k) at slot k % hist_cap
    int32_t *bins;             // [bin_ring][n]
    const int32_t *in_off;     // [n+1] CSR of edges by destination
    const int32_t *e_src;      // 0-based source region
    const double *e_gain;
    const int32_t *e_delay;
    int64_t n_inputs;
    const int32_t *inp_region;
    const int32_t *inp_source; // 0-based micro source
    const double *inp_scale;
    const int32_t *source_region;  // [n_sources] region fed by a detector source, or -1
    double *trace;             // [samples][n] out(k) for the run's macro boundaries
    int64_t trace_k0;          // macro step of trace sample 0
    int64_t trace_samples;
};

__host__ __device__ inline double jr_sigmoid(double v, double e0, double r, double v0) {
    return (2.0 * e0) / (1.0 + mind_exp(r * (v0 - v)));
}

/* Jansen-Rit right-hand side (time in s). par = A, B, a, b, e0, r, v0, C, p0. */
__host__ __device__ inline void jr_rhs(const double y[6], double p, const double *par, double dy[6]) {
    const double A = par[0], B = par[1], a = par[2], b = par[3], e0 = par[4], r = par[5], v0 = par[6],
                 C = par[7];
    dy[0] = y[3];
    dy[1] = y[4];
    dy[2] = y[5];
    dy[3] = ((A * a) * jr_sigmoid(y[1] - y[2], e0, r, v0) - (2.0 * a) * y[3]) - (a * a) * y[0];
    dy[4] = ((A * a) * (p + (0.8 * C) * jr_sigmoid(C * y[0], e0, r, v0)) - (2.0 * a) * y[4]) - (a * a) * y[1];
    dy[5] = ((B * b) * ((0.25 * C) * jr_sigmoid((0.25 * C) * y[0], e0, r, v0)) - (2.0 * b) * y[5]) -
            (b * b) * y[2];
}

/* One classical RK4 step of length h (s) with the input p held. */
__host__ __device__ inline void jr_rk4(double y[6], double p, const double *par, double h) {
    double k1[6], k2[6], k3[6], k4[6], t[6];
    jr_rhs(y, p, par, k1);
    for (int j = 0; j < 6; ++j) t[j] = y[j] + (0.5 * h) * k1[j];
    jr_rhs(t, p, par, k2);
    for (int j = 0; j < 6; ++j) t[j] = y[j] + (0.5 * h) * k2[j];
    jr_rhs(t, p, par, k3);
    for (int j = 0; j < 6; ++j) t[j] = y[j] + h * k3[j];
    jr_rhs(t, p, par, k4);
    const double w = h / 6.0;
    for (int j = 0; j < 6; ++j) y[j] = y[j] + w * (((k1[j] + 2.0 * k2[j]) + 2.0 * k3[j]) + k4[j]);
}

__host__ __device__ inline double jr_output(const double y[6], const double *par) {
    return jr_sigmoid(y[1] - y[2], par[4], par[5], par[6]);
}

/* Poisson count (inversion, at most 3) and the uniform offsets of one input's events in
 * macro step k.  Returns n; u[0..n-1] in (0, 1). */
__host__ __device__ inline int macro_input_events(uint64_t seed, int64_t input, int64_t k, double mu, double u[3]) {
    uint32_t ctr[4] = {(uint32_t)k, (uint32_t)((uint64_t)k >> 32), (uint32_t)input, 0x4D4Du};
    mind_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u0 = ((double)ctr[0] + 1.0) * MIND_INV_2P32P1;
    double p = mind_exp(-mu), F = p;
    int n = 0;
    while (u0 > F && n < 3) {
        ++n;
        p = (p * mu) / (double)n;
        F = F + p;
    }
    for (int j = 0; j < 3; ++j) u[j] = ((double)ctr[1 + j] + 1.0) * MIND_INV_2P32P1;
    return n;
}

/* Regions over macro steps [k0, k1) starting inside this window (one CTA). */
__global__ void macro_advance_kernel(const MacroParams M, int64_t k0, int64_t k1, int32_t zero_bin_slot) {
    const int32_t i = threadIdx.x;
    if (zero_bin_slot >= 0 && i < M.n) M.bins[(int64_t)zero_bin_slot * M.n + i] = 0;
    double y[6];
    if (i < M.n)
        for (int j = 0; j < 6; ++j) y[j] = M.y[(int64_t)i * 6 + j];
    for (int64_t k = k0; k < k1; ++k) {
        if (i < M.n) {
            const double *par = M.par + (int64_t)i * 9;
            const int64_t b = k / M.macro_per_bin - 1;
            const double rate =
                b >= 0 ? (double)M.bins[(b % M.bin_ring) * M.n + i] / (M.cells[i] * M.bin_s) : 0.0;
            double p = par[8] + M.micro_gain[i] * rate;
            for (int32_t e = M.in_off[i]; e < M.in_off[i + 1]; ++e) {
                int64_t m = k - M.e_delay[e];
                if (m < 0) m = 0;
                p = p + M.e_gain[e] * M.hist[(m % M.hist_cap) * M.n + M.e_src[e]];
            }
            jr_rk4(y, p, par, M.dt_s);
            const double out = jr_output(y, par);
            M.hist[((k + 1) % M.hist_cap) * M.n + i] = out;
            const int64_t sample = k + 1 - M.trace_k0;
            if (M.trace && sample >= 0 && sample < M.trace_samples) M.trace[sample * M.n + i] = out;
        }
        __syncthreads();
    }
    if (i < M.n)
        for (int j = 0; j < 6; ++j) M.y[(int64_t)i * 6 + j] = y[j];
}

/* Poisson input events of macro steps [k0, k1) through each input source's NetCons. */
__global__ void macro_input_kernel(const Params P, const MacroParams M, int64_t k0, int64_t k1, int64_t min_bin) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < M.n_inputs;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int32_t region = M.inp_region[q];
        const int32_t source = M.inp_source[q];
        for (int64_t k = k0; k < k1; ++k) {
            const double out = M.hist[(k % M.hist_cap) * M.n + region];
            const double mu = (M.inp_scale[q] * out) * M.dt_s;
            double u[3];
            const int n = macro_input_events(M.seed, q, k, mu, u);
            for (int j = 0; j < n; ++j) fan_out(P, source, (double)k * M.dt_ms + M.dt_ms * u[j], min_bin);
        }
    }
}

/* out(k0) for the first trace sample of a run (the regions' state at its start). */
__global__ void macro_trace_start_kernel(const MacroParams M, int64_t k) {
    const int32_t i = threadIdx.x;
    if (i < M.n && M.trace && M.trace_samples > 0 && k == M.trace_k0)
        M.trace[i] = M.hist[(k % M.hist_cap) * M.n + i];
}

/* initialize!: states, output history (every slot holds out(0)) and rate bins. */
__global__ void macro_init_kernel(const MacroParams M, const double *y0) {
    const int32_t i = threadIdx.x;
    if (i >= M.n) return;
    double y[6];
    for (int j = 0; j < 6; ++j) y[j] = M.y[(int64_t)i * 6 + j] = y0[(int64_t)i * 6 + j];
    const double out = jr_output(y, M.par + (int64_t)i * 9);
    for (int32_t s = 0; s < M.hist_cap; ++s) M.hist[(int64_t)s * M.n + i] = out;
    for (int32_t s = 0; s < M.bin_ring; ++s) M.bins[(int64_t)s * M.n + i] = 0;
}

}  // namespace mind

namespace mind {

/* Surrogate cells' inputs for the bin `b` that starts now: the drive of bins b-20..b-1
 * (times `scale`, 0 before the run's first bin) and their own spikes in bins b-5..b-1. */
__global__ void surrogate_features_kernel(const Params P, const int32_t *cells, int32_t n, const int32_t *spikes,
                                          float scale, int64_t b, float *x) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)n * 645;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = k / 645, j = k % 645;
        const int32_t c = cells[i];
        float v = 0.0f;
        if (j < 640) {
            const int64_t bin = b - 20 + j / 32;
            if (bin >= 0) v = scale * P.sur_drive[((bin % kSurrogateRing) * P.ncells + c) * 32 + (j % 32)];
        } else {
            const int64_t bin = b - 5 + (j - 640);
            if (bin >= 0) v = (float)spikes[(bin % 6) * (int64_t)n + i];
        }
        x[k] = v;
    }
}

/* Each surrogate cell spikes in bin b with the predicted probability, its logit shifted by
 * the cell's calibration offset (u0 < p, Philox on (b, cell)), at b * bin_ms + bin_ms * u1;
 * the spike is recorded, fanned out through the cell's NetCons and counted in its region's
 * bin like a detected spike. */
__global__ void surrogate_spike_kernel(const Params P, const int32_t *cells, const int32_t *sources, int32_t n,
                                       const float *prob, const float *offset, int32_t *spikes, int64_t b,
                                       double bin_ms,
                                       const int32_t *source_region, int32_t *bins, int32_t n_regions,
                                       int32_t bin_ring, int64_t min_bin) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t ctr[4] = {(uint32_t)b, (uint32_t)((uint64_t)b >> 32), (uint32_t)cells[i], 0x5355u};
        mind_philox4x32_10(ctr, (uint32_t)P.seed, (uint32_t)(P.seed >> 32));
        const double u0 = ((double)ctr[0] + 1.0) * MIND_INV_2P32P1, u1 = ((double)ctr[1] + 1.0) * MIND_INV_2P32P1;
        double p = prob[i];
        const double shift = offset[cells[i]];
        if (shift != 0.0) {   // sigmoid(logit + shift) from sigmoid(logit)
            const double e = exp(shift);
            p = p * e / (1.0 - p + p * e);
        }
        const bool fire = u0 < p;
        spikes[(b % 6) * (int64_t)n + i] = fire ? 1 : 0;
        const int32_t src = sources[i];
        if (!fire || src < 0) continue;
        const double t = (double)b * bin_ms + bin_ms * u1;
        record_spike(P, src, t);
        fan_out(P, src, t, min_bin);
        if (n_regions > 0) {
            const int32_t region = source_region[src];
            if (region >= 0) atomicAdd(&bins[(b % bin_ring) * n_regions + region], 1);
        }
    }
}

}  // namespace mind
