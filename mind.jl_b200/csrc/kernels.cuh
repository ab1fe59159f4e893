/*
 * kernels.cuh — the sm_100a kernels of the per-micro-step loop.
 *
 *   netstim_kernel   NetStim self-events up to the window horizon; spikes are
 *                    recorded and routed into the delivery ring
 *                    (mod/NetStim.mod; src/runtime/events.jl:57-165).
 *   bucket_kernel    moves the window's delivery bins into per-cell inboxes.
 *   window_kernel    one CTA per cell, W micro steps with the cell resident in
 *                    shared memory: threshold detection, event delivery,
 *                    BREAKPOINT currents, cable assembly, Hines solve, voltage
 *                    update, cnexp advance, recording
 *                    (src/runtime/step.jl:91-151; src/runtime/cuda/micro.jl:285-749).
 *   route_kernel     fans the window's cell spikes out to the ring
 *                    (src/runtime/utils/events.jl:52-62).
 */
#pragma once

#include "device.cuh"

namespace mind {

__device__ __forceinline__ void raise_error(int32_t *error, int code) { atomicMax(error, code); }

/* Smallest delivery bin m >= 0 whose cutoff m*dt + dt/2 is at or after `time`. */
__host__ __device__ inline int64_t delivery_bin(double time, double dt) {
    double half = 0.5 * dt;
    double estimate = ceil((time - half) / dt);
    int64_t m = estimate < 0.0 ? 0 : (int64_t)estimate;
    for (int k = 0; k < 4 && m > 0 && time <= (double)(m - 1) * dt + half; ++k) --m;
    for (int k = 0; k < 4 && time > (double)m * dt + half; ++k) ++m;
    return m;
}

__device__ __forceinline__ void ring_insert(const Params &P, double time, int32_t edge, int32_t point,
                                            int64_t min_bin) {
    int64_t bin = delivery_bin(time, P.dt);
    if (bin < min_bin) {
        raise_error(P.error, MIND_ESELFEVENT);
        return;
    }
    int32_t slot = (int32_t)(bin % P.ring_slots);
    int32_t idx = atomicAdd(&P.ring_count[slot], 1);
    if (idx < P.ring_cap) {
        RingEvent e;
        e.time = time;
        e.edge = edge;
        e.point = point;
        P.ring[(int64_t)slot * P.ring_cap + idx] = e;
    } else {
        raise_error(P.error, MIND_ECAPACITY);
    }
}

__device__ __forceinline__ void record_spike(const Params &P, int32_t source, double time) {
    if (!P.record_spikes) return;
    int32_t idx = atomicAdd(P.rec_spike_count, 1);
    if (idx < P.rec_spike_cap) {
        P.rec_spike_source[idx] = source;
        P.rec_spike_time[idx] = time;
    } else {
        raise_error(P.error, MIND_ECAPACITY);
    }
}

__device__ __forceinline__ void fan_out(const Params &P, int32_t source, double time, int64_t min_bin) {
    for (int64_t e = P.fanout_off[source]; e < P.fanout_off[source + 1]; ++e)
        ring_insert(P, time + P.edge_delay[e], (int32_t)e, P.edge_target[e], min_bin);
}

/* ---------------- hh (mod/hh.mod) ---------------- */

__device__ __forceinline__ double vtrap(double x, double y) {
    if (fabs(x / y) < 1e-6) return y * (1.0 - x / y / 2.0);
    return x / (mind_exp(x / y) - 1.0);
}

struct HHRates {
    double minf, hinf, ninf, mtau, htau, ntau;
};

__device__ __forceinline__ HHRates hh_rates(double v, double celsius) {
    HHRates R;
    double q10 = mind_pow(3.0, (celsius - 6.3) / 10.0);
    double alpha = 0.1 * vtrap(-(v + 40.0), 10.0);
    double beta = 4.0 * mind_exp(-(v + 65.0) / 18.0);
    double sum = alpha + beta;
    R.mtau = 1.0 / (q10 * sum);
    R.minf = alpha / sum;
    alpha = 0.07 * mind_exp(-(v + 65.0) / 20.0);
    beta = 1.0 / (mind_exp(-(v + 35.0) / 10.0) + 1.0);
    sum = alpha + beta;
    R.htau = 1.0 / (q10 * sum);
    R.hinf = alpha / sum;
    alpha = 0.01 * vtrap(-(v + 55.0), 10.0);
    beta = 0.125 * mind_exp(-(v + 65.0) / 80.0);
    sum = alpha + beta;
    R.ntau = 1.0 / (q10 * sum);
    R.ninf = alpha / sum;
    return R;
}

/* One gate of hh_rates (0 = m, 1 = h, 2 = n) with the identical operations, so the
 * three gates of a row can advance on three threads; q10 = 3^((celsius - 6.3)/10)
 * is computed once by the caller with the same pow. */
__device__ __forceinline__ void hh_gate(double v, double q10, int gate, double &inf, double &tau) {
    double alpha, beta;
    if (gate == 0) {
        alpha = 0.1 * vtrap(-(v + 40.0), 10.0);
        beta = 4.0 * mind_exp(-(v + 65.0) / 18.0);
    } else if (gate == 1) {
        alpha = 0.07 * mind_exp(-(v + 65.0) / 20.0);
        beta = 1.0 / (mind_exp(-(v + 35.0) / 10.0) + 1.0);
    } else {
        alpha = 0.01 * vtrap(-(v + 55.0), 10.0);
        beta = 0.125 * mind_exp(-(v + 65.0) / 80.0);
    }
    const double sum = alpha + beta;
    tau = 1.0 / (q10 * sum);
    inf = alpha / sum;
}

__device__ __forceinline__ double cnexp(double s, double inf, double tau, double dt) {
    return s + (1.0 - mind_exp(dt * (-1.0 / tau))) * (inf - s);
}

/* (x)/0.001 of the current probe: the IEEE quotient in FP64 mode (division-free,
 * mind_div_milli); in the mixed mode a multiplication by 1000, within one ulp. */
template <bool MIXED>
__device__ __forceinline__ double milli_quotient(double x) {
    return MIXED ? x * 1000.0 : mind_div_milli(x);
}

/* 1/x for the mixed mode's Hines solve: the hardware reciprocal seed (relative error
 * below 2^-19.9 measured over 4M operands on B200) refined by one Newton-Raphson step
 * y <- y + y(1 - x y), which squares the error to below 2^-39 (1e-12 relative), in FP64
 * arithmetic.  Replacing it by the correctly rounded quotient changes the mixed mode's
 * 1 s config-3 max |dV| against FP64 in the tenth digit: the FP32 gating dominates. */
__device__ __forceinline__ double approx_reciprocal(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

/* FP32 gating for the mixed mode: hh's rate equations in single precision.  The cnexp
 * factor 1 - exp(-dt/tau) is formed as -expm1f(-dt/tau) and vtrap's x/(exp(x/y) - 1) as
 * x/expm1f(x/y): 1 - exp(-x) for the x = dt/tau ~ 0.005-0.2 of a step would lose up to
 * four of FP32's seven digits to cancellation, and the gate increment is that product. */
__device__ __forceinline__ float vtrapf(float x, float y) {
    if (fabsf(x / y) < 1e-6f) return y * (1.0f - x / y / 2.0f);
    return x / expm1f(x / y);
}

__device__ __forceinline__ float cnexp_factor_f32(float dt, float tau) { return -expm1f(dt * (-1.0f / tau)); }

/* One gate's steady state and cnexp factor in FP32 (0 = m, 1 = h, 2 = n); the caller
 * applies s + factor * (inf - s) to the FP64 state, so rounding does not accumulate in
 * the stored gates over a long run. */
__device__ __forceinline__ void hh_gate_f32(double v, float q10, float dt, int gate, float &inf, float &factor) {
    // The voltage offsets are formed in FP64 before rounding to FP32, so a membrane near
    // rest keeps its small distance from each rate's midpoint exactly.
    float alpha, beta;
    if (gate == 0) {
        alpha = 0.1f * vtrapf((float)(-(v + 40.0)), 10.0f);
        beta = 4.0f * expf((float)(-(v + 65.0)) / 18.0f);
    } else if (gate == 1) {
        alpha = 0.07f * expf((float)(-(v + 65.0)) / 20.0f);
        beta = 1.0f / (expf((float)(-(v + 35.0)) / 10.0f) + 1.0f);
    } else {
        alpha = 0.01f * vtrapf((float)(-(v + 55.0)), 10.0f);
        beta = 0.125f * expf((float)(-(v + 65.0)) / 80.0f);
    }
    const float sum = alpha + beta;
    inf = alpha / sum;
    factor = cnexp_factor_f32(dt, 1.0f / (q10 * sum));
}

/* Sum of hh's current fields in the reference's order: il, then ina, then ik. */
__device__ __forceinline__ double hh_current(double u, double m, double h, double n, double gnabar,
                                             double gkbar, double gl, double el, double ena, double ek) {
    double gna = gnabar * m * m * m * h;
    double ina = gna * (u - ena);
    double gk = gkbar * n * n * n * n;
    double ik = gk * (u - ek);
    double il = gl * (u - el);
    return ((0.0 + il) + ina) + ik;
}

/* ---------------- NetStim (mod/NetStim.mod) ---------------- */

struct NetStimRow {
    double interval, number, noise, event, on, ispike, next_t, next_flag;
};

__device__ __forceinline__ double ns_invl(NetStimRow &s, MindRan &ran, uint64_t seed, double mean) {
    if (mean <= 0.0) mean = 0.01;
    if (s.noise == 0.0) return mean;
    double erand = mind_ran_negexp(&ran, seed);
    return (1.0 - s.noise) * mean + s.noise * mean * erand;
}

__device__ __forceinline__ bool ns_send(const Params &P, NetStimRow &s, double t, double delay, double flag) {
    if (delay < 0.0 || !isfinite(delay)) {
        raise_error(P.error, MIND_ESELFEVENT);
        return false;
    }
    s.next_t = t + delay;
    s.next_flag = flag;
    return true;
}

/* Processes every self-event with time <= horizon.  Events never target a
 * NetStim from outside (rejected at mind_create), so at most one self-event
 * is pending per row. */
__global__ void netstim_kernel(const Params P, double horizon, int64_t min_bin) {
    const DevGroup &G = P.groups[P.ns_group];
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < G.rows; r += gridDim.x * blockDim.x) {
        NetStimRow s;
        s.next_flag = G.f[NS_NEXT_FLAG][r];
        s.next_t = G.f[NS_NEXT_T][r];
        if (s.next_flag < 0.0 || s.next_t > horizon) continue;
        s.interval = G.f[NS_INTERVAL][r];
        s.number = G.f[NS_NUMBER][r];
        s.noise = G.f[NS_NOISE][r];
        s.event = G.f[NS_EVENT][r];
        s.on = G.f[NS_ON][r];
        s.ispike = G.f[NS_ISPIKE][r];
        MindRan ran = P.ns_ran[r];
        const int32_t source = P.ns_source[r];
        for (int guard = 0; guard < (1 << 20) && s.next_flag >= 0.0 && s.next_t <= horizon; ++guard) {
            double t = s.next_t;
            double flag = s.next_flag;
            s.next_flag = -1.0;
            if (flag == 3.0) {
                if (s.on == 1.0) {
                    if (s.number > 0.0) {
                        s.on = 1.0;
                        s.event = 0.0;
                        s.ispike = 0.0;
                    }
                    ns_send(P, s, t, 0.0, 1.0);
                }
            }
            if (flag == 1.0 && s.on == 1.0) {
                s.ispike = s.ispike + 1.0;
                if (source >= 0) {
                    record_spike(P, source, t);
                    fan_out(P, source, t, min_bin);
                }
                if (s.number > 0.0) s.event = ns_invl(s, ran, P.seed, s.interval);
                if (s.ispike >= s.number) s.on = 0.0;
                if (s.on == 1.0) ns_send(P, s, t, s.event, 1.0);
            }
        }
        G.f[NS_EVENT][r] = s.event;
        G.f[NS_ON][r] = s.on;
        G.f[NS_ISPIKE][r] = s.ispike;
        G.f[NS_NEXT_T][r] = s.next_t;
        G.f[NS_NEXT_FLAG][r] = s.next_flag;
        P.ns_ran[r] = ran;
    }
}

/* NetStim INITIAL at t = 0 (mod/NetStim.mod INITIAL; micro.jl:79-91 for the stream ids). */
__global__ void netstim_init_kernel(const Params P, uint64_t digest, const uint64_t *logical) {
    const DevGroup &G = P.groups[P.ns_group];
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < G.rows; r += gridDim.x * blockDim.x) {
        MindRan ran;
        mind_ran_init(&ran, logical[r], digest, 0u, P.seed);
        mind_ran_setseq(&ran, 0.0, P.seed);
        NetStimRow s;
        s.interval = G.f[NS_INTERVAL][r];
        s.number = G.f[NS_NUMBER][r];
        s.noise = G.f[NS_NOISE][r];
        double start = G.f[NS_START][r];
        s.event = G.f[NS_EVENT][r];
        s.on = 0.0;
        s.ispike = 0.0;
        s.next_t = 0.0;
        s.next_flag = -1.0;
        if (s.noise < 0.0) s.noise = 0.0;
        if (s.noise > 1.0) s.noise = 1.0;
        if (start >= 0.0 && s.number > 0.0) {
            s.on = 1.0;
            double ev = start + ns_invl(s, ran, P.seed, s.interval) - s.interval * (1.0 - s.noise);
            if (ev < 0.0) ev = 0.0;
            s.event = ev;
            ns_send(P, s, 0.0, ev, 3.0);
        }
        G.f[NS_NOISE][r] = s.noise;
        G.f[NS_EVENT][r] = s.event;
        G.f[NS_ON][r] = s.on;
        G.f[NS_ISPIKE][r] = s.ispike;
        G.f[NS_NEXT_T][r] = s.next_t;
        G.f[NS_NEXT_FLAG][r] = s.next_flag;
        P.ns_ran[r] = ran;
    }
}

/* INITIAL of a group emitted from a MOD file, at t = 0 on the initial voltage. */
__device__ __forceinline__ void generated_init_rows(const Params &P, int32_t g) {
    const DevGroup &G = P.groups[g];
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < G.rows; r += gridDim.x * blockDim.x) {
        const MindGenRow row{G.cols, G.rows, r, P.v[G.node[r]], 0.0, P.dt, P.celsius};
        gen_initial(G.gen, row);
    }
}

/* INITIAL blocks of the cell mechanisms; decay factors of the synapses. */
__global__ void mechanism_init_kernel(const Params P, int32_t g) {
    const DevGroup &G = P.groups[g];
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < G.rows; r += gridDim.x * blockDim.x) {
        if (G.gen >= 0) {   // emitted from a MOD file: INITIAL at t = 0 on the initial voltage
            const MindGenRow row{G.cols, G.rows, r, P.v[G.node[r]], 0.0, P.dt, P.celsius};
            gen_initial(G.gen, row);
            continue;
        }
        switch (G.kind) {
            case MIND_MECH_HH: {
                HHRates R = hh_rates(P.v[G.node[r]], P.celsius);
                G.f[HH_M][r] = R.minf;
                G.f[HH_H][r] = R.hinf;
                G.f[HH_N][r] = R.ninf;
            } break;
            case MIND_MECH_EXPSYN: {
                G.f[ES_G][r] = 0.0;
                double decay = 1.0 - mind_exp(P.dt * (-1.0 / G.f[ES_TAU][r]));
                G.f[ES_DECAY][r] = decay;
                G.s[ESS_DECAY][r] = (float)decay;
            } break;
            case MIND_MECH_EXP2SYN: {
                double tau1 = G.f[E2_TAU1][r];
                double tau2 = G.f[E2_TAU2][r];
                if (tau1 / tau2 > 0.9999) tau1 = 0.9999 * tau2;
                if (tau1 / tau2 < 1e-9) tau1 = tau2 * 1e-9;
                G.f[E2_TAU1][r] = tau1;
                G.f[E2_A][r] = 0.0;
                G.f[E2_B][r] = 0.0;
                double tp = (tau1 * tau2) / (tau2 - tau1) * mind_log(tau2 / tau1);
                double factor = -mind_exp(-tp / tau1) + mind_exp(-tp / tau2);
                G.f[E2_FACTOR][r] = 1.0 / factor;
                double d1 = 1.0 - mind_exp(P.dt * (-1.0 / tau1));
                double d2 = 1.0 - mind_exp(P.dt * (-1.0 / tau2));
                G.f[E2_DECAY1][r] = d1;
                G.f[E2_DECAY2][r] = d2;
                G.s[E2S_DECAY1][r] = (float)d1;
                G.s[E2S_DECAY2][r] = (float)d2;
            } break;
            default:
                break;
        }
    }
}

/* First pass of the window's inbox: events per cell in bins n0 .. n0+W-1 (grid y = bin). */
__global__ void inbox_count_kernel(const Params P, int64_t n0) {
    const int64_t bin = n0 + blockIdx.y;
    const int32_t slot = (int32_t)(bin % P.ring_slots);
    const int32_t count = min(P.ring_count[slot], P.ring_cap);
    const RingEvent *events = P.ring + (int64_t)slot * P.ring_cap;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        atomicAdd(&P.inbox_count[P.point_cell[events[i].point]], 1);
}

/* Exclusive prefix sum of the per-cell counts into inbox_start[0 .. ncells], one block of
 * kScanThreads threads, each summing a contiguous run of cells.  A window whose events
 * exceed the inbox raises status 3 (its cells then read no events). */
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) inbox_scan_kernel(const Params P) {
    __shared__ int32_t warp_total[kScanThreads / 32];
    const int32_t n = P.ncells;
    const int32_t per = (n + kScanThreads - 1) / kScanThreads;
    const int32_t lo = min(n, (int32_t)threadIdx.x * per), hi = min(n, lo + per);
    int32_t local = 0;
    for (int32_t i = lo; i < hi; ++i) local += P.inbox_count[i];
    const int32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t x = local;   // inclusive scan within the warp
    for (int32_t off = 1; off < 32; off <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warp_total[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int32_t w = warp_total[lane];   // kScanThreads / 32 == 32 warps
        for (int32_t off = 1; off < 32; off <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        warp_total[lane] = w;
    }
    __syncthreads();
    int32_t base = (warp > 0 ? warp_total[warp - 1] : 0) + x - local;
    for (int32_t i = lo; i < hi; ++i) {
        P.inbox_start[i] = base;
        base += P.inbox_count[i];
    }
    if (threadIdx.x == kScanThreads - 1) {
        const int32_t total = warp_total[31];
        P.inbox_start[n] = total;
        if (total > P.inbox_total) raise_error(P.error, MIND_ECAPACITY);
    }
}

/* Second pass: moves bins n0 .. n0+W-1 from the ring into the cells' inbox slices. */
__global__ void bucket_kernel(const Params P, int64_t n0) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *P.win_spike_count = 0;
    const int64_t bin = n0 + blockIdx.y;
    const int32_t slot = (int32_t)(bin % P.ring_slots);
    int32_t count = P.ring_count[slot];
    if (count > P.ring_cap) count = P.ring_cap;
    const RingEvent *events = P.ring + (int64_t)slot * P.ring_cap;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        RingEvent e = events[i];
        int32_t cell = P.point_cell[e.point];
        const int64_t idx = (int64_t)P.inbox_start[cell] + atomicAdd(&P.inbox_fill[cell], 1);
        if (idx < P.inbox_total) {
            InboxEvent x;
            x.time = e.time;
            x.edge = e.edge;
            x.point = e.point;
            x.bin = bin;
            P.inbox[idx] = x;
        }
    }
}

/* Routes the window's cell spikes (detected at step s, time s*dt + 1e-10); with regions
 * attached, also counts each spike into its region's rate bin (bin_steps micro steps). */
__global__ void route_kernel(const Params P, int64_t window_end, const int32_t *source_region, int32_t *bins,
                             int32_t n_regions, int32_t bin_steps, int32_t bin_ring) {
    const int32_t count = min(*P.win_spike_count, P.win_spike_cap);
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        int32_t source = P.win_spike_source[i];
        const int64_t step = P.win_spike_step[i];
        double time = (double)step * P.dt + 1.0e-10;
        record_spike(P, source, time);
        fan_out(P, source, time, window_end);
        if (n_regions > 0) {
            const int32_t region = source_region[source];
            if (region >= 0) atomicAdd(&bins[((step / bin_steps) % bin_ring) * n_regions + region], 1);
        }
    }
}

__device__ __forceinline__ bool event_before(const InboxEvent &x, const InboxEvent &y) {
    if (x.bin != y.bin) return x.bin < y.bin;
    if (x.point != y.point) return x.point < y.point;
    if (x.time != y.time) return x.time < y.time;
    return x.edge < y.edge;
}

/* order[rank] = k for the m events ev[0..m) sorted by event_before, ties by index: each thread
 * ranks its events against all others.  ev and order are the staged copies in shared memory,
 * or the cell's inbox slice and order slice in HBM when its events exceed the staging. */
template <int NT>
__device__ __forceinline__ void sort_events(const InboxEvent *ev, int32_t m, int32_t *order) {
    for (int32_t k = threadIdx.x; k < m; k += NT) {
        int32_t rank = 0;
        const InboxEvent mine = ev[k];
        for (int32_t j = 0; j < m; ++j) {
            const InboxEvent other = ev[j];
            if (event_before(other, mine) || (j < k && !event_before(mine, other))) ++rank;
        }
        order[rank] = k;
    }
}

/* One mechanism group of the resident cell: staged state in shared memory, the rest in HBM. */
struct StagedGroup {
    int32_t kind, rows, r0;   // r0 = first device row of the cell
    double *f;                // staged FP64 slots [slots][rows]
    int32_t *node;            // local node per row
    __device__ __forceinline__ double &at(int slot, int r) const { return f[slot * rows + r]; }
};

/* NET_RECEIVE of the synapses (mod/ExpSyn.mod: g += w; mod/Exp2Syn.mod: A += w*factor,
 * B += w*factor) on a staged row; `inc` is w, or w*factor for Exp2Syn. */
__device__ __forceinline__ void apply_event(const StagedGroup &G, int32_t row, double inc) {
    if (G.kind == MIND_MECH_EXPSYN) {
        G.at(0, row) = G.at(0, row) + inc;
    } else if (G.kind == MIND_MECH_EXP2SYN) {
        G.at(0, row) = G.at(0, row) + inc;
        G.at(1, row) = G.at(1, row) + inc;
    }
}

/*
 * Hines solve of one resident cell, FP64 mode: the reference's operations in the
 * canonical order (gather-form elimination, f = a/D, back-substitution (R + a x_p)/D).
 * Level by level, one path per thread (a path is one chain, or a chain and the child chains
 * it continues when the cell's plan merged them): a path's chains are eliminated deepest
 * first and back-substituted in the reverse order, each child chain ready before its parent
 * (on the path, by the same thread; off it, in a lower level).  Along a chain only subtract
 * -> divide -> multiply stays on the dependency chain, the next node's operands being
 * loaded before the current division.  pch null: the cell's paths are its chains (lvp holds
 * chain starts), the loops are the one-chain-per-thread loops.
 */
template <int NT>
__device__ __forceinline__ void hines_exact(double *sd, double *sr, const double *sa, double *sv, double *sxd,
                                            double *sxr, const int32_t *ctop, const int32_t *clen,
                                            const int32_t *cpar, const int32_t *ckoff, const int32_t *ckids,
                                            const int32_t *lvp, const int32_t *pch, int32_t nlev, double vscale,
                                            bool &singular) {
    constexpr int32_t T = NT;
    const int32_t tid = threadIdx.x;
    for (int32_t lv = 0; lv < nlev; ++lv) {
        for (int32_t p = lvp[lv] + tid; p < lvp[lv + 1]; p += T)
        for (int32_t ch = pch ? pch[p] : p, end = pch ? pch[p + 1] : p + 1; ch < end; ++ch) {
            const int32_t top = ctop[ch];
            const int32_t bottom = top + clen[ch] - 1;
            const bool rooted = cpar[ch] < 0;
            double D = sd[bottom], R = sr[bottom];
            for (int32_t q = ckoff[ch]; q < ckoff[ch + 1]; ++q) {
                const int32_t cc = ckids[q];
                D = D - sxd[cc];
                R = R + sxr[cc];
            }
            singular |= (D == 0.0) | !isfinite(D);
            sd[bottom] = D;
            sr[bottom] = R;
            double pxd = 0.0, pxr = 0.0;
            if (bottom > top || !rooted) {
                const double ab = sa[bottom];
                double dn = 0.0, rn = 0.0, an = 0.0;
                if (bottom > top) {
                    dn = sd[bottom - 1];
                    rn = sr[bottom - 1];
                    an = sa[bottom - 1];
                }
                const double f = ab / D;
                pxd = f * ab;
                pxr = f * R;
                // interior nodes: every one has its parent at i - 1
                int32_t i = bottom - 1;
                for (; i > top; --i) {
                    const double Di = dn - pxd, Ri = rn + pxr, ai = an;
                    dn = sd[i - 1];
                    rn = sr[i - 1];
                    an = sa[i - 1];
                    singular |= (Di == 0.0) | !isfinite(Di);
                    sd[i] = Di;
                    sr[i] = Ri;
                    const double fi = ai / Di;
                    pxd = fi * ai;
                    pxr = fi * Ri;
                }
                if (i == top && bottom > top) {
                    const double Dt = dn - pxd, Rt = rn + pxr;
                    singular |= (Dt == 0.0) | !isfinite(Dt);
                    sd[top] = Dt;
                    sr[top] = Rt;
                    if (!rooted) {
                        const double ft = an / Dt;
                        pxd = ft * an;
                        pxr = ft * Rt;
                    }
                }
            }
            sxd[ch] = pxd;
            sxr[ch] = pxr;
        }
        __syncthreads();
    }
    for (int32_t lv = nlev - 1; lv >= 0; --lv) {
        for (int32_t p = lvp[lv] + tid; p < lvp[lv + 1]; p += T)
        for (int32_t ch = (pch ? pch[p + 1] : p + 1) - 1, first = pch ? pch[p] : p; ch >= first; --ch) {
            const int32_t top = ctop[ch];
            const int32_t bottom = top + clen[ch] - 1;
            const int32_t par = cpar[ch];
            double rn = sr[top], an = sa[top], dn = sd[top];
            double x;
            {
                const double ri = rn, ai = an, di = dn;
                const double xp = par >= 0 ? sr[par] : 0.0;
                if (top < bottom) {
                    rn = sr[top + 1];
                    an = sa[top + 1];
                    dn = sd[top + 1];
                }
                x = (par >= 0 ? ri + ai * xp : ri) / di;
                sr[top] = x;
                sv[top] = sv[top] + vscale * x;
            }
            for (int32_t i = top + 1; i <= bottom; ++i) {
                const double ri = rn, ai = an, di = dn;
                if (i < bottom) {
                    rn = sr[i + 1];
                    an = sa[i + 1];
                    dn = sd[i + 1];
                }
                x = (ri + ai * x) / di;
                sr[i] = x;
                sv[i] = sv[i] + vscale * x;
            }
        }
        __syncthreads();
    }
}

/*
 * Hines solve, mixed mode: FP64 arithmetic with reciprocals.  Elimination keeps, per
 * node, f = a/D in place of D and R/D in place of R, so the back-substitution is one
 * FMA per node, x = f x_p + R/D; the pivot chain is D -> 1/D -> (a^2)(1/D) -> next D.
 * One path per thread, level by level, as in the FP64 solve.
 */
template <int NT>
__device__ __forceinline__ void hines_mixed(double *sd, double *sr, const double *sa, double *sv, double *sxd,
                                            double *sxr, const int32_t *ctop, const int32_t *clen,
                                            const int32_t *cpar, const int32_t *ckoff, const int32_t *ckids,
                                            const int32_t *lvp, const int32_t *pch, int32_t nlev, double vscale,
                                            bool &singular) {
    constexpr int32_t T = NT;
    const int32_t tid = threadIdx.x;
    for (int32_t lv = 0; lv < nlev; ++lv) {
        for (int32_t p = lvp[lv] + tid; p < lvp[lv + 1]; p += T)
        for (int32_t ch = pch ? pch[p] : p, end = pch ? pch[p + 1] : p + 1; ch < end; ++ch) {
            const int32_t top = ctop[ch];
            const int32_t bottom = top + clen[ch] - 1;
            const bool rooted = cpar[ch] < 0;
            double D = sd[bottom], R = sr[bottom];
            for (int32_t q = ckoff[ch]; q < ckoff[ch + 1]; ++q) {
                const int32_t cc = ckids[q];
                D = D - sxd[cc];
                R = R + sxr[cc];
            }
            singular |= (D == 0.0) | !isfinite(D);
            const double ab = sa[bottom];
            double dn = 0.0, rn = 0.0, an = 0.0;
            if (bottom > top) {
                dn = sd[bottom - 1];
                rn = sr[bottom - 1];
                an = sa[bottom - 1];
            }
            const double y = approx_reciprocal(D);
            const double f = ab * y;
            sd[bottom] = f;
            sr[bottom] = R * y;
            double pxd = (ab * ab) * y, pxr = f * R;
            int32_t i = bottom - 1;
            for (; i > top; --i) {
                const double Di = dn - pxd, Ri = rn + pxr, ai = an, asq = an * an;
                dn = sd[i - 1];
                rn = sr[i - 1];
                an = sa[i - 1];
                singular |= (Di == 0.0) | !isfinite(Di);
                const double yi = approx_reciprocal(Di);
                const double fi = ai * yi;
                sd[i] = fi;
                sr[i] = Ri * yi;
                pxd = asq * yi;
                pxr = fi * Ri;
            }
            if (bottom > top) {
                const double Dt = dn - pxd, Rt = rn + pxr;
                singular |= (Dt == 0.0) | !isfinite(Dt);
                const double yt = approx_reciprocal(Dt);
                const double ft = an * yt;
                sd[top] = ft;
                sr[top] = Rt * yt;
                pxd = (an * an) * yt;
                pxr = ft * Rt;
            }
            sxd[ch] = rooted ? 0.0 : pxd;
            sxr[ch] = rooted ? 0.0 : pxr;
        }
        __syncthreads();
    }
    for (int32_t lv = nlev - 1; lv >= 0; --lv) {
        for (int32_t p = lvp[lv] + tid; p < lvp[lv + 1]; p += T)
        for (int32_t ch = (pch ? pch[p + 1] : p + 1) - 1, first = pch ? pch[p] : p; ch >= first; --ch) {
            const int32_t top = ctop[ch];
            const int32_t bottom = top + clen[ch] - 1;
            const int32_t par = cpar[ch];
            double fn = sd[top], qn = sr[top];
            double x = par >= 0 ? fma(fn, sr[par], qn) : qn;
            sr[top] = x;
            sv[top] = sv[top] + vscale * x;
            if (top < bottom) {
                fn = sd[top + 1];
                qn = sr[top + 1];
            }
            for (int32_t i = top + 1; i <= bottom; ++i) {
                const double fi = fn, qi = qn;
                if (i < bottom) {
                    fn = sd[i + 1];
                    qn = sr[i + 1];
                }
                x = fma(fi, x, qi);
                sr[i] = x;
                sv[i] = sv[i] + vscale * x;
            }
        }
        __syncthreads();
    }
}

/*
 * One CTA of four warps advances one cell through W micro steps.  Shared memory
 * holds what the serial parts of the step touch: v, d, rhs and axial
 * conductance of every node, the chain tables of the Hines solve, the state
 * that changes every step (hh gates, synaptic conductances) and the window's
 * events.  Parameter-only data (pas rows, synapse constants, IClamp rows,
 * C/dt, axial_diagonal) is streamed from HBM each step with coalesced loads.
 *
 * The Hines solve runs level by level, one path per thread (a chain, or on cells the plan
 * gave paths a chain and the child chains it continues); along a chain only subtract ->
 * divide -> multiply stays on the dependency chain, the next node's operands being loaded
 * ahead.  PATHS false compiles the one-chain-per-thread loops only, for launches whose
 * cells all have the chain schedule.
 */
template <bool MIXED, int NT, bool GLOBAL_IMAGE = false, bool GEN = false, bool PATHS = true>
__device__ __forceinline__ void window_body(const Params &P, const int32_t *cells, int64_t n0, int32_t W) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ StagedGroup sg[kMaxGroups];
    const int32_t c = cells[blockIdx.x];
    const int32_t tid = threadIdx.x;
    constexpr int32_t T = NT;            // threads of this launch
    constexpr int32_t O = kCellThreads;  // owner slots: node i belongs to slot i % O
    static_assert(O % T == 0, "a thread serves whole owner slots");
    const int64_t nb = P.node_off[c];
    const int32_t n = (int32_t)(P.node_off[c + 1] - nb);
    const int32_t cb = P.chain_off[c];
    const int32_t nch = P.chain_off[c + 1] - cb;
    const int32_t kb = P.chain_kid_off[cb];
    const int32_t nkids = P.chain_kid_off[cb + nch] - kb;
    const int32_t lv0 = P.level_off[c];
    const int32_t nlev = P.level_off[c + 1] - lv0 - 1;
    const int32_t pb = P.path_off[c];
    const int32_t npath = P.path_off[c + 1] - pb - 1;

    // ---- carve the cell image (order fixed by cell_smem_bytes): shared memory, or for a
    //      cell larger than one CTA's shared memory its own slot of an HBM buffer ----
    unsigned char *image = smem_raw;
    if (GLOBAL_IMAGE) image = P.big_image + (int64_t)P.big_slot[c] * P.big_stride;
    double *dp = reinterpret_cast<double *>(image);
    double *sv = dp; dp += n;
    double *sd = dp; dp += n;
    double *sr = dp; dp += n;
    double *sa = dp; dp += n;
    double *sxd = dp; dp += nch;
    double *sxr = dp; dp += nch;
    double *sw = dp; dp += P.inbox_cap;
    for (int32_t g = 0; g < P.ngroups; ++g) {
        const DevGroup &G = P.groups[g];
        const bool staged = kind_staged(G.kind);
        const int32_t r0 = G.row_off[c];
        const int32_t rows = G.kind == MIND_MECH_NETSTIM ? 0 : G.row_off[c + 1] - r0;
        if (tid == 0) {
            sg[g].kind = G.kind;
            sg[g].rows = rows;
            sg[g].r0 = r0;
            sg[g].f = dp;
        }
        if (staged) dp += (size_t)staged_doubles(G.kind) * rows;
    }
    InboxEvent *sev = reinterpret_cast<InboxEvent *>(dp);
    int32_t *ip = reinterpret_cast<int32_t *>(sev + P.inbox_cap);
    for (int32_t g = 0; g < P.ngroups; ++g) {
        const DevGroup &G = P.groups[g];
        const int32_t rows = kind_staged(G.kind) ? G.row_off[c + 1] - G.row_off[c] : 0;
        if (tid == 0) sg[g].node = ip;
        ip += rows;
    }
    int32_t *ctop = ip; ip += nch;
    int32_t *clen = ip; ip += nch;
    int32_t *cpar = ip; ip += nch;
    int32_t *ckoff = ip; ip += nch + 1;
    int32_t *ckids = ip; ip += nkids;
    int32_t *lvp = ip; ip += nlev + 1;
    int32_t *pch = ip; ip += npath + 1;
    int32_t *sorder = ip; ip += P.inbox_cap;
    int32_t *spart = ip; ip += P.ngroups * (O + 1);   // the threads' row ranges per group
    int16_t *chain_of = reinterpret_cast<int16_t *>(ip);
    {
        // The launch sized the image for this cell's bin; refuse rather than overrun.
        uint32_t dynamic_bytes;
        if (GLOBAL_IMAGE)
            dynamic_bytes = (uint32_t)P.big_stride;
        else
            asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dynamic_bytes));
        const size_t used = (size_t)(reinterpret_cast<unsigned char *>(chain_of + n) - image);
        if (used > dynamic_bytes) {
            if (tid == 0) raise_error(P.error, MIND_ELAYOUT);
            return;
        }
    }

    // ---- stage the cell ----
    if (blockIdx.x == 0)
        for (int32_t k = tid; k < W; k += T) P.ring_count[(n0 + k) % P.ring_slots] = 0;
    // The cell's events of this window: its slice of the window's inbox.  Up to inbox_cap of
    // them are staged and sorted in shared memory; more are sorted in place in HBM.
    const int32_t ib = P.inbox_start[c];
    int32_t nev = P.inbox_start[c + 1] - ib;
    if (ib < 0 || nev < 0 || (int64_t)ib + nev > P.inbox_total) nev = 0;   // window overflow: status 3 raised
    const bool staged_ev = nev <= P.inbox_cap;
    const InboxEvent *gev = P.inbox + (staged_ev ? 0 : ib);
    int32_t *gorder = P.inbox_order + (staged_ev ? 0 : ib);
    const InboxEvent *ev = staged_ev ? sev : gev;
    int32_t *evorder = staged_ev ? sorder : gorder;
    if (tid == 0) {   // the next window counts afresh
        P.inbox_count[c] = 0;
        P.inbox_fill[c] = 0;
    }
    if (staged_ev)
        for (int32_t k = tid; k < nev; k += T) sev[k] = P.inbox[(int64_t)ib + k];
    if (P.cell_mode && P.cell_mode[c]) {
        // A cell the surrogate stands in for: its membrane is not simulated; its window's
        // events only add their NetCon weights to its drive, per rate bin and synapse group,
        // in the canonical event order (so the sums, and the run, are reproducible).
        __syncthreads();
        sort_events<T>(ev, nev, evorder);
        __syncthreads();
        if (tid == 0)
            for (int32_t k = 0; k < nev; ++k) {
                const InboxEvent e = ev[evorder[k]];
                if (e.edge < 0) continue;
                const int32_t g = P.point_group[e.point];
                const int32_t row = P.point_row[e.point] - P.groups[g].row_off[c];
                const int64_t bin = e.bin / P.sur_bin_steps;
                P.sur_drive[((bin % kSurrogateRing) * P.ncells + c) * 32 + (row & 31)] += (float)P.edge_weight[e.edge];
            }
        return;
    }
    for (int32_t i = tid; i < n; i += T) {
        sv[i] = P.v[nb + i];
        sa[i] = P.a[nb + i];
    }
    for (int32_t k = tid; k < nch; k += T) {
        ctop[k] = P.chain_top[cb + k];
        clen[k] = P.chain_len[cb + k];
        cpar[k] = P.chain_par[cb + k];
        ckoff[k] = P.chain_kid_off[cb + k] - kb;
    }
    if (tid == 0) ckoff[nch] = nkids;
    for (int32_t k = tid; k < nkids; k += T) ckids[k] = P.chain_kids[kb + k];
    for (int32_t k = tid; k <= nlev; k += T) lvp[k] = P.level_path[lv0 + k];
    for (int32_t k = tid; k <= npath; k += T) pch[k] = P.path_chain[pb + k];
    for (int32_t k = tid; k < P.ngroups * (O + 1); k += T) spart[k] = P.part[(int64_t)c * P.ngroups * (O + 1) + k];
    __syncthreads();
    for (int32_t k = tid; k < nch; k += T)
        for (int32_t i = ctop[k]; i < ctop[k] + clen[k]; ++i) chain_of[i] = (int16_t)k;
    for (int32_t g = 0; g < P.ngroups; ++g) {
        const DevGroup &G = P.groups[g];
        const StagedGroup &S = sg[g];
        if (!kind_staged(S.kind) || S.rows == 0) continue;
        for (int32_t r = tid; r < S.rows; r += T) {
            const int32_t row = S.r0 + r;
            switch (S.kind) {
                case MIND_MECH_HH:
                    for (int k = 0; k < HH_NSLOT; ++k) S.at(k, r) = G.f[k][row];
                    break;
                case MIND_MECH_EXPSYN:
                    S.at(0, r) = G.f[ES_G][row];
                    break;
                case MIND_MECH_EXP2SYN:
                    S.at(0, r) = G.f[E2_A][row];
                    S.at(1, r) = G.f[E2_B][row];
                    break;
            }
            S.node[r] = (int32_t)(G.node[row] - nb);
        }
    }
    // Detectors stay in registers for the window (at most one per lane; checked at mind_create).
    const int32_t d0 = P.det_off[c], d1 = P.det_off[c + 1];
    int32_t my_det = -1, my_src = 0;
    double my_thr = 0.0;
    bool my_above = false;
    if (tid < d1 - d0) {
        my_det = P.det_node[d0 + tid];
        my_src = P.det_source[d0 + tid];
        my_thr = P.det_thr[d0 + tid];
        my_above = P.above[my_src] != 0;
    }
    __syncthreads();
    sort_events<T>(ev, nev, evorder);
    __syncthreads();
    // Resolve each staged event's target to (group, staged row) and its increment once per
    // window (events read from HBM are resolved as they are applied, with the same operations).
    for (int32_t k = tid; k < (staged_ev ? nev : 0); k += T) {
        InboxEvent &e = sev[k];
        const int32_t g = P.point_group[e.point];
        const int32_t drow = P.point_row[e.point];
        const double w = e.edge >= 0 ? P.edge_weight[e.edge] : 0.0;
        sw[k] = P.groups[g].kind == MIND_MECH_EXP2SYN ? w * P.groups[g].f[E2_FACTOR][drow] : w;
        e.point = (g << 24) | (drow - sg[g].r0);
    }
    __syncthreads();

    const double q10 = mind_pow(3.0, (P.celsius - 6.3) / 10.0);
    const float q10f = (float)q10;
    int32_t cursor = 0;
    bool singular = false;

    for (int32_t s = 0; s < W; ++s) {
        const int64_t step = n0 + s;
        const double t = (double)step * P.dt;

        // 1. Threshold detection from the completed boundary.
        if (my_det >= 0) {
            const bool current = sv[my_det] > my_thr;
            if (current && !my_above) {
                int32_t idx = atomicAdd(P.win_spike_count, 1);
                if (idx < P.win_spike_cap) {
                    P.win_spike_source[idx] = my_src;
                    P.win_spike_step[idx] = step;
                } else {
                    raise_error(P.error, MIND_ECAPACITY);
                }
            }
            my_above = current;
        }
        // 2. Deliver this step's bin in (target, time, edge) order.
        if (tid == 0) {
            while (cursor < nev) {
                InboxEvent e;
                int32_t g, row;
                double inc;
                if (staged_ev) {
                    const int32_t k = sorder[cursor];
                    e = sev[k];
                    g = e.point >> 24;
                    row = e.point & 0xffffff;
                    inc = sw[k];
                } else {
                    e = gev[gorder[cursor]];
                    g = P.point_group[e.point];
                    const int32_t drow = P.point_row[e.point];
                    row = drow - sg[g].r0;
                    const double w = e.edge >= 0 ? P.edge_weight[e.edge] : 0.0;
                    inc = P.groups[g].kind == MIND_MECH_EXP2SYN ? w * P.groups[g].f[E2_FACTOR][drow] : w;
                }
                if (e.bin > step) break;
                if (e.bin < step) raise_error(P.error, MIND_ESELFEVENT);
                if (GEN && P.groups[g].gen >= 0) {   // emitted NET_RECEIVE, flag 0, at the event's time
                    const DevGroup &GG = P.groups[g];
                    const int64_t grow = (int64_t)sg[g].r0 + row;
                    const MindGenRow gr{GG.cols, GG.rows, grow, sv[(int32_t)(GG.node[grow] - nb)], e.time, P.dt,
                                        P.celsius};
                    gen_receive(GG.gen, gr, inc, 0.0);
                } else {
                    apply_event(sg[g], row, inc);
                }
                if (P.drive && e.edge >= 0) {
                    // synaptic drive for the surrogate's training data: NetCon weight by
                    // (run bin, cell, synapse row mod 32)
                    const int64_t b = (step - P.run_start) / P.drive_bin_steps;
                    if (b < P.drive_bins)
                        P.drive[(b * P.ncells + c) * 32 + (row & 31)] += (float)P.edge_weight[e.edge];
                }
                ++cursor;
            }
        }
        __syncthreads();  // NET_RECEIVE above wrote staged synapse state

        // 3-5. Node i belongs to owner slot i % O and thread t serves the slots t, t + T, ...
        //      (a warp's lanes touch consecutive nodes, so shared memory serves them without
        //      bank conflicts), with the rows of every group on those nodes, which the device
        //      row order keeps as one range per slot.  The mechanism sums of a node are
        //      accumulated in group order, rows in row order, by one thread, and its assembly
        //      follows without a barrier (it reads only the unchanged v of neighbours).
        //      Parameters are streamed from HBM through the read-only path.
        for (int32_t i = tid; i < n; i += T) {
            sd[i] = 0.0;
            sr[i] = 0.0;
        }
        const double tc = t + 0.5 * P.dt;
        for (int32_t g = 0; g < P.ngroups; ++g) {
            const DevGroup &GG = P.groups[g];
            const StagedGroup G = sg[g];
            for (int32_t slot = tid; slot < O; slot += T) {
                const int32_t lo = spart[g * (O + 1) + slot], hi = spart[g * (O + 1) + slot + 1];
                if (lo >= hi) continue;
                if (G.kind == MIND_MECH_PAS) {
                    if (MIXED) continue;  // folded into the node constants of the assembly below
                    const double *pg = GG.f[PAS_G] + G.r0, *pe = GG.f[PAS_E] + G.r0, *ps = GG.f[PAS_SCALE] + G.r0;
                    const int32_t *pn = GG.node + G.r0;
                    for (int32_t r = lo; r < hi; ++r) {
                        const int32_t node = (int32_t)(__ldg(pn + r) - nb);
                        const double gp = __ldg(pg + r), ep = __ldg(pe + r), scale = __ldg(ps + r);
                        const double vv = sv[node];
                        const double probe = vv + 0.001;
                        const double shifted = 0.0 + gp * (probe - ep);
                        const double value = 0.0 + gp * (vv - ep);
                        sr[node] = sr[node] - scale * value;
                        sd[node] = sd[node] + milli_quotient<MIXED>(scale * (shifted - value));
                    }
                } else if (G.kind == MIND_MECH_ICLAMP) {
                    const int32_t *pn = GG.node + G.r0;
                    for (int32_t r = lo; r < hi; ++r) {
                        const int32_t node = (int32_t)(__ldg(pn + r) - nb);
                        const int64_t q = (int64_t)G.r0 + r;
                        const double del = __ldg(GG.f[IC_DEL] + q);
                        const double i = (tc < del + __ldg(GG.f[IC_DUR] + q) && tc >= del) ? __ldg(GG.f[IC_AMP] + q) : 0.0;
                        const double shifted = 0.0 - i;
                        const double value = 0.0 - i;
                        sr[node] = sr[node] + -1.0 * value;
                        sd[node] = sd[node] + milli_quotient<MIXED>(1.0 * (shifted - value));
                    }
                } else if (G.kind == MIND_MECH_ALPHASYN) {
                    // g = gmax alpha((t - onset)/tau), i = g (v - e) at the step's mid time
                    const int32_t *pn = GG.node + G.r0;
                    for (int32_t r = lo; r < hi; ++r) {
                        const int32_t node = (int32_t)(__ldg(pn + r) - nb);
                        const int64_t q = (int64_t)G.r0 + r;
                        const double gs = __ldg(GG.f[AS_GMAX] + q) *
                                          mind_alpha((tc - __ldg(GG.f[AS_ONSET] + q)) / __ldg(GG.f[AS_TAU] + q));
                        const double e = __ldg(GG.f[AS_E] + q);
                        const double vv = sv[node];
                        if (MIXED) {  // linear in v: the probe's difference quotient is g
                            sr[node] = sr[node] - gs * (vv - e);
                            sd[node] = sd[node] + gs;
                            continue;
                        }
                        const double probe = vv + 0.001;
                        const double shifted = 0.0 + gs * (probe - e);
                        const double value = 0.0 + gs * (vv - e);
                        sr[node] = sr[node] + -1.0 * value;
                        sd[node] = sd[node] + milli_quotient<MIXED>(1.0 * (shifted - value));
                    }
                } else if (GEN && GG.gen >= 0) {
                    // emitted from a MOD file: BREAKPOINT probed at v + 0.001 and at v
                    // (src/runtime/cuda/micro.jl:427-500); the second call's writes persist
                    const int32_t *pn = GG.node + G.r0;
                    const double *pscale = GG.cols + (int64_t)GG.ncols * GG.rows + G.r0;
                    for (int32_t r = lo; r < hi; ++r) {
                        const int32_t node = (int32_t)(__ldg(pn + r) - nb);
                        const double vv = sv[node];
                        MindGenRow row{GG.cols, GG.rows, (int64_t)G.r0 + r, vv + 0.001, tc, P.dt, P.celsius};
                        const double shifted = gen_current(GG.gen, row);
                        row.v = vv;
                        const double value = gen_current(GG.gen, row);
                        const double scale = pscale[r];
                        sr[node] = sr[node] - scale * value;
                        sd[node] = sd[node] + milli_quotient<MIXED>(scale * (shifted - value));
                    }
                } else if (G.kind == MIND_MECH_HH) {
                    for (int32_t r = lo; r < hi; ++r) {
                        const int32_t node = G.node[r];
                        const double vv = sv[node];
                        const double probe = vv + 0.001;
                        const double m = G.at(HH_M, r), h = G.at(HH_H, r), nn = G.at(HH_N, r);
                        if (MIXED) {
                            // at fixed gates the current is linear in v: dI/dv is the summed conductance
                            const double gna = G.at(HH_GNABAR, r) * m * m * m * h;
                            const double gk = G.at(HH_GKBAR, r) * nn * nn * nn * nn;
                            const double gl = G.at(HH_GL, r);
                            const double i = gl * (vv - G.at(HH_EL, r)) + gna * (vv - G.at(HH_ENA, r)) +
                                             gk * (vv - G.at(HH_EK, r));
                            const double scale = G.at(HH_SCALE, r);
                            sr[node] = sr[node] - scale * i;
                            sd[node] = sd[node] + scale * (gna + gk + gl);
                            continue;
                        }
                        const double shifted = hh_current(probe, m, h, nn, G.at(HH_GNABAR, r), G.at(HH_GKBAR, r),
                                                          G.at(HH_GL, r), G.at(HH_EL, r), G.at(HH_ENA, r), G.at(HH_EK, r));
                        const double value = hh_current(vv, m, h, nn, G.at(HH_GNABAR, r), G.at(HH_GKBAR, r),
                                                        G.at(HH_GL, r), G.at(HH_EL, r), G.at(HH_ENA, r), G.at(HH_EK, r));
                        const double scale = G.at(HH_SCALE, r);
                        sr[node] = sr[node] - scale * value;
                        sd[node] = sd[node] + milli_quotient<MIXED>(scale * (shifted - value));
                    }
                } else if (G.kind == MIND_MECH_EXPSYN || G.kind == MIND_MECH_EXP2SYN) {
                    const bool two = G.kind == MIND_MECH_EXP2SYN;
                    const double *pe = GG.f[two ? E2_E : ES_E] + G.r0;
                    for (int32_t r = lo; r < hi; ++r) {
                        const int32_t node = G.node[r];
                        const double e = __ldg(pe + r);
                        double gs;
                        if (two)
                            gs = G.at(1, r) - G.at(0, r);
                        else
                            gs = G.at(0, r);
                        const double vv = sv[node];
                        if (MIXED) {  // linear in v: the probe's difference quotient is the conductance
                            sr[node] = sr[node] - gs * (vv - e);
                            sd[node] = sd[node] + gs;
                            continue;
                        }
                        const double probe = vv + 0.001;
                        const double shifted = 0.0 + gs * (probe - e);
                        const double value = 0.0 + gs * (vv - e);
                        sr[node] = sr[node] + -1.0 * value;
                        sd[node] = sd[node] + milli_quotient<MIXED>(1.0 * (shifted - value));
                    }
                }
            }
        }
        // Cable assembly of the owned nodes: d = C/dt + d + axial_diagonal; own axial term, then children.
        for (int32_t i = tid; i < n; i += T) {
            const int64_t gi = nb + i;
            const int32_t k = chain_of[i];
            const int32_t top = ctop[k];
            const int32_t bottom = top + clen[k] - 1;
            const double vi = sv[i];
            double R = sr[i];
            if (MIXED) {
                sd[i] = __ldg(P.mix_dc + gi) + sd[i];
                R = R + (__ldg(P.mix_gse + gi) - __ldg(P.mix_gs + gi) * vi);
            } else {
                sd[i] = (__ldg(P.cdt + gi) + sd[i]) + __ldg(P.ad + gi);
            }
            const int32_t p = i == top ? cpar[k] : i - 1;
            if (p >= 0) R = R + sa[i] * (sv[p] - vi);
            if (i < bottom) {
                R = R - sa[i + 1] * (vi - sv[i + 1]);
            } else {
                for (int32_t q = ckoff[k]; q < ckoff[k + 1]; ++q) {
                    const int32_t kt = ctop[ckids[q]];
                    R = R - sa[kt] * (vi - sv[kt]);
                }
            }
            sr[i] = R;
        }
        __syncthreads();

        // 6-7. Hines elimination level by level, each chain bottom to top into its parent,
        //      then back-substitution root chain first with the voltage update.
        if (MIXED) {
            hines_mixed<NT>(sd, sr, sa, sv, sxd, sxr, ctop, clen, cpar, ckoff, ckids, lvp,
                          PATHS && npath ? pch : nullptr, nlev, P.vscale, singular);
        } else {
            hines_exact<NT>(sd, sr, sa, sv, sxd, sxr, ctop, clen, cpar, ckoff, ckids, lvp,
                          PATHS && npath ? pch : nullptr, nlev, P.vscale, singular);
        }

        // 8. cnexp state advance on the new voltage (time t + dt).
        for (int32_t g = 0; g < P.ngroups; ++g) {
            const DevGroup &GG = P.groups[g];
            const StagedGroup G = sg[g];
            if (GEN && GG.gen >= 0) {   // emitted from a MOD file: its hoisted SOLVE statements
                for (int32_t r = tid; r < G.rows; r += T) {
                    const int64_t row = (int64_t)G.r0 + r;
                    const MindGenRow gr{GG.cols, GG.rows, row, sv[(int32_t)(__ldg(GG.node + row) - nb)], t + P.dt, P.dt,
                                        P.celsius};
                    gen_advance(GG.gen, gr);
                }
                continue;
            }
            switch (G.kind) {
                case MIND_MECH_HH:
                    // one thread per (row, gate): m, h and n advance independently
                    if (MIXED) {
                        for (int32_t w = tid; w < 3 * G.rows; w += T) {
                            const int32_t r = w / 3, gate = w - 3 * r;
                            float inf, factor;
                            hh_gate_f32(sv[G.node[r]], q10f, (float)P.dt, gate, inf, factor);
                            const int slot = HH_M + gate;
                            const double state = G.at(slot, r);
                            G.at(slot, r) = state + (double)factor * ((double)inf - state);
                        }
                    } else {
                        for (int32_t w = tid; w < 3 * G.rows; w += T) {
                            const int32_t r = w / 3, gate = w - 3 * r;
                            const double vv = sv[G.node[r]];
                            double inf, tau;
                            hh_gate(vv, q10, gate, inf, tau);
                            const int slot = HH_M + gate;
                            G.at(slot, r) = cnexp(G.at(slot, r), inf, tau, P.dt);
                        }
                    }
                    break;
                case MIND_MECH_EXPSYN: {
                    const double *pdec = GG.f[ES_DECAY] + G.r0;
                    const float *pdecf = GG.s[ESS_DECAY] + G.r0;
                    for (int32_t r = tid; r < G.rows; r += T) {
                        if (MIXED) {
                            // FP32 decrement, FP64 accumulation
                            const double gs = G.at(0, r);
                            G.at(0, r) = gs + (double)(pdecf[r] * (0.0f - (float)gs));
                        } else {
                            const double gs = G.at(0, r);
                            G.at(0, r) = gs + pdec[r] * (0.0 - gs);
                        }
                    }
                } break;
                case MIND_MECH_EXP2SYN: {
                    const double *pd1 = GG.f[E2_DECAY1] + G.r0, *pd2 = GG.f[E2_DECAY2] + G.r0;
                    const float *pd1f = GG.s[E2S_DECAY1] + G.r0, *pd2f = GG.s[E2S_DECAY2] + G.r0;
                    for (int32_t r = tid; r < G.rows; r += T) {
                        if (MIXED) {
                            // FP32 decrements, FP64 accumulation
                            const double A = G.at(0, r), B = G.at(1, r);
                            G.at(0, r) = A + (double)(pd1f[r] * (0.0f - (float)A));
                            G.at(1, r) = B + (double)(pd2f[r] * (0.0f - (float)B));
                        } else {
                            const double A = G.at(0, r), B = G.at(1, r);
                            G.at(0, r) = A + pd1[r] * (0.0 - A);
                            G.at(1, r) = B + pd2[r] * (0.0 - B);
                        }
                    }
                } break;
                default:
                    break;
            }
        }
        // 9. Record the completed boundary.
        if (P.nrec) {
            const int64_t sample = step + 1 - P.run_start;
            for (int32_t k = P.rec_off[c] + tid; k < P.rec_off[c + 1]; k += T) {
                const double *gp = P.rec_ptr[k];
                const int32_t code = P.rec_node[k];
                double value;
                if (gp) {
                    value = *gp;
                } else if (code >= 0) {
                    value = sv[code];
                } else {
                    const int32_t x = -1 - code;
                    value = sg[x >> 24].at((x >> 20) & 15, x & 0xFFFFF);
                }
                P.trace[sample * P.nrec + P.rec_col[k]] = value;
            }
        }
        __syncthreads();
    }
    if (singular) raise_error(P.error, MIND_ESINGULAR);

    // ---- write back, with validate_device_state!'s finite check (src/runtime/utils/step.jl:168-197)
    //      of the written voltage and state; an earlier error code is kept ----
    if (my_det >= 0) P.above[my_src] = my_above ? 1 : 0;
    bool finite = true;
    for (int32_t i = tid; i < n; i += T) {
        P.v[nb + i] = sv[i];
        finite &= isfinite(sv[i]);
    }
    for (int32_t g = 0; g < P.ngroups; ++g) {
        const DevGroup &G = P.groups[g];
        const StagedGroup &S = sg[g];
        if (!kind_staged(S.kind)) continue;
        for (int32_t r = tid; r < S.rows; r += T) {
            const int32_t row = S.r0 + r;
            switch (S.kind) {
                case MIND_MECH_HH:
                    G.f[HH_M][row] = S.at(HH_M, r);
                    G.f[HH_H][row] = S.at(HH_H, r);
                    G.f[HH_N][row] = S.at(HH_N, r);
                    finite &= isfinite(S.at(HH_M, r)) && isfinite(S.at(HH_H, r)) && isfinite(S.at(HH_N, r));
                    break;
                case MIND_MECH_EXPSYN:
                    G.f[ES_G][row] = S.at(0, r);
                    finite &= isfinite(S.at(0, r));
                    break;
                case MIND_MECH_EXP2SYN:
                    G.f[E2_A][row] = S.at(0, r);
                    G.f[E2_B][row] = S.at(1, r);
                    finite &= isfinite(S.at(0, r)) && isfinite(S.at(1, r));
                    break;
            }
        }
    }
    if (!finite) atomicCAS(P.error, 0, MIND_ENONFINITE);
}

template <bool MIXED, int NT, bool GLOBAL_IMAGE = false, bool GEN = false,
          int MINB = default_min_blocks(NT), bool PATHS = true>
__global__ void __launch_bounds__(NT, MINB) window_kernel(const Params P, const int32_t *cells, int64_t n0,
                                                           int32_t W) {
    window_body<MIXED, NT, GLOBAL_IMAGE, GEN, PATHS>(P, cells, n0, W);
}

/* dst [records x samples] = src [samples x records], through 32 x 32 shared-memory tiles
 * (both sides read and written along rows). */
__global__ void trace_transpose_kernel(const double *src, double *dst, int64_t samples, int32_t records) {
    __shared__ double tile[32][33];
    const int64_t s0 = (int64_t)blockIdx.x * 32;
    const int32_t r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int64_t s = s0 + k;
        const int32_t r = r0 + threadIdx.x;
        if (s < samples && r < records) tile[k][threadIdx.x] = src[s * records + r];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int32_t r = r0 + k;
        const int64_t s = s0 + threadIdx.x;
        if (r < records && s < samples) dst[(int64_t)r * samples + s] = tile[threadIdx.x][k];
    }
}

/* The run's first sample: every recorded value as it stands in HBM between runs. */
__global__ void record_initial_kernel(const Params P, const double *const *rec_initial, int32_t nrec) {
    for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nrec; k += gridDim.x * blockDim.x)
        P.trace[k] = *rec_initial[k];
}

/* Host-injected events of one window: NetCon events into the ring, and the raster
 * entries of external spike inputs (edge < 0, point = 0-based source). */
/* ---- spike exchange between ranks (one network sharded by cell) ----
 *
 * After a window, each rank packs its cells' spikes of the window into a fixed-width block
 * (send[0] = count, then (sid, step) pairs), the blocks of all ranks are gathered
 * (ncclAllGather, or a device copy when the host drives the exchange), and every rank
 * enters the spikes of the sids it receives into its ring through the NetCons of the
 * matching external sources -- the fan-out route_kernel does for local spikes, so events,
 * bins and canonical orders are those of the unsharded run. */
__global__ void exchange_pack_kernel(const Params P, const int32_t *sid_of_source, int64_t *send, int32_t width) {
    __shared__ int32_t n;
    if (threadIdx.x == 0) n = 0;
    __syncthreads();
    const int32_t count = min(*P.win_spike_count, P.win_spike_cap);
    for (int32_t i = threadIdx.x; i < count; i += blockDim.x) {
        const int32_t sid = sid_of_source[P.win_spike_source[i]];
        if (sid < 0) continue;
        const int32_t k = atomicAdd(&n, 1);
        if (k < width) {
            send[1 + 2 * (int64_t)k] = sid;
            send[2 + 2 * (int64_t)k] = P.win_spike_step[i];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (n > width) raise_error(P.error, MIND_ECAPACITY);
        send[0] = min(n, width);
    }
}

__global__ void exchange_inject_kernel(const Params P, const int64_t *recv, int32_t world, int32_t width,
                                       const int32_t *ext_sid, const int32_t *ext_source, int32_t n_ext,
                                       int64_t window_end) {
    const int64_t stride = 1 + 2 * (int64_t)width;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)world * width;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = k / width, j = k - r * width;
        const int64_t *block = recv + r * stride;
        const int64_t n = block[0];
        if (j >= n || n > width) continue;
        const int64_t sid = block[1 + 2 * j];
        const int64_t step = block[2 + 2 * j];
        int32_t lo = 0, hi = n_ext;   // ext_sid ascending
        while (lo < hi) {
            const int32_t mid = (lo + hi) >> 1;
            if (ext_sid[mid] < sid)
                lo = mid + 1;
            else
                hi = mid;
        }
        if (lo == n_ext || ext_sid[lo] != sid) continue;
        fan_out(P, ext_source[lo], (double)step * P.dt + 1.0e-10, window_end);
    }
}

__global__ void inject_kernel(const Params P, const InjectedEvent *events, int32_t n, int64_t min_bin) {
    for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const InjectedEvent e = events[k];
        if (e.edge >= 0)
            ring_insert(P, e.time, e.edge, e.point, min_bin);
        else
            record_spike(P, e.point, e.time);
    }
}

}  // namespace mind
