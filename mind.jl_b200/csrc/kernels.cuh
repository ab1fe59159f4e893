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

__device__ __forceinline__ double cnexp(double s, double inf, double tau, double dt) {
    return s + (1.0 - mind_exp(dt * (-1.0 / tau))) * (inf - s);
}

/* FP32 gating for the mixed mode: same equations, single precision, fast exp. */
__device__ __forceinline__ float vtrapf(float x, float y) {
    if (fabsf(x / y) < 1e-6f) return y * (1.0f - x / y / 2.0f);
    return x / (__expf(x / y) - 1.0f);
}

__device__ __forceinline__ void hh_advance_f32(float v, float q10, float dt, float &m, float &h, float &n) {
    float alpha = 0.1f * vtrapf(-(v + 40.0f), 10.0f);
    float beta = 4.0f * __expf(-(v + 65.0f) / 18.0f);
    float sum = alpha + beta;
    float tau = 1.0f / (q10 * sum);
    m = m + (1.0f - __expf(dt * (-1.0f / tau))) * (alpha / sum - m);
    alpha = 0.07f * __expf(-(v + 65.0f) / 20.0f);
    beta = 1.0f / (__expf(-(v + 35.0f) / 10.0f) + 1.0f);
    sum = alpha + beta;
    tau = 1.0f / (q10 * sum);
    h = h + (1.0f - __expf(dt * (-1.0f / tau))) * (alpha / sum - h);
    alpha = 0.01f * vtrapf(-(v + 55.0f), 10.0f);
    beta = 0.125f * __expf(-(v + 65.0f) / 80.0f);
    sum = alpha + beta;
    tau = 1.0f / (q10 * sum);
    n = n + (1.0f - __expf(dt * (-1.0f / tau))) * (alpha / sum - n);
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

/* INITIAL blocks of the cell mechanisms; decay factors of the synapses. */
__global__ void mechanism_init_kernel(const Params P, int32_t g) {
    const DevGroup &G = P.groups[g];
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < G.rows; r += gridDim.x * blockDim.x) {
        switch (G.kind) {
            case MIND_MECH_HH: {
                HHRates R = hh_rates(P.v[G.node[r]], P.celsius);
                G.f[HH_M][r] = R.minf;
                G.f[HH_H][r] = R.hinf;
                G.f[HH_N][r] = R.ninf;
                G.s[HHS_M][r] = (float)R.minf;
                G.s[HHS_H][r] = (float)R.hinf;
                G.s[HHS_N][r] = (float)R.ninf;
            } break;
            case MIND_MECH_EXPSYN: {
                G.f[ES_G][r] = 0.0;
                double decay = 1.0 - mind_exp(P.dt * (-1.0 / G.f[ES_TAU][r]));
                G.f[ES_DECAY][r] = decay;
                G.s[ESS_G][r] = 0.0f;
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
                G.s[E2S_A][r] = 0.0f;
                G.s[E2S_B][r] = 0.0f;
                G.s[E2S_DECAY1][r] = (float)d1;
                G.s[E2S_DECAY2][r] = (float)d2;
            } break;
            default:
                break;
        }
    }
}

/* Moves bins n0 .. n0+W-1 from the ring into per-cell inboxes. */
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
        int32_t pos = atomicAdd(&P.inbox_count[cell], 1);
        if (pos < P.inbox_cap) {
            InboxEvent x;
            x.time = e.time;
            x.edge = e.edge;
            x.point = e.point;
            x.bin = bin;
            P.inbox[(int64_t)cell * P.inbox_cap + pos] = x;
        }
    }
}

/* Routes the window's cell spikes (detected at step s, time s*dt + 1e-10). */
__global__ void route_kernel(const Params P, int64_t window_end) {
    const int32_t count = min(*P.win_spike_count, P.win_spike_cap);
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        int32_t source = P.win_spike_source[i];
        double time = (double)P.win_spike_step[i] * P.dt + 1.0e-10;
        record_spike(P, source, time);
        fan_out(P, source, time, window_end);
    }
}

__device__ __forceinline__ bool event_before(const InboxEvent &x, const InboxEvent &y) {
    if (x.bin != y.bin) return x.bin < y.bin;
    if (x.point != y.point) return x.point < y.point;
    if (x.time != y.time) return x.time < y.time;
    return x.edge < y.edge;
}

__device__ __forceinline__ void apply_event(const Params &P, const InboxEvent &e, bool mixed) {
    const int32_t g = P.point_group[e.point];
    const int32_t row = P.point_row[e.point];
    const DevGroup &G = P.groups[g];
    const double w = e.edge >= 0 ? P.edge_weight[e.edge] : 0.0;
    if (G.kind == MIND_MECH_EXPSYN) {
        if (mixed)
            G.s[ESS_G][row] = G.s[ESS_G][row] + (float)w;
        else
            G.f[ES_G][row] = G.f[ES_G][row] + w;
    } else if (G.kind == MIND_MECH_EXP2SYN) {
        if (mixed) {
            float wf = (float)(w * G.f[E2_FACTOR][row]);
            G.s[E2S_A][row] = G.s[E2S_A][row] + wf;
            G.s[E2S_B][row] = G.s[E2S_B][row] + wf;
        } else {
            G.f[E2_A][row] = G.f[E2_A][row] + w * G.f[E2_FACTOR][row];
            G.f[E2_B][row] = G.f[E2_B][row] + w * G.f[E2_FACTOR][row];
        }
    }
}

template <bool MIXED>
__global__ void __launch_bounds__(kThreads) window_kernel(const Params P, int64_t n0, int32_t W) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int32_t s_nev;
    const int32_t c = blockIdx.x;
    const int32_t tid = threadIdx.x;
    const int32_t T = blockDim.x;
    const int64_t nb = P.node_off[c];
    const int32_t n = (int32_t)(P.node_off[c + 1] - nb);
    const int32_t cb = P.chain_off[c];
    const int32_t nch = P.chain_off[c + 1] - cb;
    double *sv = reinterpret_cast<double *>(smem_raw);
    double *sd = sv + n;
    double *sr = sd + n;
    double *sa = sr + n;
    double *sxd = sa + n;
    double *sxr = sxd + nch;
    InboxEvent *sev = reinterpret_cast<InboxEvent *>(sxr + nch);
    int32_t *sorder = reinterpret_cast<int32_t *>(sev + P.inbox_cap);

    if (c == 0 && tid < W) P.ring_count[(n0 + tid) % P.ring_slots] = 0;
    for (int32_t i = tid; i < n; i += T) {
        sv[i] = P.v[nb + i];
        sa[i] = P.a[nb + i];
    }
    if (tid == 0) {
        int32_t count = P.inbox_count[c];
        if (count > P.inbox_cap) {
            raise_error(P.error, MIND_ECAPACITY);
            count = P.inbox_cap;
        }
        s_nev = count;
        P.inbox_count[c] = 0;
    }
    __syncthreads();
    const int32_t nev = s_nev;
    for (int32_t k = tid; k < nev; k += T) sev[k] = P.inbox[(int64_t)c * P.inbox_cap + k];
    __syncthreads();
    for (int32_t k = tid; k < nev; k += T) {
        int32_t rank = 0;
        const InboxEvent mine = sev[k];
        for (int32_t j = 0; j < nev; ++j) {
            const InboxEvent other = sev[j];
            if (event_before(other, mine) || (j < k && !event_before(mine, other))) ++rank;
        }
        sorder[rank] = k;
    }
    __syncthreads();

    const int32_t lv0 = P.level_off[c];
    const int32_t nlev = P.level_off[c + 1] - lv0 - 1;
    const float q10f = (float)mind_pow(3.0, (P.celsius - 6.3) / 10.0);
    int32_t cursor = 0;

    for (int32_t s = 0; s < W; ++s) {
        const int64_t step = n0 + s;
        const double t = (double)step * P.dt;

        // 1. Threshold detection from the completed boundary.
        for (int32_t k = P.det_off[c] + tid; k < P.det_off[c + 1]; k += T) {
            const int32_t src = P.det_source[k];
            const bool current = sv[P.det_node[k]] > P.det_thr[k];
            if (current && !P.above[src]) {
                int32_t idx = atomicAdd(P.win_spike_count, 1);
                if (idx < P.win_spike_cap) {
                    P.win_spike_source[idx] = src;
                    P.win_spike_step[idx] = step;
                } else {
                    raise_error(P.error, MIND_ECAPACITY);
                }
            }
            P.above[src] = current ? 1 : 0;
        }
        // 2. Deliver this step's bin in (target, time, edge) order.
        if (tid == 0) {
            while (cursor < nev) {
                const InboxEvent &e = sev[sorder[cursor]];
                if (e.bin > step) break;
                if (e.bin < step) raise_error(P.error, MIND_ESELFEVENT);
                apply_event(P, e, MIXED);
                ++cursor;
            }
        }
        // 3. Clear the membrane sums.
        for (int32_t i = tid; i < n; i += T) {
            sd[i] = 0.0;
            sr[i] = 0.0;
        }
        __syncthreads();

        // 4. BREAKPOINT currents at v + 0.001 and v, group by group.
        const double tc = t + 0.5 * P.dt;
        for (int32_t g = 0; g < P.ngroups; ++g) {
            const DevGroup &G = P.groups[g];
            if (G.kind == MIND_MECH_NETSTIM) continue;
            const int32_t r0 = G.row_off[c], r1 = G.row_off[c + 1];
            if (r0 == r1) continue;
            for (int32_t r = r0 + tid; r < r1; r += T) {
                const int32_t len = G.seg[r];
                if (len == 0) continue;
                const int32_t node = (int32_t)(G.node[r] - nb);
                const double vv = sv[node];
                const double probe = vv + 0.001;
                double R = sr[node], D = sd[node];
                for (int32_t q = r; q < r + len; ++q) {
                    double shifted, value;
                    bool density = false;
                    switch (G.kind) {
                        case MIND_MECH_HH: {
                            density = true;
                            double m, h, nn;
                            if (MIXED) {
                                m = (double)G.s[HHS_M][q];
                                h = (double)G.s[HHS_H][q];
                                nn = (double)G.s[HHS_N][q];
                            } else {
                                m = G.f[HH_M][q];
                                h = G.f[HH_H][q];
                                nn = G.f[HH_N][q];
                            }
                            shifted = hh_current(probe, m, h, nn, G.f[HH_GNABAR][q], G.f[HH_GKBAR][q],
                                                 G.f[HH_GL][q], G.f[HH_EL][q], G.f[HH_ENA][q], G.f[HH_EK][q]);
                            value = hh_current(vv, m, h, nn, G.f[HH_GNABAR][q], G.f[HH_GKBAR][q],
                                               G.f[HH_GL][q], G.f[HH_EL][q], G.f[HH_ENA][q], G.f[HH_EK][q]);
                        } break;
                        case MIND_MECH_PAS: {
                            density = true;
                            shifted = 0.0 + G.f[PAS_G][q] * (probe - G.f[PAS_E][q]);
                            value = 0.0 + G.f[PAS_G][q] * (vv - G.f[PAS_E][q]);
                        } break;
                        case MIND_MECH_EXPSYN: {
                            double gs = MIXED ? (double)G.s[ESS_G][q] : G.f[ES_G][q];
                            shifted = 0.0 + gs * (probe - G.f[ES_E][q]);
                            value = 0.0 + gs * (vv - G.f[ES_E][q]);
                        } break;
                        case MIND_MECH_EXP2SYN: {
                            double gs = MIXED ? (double)(G.s[E2S_B][q] - G.s[E2S_A][q])
                                              : G.f[E2_B][q] - G.f[E2_A][q];
                            shifted = 0.0 + gs * (probe - G.f[E2_E][q]);
                            value = 0.0 + gs * (vv - G.f[E2_E][q]);
                        } break;
                        case MIND_MECH_ICLAMP: {
                            const double del = G.f[IC_DEL][q];
                            const double i = (tc < del + G.f[IC_DUR][q] && tc >= del) ? G.f[IC_AMP][q] : 0.0;
                            shifted = 0.0 - i;
                            value = 0.0 - i;
                        } break;
                        default:
                            shifted = value = 0.0;
                    }
                    if (density) {
                        const double scale = G.f[G.kind == MIND_MECH_HH ? HH_SCALE : PAS_SCALE][q];
                        R = R - scale * value;
                        D = D + scale * (shifted - value) / 0.001;
                    } else {
                        R = R + -1.0 * value;
                        D = D + 1.0 * (shifted - value) / 0.001;
                    }
                }
                sr[node] = R;
                sd[node] = D;
            }
            __syncthreads();
        }

        // 5. Cable assembly: d = C/dt + d + axial_diagonal; own axial term, then children.
        for (int32_t i = tid; i < n; i += T) {
            const int64_t gi = nb + i;
            sd[i] = (P.cdt[gi] + sd[i]) + P.ad[gi];
            double R = sr[i];
            const int32_t p = P.parent[gi];
            if (p >= 0) R = R + sa[i] * (sv[p] - sv[i]);
            for (int32_t k = P.kid_off[gi]; k < P.kid_off[gi + 1]; ++k) {
                const int32_t kk = P.kids[k];
                R = R - sa[kk] * (sv[i] - sv[kk]);
            }
            sr[i] = R;
        }
        __syncthreads();

        // 6. Hines elimination, chains level by level, each chain bottom to top.
        for (int32_t lv = 0; lv < nlev; ++lv) {
            const int32_t c0 = P.level_chain[lv0 + lv], c1 = P.level_chain[lv0 + lv + 1];
            for (int32_t ch = c0 + tid; ch < c1; ch += T) {
                const int32_t top = P.chain_top[cb + ch];
                const int32_t bottom = top + P.chain_len[cb + ch] - 1;
                double D = sd[bottom], R = sr[bottom];
                for (int32_t k = P.chain_kid_off[cb + ch]; k < P.chain_kid_off[cb + ch + 1]; ++k) {
                    const int32_t cc = P.chain_kids[k];
                    D = D - sxd[cc];
                    R = R + sxr[cc];
                }
                if (D == 0.0 || !isfinite(D)) raise_error(P.error, MIND_ESINGULAR);
                sd[bottom] = D;
                sr[bottom] = R;
                double pxd = 0.0, pxr = 0.0;
                if (P.parent[nb + bottom] >= 0) {
                    const double f = sa[bottom] / D;
                    pxd = f * sa[bottom];
                    pxr = f * R;
                }
                for (int32_t i = bottom - 1; i >= top; --i) {
                    D = sd[i] - pxd;
                    R = sr[i] + pxr;
                    if (D == 0.0 || !isfinite(D)) raise_error(P.error, MIND_ESINGULAR);
                    sd[i] = D;
                    sr[i] = R;
                    if (P.parent[nb + i] >= 0) {
                        const double f = sa[i] / D;
                        pxd = f * sa[i];
                        pxr = f * R;
                    }
                }
                sxd[ch] = pxd;
                sxr[ch] = pxr;
            }
            __syncthreads();
        }
        // 7. Back-substitution, root chain first.
        for (int32_t lv = nlev - 1; lv >= 0; --lv) {
            const int32_t c0 = P.level_chain[lv0 + lv], c1 = P.level_chain[lv0 + lv + 1];
            for (int32_t ch = c0 + tid; ch < c1; ch += T) {
                const int32_t top = P.chain_top[cb + ch];
                const int32_t bottom = top + P.chain_len[cb + ch] - 1;
                const int32_t p = P.parent[nb + top];
                double x = p >= 0 ? sr[p] : 0.0;
                for (int32_t i = top; i <= bottom; ++i) {
                    double value = sr[i];
                    if (P.parent[nb + i] >= 0) value = value + sa[i] * x;
                    x = value / sd[i];
                    sr[i] = x;
                }
            }
            __syncthreads();
        }
        // 8. Voltage update.
        for (int32_t i = tid; i < n; i += T) sv[i] = sv[i] + sr[i];
        __syncthreads();

        // 9. cnexp state advance on the new voltage (time t + dt).
        for (int32_t g = 0; g < P.ngroups; ++g) {
            const DevGroup &G = P.groups[g];
            const int32_t r0 = G.row_off[c], r1 = G.row_off[c + 1];
            switch (G.kind) {
                case MIND_MECH_HH:
                    for (int32_t r = r0 + tid; r < r1; r += T) {
                        const double vv = sv[G.node[r] - nb];
                        if (MIXED) {
                            float m = G.s[HHS_M][r], h = G.s[HHS_H][r], nn = G.s[HHS_N][r];
                            hh_advance_f32((float)vv, q10f, (float)P.dt, m, h, nn);
                            G.s[HHS_M][r] = m;
                            G.s[HHS_H][r] = h;
                            G.s[HHS_N][r] = nn;
                        } else {
                            HHRates R = hh_rates(vv, P.celsius);
                            G.f[HH_M][r] = cnexp(G.f[HH_M][r], R.minf, R.mtau, P.dt);
                            G.f[HH_H][r] = cnexp(G.f[HH_H][r], R.hinf, R.htau, P.dt);
                            G.f[HH_N][r] = cnexp(G.f[HH_N][r], R.ninf, R.ntau, P.dt);
                        }
                    }
                    break;
                case MIND_MECH_EXPSYN:
                    for (int32_t r = r0 + tid; r < r1; r += T) {
                        if (MIXED) {
                            float gs = G.s[ESS_G][r];
                            G.s[ESS_G][r] = gs + G.s[ESS_DECAY][r] * (0.0f - gs);
                        } else {
                            double gs = G.f[ES_G][r];
                            G.f[ES_G][r] = gs + G.f[ES_DECAY][r] * (0.0 - gs);
                        }
                    }
                    break;
                case MIND_MECH_EXP2SYN:
                    for (int32_t r = r0 + tid; r < r1; r += T) {
                        if (MIXED) {
                            float A = G.s[E2S_A][r], B = G.s[E2S_B][r];
                            G.s[E2S_A][r] = A + G.s[E2S_DECAY1][r] * (0.0f - A);
                            G.s[E2S_B][r] = B + G.s[E2S_DECAY2][r] * (0.0f - B);
                        } else {
                            double A = G.f[E2_A][r], B = G.f[E2_B][r];
                            G.f[E2_A][r] = A + G.f[E2_DECAY1][r] * (0.0 - A);
                            G.f[E2_B][r] = B + G.f[E2_DECAY2][r] * (0.0 - B);
                        }
                    }
                    break;
                default:
                    break;
            }
        }
        // 10. Record the completed boundary.
        if (P.nrec) {
            const int64_t sample = step + 1 - P.run_start;
            for (int32_t k = P.rec_off[c] + tid; k < P.rec_off[c + 1]; k += T)
                P.trace[sample * P.nrec + P.rec_col[k]] = sv[P.rec_node[k]];
        }
        __syncthreads();
    }
    for (int32_t i = tid; i < n; i += T) P.v[nb + i] = sv[i];
}

__global__ void record_initial_kernel(const Params P, const int64_t *rec_global, int32_t nrec) {
    for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nrec; k += gridDim.x * blockDim.x)
        P.trace[k] = P.v[rec_global[k]];
}

__global__ void finite_kernel(const double *values, int64_t count, int32_t *error) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x)
        if (!isfinite(values[i])) atomicCAS(error, 0, MIND_ENONFINITE);
}

__global__ void inject_kernel(const Params P, double time, int32_t edge, int32_t point, int64_t min_bin) {
    ring_insert(P, time, edge, point, min_bin);
}

}  // namespace mind
