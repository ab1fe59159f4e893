/*
 * mind_oracle.cpp — CPU FP64 restatement of MIND.jl's per-micro-step loop.
 *
 * TEST INFRASTRUCTURE.  This is the checker for libmindgpu.so's FP64 mode and
 * the timed CPU baseline; only tests/, __graft_entry__.smoke() and bench.py's
 * CPU legs load it.  The product never calls it.
 *
 * It consumes the same MindLayout the library receives (include/mindgpu.h)
 * and follows the reference's algorithm, not the library's:
 *   - step order of advance_micro! (src/runtime/step.jl:91-151): detection at
 *     t + 1e-10 from the completed boundary (src/runtime/utils/step.jl:143-156,
 *     src/runtime/cuda/micro.jl:285-302), routing, delivery through t + dt/2,
 *     currents at t + dt/2, assembly, Hines solve, voltage update, state
 *     advance at t + dt, recording, delivery through the new boundary;
 *   - a CPU binary heap keyed (time, order, target) with order assigned at
 *     enqueue (src/runtime/utils/events.jl:7-62) and NET_RECEIVE applied in
 *     pop order (src/runtime/events.jl:57-165), NetStim self-events and
 *     net_event fanout re-entering the heap before the next pop;
 *   - the current probe at v + 0.001 and v with rhs -= s*i, d += s*di/0.001,
 *     s = area*0.01 for density and 1 for point mechanisms
 *     (src/runtime/cuda/micro.jl:427-500), currents summed in the MOD's
 *     order (NONSPECIFIC then USEION writes, src/runtime/initialize.jl:496-501);
 *   - assembly d = C/dt + d + axial_diagonal, rhs += a (v_p - v)
 *     (src/runtime/cuda/micro.jl:633-657), Hines elimination
 *     d_p -= (a/d) a, rhs_p += (a/d) rhs and back-substitution
 *     x = (rhs + a x_p)/d (src/runtime/cuda/micro.jl:688-749);
 *   - cnexp as the reference lowers relaxation equations:
 *     s += (1 - exp(dt * (-1/tau))) (s_inf - s) (src/compiler/codegen.jl:569-641);
 *   - mechanism equations of mod/{hh,pas,ExpSyn,Exp2Syn,NetStim,IClamp}.mod;
 *   - NetStim's Philox streams (src/runtime/cuda/micro.jl:3-91).
 * Where the reference's result depends on the order of concurrent FP64
 * atomics (siblings eliminated into one parent, several point processes or
 * children adding into one node) this restatement fixes the order: a node's
 * own term first, then children in ascending node index; mechanism groups in
 * layout order; rows in row order.  The library uses the same order, which
 * makes FP64 parity bit-exact.  Both sides call mind_math.h for exp/log/pow.
 * Built with -DMIND_ORACLE_LIBM (liboracle_libm.so, the Makefile's second target) the
 * oracle takes exp, log and pow from the C library instead: a second, independently
 * written faithful math library, against which the tests bound how much a run depends on
 * the choice of math library (MIND.jl's device math being a third one).  Built with
 * -DMIND_ORACLE_REVERSED (liboracle_rev.so) it sums every order-dependent term in the
 * opposite order (mechanism groups and rows into a node, children into a parent in the
 * assembly and the elimination): another order the reference's atomics may take, against
 * which the tests bound how much a run depends on that order.
 *
 * Threads: cells are independent between two event deliveries, so each step hands
 * whole cells (currents, cable assembly and solve, state advance) to a pool of worker
 * threads created once per run; detection, the event heap and the regions stay serial.
 * Every node is summed by one thread in the fixed order above, so the result does not
 * depend on the thread count.
 */
#include "../include/mindgpu.h"
#include "../mind.jl_b200/csrc/mind_math.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <queue>
#include <string>
#include <vector>

#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>

namespace {

// The oracle's elementary functions (see the header comment).
#ifdef MIND_ORACLE_LIBM
inline double oexp(double x) { return std::exp(x); }
inline double olog(double x) { return std::log(x); }
inline double opow(double x, double y) { return std::pow(x, y); }
#else
inline double oexp(double x) { return mind_exp(x); }
inline double olog(double x) { return mind_log(x); }
inline double opow(double x, double y) { return mind_pow(x, y); }
#endif
// alpha(x) = x e^(1-x) on [0, 10] (mod/AlphaSynapse.mod), and random_negexp = -log(u)
inline double oalpha(double x) { return (x < 0.0 || x > 10.0) ? 0.0 : x * oexp(1.0 - x); }
inline double onegexp(MindRan *s, uint64_t seed) { return -olog(mind_ran_uniform(s, seed)) * 1.0; }

struct Event {
    double time;
    double flag;
    int64_t edge;   // 1-based, 0 = self event
    int64_t order;
    int32_t target; // 1-based point index
};

struct Later {
    bool operator()(const Event &a, const Event &b) const {
        // priority_queue pops the largest; "largest" = earliest by event_before.
        if (a.time != b.time) return a.time > b.time;
        if (a.order != b.order) return a.order > b.order;
        return a.target > b.target;
    }
};

/* A fixed set of worker threads, created once per run and reused every step: run(job)
 * calls job(k) for k = 0 .. n-1 on the workers and the caller, and returns when all are
 * done.  No thread is created or joined inside the step loop. */
class ThreadPool {
  public:
    explicit ThreadPool(int n) : n_(n < 1 ? 1 : n) {
        for (int k = 1; k < n_; ++k) workers_.emplace_back([this, k] { loop(k); });
    }
    ~ThreadPool() {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            stop_ = true;
            ++generation_;
        }
        wake_.notify_all();
        for (auto &t : workers_) t.join();
    }
    int size() const { return n_; }
    void run(const std::function<void(int)> &job) {
        if (n_ == 1) {
            job(0);
            return;
        }
        {
            std::lock_guard<std::mutex> lock(mutex_);
            job_ = &job;
            pending_ = n_ - 1;
            ++generation_;
        }
        wake_.notify_all();
        job(0);
        std::unique_lock<std::mutex> lock(mutex_);
        done_.wait(lock, [this] { return pending_ == 0; });
        job_ = nullptr;
    }

  private:
    void loop(int k) {
        uint64_t seen = 0;
        for (;;) {
            const std::function<void(int)> *job;
            {
                std::unique_lock<std::mutex> lock(mutex_);
                wake_.wait(lock, [&] { return generation_ != seen; });
                seen = generation_;
                if (stop_) return;
                job = job_;
            }
            (*job)(k);
            std::lock_guard<std::mutex> lock(mutex_);
            if (--pending_ == 0) done_.notify_one();
        }
    }
    int n_;
    std::vector<std::thread> workers_;
    std::mutex mutex_;
    std::condition_variable wake_, done_;
    const std::function<void(int)> *job_ = nullptr;
    uint64_t generation_ = 0;
    int pending_ = 0;
    bool stop_ = false;
};

struct Group {
    int32_t kind;
    int64_t rows;
    std::vector<int32_t> node;     // 0-based, -1 for artificial
    std::vector<std::vector<double>> f;  // fields by canonical slot
    uint64_t digest;
    std::vector<uint64_t> logical;
};

enum { HH_GNABAR, HH_GKBAR, HH_GL, HH_EL, HH_M, HH_H, HH_N, HH_ENA, HH_EK, HH_NF };
enum { PAS_G, PAS_E, PAS_NF };
enum { ES_TAU, ES_E, ES_G, ES_NF };
enum { E2_TAU1, E2_TAU2, E2_E, E2_A, E2_B, E2_FACTOR, E2_NF };
enum { NS_INTERVAL, NS_NUMBER, NS_START, NS_NOISE, NS_EVENT, NS_ON, NS_ISPIKE, NS_NF };
enum { IC_DEL, IC_DUR, IC_AMP, IC_NF };
enum { AS_ONSET, AS_TAU, AS_GMAX, AS_E, AS_NF };

const char *const HH_NAMES[] = {"gnabar", "gkbar", "gl", "el", "m", "h", "n", "ena", "ek"};
const char *const PAS_NAMES[] = {"g", "e"};
const char *const ES_NAMES[] = {"tau", "e", "g"};
const char *const E2_NAMES[] = {"tau1", "tau2", "e", "A", "B", "factor"};
const char *const NS_NAMES[] = {"interval", "number", "start", "noise", "event", "on", "ispike"};
const char *const IC_NAMES[] = {"del", "dur", "amp"};
const char *const AS_NAMES[] = {"onset", "tau", "gmax", "e"};

/* Electrode clamps of mod/SEClamp.mod and mod/VClamp.mod, restated by hand (the library runs
 * them through CUDA C emitted from the MOD files; oracle.py hands them to this file under
 * these kind codes).  Fields by MOD name; VClamp's dur/amp arrays as dur[0..2], amp[0..2]. */
constexpr int32_t ORACLE_SECLAMP = 1001, ORACLE_VCLAMP = 1002;
enum { SE_RS, SE_DUR1, SE_AMP1, SE_DUR2, SE_AMP2, SE_DUR3, SE_AMP3, SE_I, SE_VC, SE_TC2, SE_TC3, SE_ON, SE_NF };
const char *const SE_NAMES[] = {"rs", "dur1", "amp1", "dur2", "amp2", "dur3", "amp3", "i", "vc", "tc2", "tc3", "on"};
enum { VC_DUR, VC_AMP = VC_DUR + 3, VC_GAIN = VC_AMP + 3, VC_RSTIM, VC_TAU1, VC_TAU2, VC_E0, VC_VO0, VC_VI0, VC_FAC,
       VC_E, VC_VO, VC_VI, VC_I, VC_STIM, VC_TC, VC_NF };
const char *const VC_NAMES[] = {"dur[0]", "dur[1]", "dur[2]", "amp[0]", "amp[1]", "amp[2]", "gain", "rstim", "tau1",
                                "tau2", "e0", "vo0", "vi0", "fac", "e", "vo", "vi", "i", "stim", "tc"};

struct Oracle {
    const MindLayout *L;
    int64_t n;
    double dt, celsius;
    uint64_t seed;
    std::vector<int32_t> parent;  // 0-based, -1 root
    std::vector<double> v, d, rhs, cap, a, ad, area, xd, xr;
    std::vector<int64_t> child_off;
    std::vector<int32_t> child;   // ascending
    std::vector<std::vector<int32_t>> cell_up;    // per cell: nodes children-before-parent
    std::vector<int32_t> cell_of;                 // per node: its cell
    // per cell and group: the group's rows on the cell's nodes, ascending (row order)
    std::vector<std::vector<std::vector<int64_t>>> cell_rows;
    std::vector<int64_t> detector_sources;        // sources with a threshold detector, ascending
    ThreadPool *pool = nullptr;
    std::vector<Group> groups;
    std::vector<MindRan> ran;     // per NetStim row, indexed via group
    std::vector<char> above;
    std::priority_queue<Event, std::vector<Event>, Later> heap;
    int64_t next_order = 0;
    int64_t step = 0;
    int error = 0;
    std::string message;
    std::vector<double> spike_t;
    std::vector<int64_t> spike_sid;
    std::vector<int64_t> point_source;  // per point (0-based) -> source index (0-based) or -1

    // ---- regions (mind_attach_macro's specification in include/mindgpu.h) ----
    const MindMacroLayout *ML = nullptr;
    int32_t spm = 0, mpb = 0, bin_steps = 0;
    std::vector<double> ry;                       // [n][6]
    std::vector<std::vector<double>> out_hist;    // out(k) per macro step
    std::vector<std::vector<int64_t>> bin_count;  // spikes per rate bin and region
    std::vector<int32_t> source_region;           // detector source -> region or -1
    std::vector<double> region_cells;
    std::vector<std::vector<int64_t>> edges_in;   // per region: edge indices into it, in edge order

    int load_macro(const MindMacroLayout *M) {
        ML = M;
        spm = (int32_t)std::llround(M->dt_macro / dt);
        mpb = (int32_t)std::llround(M->bin_ms / M->dt_macro);
        bin_steps = spm * mpb;
        const int32_t nr = M->n_regions;
        ry.assign(M->y0, M->y0 + (size_t)nr * 6);
        source_region.assign(L->n_sources, -1);
        region_cells.assign(nr, 0.0);
        for (int64_t q = 0; q < M->n_outputs; ++q) {
            source_region[M->output_source[q] - 1] = M->output_region[q] - 1;
            region_cells[M->output_region[q] - 1] += 1.0;
        }
        for (auto &c : region_cells)
            if (c == 0.0) c = 1.0;
        edges_in.assign(nr, {});
        for (int64_t e = 0; e < M->n_edges; ++e) edges_in[M->edge_dst[e] - 1].push_back(e);
        std::vector<double> out0(nr);
        for (int32_t i = 0; i < nr; ++i) out0[i] = region_output(&ry[(size_t)i * 6], M->params + (size_t)i * 9);
        out_hist.assign(1, out0);
        return 0;
    }

    static double sigmoid(double v, double e0, double r, double v0) {
        return (2.0 * e0) / (1.0 + oexp(r * (v0 - v)));
    }
    static double region_output(const double *y, const double *par) { return sigmoid(y[1] - y[2], par[4], par[5], par[6]); }
    static void region_rhs(const double *y, double p, const double *par, double *dy) {
        const double A = par[0], B = par[1], a = par[2], b = par[3], e0 = par[4], r = par[5], v0 = par[6], C = par[7];
        dy[0] = y[3];
        dy[1] = y[4];
        dy[2] = y[5];
        dy[3] = ((A * a) * sigmoid(y[1] - y[2], e0, r, v0) - (2.0 * a) * y[3]) - (a * a) * y[0];
        dy[4] = ((A * a) * (p + (0.8 * C) * sigmoid(C * y[0], e0, r, v0)) - (2.0 * a) * y[4]) - (a * a) * y[1];
        dy[5] = ((B * b) * ((0.25 * C) * sigmoid((0.25 * C) * y[0], e0, r, v0)) - (2.0 * b) * y[5]) - (b * b) * y[2];
    }
    static void region_rk4(double *y, double p, const double *par, double h) {
        double k1[6], k2[6], k3[6], k4[6], t[6];
        region_rhs(y, p, par, k1);
        for (int j = 0; j < 6; ++j) t[j] = y[j] + (0.5 * h) * k1[j];
        region_rhs(t, p, par, k2);
        for (int j = 0; j < 6; ++j) t[j] = y[j] + (0.5 * h) * k2[j];
        region_rhs(t, p, par, k3);
        for (int j = 0; j < 6; ++j) t[j] = y[j] + h * k3[j];
        region_rhs(t, p, par, k4);
        const double w = h / 6.0;
        for (int j = 0; j < 6; ++j) y[j] = y[j] + w * (((k1[j] + 2.0 * k2[j]) + 2.0 * k3[j]) + k4[j]);
    }

    /* Macro step k begins: advance every region over it, then queue its input spikes. */
    void macro_step(int64_t k) {
        const int32_t nr = ML->n_regions;
        const double dt_s = ML->dt_macro * 1e-3, bin_s = ML->bin_ms * 1e-3;
        std::vector<double> next(nr);
        for (int32_t i = 0; i < nr; ++i) {
            const double *par = ML->params + (size_t)i * 9;
            const int64_t b = k / mpb - 1;
            double rate = 0.0;
            if (b >= 0 && b < (int64_t)bin_count.size()) rate = (double)bin_count[b][i] / (region_cells[i] * bin_s);
            double p = par[8] + ML->micro_gain[i] * rate;
            for (int64_t e : edges_in[i]) {
                int64_t m = k - ML->edge_delay[e];
                if (m < 0) m = 0;
                p = p + ML->edge_gain[e] * out_hist[m][ML->edge_src[e] - 1];
            }
            region_rk4(&ry[(size_t)i * 6], p, par, dt_s);
            next[i] = region_output(&ry[(size_t)i * 6], par);
        }
        // inputs over [k dt_macro, (k+1) dt_macro) from out(k)
        for (int64_t q = 0; q < ML->n_inputs; ++q) {
            const double out = out_hist[k][ML->input_region[q] - 1];
            const double mu = (ML->input_scale[q] * out) * dt_s;
            uint32_t ctr[4] = {(uint32_t)k, (uint32_t)((uint64_t)k >> 32), (uint32_t)q, 0x4D4Du};
            mind_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
            const double u0 = ((double)ctr[0] + 1.0) * MIND_INV_2P32P1;
            double pr = oexp(-mu), F = pr;
            int count = 0;
            while (u0 > F && count < 3) {
                ++count;
                pr = (pr * mu) / (double)count;
                F = F + pr;
            }
            const int64_t source = ML->input_source[q] - 1;
            for (int j = 0; j < count; ++j) {
                const double t = (double)k * ML->dt_macro + ML->dt_macro * (((double)ctr[1 + j] + 1.0) * MIND_INV_2P32P1);
                for (int64_t e = L->fanout_offsets[source] - 1; e < L->fanout_offsets[source + 1] - 1; ++e)
                    enqueue(t + L->edge_delays[e], 0.0, e + 1, L->edge_targets[e]);
            }
        }
        out_hist.push_back(next);
    }

    void count_spike(int64_t source) {
        if (!ML || source_region[source] < 0) return;
        const int64_t b = step / bin_steps;
        while ((int64_t)bin_count.size() <= b) bin_count.emplace_back(ML->n_regions, 0);
        bin_count[b][source_region[source]] += 1;
    }

    int fail(int code, const std::string &why) {
        if (!error) {
            error = code;
            message = why;
        }
        return code;
    }

    int load(const MindLayout *layout) {
        L = layout;
        if (L->abi_version != MIND_ABI_VERSION) return fail(MIND_ELAYOUT, "ABI version");
        if (L->secondorder < 0 || L->secondorder > 2) return fail(MIND_ELAYOUT, "secondorder must be 0, 1 or 2");
        n = L->n_nodes;
        dt = L->dt;
        celsius = L->celsius;
        seed = L->seed;
        parent.resize(n);
        for (int64_t i = 0; i < n; ++i) parent[i] = L->parent[i] - 1;
        v.assign(L->voltage, L->voltage + n);
        cap.assign(L->capacitance, L->capacitance + n);
        a.assign(L->axial, L->axial + n);
        ad.assign(L->axial_diagonal, L->axial_diagonal + n);
        area.assign(L->area, L->area + n);
        d.assign(n, 0.0);
        rhs.assign(n, 0.0);
        xd.assign(n, 0.0);
        xr.assign(n, 0.0);
        // children CSR, ascending
        std::vector<int64_t> count(n + 1, 0);
        for (int64_t i = 0; i < n; ++i)
            if (parent[i] >= 0) count[parent[i] + 1]++;
        child_off.assign(n + 1, 0);
        for (int64_t i = 0; i < n; ++i) child_off[i + 1] = child_off[i] + count[i + 1];
        child.assign(child_off[n], 0);
        std::vector<int64_t> cursor(child_off.begin(), child_off.end() - 1);
        for (int64_t i = 0; i < n; ++i)
            if (parent[i] >= 0) child[cursor[parent[i]]++] = (int32_t)i;
        // cells: BFS from each root; up-order = reverse BFS
        for (int64_t r = 0; r < n; ++r) {
            if (parent[r] >= 0) continue;
            std::vector<int32_t> bfs{(int32_t)r};
            for (size_t k = 0; k < bfs.size(); ++k)
                for (int64_t c = child_off[bfs[k]]; c < child_off[bfs[k] + 1]; ++c) bfs.push_back(child[c]);
            std::reverse(bfs.begin(), bfs.end());
            cell_up.push_back(std::move(bfs));
        }
        // mechanisms
        for (int32_t g = 0; g < L->n_mechanisms; ++g) {
            const MindMechanism &m = L->mechanisms[g];
            Group G;
            G.kind = m.kind;
            G.rows = m.rows;
            G.digest = m.digest;
            const char *const *names = nullptr;
            int nf = 0;
            switch (m.kind) {
                case MIND_MECH_HH: names = HH_NAMES; nf = HH_NF; break;
                case MIND_MECH_PAS: names = PAS_NAMES; nf = PAS_NF; break;
                case MIND_MECH_EXPSYN: names = ES_NAMES; nf = ES_NF; break;
                case MIND_MECH_EXP2SYN: names = E2_NAMES; nf = E2_NF; break;
                case MIND_MECH_NETSTIM: names = NS_NAMES; nf = NS_NF; break;
                case MIND_MECH_ICLAMP: names = IC_NAMES; nf = IC_NF; break;
                case MIND_MECH_ALPHASYN: names = AS_NAMES; nf = AS_NF; break;
                case ORACLE_SECLAMP: names = SE_NAMES; nf = SE_NF; break;
                case ORACLE_VCLAMP: names = VC_NAMES; nf = VC_NF; break;
                case MIND_MECH_PATTERNSTIM: names = nullptr; nf = 0; break;
                default: return fail(MIND_ELAYOUT, "unsupported mechanism kind");
            }
            G.f.resize(nf);
            for (int k = 0; k < nf; ++k) {
                int found = -1;
                for (int j = 0; j < m.n_fields; ++j)
                    if (std::strcmp(m.field_names[j], names[k]) == 0) found = j;
                if (found < 0) return fail(MIND_ELAYOUT, std::string("missing field ") + names[k]);
                G.f[k].assign(m.data + (int64_t)found * m.rows, m.data + (int64_t)(found + 1) * m.rows);
            }
            G.node.resize(m.rows);
            for (int64_t r = 0; r < m.rows; ++r) G.node[r] = m.nodes[r] - 1;
            G.logical.assign(m.logical_ids, m.logical_ids + m.rows);
            groups.push_back(std::move(G));
        }
        point_source.assign(L->n_points, -1);
        for (int64_t s = 0; s < L->n_sources; ++s)
            if (L->source_points[s] > 0) point_source[L->source_points[s] - 1] = s;
        above.assign(L->n_sources, 0);
        cell_of.assign(n, -1);
        for (size_t c = 0; c < cell_up.size(); ++c)
            for (int32_t i : cell_up[c]) cell_of[i] = (int32_t)c;
        cell_rows.assign(cell_up.size(), std::vector<std::vector<int64_t>>(groups.size()));
        for (size_t g = 0; g < groups.size(); ++g)
            for (int64_t r = 0; r < groups[g].rows; ++r)
                if (groups[g].node[r] >= 0) cell_rows[cell_of[groups[g].node[r]]][g].push_back(r);
        for (int64_t s = 0; s < L->n_sources; ++s)
            if (L->source_nodes[s] > 0) detector_sources.push_back(s);
        return 0;
    }

    void enqueue(double time, double flag, int64_t edge, int32_t target) {
        heap.push(Event{time, flag, edge, ++next_order, target});
    }

    void emit_spike(int64_t source, double time) {
        spike_t.push_back(time);
        spike_sid.push_back(L->source_ids[source]);
        for (int64_t e = L->fanout_offsets[source] - 1; e < L->fanout_offsets[source + 1] - 1; ++e)
            enqueue(time + L->edge_delays[e], 0.0, e + 1, L->edge_targets[e]);
    }

    // ---- NetStim (mod/NetStim.mod) ----
    double invl(Group &G, int64_t r, double mean) {
        if (mean <= 0.0) mean = 0.01;
        double noise = G.f[NS_NOISE][r];
        if (noise == 0.0) return mean;
        double erand = onegexp(&ran[r], seed);
        return (1.0 - noise) * mean + noise * mean * erand;
    }
    void init_sequence(Group &G, int64_t r) {
        if (G.f[NS_NUMBER][r] > 0.0) {
            G.f[NS_ON][r] = 1.0;
            G.f[NS_EVENT][r] = 0.0;
            G.f[NS_ISPIKE][r] = 0.0;
        }
    }
    void next_invl(Group &G, int64_t r) {
        if (G.f[NS_NUMBER][r] > 0.0) G.f[NS_EVENT][r] = invl(G, r, G.f[NS_INTERVAL][r]);
        if (G.f[NS_ISPIKE][r] >= G.f[NS_NUMBER][r]) G.f[NS_ON][r] = 0.0;
    }
    void net_send(double t, double delay, double flag, int32_t point) {
        if (delay < 0.0 || !std::isfinite(delay)) {
            fail(MIND_ESELFEVENT, "invalid self-event delay");
            return;
        }
        enqueue(t + delay, flag, 0, point);
    }
    void netstim_receive(Group &G, int64_t r, int32_t point, double t, double flag, double w) {
        if (flag == 0.0) {
            if (w > 0.0 && G.f[NS_ON][r] == 0.0) {
                init_sequence(G, r);
                next_invl(G, r);
                G.f[NS_EVENT][r] = G.f[NS_EVENT][r] - G.f[NS_INTERVAL][r] * (1.0 - G.f[NS_NOISE][r]);
                net_send(t, G.f[NS_EVENT][r], 1.0, point);
            } else if (w < 0.0) {
                G.f[NS_ON][r] = 0.0;
            }
        }
        if (flag == 3.0) {
            if (G.f[NS_ON][r] == 1.0) {
                init_sequence(G, r);
                net_send(t, 0.0, 1.0, point);
            }
        }
        if (flag == 1.0 && G.f[NS_ON][r] == 1.0) {
            G.f[NS_ISPIKE][r] = G.f[NS_ISPIKE][r] + 1.0;
            int64_t source = point_source[point - 1];
            if (source >= 0) emit_spike(source, t);
            next_invl(G, r);
            if (G.f[NS_ON][r] == 1.0) net_send(t, G.f[NS_EVENT][r], 1.0, point);
        }
    }

    // ---- hh rates (mod/hh.mod) ----
    static double vtrap(double x, double y) {
        if (std::fabs(x / y) < 1e-6) return y * (1.0 - x / y / 2.0);
        return x / (oexp(x / y) - 1.0);
    }
    struct Rates { double minf, hinf, ninf, mtau, htau, ntau; };
    Rates rates(double vv) const {
        Rates R;
        double q10 = opow(3.0, (celsius - 6.3) / 10.0);
        double alpha = 0.1 * vtrap(-(vv + 40.0), 10.0);
        double beta = 4.0 * oexp(-(vv + 65.0) / 18.0);
        double sum = alpha + beta;
        R.mtau = 1.0 / (q10 * sum);
        R.minf = alpha / sum;
        alpha = 0.07 * oexp(-(vv + 65.0) / 20.0);
        beta = 1.0 / (oexp(-(vv + 35.0) / 10.0) + 1.0);
        sum = alpha + beta;
        R.htau = 1.0 / (q10 * sum);
        R.hinf = alpha / sum;
        alpha = 0.01 * vtrap(-(vv + 55.0), 10.0);
        beta = 0.125 * oexp(-(vv + 65.0) / 80.0);
        sum = alpha + beta;
        R.ntau = 1.0 / (q10 * sum);
        R.ninf = alpha / sum;
        return R;
    }
    static double cnexp(double s, double inf, double tau, double step_dt) {
        return s + (1.0 - oexp(step_dt * (-1.0 / tau))) * (inf - s);
    }

    void initialize() {
        step = 0;
        for (auto &G : groups) {
            for (int64_t r = 0; r < G.rows; ++r) {
                switch (G.kind) {
                    case MIND_MECH_HH: {
                        Rates R = rates(v[G.node[r]]);
                        G.f[HH_M][r] = R.minf;
                        G.f[HH_H][r] = R.hinf;
                        G.f[HH_N][r] = R.ninf;
                    } break;
                    case MIND_MECH_EXPSYN: G.f[ES_G][r] = 0.0; break;
                    case ORACLE_SECLAMP:
                        G.f[SE_TC2][r] = G.f[SE_DUR1][r] + G.f[SE_DUR2][r];
                        G.f[SE_TC3][r] = G.f[SE_TC2][r] + G.f[SE_DUR3][r];
                        G.f[SE_ON][r] = 0.0;
                        break;
                    case ORACLE_VCLAMP: {
                        const double vv = v[G.node[r]];
                        G.f[VC_E0][r] = 0.0;
                        G.f[VC_VO][r] = vv;
                        G.f[VC_VO0][r] = vv;
                        G.f[VC_VI][r] = vv;
                        G.f[VC_VI0][r] = vv;
                        G.f[VC_E][r] = 0.0;
                    } break;
                    case MIND_MECH_EXP2SYN: {
                        double &tau1 = G.f[E2_TAU1][r];
                        double tau2 = G.f[E2_TAU2][r];
                        if (tau1 / tau2 > 0.9999) tau1 = 0.9999 * tau2;
                        if (tau1 / tau2 < 1e-9) tau1 = tau2 * 1e-9;
                        G.f[E2_A][r] = 0.0;
                        G.f[E2_B][r] = 0.0;
                        double tp = (tau1 * tau2) / (tau2 - tau1) * olog(tau2 / tau1);
                        double factor = -oexp(-tp / tau1) + oexp(-tp / tau2);
                        G.f[E2_FACTOR][r] = 1.0 / factor;
                    } break;
                    default: break;
                }
            }
        }
        // PatternStim: each prescribed time fires the sources its point feeds
        // (src/runtime/utils/events.jl:92-110), queued in time order.
        for (int64_t k = 0; k < L->n_pattern; ++k)
            for (int64_t s = 0; s < L->n_sources; ++s)
                if (L->source_points[s] == L->pattern_points[k]) enqueue(L->pattern_times[k], 0.0, 0, -(int32_t)(s + 1));
        // NetStim INITIAL, groups in order, rows in order (t = 0).
        for (size_t g = 0; g < groups.size(); ++g) {
            Group &G = groups[g];
            if (G.kind != MIND_MECH_NETSTIM) continue;
            ran.assign(G.rows, MindRan{});
            for (int64_t r = 0; r < G.rows; ++r) {
                mind_ran_init(&ran[r], G.logical[r], G.digest, 0u, seed);
                mind_ran_setseq(&ran[r], 0.0, seed);
                G.f[NS_ON][r] = 0.0;
                G.f[NS_ISPIKE][r] = 0.0;
                if (G.f[NS_NOISE][r] < 0.0) G.f[NS_NOISE][r] = 0.0;
                if (G.f[NS_NOISE][r] > 1.0) G.f[NS_NOISE][r] = 1.0;
                if (G.f[NS_START][r] >= 0.0 && G.f[NS_NUMBER][r] > 0.0) {
                    G.f[NS_ON][r] = 1.0;
                    double ev = G.f[NS_START][r] + invl(G, r, G.f[NS_INTERVAL][r]) -
                                G.f[NS_INTERVAL][r] * (1.0 - G.f[NS_NOISE][r]);
                    if (ev < 0.0) ev = 0.0;
                    G.f[NS_EVENT][r] = ev;
                    net_send(0.0, ev, 3.0, point_of(g, r));
                }
            }
        }
        deliver(0.0);
    }

    std::vector<std::vector<int32_t>> row_point;  // group -> row -> point (1-based)
    int32_t point_of(size_t g, int64_t r) { return row_point[g][r]; }

    void build_row_points() {
        row_point.assign(groups.size(), {});
        for (size_t g = 0; g < groups.size(); ++g) row_point[g].assign(groups[g].rows, 0);
        for (int64_t p = 0; p < L->n_points; ++p)
            row_point[L->point_group[p] - 1][L->point_row[p] - 1] = (int32_t)(p + 1);
    }

    void receive(const Event &e) {
        if (e.target < 0) {   // a PatternStim firing of source -target - 1 (events.jl:92-110)
            emit_spike(-(int64_t)e.target - 1, e.time);
            return;
        }
        int32_t point = e.target;
        int32_t g = L->point_group[point - 1] - 1;
        int64_t r = L->point_row[point - 1] - 1;
        Group &G = groups[g];
        double w = e.edge == 0 ? 0.0 : L->edge_weights[e.edge - 1];
        switch (G.kind) {
            case MIND_MECH_EXPSYN: G.f[ES_G][r] = G.f[ES_G][r] + w; break;
            case MIND_MECH_EXP2SYN:
                G.f[E2_A][r] = G.f[E2_A][r] + w * G.f[E2_FACTOR][r];
                G.f[E2_B][r] = G.f[E2_B][r] + w * G.f[E2_FACTOR][r];
                break;
            case MIND_MECH_NETSTIM: netstim_receive(G, r, point, e.time, e.flag, w); break;
            default: break;
        }
    }

    void deliver(double cutoff) {
        while (!heap.empty() && heap.top().time <= cutoff) {
            Event e = heap.top();
            heap.pop();
            receive(e);
        }
    }

    // ---- SEClamp (mod/SEClamp.mod): vstim() then icur() in BREAKPOINT; icur() after the solve
    static void seclamp_icur(Group &G, int64_t r, double vv) {
        if (G.f[SE_ON][r] != 0.0)
            G.f[SE_I][r] = (G.f[SE_VC][r] - vv) / G.f[SE_RS][r];
        else
            G.f[SE_I][r] = 0.0;
    }
    static void seclamp_vstim(Group &G, int64_t r, double t, double vv) {
        G.f[SE_ON][r] = 1.0;
        if (t < G.f[SE_DUR1][r]) {
            G.f[SE_VC][r] = G.f[SE_AMP1][r];
        } else if (t < G.f[SE_TC2][r]) {
            G.f[SE_VC][r] = G.f[SE_AMP2][r];
        } else if (t < G.f[SE_TC3][r]) {
            G.f[SE_VC][r] = G.f[SE_AMP3][r];
        } else {
            G.f[SE_VC][r] = 0.0;
            G.f[SE_ON][r] = 0.0;
        }
        seclamp_icur(G, r, vv);
    }

    // ---- VClamp (mod/VClamp.mod): the three-level clamp with its amplifier eliminated
    static void vclamp_vstim(Group &G, int64_t r, double t) {
        G.f[VC_TC][r] = 0.0;
        for (int j = 0; j < 3; ++j) {
            G.f[VC_STIM][r] = G.f[VC_AMP + j][r];
            G.f[VC_TC][r] = G.f[VC_TC][r] + G.f[VC_DUR + j][r];
            if (t < G.f[VC_TC][r]) {
                G.f[VC_TC][r] = G.f[VC_TC][r] + 100.0;
                break;
            }
        }
    }
    static void vclamp_clamp(Group &G, int64_t r, double vv, double step_dt) {
        const double t1 = G.f[VC_TAU1][r] / step_dt, t2 = G.f[VC_TAU2][r] / step_dt;
        const double fac = G.f[VC_FAC][r], gain = G.f[VC_GAIN][r], vo0 = G.f[VC_VO0][r];
        const double e = ((1.0 + t1) * ((1.0 - fac) * vv + fac * t2 * vo0 / (1.0 + t2)) - G.f[VC_STIM][r] -
                          t1 * (G.f[VC_VI0][r] - G.f[VC_E0][r])) /
                         (2.0 + t1 + (1.0 + t1) * fac * gain / (1.0 + t2));
        G.f[VC_E][r] = e;
        G.f[VC_VO][r] = (t2 * vo0 - gain * e) / (1.0 + t2);
        G.f[VC_VI][r] = vv + fac * G.f[VC_VO][r] - fac * vv;
    }
    static double vclamp_icur(Group &G, int64_t r, double t, double vv, double step_dt) {
        if (t > G.f[VC_TC][r]) {
            G.f[VC_E0][r] = 0.0;
            G.f[VC_VO0][r] = 0.0;
            return 0.0;
        }
        vclamp_clamp(G, r, vv, step_dt);
        return (G.f[VC_VO][r] - vv) / G.f[VC_RSTIM][r];
    }

    /* BREAKPOINT currents of one row at v + 0.001 and v into rhs and d of its node. */
    void current_row(Group &G, int64_t r, double tc) {
        int32_t node = G.node[r];
        if (node < 0) return;
        double vv = v[node];
        double probe = vv + 0.001;
        double shifted = 0.0, value = 0.0;
        double scale = 1.0;
        bool density = false;
        switch (G.kind) {
            case MIND_MECH_HH: {
                density = true;
                auto eval = [&](double u) {
                    double m = G.f[HH_M][r], h = G.f[HH_H][r], nn = G.f[HH_N][r];
                    double gna = G.f[HH_GNABAR][r] * m * m * m * h;
                    double ina = gna * (u - G.f[HH_ENA][r]);
                    double gk = G.f[HH_GKBAR][r] * nn * nn * nn * nn;
                    double ik = gk * (u - G.f[HH_EK][r]);
                    double il = G.f[HH_GL][r] * (u - G.f[HH_EL][r]);
                    return ((0.0 + il) + ina) + ik;
                };
                shifted = eval(probe);
                value = eval(vv);
            } break;
            case MIND_MECH_PAS: {
                density = true;
                shifted = 0.0 + G.f[PAS_G][r] * (probe - G.f[PAS_E][r]);
                value = 0.0 + G.f[PAS_G][r] * (vv - G.f[PAS_E][r]);
            } break;
            case MIND_MECH_EXPSYN: {
                shifted = 0.0 + G.f[ES_G][r] * (probe - G.f[ES_E][r]);
                value = 0.0 + G.f[ES_G][r] * (vv - G.f[ES_E][r]);
            } break;
            case MIND_MECH_EXP2SYN: {
                double gs = G.f[E2_B][r] - G.f[E2_A][r];
                shifted = 0.0 + gs * (probe - G.f[E2_E][r]);
                value = 0.0 + gs * (vv - G.f[E2_E][r]);
            } break;
            case MIND_MECH_ICLAMP: {
                double del = G.f[IC_DEL][r];
                double i = (tc < del + G.f[IC_DUR][r] && tc >= del) ? G.f[IC_AMP][r] : 0.0;
                shifted = 0.0 - i;
                value = 0.0 - i;
            } break;
            case MIND_MECH_ALPHASYN: {  // mod/AlphaSynapse.mod BREAKPOINT
                double g = G.f[AS_GMAX][r] * oalpha((tc - G.f[AS_ONSET][r]) / G.f[AS_TAU][r]);
                shifted = 0.0 + g * (probe - G.f[AS_E][r]);
                value = 0.0 + g * (vv - G.f[AS_E][r]);
            } break;
            case ORACLE_SECLAMP: {   // electrode current: the MOD's i counts negative
                seclamp_vstim(G, r, tc, probe);
                shifted = 0.0 - G.f[SE_I][r];
                seclamp_vstim(G, r, tc, vv);
                value = 0.0 - G.f[SE_I][r];
            } break;
            case ORACLE_VCLAMP: {
                vclamp_vstim(G, r, tc);
                G.f[VC_I][r] = vclamp_icur(G, r, tc, probe, dt);
                shifted = 0.0 - G.f[VC_I][r];
                vclamp_vstim(G, r, tc);
                G.f[VC_I][r] = vclamp_icur(G, r, tc, vv, dt);
                value = 0.0 - G.f[VC_I][r];
            } break;
            default: return;
        }
        if (density) {
            scale = area[node] * 0.01;
            rhs[node] -= scale * value;
            d[node] += scale * (shifted - value) / 0.001;
        } else {
            rhs[node] += -scale * value;
            d[node] += scale * (shifted - value) / 0.001;
        }
    }

    /* Currents of one cell: its nodes cleared, then groups in layout order and each group's
     * rows in row order -- per node the order of the reference's serial loop
     * (src/runtime/cuda/micro.jl:427-500 with the atomics' order fixed). */
    void currents_cell(int64_t c, double tc) {
        for (int32_t i : cell_up[c]) {
            rhs[i] = 0.0;
            d[i] = 0.0;
        }
#ifdef MIND_ORACLE_REVERSED
        for (size_t g = groups.size(); g-- > 0;)
            for (auto r = cell_rows[c][g].rbegin(); r != cell_rows[c][g].rend(); ++r) current_row(groups[g], *r, tc);
#else
        for (size_t g = 0; g < groups.size(); ++g)
            for (int64_t r : cell_rows[c][g]) current_row(groups[g], r, tc);
#endif
    }

    /* The children of node i in the order their terms are summed into it: ascending, or
     * descending in the reversed-order variant. */
    template <class F>
    void each_child(int32_t i, F f) const {
#ifdef MIND_ORACLE_REVERSED
        for (int64_t c = child_off[i + 1]; c-- > child_off[i];) f(child[c]);
#else
        for (int64_t c = child_off[i]; c < child_off[i + 1]; ++c) f(child[c]);
#endif
    }

    int cable(int64_t cell) {
        const std::vector<int32_t> &up = cell_up[cell];
        // secondorder 1 and 2 (src/runtime/step.jl:112): capacitance over dt/2
        const double step_dt = L->secondorder == 0 ? dt : 0.5 * dt;
        for (int32_t i : up) d[i] = cap[i] / step_dt + d[i] + ad[i];
        for (int32_t i : up) {
            double R = rhs[i];
            if (parent[i] >= 0) R = R + a[i] * (v[parent[i]] - v[i]);
            each_child(i, [&](int32_t k) { R = R - a[k] * (v[i] - v[k]); });
            rhs[i] = R;
        }
        int status = 0;
        for (int32_t i : up) {
            double D = d[i], R = rhs[i];
            each_child(i, [&](int32_t k) {
                D = D - xd[k];
                R = R + xr[k];
            });
            d[i] = D;
            rhs[i] = R;
            if (D == 0.0 || !std::isfinite(D)) status = MIND_ESINGULAR;
            if (parent[i] >= 0) {
                double f = a[i] / D;
                xd[i] = f * a[i];
                xr[i] = f * R;
            }
        }
        for (auto it = up.rbegin(); it != up.rend(); ++it) {
            int32_t i = *it;
            double value = rhs[i];
            if (parent[i] >= 0) value = value + a[i] * rhs[parent[i]];
            rhs[i] = value / d[i];
        }
        // micro.jl:660-679: v += x, or v += 2 x for secondorder 1 and 2
        if (L->secondorder == 0)
            for (int32_t i : up) v[i] = v[i] + rhs[i];
        else
            for (int32_t i : up) v[i] = v[i] + 2.0 * rhs[i];
        return status;
    }

    /* cnexp state advance of one row on the new voltage at time ta = t + dt
     * (src/compiler/codegen.jl:569-641). */
    void advance_row(Group &G, int64_t r, double ta) {
        switch (G.kind) {
            case MIND_MECH_HH: {
                Rates R = rates(v[G.node[r]]);
                G.f[HH_M][r] = cnexp(G.f[HH_M][r], R.minf, R.mtau, dt);
                G.f[HH_H][r] = cnexp(G.f[HH_H][r], R.hinf, R.htau, dt);
                G.f[HH_N][r] = cnexp(G.f[HH_N][r], R.ninf, R.ntau, dt);
            } break;
            case MIND_MECH_EXPSYN:
                G.f[ES_G][r] = cnexp(G.f[ES_G][r], 0.0, G.f[ES_TAU][r], dt);
                break;
            case MIND_MECH_EXP2SYN:
                G.f[E2_A][r] = cnexp(G.f[E2_A][r], 0.0, G.f[E2_TAU1][r], dt);
                G.f[E2_B][r] = cnexp(G.f[E2_B][r], 0.0, G.f[E2_TAU2][r], dt);
                break;
            case ORACLE_SECLAMP:   // SOLVE icur METHOD after_cvode, on the new voltage
                seclamp_icur(G, r, v[G.node[r]]);
                break;
            case ORACLE_VCLAMP: {  // SOLVE update METHOD after_cvode at t + dt
                G.f[VC_I][r] = vclamp_icur(G, r, ta, v[G.node[r]], dt);
                G.f[VC_E0][r] = G.f[VC_E][r];
                G.f[VC_VO0][r] = G.f[VC_VO][r];
                G.f[VC_VI0][r] = G.f[VC_VI][r];
            } break;
            default: break;
        }
    }

    void advance_cell(int64_t c, double ta) {
        for (size_t g = 0; g < groups.size(); ++g)
            for (int64_t r : cell_rows[c][g]) advance_row(groups[g], r, ta);
    }

    void detect(double t) {
        double time = t + 1.0e-10;
        for (int64_t s : detector_sources) {
            int32_t node = L->source_nodes[s];
            bool current = v[node - 1] > L->source_thresholds[s];
            if (current && !above[s]) {
                emit_spike(s, time);
                count_spike(s);
            }
            above[s] = current;
        }
    }

    /* One micro step (src/runtime/step.jl:91-151).  Detection, the macro step and event
     * delivery are serial (heap order); the cells are independent between deliveries, so
     * each cell's currents, cable solve and state advance run on one worker of the pool,
     * cells handed out in small chunks. */
    int advance_step() {
        double t = (double)step * dt;
        if (ML && step % spm == 0) macro_step(step / spm);
        detect(t);
        deliver(t + 0.5 * dt);
        const double tc = t + 0.5 * dt;
        const int64_t cells = (int64_t)cell_up.size();
        std::atomic<int64_t> next{0};
        std::atomic<int> worst{0};
        pool->run([&](int) {
            for (;;) {
                const int64_t lo = next.fetch_add(4);
                if (lo >= cells) break;
                const int64_t hi = std::min(cells, lo + 4);
                for (int64_t c = lo; c < hi; ++c) {
                    currents_cell(c, tc);
                    const int s = cable(c);
                    advance_cell(c, t + dt);
                    int w = worst.load();
                    while (s > w && !worst.compare_exchange_weak(w, s)) {
                    }
                }
            }
        });
        const int status = worst.load();
        if (status) return fail(status, "singular or non-finite cable system");
        step += 1;
        return 0;
    }
};

}  // namespace

extern "C" {

/* Initialize from the layout (and regions, if `macro` is given) and run `steps` micro
 * steps.  trace is [(steps+1) x nrec] sample-major; spikes sorted by (time, sid);
 * macro_trace is [(steps / steps per macro step + 1) x regions] region outputs; run_ms
 * is the wall time of steps timed_from .. steps-1 (a settle period before it is untimed). */
int oracle_run_macro(const MindLayout *layout, const MindMacroLayout *macro, int64_t steps, const MindRecord *records,
                     int32_t nrec, int32_t threads, double *trace, double *spike_t, int64_t *spike_sid, int64_t cap,
                     int64_t *nspikes, double *macro_trace, double *run_ms, char *message, int32_t message_len,
                     int64_t timed_from) {
    Oracle o;
    ThreadPool pool(threads);
    o.pool = &pool;
    int status = o.load(layout);
    if (!status && macro) status = o.load_macro(macro);
    if (!status) {
        o.build_row_points();
        o.initialize();
        status = o.error;
    }
    // Recorded values: a node's v, or a kept mechanism field of a layout row (the MindRecord
    // reference rules of include/mindgpu.h; NetStim fields are not recorded).
    std::vector<const std::vector<double> *> rec_vec(nrec, nullptr);
    std::vector<int64_t> rec_idx(nrec, 0);
    for (int32_t k = 0; k < nrec && !status; ++k) {
        const MindRecord &r = records[k];
        if (r.kind == MIND_RECORD_VOLTAGE) {
            if (r.node < 1 || r.node > o.n) status = o.fail(MIND_EARG, "record node out of range");
            rec_vec[k] = &o.v;
            rec_idx[k] = r.node - 1;
            continue;
        }
        if (r.kind != MIND_RECORD_MECHANISM || r.group < 1 || r.group > layout->n_mechanisms) {
            status = o.fail(MIND_EARG, "unsupported record");
            break;
        }
        const MindMechanism &m = layout->mechanisms[r.group - 1];
        const Group &G = o.groups[r.group - 1];
        if (r.row < 1 || r.row > G.rows || r.field < 1 || r.field > m.n_fields || m.kind == MIND_MECH_NETSTIM) {
            status = o.fail(MIND_EARG, "mechanism record out of range");
            break;
        }
        const char *const *names = m.kind == MIND_MECH_HH       ? HH_NAMES
                                   : m.kind == MIND_MECH_PAS    ? PAS_NAMES
                                   : m.kind == MIND_MECH_EXPSYN ? ES_NAMES
                                   : m.kind == MIND_MECH_EXP2SYN ? E2_NAMES
                                   : m.kind == MIND_MECH_ALPHASYN ? AS_NAMES
                                   : m.kind == ORACLE_SECLAMP    ? SE_NAMES
                                   : m.kind == ORACLE_VCLAMP     ? VC_NAMES
                                                                 : IC_NAMES;
        for (size_t slot = 0; slot < G.f.size(); ++slot)
            if (std::strcmp(names[slot], m.field_names[r.field - 1]) == 0) rec_vec[k] = &G.f[slot];
        if (!rec_vec[k]) {
            status = o.fail(MIND_EARG, "mechanism field is not kept");
            break;
        }
        rec_idx[k] = r.row - 1;
    }
    auto record = [&](int64_t sample) {
        for (int32_t k = 0; k < nrec; ++k) trace[sample * nrec + k] = (*rec_vec[k])[rec_idx[k]];
    };
    auto t0 = std::chrono::steady_clock::now();
    if (!status) {
        if (nrec) record(0);
        for (int64_t s = 0; s < steps && !status; ++s) {
            if (s == timed_from) t0 = std::chrono::steady_clock::now();   // steps before it are not timed
            status = o.advance_step();
            if (status) break;
            if (nrec) record(s + 1);
            o.deliver((double)o.step * o.dt);
            status = o.error;
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    if (run_ms) *run_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (!status) {
        for (int64_t i = 0; i < o.n; ++i)
            if (!std::isfinite(o.v[i])) status = o.fail(MIND_ENONFINITE, "non-finite voltage");
    }
    if (!status && macro && macro_trace) {
        // out(k) for k = 0 .. steps / spm; the last boundary's out needs macro step k-1 done
        const int64_t last = steps / o.spm;
        while ((int64_t)o.out_hist.size() <= last) o.macro_step((int64_t)o.out_hist.size() - 1);
        for (int64_t k = 0; k <= last; ++k)
            for (int32_t i = 0; i < macro->n_regions; ++i) macro_trace[k * macro->n_regions + i] = o.out_hist[k][i];
    }
    std::vector<int64_t> idx(o.spike_t.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int64_t)i;
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t x, int64_t y) {
        if (o.spike_t[x] != o.spike_t[y]) return o.spike_t[x] < o.spike_t[y];
        return o.spike_sid[x] < o.spike_sid[y];
    });
    *nspikes = (int64_t)idx.size();
    for (int64_t i = 0; i < (int64_t)idx.size() && i < cap; ++i) {
        spike_t[i] = o.spike_t[idx[i]];
        spike_sid[i] = o.spike_sid[idx[i]];
    }
    if (message && message_len > 0) {
        std::strncpy(message, o.message.c_str(), (size_t)message_len - 1);
        message[message_len - 1] = 0;
    }
    return status;
}

int oracle_run(const MindLayout *layout, int64_t steps, const MindRecord *records, int32_t nrec,
               int32_t threads, double *trace, double *spike_t, int64_t *spike_sid, int64_t cap,
               int64_t *nspikes, double *run_ms, char *message, int32_t message_len) {
    return oracle_run_macro(layout, nullptr, steps, records, nrec, threads, trace, spike_t, spike_sid, cap, nspikes,
                            nullptr, run_ms, message, message_len, 0);
}

}  // extern "C"

extern "C" {

/* The project-owned elementary functions and Philox, exposed for the tests that
 * pin them against glibc and the published Random123 known-answer vectors. */
double oracle_exp(double x) { return mind_exp(x); }
double oracle_log(double x) { return mind_log(x); }
double oracle_pow(double x, double y) { return mind_pow(x, y); }
/* The division-free x/0.001 of the CUDA path, exported so its equality with x/0.001 can be tested. */
void oracle_div_milli(const double *x, double *out, int64_t n) {
    for (int64_t i = 0; i < n; ++i) out[i] = mind_div_milli(x[i]);
}
void oracle_philox(uint32_t *ctr, uint32_t key0, uint32_t key1) { mind_philox4x32_10(ctr, key0, key1); }

/* The region inputs' per-step Poisson counts (the rule of mind_attach_macro), for statistics tests. */
int32_t oracle_region_input_count(uint64_t seed, int64_t input, int64_t k, double mu) {
    uint32_t ctr[4] = {(uint32_t)k, (uint32_t)((uint64_t)k >> 32), (uint32_t)input, 0x4D4Du};
    mind_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u0 = ((double)ctr[0] + 1.0) * MIND_INV_2P32P1;
    double p = mind_exp(-mu), F = p;
    int32_t n = 0;
    while (u0 > F && n < 3) {
        ++n;
        p = (p * mu) / (double)n;
        F = F + p;
    }
    return n;
}

/* One random stream in the nrnran123 layout: `n` negexp draws from a fresh
 * stream keyed by (logical id, digest, stream 0, seed). */
void oracle_negexp_stream(uint64_t logical_id, uint64_t digest, uint64_t seed, int64_t n, double *out) {
    MindRan ran;
    mind_ran_init(&ran, logical_id, digest, 0u, seed);
    for (int64_t i = 0; i < n; ++i) out[i] = mind_ran_negexp(&ran, seed);
}

}  // extern "C"
