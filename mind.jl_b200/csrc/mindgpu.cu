/*
 * mindgpu.cu — host runtime and C-ABI of libmindgpu.so (include/mindgpu.h).
 *
 * mind_create validates the layout and packs it for the device:
 *   cells      connected components of the parent forest;
 *   chains     per cell, maximal unbranched paths, ordered by level so that a
 *              level's chains can be eliminated in parallel after the level
 *              below (the role of the reference's DHS rounds,
 *              src/model/micro/model.jl:906-1077);
 *   kids       per node, children in ascending layout index (the order in
 *              which their axial currents and eliminated pivots are added);
 *   rows       mechanism rows per group sorted by (cell, node, layout row);
 *   events     a ring of delivery bins sized for the longest NetCon delay.
 * mind_run advances in windows of W steps, W bounded by the shortest NetCon
 * delay out of a cell detector: a spike detected inside a window can only be
 * delivered after it, so each cell advances a whole window on its own.
 */
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <array>
#include <memory>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "kernels.cuh"
#include "macro.cuh"

using namespace mind;

int mind_mlp_forward_device(MindMlp *m, const float *x, int64_t n, float *prob, cudaStream_t stream, int32_t *err);
int mind_mlp_reserve_device(MindMlp *m, int64_t rows);
int32_t mind_mlp_inputs(const MindMlp *m);

namespace {

constexpr int32_t kMaxWindow = 64;
thread_local std::string g_create_error;

struct DeviceBuffers {
    std::vector<void *> owned;
    ~DeviceBuffers() {
        for (void *p : owned) cudaFree(p);
    }
};

}  // namespace

struct MindHandle {
    // host copies
    int32_t ncells = 0;
    int64_t n_nodes = 0;
    double dt = 0.0;
    std::vector<int64_t> packed_of_layout;   // layout node -> packed index
    std::vector<int64_t> node_off;           // [ncells+1] packed node ranges
    std::vector<int32_t> edge_target;        // 0-based point per edge
    struct Injected {
        int64_t bin;
        InjectedEvent event;                 // edge < 0: the raster entry of external source `point`
    };
    // Events from inject_event!/inject_spike! wait on the host until the window that
    // delivers them (the ring holds one window plus the longest delay); appended in
    // call order and stably sorted by bin before a window drains them.
    std::vector<Injected> injected;
    bool injected_sorted = true;
    InjectedEvent *inject_dev = nullptr;     // staging for one window's due events
    size_t inject_cap = 0;
    std::vector<int64_t> fanout;             // [n_sources+1] 0-based edge ranges
    std::vector<double> edge_delay;
    std::vector<uint8_t> source_external;    // no detector and no point: an inject_spike! input
    struct PatternSpike {
        double time;
        int32_t source;                      // 0-based source fed by a PatternStim
    };
    std::vector<PatternSpike> pattern;       // PatternStim firings, in time order
    std::vector<uint8_t> source_detector;
    // regions coupled to the cells (mind_attach_macro)
    MacroParams M{};
    double *macro_y0 = nullptr;
    int32_t bin_steps = 0;                   // micro steps per rate bin
    int32_t macro_threads = 32;
    double *macro_trace_dev = nullptr;
    size_t macro_trace_cap = 0;
    std::vector<double> macro_trace;
    int64_t macro_trace_samples = 0;
    std::vector<int32_t> cell_detector;      // first detector source of each cell, or -1
    // cells the surrogate stands in for (mind_attach_surrogate)
    MindMlp *sur_mlp = nullptr;
    int32_t n_sur = 0;
    std::vector<uint8_t> sur_attached;   // cells named at mind_attach_surrogate (buffer capacity)
    int32_t sur_cap = 0;
    float sur_scale = 1.0f;
    int32_t *sur_cells = nullptr, *sur_sources = nullptr, *sur_spikes = nullptr;
    float *sur_x = nullptr, *sur_prob = nullptr;
    float *sur_offset = nullptr;         // per cell (layout order): logit calibration offset
    // spike exchange between ranks (mind_attach_exchange)
    int32_t ex_world = 0, ex_rank = 0, ex_width = 0, ex_n_ext = 0;
    int32_t *ex_sid_of_source = nullptr;   // [n_sources]: global sid of a local detector, else -1
    int32_t *ex_ext_sid = nullptr, *ex_ext_source = nullptr;   // received sids (ascending) -> local source
    int64_t *ex_send = nullptr, *ex_recv = nullptr;            // [1 + 2 width], [world][1 + 2 width]
    ncclComm_t ex_comm = nullptr;
    // synaptic drive recording (mind_set_drive_recording)
    int32_t drive_bin_steps = 0;
    float *drive_dev = nullptr;
    size_t drive_cap = 0;
    std::vector<float> drive;
    int64_t drive_bins = 0;
    std::vector<double> v0_packed;
    bool has_generated = false;              // some group runs CUDA C emitted from a MOD file
    bool gen_runtime = false;                // ... one compiled at run time (mind_load_mechanisms)
    cudaKernel_t rt_window[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // that module's kernels
    cudaKernel_t rt_init = nullptr;
    int32_t device = -1;                     // the device current at the first allocation: state and stream live there
    int64_t n_sources = 0;
    std::vector<int64_t> source_ids;
    int32_t precision = MIND_FP64;
    bool initialized = false;
    int64_t step = 0;
    int32_t window = 1;
    int32_t max_delay_bins = 0;
    std::string error;
    double last_ms = 0.0;
    // per-group initial data for restore at initialize
    struct GroupInit {
        int32_t kind;
        int32_t rows;
        std::vector<std::vector<double>> f;   // device slot order
        uint64_t digest;
        std::vector<uint64_t> logical;        // device row order (NetStim)
    };
    std::vector<GroupInit> group_init;
    // references (MindRecord): per group, layout row -> device row, layout column -> device
    // slot (-1: not kept), and each cell's first device row
    std::vector<std::vector<int32_t>> dev_row_of;
    std::vector<std::vector<int32_t>> field_slot;
    std::vector<std::vector<int32_t>> group_row_off;
    // results
    const double *trace_result = nullptr;   // the last run's traces (device), [samples x records]
    double *trace_by_record = nullptr;      // their transpose for mind_get_trace_by_record (grow-only)
    size_t trace_by_record_cap = 0;
    int64_t trace_samples = 0;
    int32_t trace_records = 0;
    std::vector<double> spike_times;
    std::vector<int64_t> spike_sids;
    // device
    DeviceBuffers buffers;
    Params P{};
    uint64_t *ns_logical = nullptr;
    size_t smem_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    int32_t *rec_off_dev = nullptr;
    int32_t *rec_node_dev = nullptr;
    int32_t *rec_col_dev = nullptr;
    const double **rec_initial_dev = nullptr;   // per record: its value in HBM (first sample)
    const double **rec_ptr_dev = nullptr;       // per cell-sorted record: HBM parameter or null
    double *trace_dev = nullptr;
    size_t trace_capacity = 0;
    size_t rec_capacity = 0, rec_off_cap = 0, rec_col_cap = 0, rec_ptr_cap = 0, rec_initial_cap = 0;
    std::vector<MindRecord> rec_last;             // the record set whose tables are on the device
    struct Bin {
        int32_t first, count;
        size_t smem_bytes;
        int32_t threads = kCellThreads;   // CTA size of the bin's launches (kCellThreads or half)
        bool tight = false;               // 128 threads, compiled for kTightBlocks CTAs per SM
        int32_t max_detectors = 0;        // most threshold detectors on one of its cells
        bool global_image = false;        // cells too large for shared memory: image in HBM
        bool paths = false;               // some cell has the path schedule of the solve
    };
    std::vector<Bin> bins;           // cells grouped by shared-memory need
    std::vector<cudaStream_t> bin_streams;   // size bins run concurrently
    std::vector<cudaEvent_t> bin_done;
    cudaEvent_t fork = nullptr;
    bool profiling = false;
    std::vector<cudaEvent_t> prof_events;
    MindRunStats stats{};
    int32_t *bin_cells = nullptr;    // cell ids, bins contiguous

    template <class T>
    T *alloc(size_t count) {
        void *p = nullptr;
        if (device < 0 && cudaGetDevice(&device) != cudaSuccess) throw std::bad_alloc();
        if (count == 0) count = 1;
        if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) throw std::bad_alloc();
        buffers.owned.push_back(p);
        return static_cast<T *>(p);
    }
    template <class T>
    T *upload(const std::vector<T> &host) {
        T *p = alloc<T>(host.size());
        if (!host.empty() &&
            cudaMemcpy(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::bad_alloc();
        return p;
    }
    void release(void *p) {
        if (!p) return;
        auto it = std::find(buffers.owned.begin(), buffers.owned.end(), p);
        if (it != buffers.owned.end()) buffers.owned.erase(it);
        cudaFree(p);
    }
};

namespace {

int fail(MindHandle *h, int code, const std::string &why) {
    if (h) {
        h->error = why;
        if (code != MIND_ELAYOUT && code != MIND_EARG) h->initialized = false;
    } else {
        g_create_error = why;
    }
    return code;
}

int cuda_fail(MindHandle *h, cudaError_t e, const char *where) {
    return fail(h, MIND_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CUDA_TRY(h, call)                                          \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) return cuda_fail((h), _e, #call);   \
    } while (0)

/* Window: a spike detected at step s arrives in bin >= s + floor((d - dt/2)/dt); keep one bin margin. */
int32_t window_for_delay(double min_delay, double dt) {
    if (!std::isfinite(min_delay)) return kMaxWindow;
    const double k = std::floor((min_delay - 0.5 * dt) / dt) - 1.0;
    return (int32_t)std::max(1.0, std::min((double)kMaxWindow, k));
}

int field_index(const MindMechanism &m, const char *name) {
    for (int32_t j = 0; j < m.n_fields; ++j)
        if (m.field_names && m.field_names[j] && std::strcmp(m.field_names[j], name) == 0) return j;
    return -1;
}

/* The generated mechanisms the library knows, by generated index (kind - MIND_MECH_GENERATED):
 * those compiled in (kGenMechanisms), then those of modules compiled at run time and
 * loaded by mind_load_mechanisms.  Append-only, so a kind keeps its meaning for the life of
 * the process; the latest module's kernels serve every runtime index (each module holds
 * all runtime mechanisms registered so far). */
struct GenEntry {
    std::string name;
    int32_t point = 0, net_receive = 0;
    std::vector<std::string> fields;
    std::vector<const char *> field_ptrs;
    std::vector<double> defaults;
    uint64_t digest = 0;
    std::string ion_reads;
};

struct GenRegistry {
    std::mutex mu;
    std::vector<std::unique_ptr<GenEntry>> entries;
    cudaKernel_t window[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [mixed][image in HBM]
    cudaKernel_t init = nullptr;
};

GenRegistry &gen_registry() {
    static GenRegistry *r = [] {
        GenRegistry *g = new GenRegistry();
        for (int32_t k = 0; k < kGeneratedCount; ++k) {
            const GenMechanism &m = kGenMechanisms[k];
            auto e = std::make_unique<GenEntry>();
            e->name = m.name;
            e->point = m.point;
            e->net_receive = m.net_receive;
            for (int32_t f = 0; f < m.n_fields; ++f) {
                e->fields.push_back(kGenFieldNames[m.first_field + f]);
                e->defaults.push_back(kGenDefaults[m.first_field + f]);
            }
            e->digest = m.digest;
            e->ion_reads = m.ion_reads;
            g->entries.push_back(std::move(e));
        }
        for (auto &e : g->entries)
            for (auto &f : e->fields) e->field_ptrs.push_back(f.c_str());
        return g;
    }();
    return *r;
}

/* The generated mechanism of `kind`, or null. */
const GenEntry *gen_entry(int32_t kind) {
    if (kind < MIND_MECH_GENERATED) return nullptr;
    GenRegistry &g = gen_registry();
    std::lock_guard<std::mutex> lock(g.mu);
    const size_t k = (size_t)(kind - MIND_MECH_GENERATED);
    return k < g.entries.size() ? g.entries[k].get() : nullptr;
}

bool generated_kind(int32_t kind) { return gen_entry(kind) != nullptr; }

struct KindSpec {
    int32_t kind;
    std::vector<const char *> fields;   // layout fields copied to device slots 0..k-1
    int32_t nslot;
    int32_t nfloat;
};

KindSpec spec_of(int32_t kind) {
    switch (kind) {
        case MIND_MECH_HH:
            return {kind, {"gnabar", "gkbar", "gl", "el", "ena", "ek"}, HH_NSLOT, 0};
        case MIND_MECH_PAS:
            return {kind, {"g", "e"}, PAS_NSLOT, 0};
        case MIND_MECH_EXPSYN:
            return {kind, {"e", "g", "tau"}, ES_NSLOT, 1};
        case MIND_MECH_EXP2SYN:
            return {kind, {"e", "A", "B", "factor", "tau1", "tau2"}, E2_NSLOT, 2};
        case MIND_MECH_ICLAMP:
            return {kind, {"del", "dur", "amp"}, IC_NSLOT, 0};
        case MIND_MECH_ALPHASYN:
            return {kind, {"onset", "tau", "gmax", "e"}, AS_NSLOT, 0};
        case MIND_MECH_NETSTIM:
            return {kind, {"interval", "number", "start", "noise", "event", "on", "ispike"}, NS_NSLOT, 0};
        case MIND_MECH_PATTERNSTIM:   // no fields: its spike times come with the layout
            return {kind, {}, 0, 0};
        default:
            if (const GenEntry *g = gen_entry(kind)) {   // every field of an emitted mechanism, in column order
                KindSpec spec{kind, {}, 0, 0};
                for (const char *f : g->field_ptrs) spec.fields.push_back(f);
                return spec;
            }
            return {0, {}, 0, 0};
    }
}

/* Device slot of each copied layout field (same order as spec_of fields). */
int slot_of(int32_t kind, int k) {
    static const int hh[] = {HH_GNABAR, HH_GKBAR, HH_GL, HH_EL, HH_ENA, HH_EK};
    static const int pas[] = {PAS_G, PAS_E};
    static const int es[] = {ES_E, ES_G, ES_TAU};
    static const int e2[] = {E2_E, E2_A, E2_B, E2_FACTOR, E2_TAU1, E2_TAU2};
    static const int ic[] = {IC_DEL, IC_DUR, IC_AMP};
    static const int as[] = {AS_ONSET, AS_TAU, AS_GMAX, AS_E};
    static const int ns[] = {NS_INTERVAL, NS_NUMBER, NS_START, NS_NOISE, NS_EVENT, NS_ON, NS_ISPIKE};
    switch (kind) {
        case MIND_MECH_HH: return hh[k];
        case MIND_MECH_PAS: return pas[k];
        case MIND_MECH_EXPSYN: return es[k];
        case MIND_MECH_EXP2SYN: return e2[k];
        case MIND_MECH_ICLAMP: return ic[k];
        case MIND_MECH_ALPHASYN: return as[k];
        case MIND_MECH_NETSTIM: return ns[k];
        default: return 0;
    }
}

/* Device slot of a MOD field that a reference may name (the PARAMETER and STATE fields
 * the kernels keep), or -1. */
int readable_slot(int32_t kind, const char *name) {
    struct Entry {
        int32_t kind;
        const char *name;
        int slot;
    };
    static const Entry table[] = {
        {MIND_MECH_HH, "gnabar", HH_GNABAR}, {MIND_MECH_HH, "gkbar", HH_GKBAR}, {MIND_MECH_HH, "gl", HH_GL},
        {MIND_MECH_HH, "el", HH_EL},         {MIND_MECH_HH, "ena", HH_ENA},     {MIND_MECH_HH, "ek", HH_EK},
        {MIND_MECH_HH, "m", HH_M},           {MIND_MECH_HH, "h", HH_H},         {MIND_MECH_HH, "n", HH_N},
        {MIND_MECH_PAS, "g", PAS_G},         {MIND_MECH_PAS, "e", PAS_E},
        {MIND_MECH_EXPSYN, "tau", ES_TAU},   {MIND_MECH_EXPSYN, "e", ES_E},     {MIND_MECH_EXPSYN, "g", ES_G},
        {MIND_MECH_EXP2SYN, "tau1", E2_TAU1}, {MIND_MECH_EXP2SYN, "tau2", E2_TAU2},
        {MIND_MECH_EXP2SYN, "e", E2_E},      {MIND_MECH_EXP2SYN, "A", E2_A},    {MIND_MECH_EXP2SYN, "B", E2_B},
        {MIND_MECH_EXP2SYN, "factor", E2_FACTOR},
        {MIND_MECH_ICLAMP, "del", IC_DEL},   {MIND_MECH_ICLAMP, "dur", IC_DUR}, {MIND_MECH_ICLAMP, "amp", IC_AMP},
        {MIND_MECH_ALPHASYN, "onset", AS_ONSET}, {MIND_MECH_ALPHASYN, "tau", AS_TAU},
        {MIND_MECH_ALPHASYN, "gmax", AS_GMAX},   {MIND_MECH_ALPHASYN, "e", AS_E},
        {MIND_MECH_NETSTIM, "interval", NS_INTERVAL}, {MIND_MECH_NETSTIM, "number", NS_NUMBER},
        {MIND_MECH_NETSTIM, "start", NS_START},       {MIND_MECH_NETSTIM, "noise", NS_NOISE},
        {MIND_MECH_NETSTIM, "event", NS_EVENT},       {MIND_MECH_NETSTIM, "on", NS_ON},
        {MIND_MECH_NETSTIM, "ispike", NS_ISPIKE},
    };
    if (!name) return -1;
    if (const GenEntry *g = gen_entry(kind)) {   // every column of an emitted mechanism is kept
        for (size_t k = 0; k < g->fields.size(); ++k)
            if (g->fields[k] == name) return (int)k;
        return -1;
    }
    for (const Entry &e : table)
        if (e.kind == kind && std::strcmp(e.name, name) == 0) return e.slot;
    return -1;
}

/* Index of a device slot in a group's staged shared-memory rows, or -1 (read from HBM). */
int staged_slot(int32_t kind, int slot) {
    switch (kind) {
        case MIND_MECH_HH: return slot;
        case MIND_MECH_EXPSYN: return slot == ES_G ? 0 : -1;
        case MIND_MECH_EXP2SYN: return slot == E2_A ? 0 : slot == E2_B ? 1 : -1;
        default: return -1;
    }
}

int launch_grid(int64_t work) {
    int64_t blocks = (work + kThreads - 1) / kThreads;
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 16) blocks = 148 * 16;
    return (int)blocks;
}

/* The window kernel's launch shapes: 128 threads per cell (kCellThreads), 64, or one warp;
 * the 128-thread shapes also without the path schedule (PATHS false). */
template <int NT, int MINB = default_min_blocks(NT), bool PATHS = true>
cudaError_t set_window_smem(int bytes) {
    cudaError_t e = cudaFuncSetAttribute(window_kernel<false, NT, false, false, MINB, PATHS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(window_kernel<true, NT, false, false, MINB, PATHS>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

/* Whether a bin's 128-thread launches start as the tight variant: when its shared memory
 * leaves room for more resident CTAs per SM than the default register bound (228 KB per SM,
 * 1 KB reserved per CTA). */
bool tight_by_default(size_t smem_bytes) { return (smem_bytes + 1024) * 6 <= 228 * 1024; }

bool valid_cell_threads(int32_t threads) {
    return threads == kCellThreads || threads == kCellThreads / 2 || threads == kCellThreads / 4;
}

int create(const MindLayout *L, MindHandle *h) {
    if (!L) return fail(h, MIND_EARG, "null layout");
    if (L->abi_version != MIND_ABI_VERSION) return fail(h, MIND_ELAYOUT, "ABI version mismatch");
    // secondorder (src/runtime/step.jl:101-136, micro.jl:660-679): 1 and 2 assemble with
    // C/(dt/2) and update v += 2 x; order 2's ion-current correction only feeds ion
    // concentration mechanisms, which this runtime does not run, so 2 acts as 1 here.
    if (L->secondorder < 0 || L->secondorder > 2) return fail(h, MIND_ELAYOUT, "secondorder must be 0, 1 or 2");
    if (!(L->dt > 0.0) || !std::isfinite(L->dt)) return fail(h, MIND_ELAYOUT, "dt must be positive");
    if (L->n_mechanisms > kMaxGroups) return fail(h, MIND_ELAYOUT, "too many mechanism groups");
    const int64_t n = L->n_nodes;
    if (n < 0 || n >= INT32_MAX) return fail(h, MIND_ELAYOUT, "node count out of range");
    h->n_nodes = n;
    h->dt = L->dt;

    // ---- cells and children (ascending layout index) ----
    std::vector<int32_t> parent(n);
    for (int64_t i = 0; i < n; ++i) {
        int32_t p = L->parent[i];
        if (p < 0 || p > n || p == i + 1) return fail(h, MIND_ELAYOUT, "parent index out of range");
        parent[i] = p - 1;
    }
    std::vector<int64_t> child_off(n + 1, 0);
    for (int64_t i = 0; i < n; ++i)
        if (parent[i] >= 0) child_off[parent[i] + 1]++;
    for (int64_t i = 0; i < n; ++i) child_off[i + 1] += child_off[i];
    std::vector<int32_t> child(child_off[n]);
    {
        std::vector<int64_t> cur(child_off.begin(), child_off.end() - 1);
        for (int64_t i = 0; i < n; ++i)
            if (parent[i] >= 0) child[cur[parent[i]]++] = (int32_t)i;
    }
    std::vector<int64_t> node_off{0};
    std::vector<int32_t> layout_of_packed;
    layout_of_packed.reserve(n);
    std::vector<int32_t> cell_of(n, -1);
    std::vector<int32_t> chain_off{0}, chain_top, chain_len, chain_par, chain_kid_off{0}, chain_kids;
    std::vector<int32_t> level_off{0}, level_path, path_off{0}, path_chain;
    h->packed_of_layout.assign(n, -1);
    // Two schedules of the solve; every chain's arithmetic is the same in both.  Levels per
    // node, carried from a chain's bottom to its top (a node with one child is inside a chain):
    //  chains (chain_level): a chain runs one level above its highest child chain, one chain
    //          per thread;
    //  paths (path_level): a chain continues the path of the child chain that finishes last,
    //          when that child is unique, so one thread eliminates both in the same level and
    //          the chain adds no level; otherwise (a leaf, or a tie) it starts a path one level
    //          above its children.
    // Cells take paths when paths cut their levels at least fourfold (pyramidal trees, a long
    // trunk with side branches: 16 levels -> 2) and such cells hold at least half of the
    // network's nodes; on bushy random trees (11 -> 4.5 levels) the chain schedule measured
    // faster at full occupancy, and a network of them keeps the chain-only kernels.
    std::vector<int32_t> chain_level(n, 0), path_level(n, 0);
    std::vector<char> path_cell(n, 0);   // by root
    bool network_paths = false;
    {
        int64_t path_nodes = 0;
        std::vector<int32_t> bfs;
        for (int64_t root = 0; root < n; ++root) {
            if (parent[root] >= 0) continue;
            bfs.assign(1, (int32_t)root);
            for (size_t k = 0; k < bfs.size(); ++k)
                for (int64_t c = child_off[bfs[k]]; c < child_off[bfs[k] + 1]; ++c) bfs.push_back(child[c]);
            for (size_t k = bfs.size(); k-- > 0;) {
                const int32_t i = bfs[k];
                const int64_t kids = child_off[i + 1] - child_off[i];
                if (kids == 1) {
                    chain_level[i] = chain_level[child[child_off[i]]];
                    path_level[i] = path_level[child[child_off[i]]];
                } else if (kids > 1) {
                    int32_t cl = 0, last = -1, ties = 0;
                    for (int64_t c = child_off[i]; c < child_off[i + 1]; ++c) {
                        const int32_t j = child[c];
                        cl = std::max(cl, chain_level[j] + 1);
                        if (path_level[j] > last) {
                            last = path_level[j];
                            ties = 1;
                        } else if (path_level[j] == last) {
                            ++ties;
                        }
                    }
                    chain_level[i] = cl;
                    path_level[i] = ties == 1 ? last : last + 1;
                }
            }
            if (chain_level[root] + 1 >= 4 * (path_level[root] + 1)) {
                path_cell[root] = 1;
                path_nodes += (int64_t)bfs.size();
            }
        }
        network_paths = 2 * path_nodes >= n;
    }
    std::vector<char> cell_paths;   // by cell: the path schedule
    for (int64_t root = 0; root < n; ++root) {
        if (parent[root] >= 0) continue;
        const int32_t cell = (int32_t)(node_off.size() - 1);
        // BFS over the cell
        std::vector<int32_t> bfs{(int32_t)root};
        for (size_t k = 0; k < bfs.size(); ++k) {
            cell_of[bfs[k]] = cell;
            for (int64_t c = child_off[bfs[k]]; c < child_off[bfs[k] + 1]; ++c) bfs.push_back(child[c]);
        }
        // chains: a node starts a chain unless it is the only child of its parent
        auto only_child = [&](int32_t i) {
            return parent[i] >= 0 && child_off[parent[i] + 1] - child_off[parent[i]] == 1;
        };
        std::vector<int32_t> tops;
        for (int32_t i : bfs)
            if (!only_child(i)) tops.push_back(i);
        std::vector<std::vector<int32_t>> chains(tops.size());
        // top node -> chain id, by binary search over (top, id) pairs
        std::vector<std::pair<int32_t, int32_t>> top_id;
        top_id.reserve(tops.size());
        for (size_t k = 0; k < tops.size(); ++k) {
            int32_t i = tops[k];
            chains[k].push_back(i);
            while (child_off[i + 1] - child_off[i] == 1) {
                i = child[child_off[i]];
                chains[k].push_back(i);
            }
            top_id.push_back({tops[k], (int32_t)k});
        }
        std::sort(top_id.begin(), top_id.end());
        auto chain_id_of = [&](int32_t top) {
            auto it = std::lower_bound(top_id.begin(), top_id.end(), std::make_pair(top, INT32_MIN));
            return it->second;
        };
        // levels of the cell's schedule; on paths, the child chain a chain continues is its
        // one child chain of the same path level
        const bool use_paths = network_paths && path_cell[root];
        cell_paths.push_back(use_paths ? 1 : 0);
        std::vector<int32_t> level(tops.size(), 0), below(tops.size(), -1);
        for (size_t k = 0; k < tops.size(); ++k) {
            level[k] = use_paths ? path_level[tops[k]] : chain_level[tops[k]];
            if (!use_paths) continue;
            const int32_t bottom = chains[k].back();
            for (int64_t c = child_off[bottom]; c < child_off[bottom + 1]; ++c)
                if (path_level[child[c]] == level[k]) below[k] = chain_id_of(child[c]);
        }
        // a path is named by its head, the chain that no parent chain continues; its chains
        // are listed deepest first (the elimination order)
        std::vector<char> continued(tops.size(), 0);
        for (size_t k = 0; k < tops.size(); ++k)
            if (below[k] >= 0) continued[below[k]] = 1;
        std::vector<std::vector<int32_t>> paths;
        std::vector<int64_t> path_nodes;
        for (size_t k = 0; k < tops.size(); ++k) {
            if (continued[k]) continue;
            std::vector<int32_t> path;
            int64_t nodes = 0;
            for (int32_t q = (int32_t)k; q >= 0; q = below[q]) {
                path.push_back(q);
                nodes += (int64_t)chains[q].size();
            }
            std::reverse(path.begin(), path.end());
            paths.push_back(std::move(path));
            path_nodes.push_back(nodes);
        }
        // paths by level (chains: in BFS order within a level; paths: the longest first, as the
        // threads take them in turn)
        std::vector<int32_t> porder(paths.size());
        for (size_t p = 0; p < porder.size(); ++p) porder[p] = (int32_t)p;
        std::stable_sort(porder.begin(), porder.end(), [&](int32_t x, int32_t y) {
            const int32_t lx = level[paths[x].front()], ly = level[paths[y].front()];
            return lx != ly ? lx < ly : use_paths && path_nodes[x] > path_nodes[y];
        });
        std::vector<int32_t> order;   // chains: the paths in that order, each deepest first
        order.reserve(tops.size());
        for (int32_t p : porder)
            for (int32_t q : paths[p]) order.push_back(q);
        std::vector<int32_t> rank(tops.size());
        for (size_t k = 0; k < order.size(); ++k) rank[order[k]] = (int32_t)k;
        // packed order: chains by rank, nodes top -> bottom
        const int64_t base = (int64_t)layout_of_packed.size();
        std::vector<int32_t> local_chain_top(tops.size());
        for (size_t k = 0; k < order.size(); ++k) {
            const auto &ch = chains[order[k]];
            local_chain_top[k] = (int32_t)(layout_of_packed.size() - base);
            for (int32_t i : ch) {
                h->packed_of_layout[i] = (int64_t)layout_of_packed.size();
                layout_of_packed.push_back(i);
            }
        }
        const int64_t cell_nodes = (int64_t)layout_of_packed.size() - base;
        node_off.push_back((int64_t)layout_of_packed.size());
        for (size_t k = 0; k < order.size(); ++k) {
            const auto &ch = chains[order[k]];
            chain_top.push_back(local_chain_top[k]);
            chain_len.push_back((int32_t)ch.size());
            int32_t top_parent = parent[ch.front()];
            chain_par.push_back(top_parent >= 0 ? (int32_t)(h->packed_of_layout[top_parent] - base) : -1);
            int32_t bottom = ch.back();
            for (int64_t c = child_off[bottom]; c < child_off[bottom + 1]; ++c)
                chain_kids.push_back(rank[chain_id_of(child[c])]);
            chain_kid_off.push_back((int32_t)chain_kids.size());
        }
        chain_off.push_back((int32_t)chain_top.size());
        int32_t nlev = 0;
        for (int32_t lv : level) nlev = std::max(nlev, lv + 1);
        const int32_t npaths = (int32_t)porder.size();
        for (int32_t lv = 0, k = 0; lv <= nlev; ++lv) {
            while (k < npaths && level[paths[porder[k]].front()] < lv) ++k;
            level_path.push_back(k);
        }
        level_off.push_back((int32_t)level_path.size());
        // a cell on the chain schedule keeps only the sentinel: its paths are its chains, and
        // level_path holds chain starts
        int32_t first_chain = 0;
        if (use_paths)
            for (int32_t p : porder) {
                path_chain.push_back(first_chain);
                first_chain += (int32_t)paths[p].size();
            }
        path_chain.push_back(first_chain);
        path_off.push_back((int32_t)path_chain.size());
    }
    if ((int64_t)layout_of_packed.size() != n) return fail(h, MIND_ELAYOUT, "parent links form a cycle");
    const int32_t ncells = (int32_t)(node_off.size() - 1);
    h->ncells = ncells;
    h->node_off = node_off;

    // ---- node coefficients in packed order ----
    std::vector<double> a(n), cdt(n), ad(n), v0(n);
    for (int64_t j = 0; j < n; ++j) {
        int32_t i = layout_of_packed[j];
        a[j] = L->axial[i];
        cdt[j] = L->capacitance[i] / (L->secondorder == 0 ? L->dt : 0.5 * L->dt);
        ad[j] = L->axial_diagonal[i];
        v0[j] = L->voltage[i];
    }
    h->v0_packed = v0;

    // ---- mechanism groups ----
    Params &P = h->P;
    P.ncells = ncells;
    P.ngroups = L->n_mechanisms;
    P.dt = L->dt;
    P.celsius = L->celsius;
    P.vscale = L->secondorder == 0 ? 1.0 : 2.0;
    P.seed = L->seed;
    P.ns_group = -1;
    std::vector<std::vector<int32_t>> &dev_row_of = h->dev_row_of;  // layout row -> device row
    dev_row_of.assign(L->n_mechanisms, {});
    h->field_slot.assign(L->n_mechanisms, {});
    // Thread t of a cell's CTA owns the local nodes i with i % kCellThreads == t, so that the
    // threads of a warp touch consecutive nodes (distinct shared-memory banks).  Each
    // group's rows are sorted by (cell, owner thread, node, layout row): a thread's rows are
    // one range, and rows of one node stay in layout order.
    std::vector<int32_t> part((size_t)ncells * L->n_mechanisms * (kCellThreads + 1), 0);
    // Mixed mode folds pas into per-node constants: its conductance g*area*0.01 and
    // that times e (the probe's (i(v+0.001)-i(v))/0.001 of a linear current is g).
    std::vector<double> mix_gs(n, 0.0), mix_gse(n, 0.0);
    std::vector<std::vector<int32_t>> row_cell(L->n_mechanisms);
    for (int32_t g = 0; g < L->n_mechanisms; ++g) {
        const MindMechanism &m = L->mechanisms[g];
        KindSpec spec = spec_of(m.kind);
        if (!spec.kind) return fail(h, MIND_ELAYOUT, "unsupported mechanism kind " + std::to_string(m.kind));
        if (m.rows < 0 || m.rows >= INT32_MAX) return fail(h, MIND_ELAYOUT, "mechanism rows out of range");
        const int32_t rows = (int32_t)m.rows;
        std::vector<int> src(spec.fields.size());
        for (size_t k = 0; k < spec.fields.size(); ++k) {
            src[k] = field_index(m, spec.fields[k]);
            if (src[k] < 0)
                return fail(h, MIND_ELAYOUT, std::string("mechanism lacks field ") + spec.fields[k]);
        }
        for (int32_t j = 0; j < m.n_fields; ++j)
            h->field_slot[g].push_back(readable_slot(m.kind, m.field_names ? m.field_names[j] : nullptr));
        const bool artificial = m.kind == MIND_MECH_NETSTIM || m.kind == MIND_MECH_PATTERNSTIM;
        if (m.kind == MIND_MECH_NETSTIM) {
            if (P.ns_group >= 0) return fail(h, MIND_ELAYOUT, "more than one NetStim group");
            P.ns_group = g;
        }
        // sort rows by (cell, owner thread, local node, layout row)
        std::vector<int64_t> key(rows), order_key(rows);
        for (int32_t r = 0; r < rows; ++r) {
            int32_t node = m.nodes[r];
            if (artificial) {
                if (node != 0) return fail(h, MIND_ELAYOUT, "artificial cell with a node");
                key[r] = r;
                order_key[r] = r;
            } else {
                if (node < 1 || node > n) return fail(h, MIND_ELAYOUT, "mechanism node out of range");
                key[r] = h->packed_of_layout[node - 1];
                const int32_t cell = cell_of[node - 1];
                const int64_t local = key[r] - node_off[cell];
                const int64_t per_thread = (node_off[cell + 1] - node_off[cell] + kCellThreads - 1) / kCellThreads;
                order_key[r] = ((int64_t)cell << 32) | ((local % kCellThreads) * per_thread + local / kCellThreads);
            }
        }
        std::vector<int32_t> perm(rows);
        for (int32_t r = 0; r < rows; ++r) perm[r] = r;
        std::stable_sort(perm.begin(), perm.end(), [&](int32_t x, int32_t y) { return order_key[x] < order_key[y]; });
        dev_row_of[g].assign(rows, 0);
        for (int32_t r = 0; r < rows; ++r) dev_row_of[g][perm[r]] = r;
        MindHandle::GroupInit init;
        init.kind = m.kind;
        init.rows = rows;
        init.digest = m.digest;
        const bool generated = generated_kind(m.kind);
        const int32_t gen_cols = (int32_t)spec.fields.size();
        // an emitted mechanism keeps every field as a column, then its current scale
        init.f.assign(generated ? gen_cols + 1 : spec.nslot, std::vector<double>(rows, generated ? 1.0 : 0.0));
        for (size_t k = 0; k < spec.fields.size(); ++k) {
            int slot = generated ? (int)k : slot_of(m.kind, (int)k);
            for (int32_t r = 0; r < rows; ++r) init.f[slot][r] = m.data[(int64_t)src[k] * m.rows + perm[r]];
        }
        std::vector<int32_t> node_dev(rows, -1), seg(rows, 1), row_off(ncells + 1, 0);
        row_cell[g].assign(rows, -1);
        if (!artificial) {
            for (int32_t r = 0; r < rows; ++r) {
                int64_t packed = key[perm[r]];
                node_dev[r] = (int32_t)packed;
                row_cell[g][r] = cell_of[layout_of_packed[packed]];
            }
            for (int32_t r = 0; r < rows; ++r) {
                if (r > 0 && node_dev[r] == node_dev[r - 1]) {
                    seg[r] = 0;
                } else {
                    int32_t len = 1;
                    while (r + len < rows && node_dev[r + len] == node_dev[r]) ++len;
                    seg[r] = len;
                }
            }
            if (generated && !gen_entry(m.kind)->point) {
                for (int32_t r = 0; r < rows; ++r)
                    if (seg[r] > 1) return fail(h, MIND_ELAYOUT, "density mechanism twice on one node");
                for (int32_t r = 0; r < rows; ++r)
                    init.f[gen_cols][r] = L->area[layout_of_packed[node_dev[r]]] * 0.01;
            }
            if ((m.kind == MIND_MECH_HH || m.kind == MIND_MECH_PAS)) {
                for (int32_t r = 0; r < rows; ++r)
                    if (seg[r] > 1) return fail(h, MIND_ELAYOUT, "density mechanism twice on one node");
                int slot = m.kind == MIND_MECH_HH ? (int)HH_SCALE : (int)PAS_SCALE;
                for (int32_t r = 0; r < rows; ++r) init.f[slot][r] = L->area[layout_of_packed[node_dev[r]]] * 0.01;
                if (m.kind == MIND_MECH_PAS)
                    for (int32_t r = 0; r < rows; ++r) {
                        const double gs = init.f[PAS_G][r] * init.f[PAS_SCALE][r];
                        mix_gs[node_dev[r]] += gs;
                        mix_gse[node_dev[r]] += gs * init.f[PAS_E][r];
                    }
            }
            for (int32_t r = 0; r < rows; ++r) row_off[row_cell[g][r] + 1]++;
            for (int32_t c = 0; c < ncells; ++c) row_off[c + 1] += row_off[c];
            // thread t's rows: the range after the rows of the owners before it
            for (int32_t c = 0; c < ncells; ++c) {
                int32_t *pc = part.data() + ((size_t)c * L->n_mechanisms + g) * (kCellThreads + 1);
                for (int32_t r = row_off[c]; r < row_off[c + 1]; ++r)
                    pc[(node_dev[r] - node_off[c]) % kCellThreads + 1]++;
                for (int32_t t = 0; t < kCellThreads; ++t) pc[t + 1] += pc[t];
            }
        }
        if (m.kind == MIND_MECH_NETSTIM) {
            init.logical.resize(rows);
            for (int32_t r = 0; r < rows; ++r) init.logical[r] = m.logical_ids[perm[r]];
        }
        DevGroup &G = P.groups[g];
        G.kind = m.kind;
        G.rows = rows;
        G.row_off = h->upload(row_off);
        G.node = h->upload(node_dev);
        G.seg = h->upload(seg);
        for (int k = 0; k < 12; ++k) G.f[k] = nullptr;
        for (int k = 0; k < 4; ++k) G.s[k] = nullptr;
        for (int k = 0; k < spec.nslot; ++k) G.f[k] = h->alloc<double>(rows);
        for (int k = 0; k < spec.nfloat; ++k) G.s[k] = h->alloc<float>(rows);
        G.gen = generated ? m.kind - MIND_MECH_GENERATED : -1;
        h->has_generated |= generated;
        h->gen_runtime |= generated && m.kind - MIND_MECH_GENERATED >= kGeneratedCount;
        G.ncols = generated ? gen_cols : 0;
        G.cols = generated ? h->alloc<double>((size_t)(gen_cols + 1) * (size_t)std::max(rows, 1)) : nullptr;
        h->group_init.push_back(std::move(init));
    }

    // ---- points, sources, detectors, edges ----
    const int64_t np = L->n_points;
    std::vector<int32_t> point_cell(np, -1), point_group(np, -1), point_row(np, -1);
    for (int64_t p = 0; p < np; ++p) {
        int32_t g = L->point_group[p] - 1, r = L->point_row[p] - 1;
        if (g < 0 || g >= L->n_mechanisms || r < 0 || r >= L->mechanisms[g].rows)
            return fail(h, MIND_ELAYOUT, "point index out of range");
        point_group[p] = g;
        point_row[p] = dev_row_of[g][r];
        point_cell[p] = row_cell[g][point_row[p]];
    }
    h->n_sources = L->n_sources;
    h->source_ids.assign(L->source_ids, L->source_ids + L->n_sources);
    std::vector<std::vector<std::pair<int32_t, int32_t>>> det_by_cell(ncells);
    std::vector<double> det_thr_by_source(L->n_sources, 0.0);
    std::vector<int32_t> ns_source(P.ns_group >= 0 ? L->mechanisms[P.ns_group].rows : 0, -1);
    std::vector<std::vector<int32_t>> pattern_sources(np);   // sources fed by each PatternStim point
    for (int64_t s = 0; s < L->n_sources; ++s) {
        int32_t node = L->source_nodes[s];
        int32_t point = L->source_points[s];
        if (node < 0 || node > n) return fail(h, MIND_ELAYOUT, "source node out of range");
        if (point < 0 || point > np) return fail(h, MIND_ELAYOUT, "source point out of range");
        if (node > 0) {
            int64_t packed = h->packed_of_layout[node - 1];
            int32_t cell = cell_of[node - 1];
            det_by_cell[cell].push_back({(int32_t)(packed - node_off[cell]), (int32_t)s});
            det_thr_by_source[s] = L->source_thresholds[s];
        } else if (point > 0) {
            int32_t g = point_group[point - 1];
            if (g == P.ns_group) ns_source[point_row[point - 1]] = (int32_t)s;
            if (L->mechanisms[g].kind == MIND_MECH_PATTERNSTIM) pattern_sources[point - 1].push_back((int32_t)s);
        }
    }
    // PatternStim: every prescribed time fires the point's sources (replayed at each initialize)
    if (L->n_pattern < 0 || (L->n_pattern > 0 && (!L->pattern_times || !L->pattern_points)))
        return fail(h, MIND_ELAYOUT, "invalid PatternStim spike list");
    for (int64_t k = 0; k < L->n_pattern; ++k) {
        const int32_t point = L->pattern_points[k];
        const double t = L->pattern_times[k];
        if (point < 1 || point > np || L->mechanisms[point_group[point - 1]].kind != MIND_MECH_PATTERNSTIM)
            return fail(h, MIND_ELAYOUT, "a PatternStim spike names a point that is not a PatternStim");
        if (!(t >= 0.0) || !std::isfinite(t)) return fail(h, MIND_ELAYOUT, "PatternStim spike times must be >= 0");
        for (int32_t s : pattern_sources[point - 1]) h->pattern.push_back({t, s});
    }
    std::vector<int32_t> det_off{0}, det_node, det_source;
    std::vector<double> det_thr;
    for (int32_t c = 0; c < ncells; ++c) {
        h->cell_detector.push_back(det_by_cell[c].empty() ? -1 : det_by_cell[c].front().second);
        if ((int32_t)det_by_cell[c].size() > kCellThreads)
            return fail(h, MIND_ELAYOUT, "more than " + std::to_string(kCellThreads) +
                                             " threshold detectors on one cell");
        for (auto &d : det_by_cell[c]) {
            det_node.push_back(d.first);
            det_source.push_back(d.second);
            det_thr.push_back(det_thr_by_source[d.second]);
        }
        det_off.push_back((int32_t)det_node.size());
    }
    const int64_t ne = L->n_edges;
    std::vector<int64_t> fanout(L->n_sources + 1);
    for (int64_t s = 0; s <= L->n_sources; ++s) fanout[s] = L->fanout_offsets[s] - 1;
    if (fanout[0] != 0 || fanout[L->n_sources] != ne) return fail(h, MIND_ELAYOUT, "fanout offsets inconsistent");
    std::vector<int32_t> edge_target(ne);
    std::vector<double> edge_delay(L->edge_delays, L->edge_delays + ne), edge_weight(L->edge_weights, L->edge_weights + ne);
    double min_cell_delay = INFINITY, max_delay = 0.0;
    for (int64_t s = 0; s < L->n_sources; ++s) {
        if (fanout[s + 1] < fanout[s]) return fail(h, MIND_ELAYOUT, "fanout offsets decrease");
        for (int64_t e = fanout[s]; e < fanout[s + 1]; ++e) {
            int32_t t = L->edge_targets[e];
            if (t < 1 || t > np) return fail(h, MIND_ELAYOUT, "edge target out of range");
            int32_t kind = L->mechanisms[point_group[t - 1]].kind;
            const bool receives = kind == MIND_MECH_EXPSYN || kind == MIND_MECH_EXP2SYN ||
                                  (generated_kind(kind) && gen_entry(kind)->net_receive > 0);
            if (!receives)
                return fail(h, MIND_ELAYOUT, "NetCon target has no NET_RECEIVE on the device (ExpSyn, Exp2Syn or an "
                                             "emitted mechanism with one)");
            double d = edge_delay[e];
            if (!(d >= 0.0) || !std::isfinite(d) || !std::isfinite(edge_weight[e]))
                return fail(h, MIND_ELAYOUT, "invalid NetCon delay or weight");
            edge_target[e] = t - 1;
            max_delay = std::max(max_delay, d);
            // cell detectors and external inputs bound the window (their spikes are routed
            // between windows); point sources (NetStim) are planned ahead on the device
            if (L->source_nodes[s] > 0 || L->source_points[s] == 0) min_cell_delay = std::min(min_cell_delay, d);
        }
    }
    h->window = window_for_delay(min_cell_delay, L->dt);
    h->edge_target = edge_target;
    h->fanout = fanout;
    h->edge_delay = edge_delay;
    h->source_external.assign(L->n_sources, 0);
    h->source_detector.assign(L->n_sources, 0);
    for (int64_t s = 0; s < L->n_sources; ++s) {
        h->source_external[s] = L->source_nodes[s] == 0 && L->source_points[s] == 0;
        h->source_detector[s] = L->source_nodes[s] > 0;
    }
    h->max_delay_bins = (int32_t)std::ceil(max_delay / L->dt) + 2;

    // ---- device arrays ----
    P.node_off = h->upload(node_off);
    P.v = h->alloc<double>(n);
    P.a = h->upload(a);
    P.cdt = h->upload(cdt);
    P.ad = h->upload(ad);
    {
        std::vector<double> mix_dc(n);
        for (int64_t j = 0; j < n; ++j) mix_dc[j] = cdt[j] + ad[j] + mix_gs[j];
        P.mix_dc = h->upload(mix_dc);
        P.mix_gs = h->upload(mix_gs);
        P.mix_gse = h->upload(mix_gse);
    }
    P.chain_off = h->upload(chain_off);
    P.chain_top = h->upload(chain_top);
    P.chain_len = h->upload(chain_len);
    P.chain_par = h->upload(chain_par);
    P.chain_kid_off = h->upload(chain_kid_off);
    P.chain_kids = h->upload(chain_kids);
    P.level_off = h->upload(level_off);
    P.level_path = h->upload(level_path);
    P.path_off = h->upload(path_off);
    P.path_chain = h->upload(path_chain);
    P.part = h->upload(part);
    P.det_off = h->upload(det_off);
    P.det_node = h->upload(det_node);
    P.det_source = h->upload(det_source);
    P.det_thr = h->upload(det_thr);
    P.above = h->alloc<uint8_t>(L->n_sources);
    P.win_spike_cap = std::max<int32_t>(1024, ncells * 4);
    P.win_spike_source = h->alloc<int32_t>(P.win_spike_cap);
    P.win_spike_step = h->alloc<int64_t>(P.win_spike_cap);
    P.win_spike_count = h->alloc<int32_t>(1);
    int64_t spike_cap = L->spike_capacity > 0 ? L->spike_capacity : (int64_t)1 << 22;
    P.rec_spike_cap = (int32_t)std::min<int64_t>(spike_cap, INT32_MAX);
    P.rec_spike_source = h->alloc<int32_t>(P.rec_spike_cap);
    P.rec_spike_time = h->alloc<double>(P.rec_spike_cap);
    P.rec_spike_count = h->alloc<int32_t>(1);
    // Room for the longest window (attaching regions can lengthen it) plus the longest delay.
    P.ring_slots = kMaxWindow + h->max_delay_bins + 4;
    int64_t ring_cap = L->event_capacity > 0 ? L->event_capacity
                                             : std::max<int64_t>(4096, std::min<int64_t>(ne / 16 + 1, 1 << 20));
    P.ring_cap = (int32_t)ring_cap;
    P.ring = h->alloc<RingEvent>((size_t)P.ring_slots * P.ring_cap);
    P.ring_count = h->alloc<int32_t>(P.ring_slots);
    // Inbox: the events of one window by cell (a CSR rebuilt per window).  A window holds at
    // most kMaxWindow bins of at most ring_cap events; each cell stages up to 32 of its events
    // in shared memory and sorts any more in HBM.
    P.inbox_cap = 32;
    P.inbox_total = (int32_t)std::min<int64_t>((int64_t)kMaxWindow * P.ring_cap, INT32_MAX / 2);
    P.inbox = h->alloc<InboxEvent>((size_t)P.inbox_total);
    P.inbox_order = h->alloc<int32_t>((size_t)P.inbox_total);
    P.inbox_count = h->alloc<int32_t>(ncells);
    P.inbox_fill = h->alloc<int32_t>(ncells);
    P.inbox_start = h->alloc<int32_t>((size_t)ncells + 1);
    P.edge_weight = h->upload(edge_weight);
    P.edge_delay = h->upload(edge_delay);
    P.edge_target = h->upload(edge_target);
    P.fanout_off = h->upload(fanout);
    P.point_cell = h->upload(point_cell);
    P.point_group = h->upload(point_group);
    P.point_row = h->upload(point_row);
    if (P.ns_group >= 0) {
        P.ns_ran = h->alloc<MindRan>(ns_source.size());
        P.ns_source = h->upload(ns_source);
        h->ns_logical = h->upload(h->group_init[P.ns_group].logical);
    }
    P.error = h->alloc<int32_t>(1);
    P.nrec = 0;
    std::vector<int32_t> zero_off(ncells + 1, 0);
    P.rec_off = h->upload(zero_off);

    // Shared-memory image per cell; cells are launched in bins of similar size so a
    // launch's dynamic shared memory matches its cells.
    std::vector<int32_t> kinds(L->n_mechanisms);
    for (int32_t g = 0; g < L->n_mechanisms; ++g) kinds[g] = L->mechanisms[g].kind;
    std::vector<std::vector<int32_t>> &group_row_off = h->group_row_off;
    group_row_off.assign(L->n_mechanisms, {});
    for (int32_t g = 0; g < L->n_mechanisms; ++g) {
        group_row_off[g].assign(ncells + 1, 0);
        if (kinds[g] == MIND_MECH_NETSTIM || kinds[g] == MIND_MECH_PATTERNSTIM) continue;
        for (int32_t r = 0; r < (int32_t)row_cell[g].size(); ++r) group_row_off[g][row_cell[g][r] + 1]++;
        for (int32_t c = 0; c < ncells; ++c) group_row_off[g][c + 1] += group_row_off[g][c];
    }
    std::vector<std::pair<size_t, int32_t>> need(ncells);
    size_t worst_any = 0;
    for (int32_t c = 0; c < ncells; ++c) {
        CellShape shape{};
        shape.n = (int32_t)(node_off[c + 1] - node_off[c]);
        shape.nch = chain_off[c + 1] - chain_off[c];
        if (shape.nch > 32767)   // the window kernel keeps a node's chain as int16
            return fail(h, MIND_ELAYOUT, "a cell has more than 32767 unbranched chains");
        shape.nkids = chain_kid_off[chain_off[c + 1]] - chain_kid_off[chain_off[c]];
        shape.nlev = level_off[c + 1] - level_off[c] - 1;
        shape.npath = path_off[c + 1] - path_off[c] - 1;
        for (int32_t g = 0; g < L->n_mechanisms; ++g) shape.rows[g] = group_row_off[g][c + 1] - group_row_off[g][c];
        const size_t bytes = cell_smem_bytes(shape, kinds.data(), L->n_mechanisms, P.inbox_cap);
        need[c] = {bytes, c};
        worst_any = std::max(worst_any, bytes);
    }
    std::stable_sort(need.begin(), need.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
    // A cell whose image exceeds what one CTA can add to the kernel's static shared memory
    // keeps its image in an HBM slot (one bin, launched without dynamic shared memory).
    const size_t smem_limit = 227 * 1024 - 1024;
    size_t n_big = 0, big_bytes = 0;
    while (n_big < need.size() && need[n_big].first > smem_limit) big_bytes = std::max(big_bytes, need[n_big++].first);
    std::vector<int32_t> big_slot(ncells, -1);
    P.big_stride = (int64_t)((big_bytes + 255) / 256 * 256);
    for (size_t k = 0; k < n_big; ++k) big_slot[need[k].second] = (int32_t)k;
    P.big_image = n_big ? h->alloc<unsigned char>(n_big * (size_t)P.big_stride) : nullptr;
    P.big_slot = h->upload(big_slot);
    size_t worst_smem = 0;
    std::vector<int32_t> bin_cells;
    for (size_t k = 0; k < need.size();) {
        size_t top = need[k].first;
        size_t first = k;
        const bool big = k < n_big;
        if (big)
            k = n_big;
        else
            while (k < need.size() && need[k].first * 4 >= top * 3) ++k;
        MindHandle::Bin bin;
        bin.first = (int32_t)first;
        bin.count = (int32_t)(k - first);
        bin.smem_bytes = big ? 0 : top;
        bin.global_image = big;
        bin.tight = !big && tight_by_default(top);
        if (!big) worst_smem = std::max(worst_smem, top);
        for (size_t q = first; q < k; ++q) {
            bin.max_detectors = std::max(bin.max_detectors, det_off[need[q].second + 1] - det_off[need[q].second]);
            bin.paths = bin.paths || cell_paths[need[q].second];
        }
        h->bins.push_back(bin);
    }
    for (auto &x : need) bin_cells.push_back(x.second);
    h->bin_cells = h->upload(bin_cells);
    h->smem_bytes = worst_smem;
    // The shared-memory opt-in is an attribute of the kernel function, shared by every handle
    // of the process (and every device it runs on): it only grows, so a handle made later
    // with smaller cells does not shrink what an earlier one launches with.
    int smem_attr = (int)std::max<size_t>(worst_smem, 1);
    {
        static std::mutex mu;
        static int largest = 0;
        std::lock_guard<std::mutex> lock(mu);
        largest = std::max(largest, smem_attr);
        smem_attr = largest;
    }
    CUDA_TRY(h, set_window_smem<kCellThreads>(smem_attr));
    CUDA_TRY(h, (set_window_smem<kCellThreads, kTightBlocks>(smem_attr)));
    CUDA_TRY(h, (set_window_smem<kCellThreads, default_min_blocks(kCellThreads), false>(smem_attr)));
    CUDA_TRY(h, (set_window_smem<kCellThreads, kTightBlocks, false>(smem_attr)));
    CUDA_TRY(h, cudaFuncSetAttribute(window_kernel<false, kCellThreads, false, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr));
    CUDA_TRY(h, cudaFuncSetAttribute(window_kernel<true, kCellThreads, false, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr));
    CUDA_TRY(h, set_window_smem<kCellThreads / 2>(smem_attr));
    CUDA_TRY(h, set_window_smem<kCellThreads / 4>(smem_attr));
    if (h->gen_runtime) {   // mechanisms compiled at run time: the kernels of the latest module
        GenRegistry &g = gen_registry();
        {
            std::lock_guard<std::mutex> lock(g.mu);
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b) h->rt_window[a][b] = g.window[a][b];
            h->rt_init = g.init;
        }
        if (!h->rt_init) return fail(h, MIND_ELAYOUT, "no mechanism module is loaded (mind_load_mechanisms)");
        for (int a = 0; a < 2; ++a)
            CUDA_TRY(h, cudaFuncSetAttribute((const void *)h->rt_window[a][0],
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr));
    }
    CUDA_TRY(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming));
    for (size_t b = 0; b < h->bins.size(); ++b) {
        cudaStream_t s;
        cudaEvent_t e;
        CUDA_TRY(h, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        CUDA_TRY(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        h->bin_streams.push_back(s);
        h->bin_done.push_back(e);
    }
    CUDA_TRY(h, cudaEventCreate(&h->ev_start));
    CUDA_TRY(h, cudaEventCreate(&h->ev_stop));
    return MIND_OK;
}

int upload_group_state(MindHandle *h) {
    for (size_t g = 0; g < h->group_init.size(); ++g) {
        const auto &init = h->group_init[g];
        DevGroup &G = h->P.groups[g];
        if (G.gen >= 0) {
            for (size_t k = 0; k < init.f.size() && init.rows; ++k)
                CUDA_TRY(h, cudaMemcpyAsync(G.cols + k * (size_t)init.rows, init.f[k].data(), init.rows * sizeof(double),
                                            cudaMemcpyHostToDevice, h->stream));
            continue;
        }
        for (size_t k = 0; k < init.f.size(); ++k)
            if (G.f[k] && init.rows)
                CUDA_TRY(h, cudaMemcpyAsync(G.f[k], init.f[k].data(), init.rows * sizeof(double),
                                            cudaMemcpyHostToDevice, h->stream));
    }
    return MIND_OK;
}

int check_device_error(MindHandle *h) {
    int32_t code = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&code, h->P.error, sizeof code, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (code == 0) return MIND_OK;
    const char *what = code == MIND_ECAPACITY   ? "event ring, window inbox or spike record capacity exhausted"
                       : code == MIND_ESELFEVENT ? "invalid self-event delay or an event behind its delivery step"
                       : code == MIND_ESINGULAR  ? "singular or non-finite cable system"
                       : code == MIND_ENONFINITE ? "non-finite numerical state"
                       : code == MIND_ETIMEOUT   ? "a device wait ran out of time"
                                                 : "device error";
    return fail(h, code, what);
}

/* Where a reference's value lives.  `cell` is the cell whose window kernel records it
 * (-1: no cell, read only); `code`/`ptr` follow Params::rec_node/rec_ptr; `initial` points
 * at the value in HBM. */
struct RecordTarget {
    int32_t cell = -1;
    int32_t code = 0;
    const double *ptr = nullptr;
    const double *initial = nullptr;
};

int resolve_record(MindHandle *h, const MindRecord &rec, RecordTarget &out) {
    const Params &P = h->P;
    if (rec.kind == MIND_RECORD_VOLTAGE) {
        if (rec.node < 1 || rec.node > h->n_nodes) return fail(h, MIND_EARG, "record node out of range");
        const int64_t packed = h->packed_of_layout[rec.node - 1];
        out.cell = (int32_t)(std::upper_bound(h->node_off.begin(), h->node_off.end(), packed) -
                             h->node_off.begin() - 1);
        out.code = (int32_t)(packed - h->node_off[out.cell]);
        out.ptr = nullptr;
        out.initial = P.v + packed;
        return MIND_OK;
    }
    if (rec.kind != MIND_RECORD_MECHANISM) return fail(h, MIND_EARG, "unsupported record kind");
    const int32_t g = rec.group - 1;
    if (g < 0 || g >= P.ngroups) return fail(h, MIND_EARG, "mechanism group out of range");
    if (rec.row < 1 || rec.row > (int64_t)h->dev_row_of[g].size()) return fail(h, MIND_EARG, "mechanism row out of range");
    if (rec.field < 1 || rec.field > (int32_t)h->field_slot[g].size())
        return fail(h, MIND_EARG, "mechanism field out of range");
    const int slot = h->field_slot[g][rec.field - 1];
    if (slot < 0) return fail(h, MIND_EARG, "mechanism field is not kept on the device (ASSIGNED in BREAKPOINT)");
    const int32_t kind = h->group_init[g].kind;
    const int32_t dev = h->dev_row_of[g][rec.row - 1];
    out.initial = generated_kind(kind) ? P.groups[g].cols + (int64_t)slot * P.groups[g].rows + dev
                                       : P.groups[g].f[slot] + dev;
    if (kind == MIND_MECH_NETSTIM || kind == MIND_MECH_PATTERNSTIM) {
        out.cell = -1;   // artificial cells belong to no cell's window
        return MIND_OK;
    }
    const std::vector<int32_t> &off = h->group_row_off[g];
    out.cell = (int32_t)(std::upper_bound(off.begin(), off.end(), dev) - off.begin() - 1);
    const int32_t local = dev - off[out.cell];
    const int ss = staged_slot(kind, slot);
    if (ss >= 0 && local < (1 << 20)) {
        out.code = -1 - ((g << 24) | (ss << 20) | local);
        out.ptr = nullptr;
    } else if (ss >= 0) {
        return fail(h, MIND_EARG, "a recorded state row lies beyond 2^20 rows of its cell");
    } else {
        out.code = 0;
        out.ptr = out.initial;   // a parameter: constant through the run
    }
    return MIND_OK;
}

/* Per-cell record tables of a run: rec_off [ncells+1], then per entry (cell-sorted) its
 * code, HBM pointer and trace column; and per record its first-sample pointer. */
struct RecordTables {
    std::vector<int32_t> off, code, col;
    std::vector<const double *> ptr, initial;
};

int build_records(MindHandle *h, const MindRecord *records, int32_t nrec, RecordTables &t) {
    std::vector<std::vector<std::pair<RecordTarget, int32_t>>> by_cell(h->ncells);
    t.initial.assign(nrec, nullptr);
    for (int32_t k = 0; k < nrec; ++k) {
        RecordTarget target;
        int status = resolve_record(h, records[k], target);
        if (status) return status;
        if (target.cell < 0) return fail(h, MIND_EARG, "NetStim fields are read with mind_read_value, not recorded");
        t.initial[k] = target.initial;
        by_cell[target.cell].push_back({target, k});
    }
    t.off.assign(1, 0);
    for (int32_t c = 0; c < h->ncells; ++c) {
        for (auto &x : by_cell[c]) {
            t.code.push_back(x.first.code);
            t.ptr.push_back(x.first.ptr);
            t.col.push_back(x.second);
        }
        t.off.push_back((int32_t)t.code.size());
    }
    return MIND_OK;
}

/* Grows a device buffer to `count` elements without shrinking (contents not kept). */
template <class T>
T *grow(MindHandle *h, T *old, size_t &capacity, size_t count) {
    if (count <= capacity && old) return old;
    const size_t cap = std::max<size_t>(count, std::max<size_t>(64, capacity + capacity / 2));
    T *p = h->alloc<T>(cap);
    h->release(const_cast<void *>(static_cast<const void *>(old)));
    capacity = cap;
    return p;
}

/* The run's record maps on the device.  A run with the same records as the last one (the
 * usual case: a host records the same set every call) reuses the uploaded tables; a new set
 * is uploaded into buffers that only ever grow, so repeated runs allocate nothing. */
int set_records(MindHandle *h, const MindRecord *records, int32_t nrec, int64_t samples) {
    Params &P = h->P;
    const bool same = nrec == (int32_t)h->rec_last.size() &&
                      (nrec == 0 || std::memcmp(records, h->rec_last.data(), (size_t)nrec * sizeof(MindRecord)) == 0);
    if (!same || !h->rec_off_dev) {
        RecordTables t;
        int status = build_records(h, records, nrec, t);
        if (status) return status;
        const size_t n = std::max<size_t>(1, t.code.size());
        h->rec_off_dev = grow(h, h->rec_off_dev, h->rec_off_cap, t.off.size());
        h->rec_node_dev = grow(h, h->rec_node_dev, h->rec_capacity, n);
        size_t cap = h->rec_capacity;   // the per-entry tables share one capacity
        h->rec_col_dev = grow(h, h->rec_col_dev, h->rec_col_cap, cap);
        h->rec_ptr_dev = grow(h, h->rec_ptr_dev, h->rec_ptr_cap, cap);
        h->rec_initial_dev = grow(h, h->rec_initial_dev, h->rec_initial_cap, std::max<size_t>(1, t.initial.size()));
        CUDA_TRY(h, cudaMemcpyAsync(h->rec_off_dev, t.off.data(), t.off.size() * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, h->stream));
        if (!t.code.empty()) {
            CUDA_TRY(h, cudaMemcpyAsync(h->rec_node_dev, t.code.data(), t.code.size() * sizeof(int32_t),
                                        cudaMemcpyHostToDevice, h->stream));
            CUDA_TRY(h, cudaMemcpyAsync(h->rec_col_dev, t.col.data(), t.col.size() * sizeof(int32_t),
                                        cudaMemcpyHostToDevice, h->stream));
            CUDA_TRY(h, cudaMemcpyAsync(h->rec_ptr_dev, t.ptr.data(), t.ptr.size() * sizeof(const double *),
                                        cudaMemcpyHostToDevice, h->stream));
            CUDA_TRY(h, cudaMemcpyAsync(h->rec_initial_dev, t.initial.data(),
                                        t.initial.size() * sizeof(const double *), cudaMemcpyHostToDevice, h->stream));
        }
        // pageable sources: the copies above have consumed the host tables when they return
        h->rec_last.assign(records, records + nrec);
    }
    P.rec_off = h->rec_off_dev;
    P.rec_node = h->rec_node_dev;
    P.rec_ptr = h->rec_ptr_dev;
    P.rec_col = h->rec_col_dev;
    P.nrec = nrec;
    size_t need = (size_t)samples * (size_t)std::max(nrec, 1);
    if (nrec > 0 && need > h->trace_capacity) {
        h->release(h->trace_dev);
        h->trace_dev = nullptr;
        h->trace_dev = h->alloc<double>(need);
        h->trace_capacity = need;
    }
    P.trace = h->trace_dev;
    P.trace_samples = samples;
    return MIND_OK;
}

/* NCCL, opened at run time (libnccl.so.2, the one the process already has when torch loaded
 * it): the library needs only these five entry points, for the exchange between ranks. */
struct NcclApi {
    decltype(&ncclGetUniqueId) get_unique_id = nullptr;
    decltype(&ncclCommInitRank) comm_init_rank = nullptr;
    decltype(&ncclAllGather) all_gather = nullptr;
    decltype(&ncclCommDestroy) comm_destroy = nullptr;
    decltype(&ncclGetErrorString) error_string = nullptr;
};

const NcclApi *nccl() {
    static NcclApi api;
    static bool ok = false;
    static std::once_flag once;
    std::call_once(once, [] {
        void *lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!lib) return;
        api.get_unique_id = reinterpret_cast<decltype(api.get_unique_id)>(dlsym(lib, "ncclGetUniqueId"));
        api.comm_init_rank = reinterpret_cast<decltype(api.comm_init_rank)>(dlsym(lib, "ncclCommInitRank"));
        api.all_gather = reinterpret_cast<decltype(api.all_gather)>(dlsym(lib, "ncclAllGather"));
        api.comm_destroy = reinterpret_cast<decltype(api.comm_destroy)>(dlsym(lib, "ncclCommDestroy"));
        api.error_string = reinterpret_cast<decltype(api.error_string)>(dlsym(lib, "ncclGetErrorString"));
        ok = api.get_unique_id && api.comm_init_rank && api.all_gather && api.comm_destroy && api.error_string;
    });
    return ok ? &api : nullptr;
}

/* The window's exchange on the handle's stream: pack, all-gather (NCCL), inject. */
int exchange_window(MindHandle *h, int64_t window_end) {
    Params &P = h->P;
    exchange_pack_kernel<<<1, 256, 0, h->stream>>>(P, h->ex_sid_of_source, h->ex_send, h->ex_width);
    const size_t block = 1 + 2 * (size_t)h->ex_width;
    const ncclResult_t r = nccl()->all_gather(h->ex_send, h->ex_recv, block, ncclInt64, h->ex_comm, h->stream);
    if (r != ncclSuccess) return fail(h, MIND_ECUDA, std::string("ncclAllGather: ") + nccl()->error_string(r));
    const int64_t total = (int64_t)h->ex_world * h->ex_width;
    exchange_inject_kernel<<<launch_grid(std::max<int64_t>(total, 1)), kThreads, 0, h->stream>>>(
        P, h->ex_recv, h->ex_world, h->ex_width, h->ex_ext_sid, h->ex_ext_source, h->ex_n_ext, window_end);
    return MIND_OK;
}

/* One size bin's window-kernel launch in its chosen shape. */
template <bool MIXED>
void launch_window(const MindHandle *h, const MindHandle::Bin &bin, cudaStream_t s, const Params &P,
                   const int32_t *cells, int64_t n0, int32_t W) {
    constexpr int T = kCellThreads;
    const size_t smem = bin.smem_bytes;
    if (h->gen_runtime) {   // the same kernel from a module compiled at run time
        const void *k = (const void *)h->rt_window[MIXED ? 1 : 0][bin.global_image ? 1 : 0];
        void *args[] = {(void *)&P, (void *)&cells, (void *)&n0, (void *)&W};
        cudaLaunchKernel(k, dim3(bin.count), dim3(T), args, bin.global_image ? 0 : smem, s);
    } else if (h->has_generated) {   // mechanisms emitted from MOD files: the variant that runs them, 128 threads
        if (bin.global_image)
            window_kernel<MIXED, T, true, true><<<bin.count, T, 0, s>>>(P, cells, n0, W);
        else
            window_kernel<MIXED, T, false, true><<<bin.count, T, smem, s>>>(P, cells, n0, W);
    } else if (bin.global_image)
        window_kernel<MIXED, T, true><<<bin.count, T, 0, s>>>(P, cells, n0, W);
    else if (bin.threads == T && bin.tight && bin.paths)
        window_kernel<MIXED, T, false, false, kTightBlocks><<<bin.count, T, smem, s>>>(P, cells, n0, W);
    else if (bin.threads == T && bin.tight)
        window_kernel<MIXED, T, false, false, kTightBlocks, false><<<bin.count, T, smem, s>>>(P, cells, n0, W);
    else if (bin.threads == T && bin.paths)
        window_kernel<MIXED, T><<<bin.count, T, smem, s>>>(P, cells, n0, W);
    else if (bin.threads == T)
        window_kernel<MIXED, T, false, false, default_min_blocks(T), false><<<bin.count, T, smem, s>>>(P, cells, n0,
                                                                                                       W);
    else if (bin.threads == T / 2)
        window_kernel<MIXED, T / 2><<<bin.count, T / 2, smem, s>>>(P, cells, n0, W);
    else
        window_kernel<MIXED, T / 4><<<bin.count, T / 4, smem, s>>>(P, cells, n0, W);
}

/* The runtime's last-error slot is per thread and shared with the host's other CUDA code
 * (a framework's lazy initialisation can leave a benign error in it): the library's launch
 * checks must see only their own errors, so each entry that launches clears it first.  A
 * sticky error (a lost context) is not cleared by this and fails the next call. */
void clear_foreign_error() { (void)cudaGetLastError(); }

/* A named NVTX range for the lifetime of a scope: runs and their windows show up by name on
 * an Nsight timeline.  Without a profiler attached the calls do nothing. */
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

int advance(MindHandle *h, int64_t steps, bool record_spikes) {
    const NvtxRange run_range("mind run");
    clear_foreign_error();
    Params &P = h->P;
    P.record_spikes = record_spikes ? 1 : 0;
    P.run_start = h->step;
    CUDA_TRY(h, cudaMemsetAsync(P.rec_spike_count, 0, sizeof(int32_t), h->stream));
    if (P.nrec)
        record_initial_kernel<<<launch_grid(P.nrec), kThreads, 0, h->stream>>>(P, h->rec_initial_dev, P.nrec);
    CUDA_TRY(h, cudaEventRecord(h->ev_start, h->stream));
    int64_t n0 = h->step;
    const int64_t end = h->step + steps;
    const int ns_blocks = P.ns_group >= 0 ? launch_grid(P.groups[P.ns_group].rows) : 0;
    MindRunStats st{};
    st.window_steps = h->window;
    st.bins = (int32_t)h->bins.size();
    st.steps = steps;
    size_t prof_used = 0;
    auto prof_event = [&]() -> cudaEvent_t {
        if (prof_used == h->prof_events.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            h->prof_events.push_back(e);
        }
        return h->prof_events[prof_used++];
    };
    const MacroParams &M = h->M;
    if (M.n > 0 && M.trace) {
        macro_trace_start_kernel<<<1, h->macro_threads, 0, h->stream>>>(M, M.trace_k0);
        ++st.launches;
    }
    while (n0 < end) {
        const NvtxRange window_range("mind window");
        int32_t W = (int32_t)std::min<int64_t>(h->window, end - n0);
        // With regions attached, a window ends at the next rate-bin boundary at the latest,
        // so every bin the regions read is complete.
        if (M.n > 0) W = (int32_t)std::min<int64_t>(W, h->bin_steps - n0 % h->bin_steps);
        // NetStim self-events through the window's end boundary, as the reference's delivery
        // at the end of every step (time <= t + dt, src/runtime/step.jl:148): their spikes
        // enter this run's raster, their NetCon events the next window's bins
        const double horizon = (double)(n0 + W) * P.dt;
        if (M.n > 0) {
            const int64_t spm = M.steps_per_macro;
            const int64_t k0 = (n0 + spm - 1) / spm, k1 = (n0 + W + spm - 1) / spm;
            const int32_t zero_slot = n0 % h->bin_steps == 0 ? (int32_t)((n0 / h->bin_steps) % M.bin_ring) : -1;
            macro_advance_kernel<<<1, h->macro_threads, 0, h->stream>>>(M, k0, k1, zero_slot);
            ++st.launches;
            if (h->n_sur > 0 && n0 % h->bin_steps == 0) {
                // bin b starts: the surrogate cells' spikes of bin b from their last 20 bins
                const int64_t b = n0 / h->bin_steps;
                CUDA_TRY(h, cudaMemsetAsync(P.sur_drive + (b % kSurrogateRing) * (int64_t)h->ncells * 32, 0,
                                            (size_t)h->ncells * 32 * sizeof(float), h->stream));
                surrogate_features_kernel<<<launch_grid((int64_t)h->n_sur * 645), kThreads, 0, h->stream>>>(
                    P, h->sur_cells, h->n_sur, h->sur_spikes, h->sur_scale, b, h->sur_x);
                if (mind_mlp_forward_device(h->sur_mlp, h->sur_x, h->n_sur, h->sur_prob, h->stream, h->P.error))
                    return fail(h, MIND_ECUDA, "surrogate inference failed");
                surrogate_spike_kernel<<<launch_grid(h->n_sur), kThreads, 0, h->stream>>>(
                    P, h->sur_cells, h->sur_sources, h->n_sur, h->sur_prob, h->sur_offset, h->sur_spikes, b,
                    (double)h->bin_steps * P.dt, M.source_region, M.bins, M.n, M.bin_ring, n0);
                st.launches += 3;
            }
            if (k1 > k0 && M.n_inputs > 0) {
                macro_input_kernel<<<launch_grid(M.n_inputs), kThreads, 0, h->stream>>>(P, M, k0, k1, n0);
                ++st.launches;
            }
        }
        if (P.ns_group >= 0) {
            netstim_kernel<<<ns_blocks, kThreads, 0, h->stream>>>(P, horizon, n0);
            ++st.launches;
        }
        // Injected events whose bin falls in this window enter the ring now, in one launch
        // (the staging buffer was sized when they were injected).
        if (!h->injected.empty()) {
            if (!h->injected_sorted) {
                std::stable_sort(h->injected.begin(), h->injected.end(),
                                 [](const MindHandle::Injected &x, const MindHandle::Injected &y) { return x.bin < y.bin; });
                h->injected_sorted = true;
            }
            size_t due = 0;
            while (due < h->injected.size() && h->injected[due].bin < n0 + W) ++due;
            if (due > 0) {
                std::vector<InjectedEvent> batch(due);
                for (size_t k = 0; k < due; ++k) batch[k] = h->injected[k].event;
                cudaMemcpyAsync(h->inject_dev, batch.data(), due * sizeof(InjectedEvent), cudaMemcpyHostToDevice,
                                h->stream);
                inject_kernel<<<(unsigned)((due + kThreads - 1) / kThreads), kThreads, 0, h->stream>>>(
                    P, h->inject_dev, (int32_t)due, n0);
                ++st.launches;
                h->injected.erase(h->injected.begin(), h->injected.begin() + due);
            }
        }
        inbox_count_kernel<<<dim3(64, W), kThreads, 0, h->stream>>>(P, n0);
        inbox_scan_kernel<<<1, kScanThreads, 0, h->stream>>>(P);
        bucket_kernel<<<dim3(64, W), kThreads, 0, h->stream>>>(P, n0);
        st.launches += 3;
        // Size bins run side by side on their own streams so SMs mix CTAs of
        // different shared-memory images; the main stream joins them.
        if (h->profiling) cudaEventRecord(prof_event(), h->stream);
        cudaEventRecord(h->fork, h->stream);
        for (size_t b = 0; b < h->bins.size(); ++b) {
            const auto &bin = h->bins[b];
            cudaStream_t s = h->bin_streams[b];
            cudaStreamWaitEvent(s, h->fork, 0);
            const int32_t *cells = h->bin_cells + bin.first;
            if (h->precision == MIND_MIXED)
                launch_window<true>(h, bin, s, P, cells, n0, W);
            else
                launch_window<false>(h, bin, s, P, cells, n0, W);
            cudaEventRecord(h->bin_done[b], s);
            cudaStreamWaitEvent(h->stream, h->bin_done[b], 0);
            ++st.launches;
            ++st.window_launches;
        }
        if (h->profiling) cudaEventRecord(prof_event(), h->stream);
        route_kernel<<<64, kThreads, 0, h->stream>>>(P, n0 + W, M.source_region, M.bins, M.n, h->bin_steps,
                                                     M.bin_ring);
        ++st.launches;
        if (h->ex_comm) {   // the other ranks' spikes of this window
            const int status = exchange_window(h, n0 + W);
            if (status) return status;
            st.launches += 2;
        }
        n0 += W;
    }
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaEventRecord(h->ev_stop, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    float ms = 0.0f;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev_start, h->ev_stop));
    h->last_ms = ms;
    st.run_ms = ms;
    for (size_t k = 0; k + 1 < prof_used; k += 2) {
        float part = 0.0f;
        CUDA_TRY(h, cudaEventElapsedTime(&part, h->prof_events[k], h->prof_events[k + 1]));
        st.window_ms += part;
    }
    h->stats = st;
    h->step = end;
    return check_device_error(h);
}

/* Device buffer for the regions' outputs at the run's macro boundaries (mind_run only). */
int set_macro_trace(MindHandle *h, int64_t steps) {
    MacroParams &M = h->M;
    M.trace = nullptr;
    h->macro_trace_samples = 0;
    if (M.n == 0) return MIND_OK;
    const int64_t spm = M.steps_per_macro;
    const int64_t k0 = (h->step + spm - 1) / spm, k1 = (h->step + steps) / spm;
    const int64_t samples = std::max<int64_t>(0, k1 - k0 + 1);
    if (samples == 0) return MIND_OK;
    const size_t need = (size_t)samples * M.n;
    if (need > h->macro_trace_cap) {
        if (h->macro_trace_dev) h->release(h->macro_trace_dev);
        h->macro_trace_dev = nullptr;
        h->macro_trace_dev = h->alloc<double>(need);
        h->macro_trace_cap = need;
    }
    M.trace = h->macro_trace_dev;
    M.trace_k0 = k0;
    M.trace_samples = samples;
    h->macro_trace_samples = samples;
    return MIND_OK;
}

/* Zeroed device buffer for the run's synaptic drive bins, when recording is on (mind_run only). */
int set_drive(MindHandle *h, int64_t steps) {
    Params &P = h->P;
    P.drive = nullptr;
    h->drive_bins = 0;
    if (h->drive_bin_steps <= 0) return MIND_OK;
    const int64_t bins = steps / h->drive_bin_steps;
    if (bins == 0) return MIND_OK;
    const size_t need = (size_t)bins * h->ncells * 32;
    if (need > h->drive_cap) {
        if (h->drive_dev) h->release(h->drive_dev);
        h->drive_dev = nullptr;
        try {
            h->drive_dev = h->alloc<float>(need);
        } catch (const std::bad_alloc &) {
            return fail(h, MIND_ECAPACITY, "no device memory for the drive recording");
        }
        h->drive_cap = need;
    }
    CUDA_TRY(h, cudaMemsetAsync(h->drive_dev, 0, need * sizeof(float), h->stream));
    P.drive = h->drive_dev;
    P.drive_bin_steps = h->drive_bin_steps;
    P.drive_bins = bins;
    h->drive_bins = bins;
    return MIND_OK;
}

int collect_drive(MindHandle *h) {
    const size_t n = (size_t)h->drive_bins * h->ncells * 32;
    h->drive.assign(n, 0.0f);
    if (n) CUDA_TRY(h, cudaMemcpy(h->drive.data(), h->drive_dev, n * sizeof(float), cudaMemcpyDeviceToHost));
    return MIND_OK;
}

int collect_macro_trace(MindHandle *h) {
    const size_t n = (size_t)h->macro_trace_samples * h->M.n;
    h->macro_trace.assign(n, 0.0);
    if (n) CUDA_TRY(h, cudaMemcpy(h->macro_trace.data(), h->macro_trace_dev, n * sizeof(double), cudaMemcpyDeviceToHost));
    return MIND_OK;
}

int collect(MindHandle *h, bool record_spikes) {
    Params &P = h->P;
    h->spike_times.clear();
    h->spike_sids.clear();
    if (record_spikes) {
        int32_t count = 0;
        CUDA_TRY(h, cudaMemcpy(&count, P.rec_spike_count, sizeof count, cudaMemcpyDeviceToHost));
        count = std::min(count, P.rec_spike_cap);
        std::vector<int32_t> src(count);
        std::vector<double> t(count);
        if (count) {
            CUDA_TRY(h, cudaMemcpy(src.data(), P.rec_spike_source, count * sizeof(int32_t), cudaMemcpyDeviceToHost));
            CUDA_TRY(h, cudaMemcpy(t.data(), P.rec_spike_time, count * sizeof(double), cudaMemcpyDeviceToHost));
        }
        std::vector<int32_t> idx(count);
        for (int32_t i = 0; i < count; ++i) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](int32_t x, int32_t y) {
            if (t[x] != t[y]) return t[x] < t[y];
            if (h->source_ids[src[x]] != h->source_ids[src[y]]) return h->source_ids[src[x]] < h->source_ids[src[y]];
            return x < y;
        });
        h->spike_times.resize(count);
        h->spike_sids.resize(count);
        for (int32_t i = 0; i < count; ++i) {
            h->spike_times[i] = t[idx[i]];
            h->spike_sids[i] = h->source_ids[src[idx[i]]];
        }
    }
    // the traces stay in device memory until mind_get_trace copies them out (one copy)
    h->trace_records = P.nrec;
    h->trace_samples = P.nrec ? P.trace_samples : 0;
    h->trace_result = P.trace;
    return MIND_OK;
}

}  // namespace

extern "C" {

int mind_create(const MindLayout *layout, MindHandle **out) {
    if (!out) return MIND_EARG;
    *out = nullptr;
    MindHandle *h = nullptr;
    try {
        h = new MindHandle();
        int status = create(layout, h);
        if (status != MIND_OK) {
            g_create_error = h->error;
            delete h;
            return status;
        }
    } catch (const std::bad_alloc &) {
        g_create_error = "device or host allocation failed";
        delete h;
        return MIND_ECUDA;
    }
    *out = h;
    return MIND_OK;
}

int mind_set_precision(MindHandle *h, int32_t mode) {
    if (!h) return MIND_EARG;
    if (mode != MIND_FP64 && mode != MIND_MIXED) return fail(h, MIND_EARG, "unknown precision mode");
    h->precision = mode;
    return MIND_OK;
}

namespace {
int reserve_injected(MindHandle *h);
void push_injected(MindHandle *h, double time, int32_t edge, int32_t point);
}  // namespace

int mind_initialize(MindHandle *h) {
    if (!h) return MIND_EARG;
    Params &P = h->P;
    h->initialized = false;
    h->step = 0;
    h->injected.clear();
    h->injected_sorted = true;
    // PatternStim firings (src/runtime/utils/events.jl:92-110): each prescribed time is a
    // spike of the point's sources -- its raster entry and every NetCon event, queued now
    // and moved into the delivery ring by the window that delivers them
    for (const auto &ps : h->pattern) {
        push_injected(h, ps.time, -1, ps.source);
        for (int64_t e = h->fanout[ps.source]; e < h->fanout[ps.source + 1]; ++e)
            push_injected(h, ps.time + h->edge_delay[e], (int32_t)e, h->edge_target[e]);
    }
    if (!h->pattern.empty()) {
        const int status = reserve_injected(h);
        if (status) return status;
    }
    CUDA_TRY(h, cudaMemcpyAsync(P.v, h->v0_packed.data(), h->n_nodes * sizeof(double), cudaMemcpyHostToDevice,
                                h->stream));
    CUDA_TRY(h, cudaMemsetAsync(P.error, 0, sizeof(int32_t), h->stream));
    CUDA_TRY(h, cudaMemsetAsync(P.above, 0, std::max<int64_t>(1, h->n_sources), h->stream));
    CUDA_TRY(h, cudaMemsetAsync(P.ring_count, 0, P.ring_slots * sizeof(int32_t), h->stream));
    CUDA_TRY(h, cudaMemsetAsync(P.inbox_count, 0, std::max(1, h->ncells) * sizeof(int32_t), h->stream));
    CUDA_TRY(h, cudaMemsetAsync(P.inbox_fill, 0, std::max(1, h->ncells) * sizeof(int32_t), h->stream));
    CUDA_TRY(h, cudaMemsetAsync(P.win_spike_count, 0, sizeof(int32_t), h->stream));
    int status = upload_group_state(h);
    if (status) return status;
    for (int32_t g = 0; g < P.ngroups; ++g) {
        if (g == P.ns_group || P.groups[g].rows == 0) continue;
        if (h->gen_runtime && P.groups[g].gen >= 0) {   // INITIAL from the run-time module
            int32_t gg = g;
            void *args[] = {(void *)&P, (void *)&gg};
            CUDA_TRY(h, cudaLaunchKernel((const void *)h->rt_init, dim3(launch_grid(P.groups[g].rows)), dim3(kThreads),
                                         args, 0, h->stream));
            continue;
        }
        mechanism_init_kernel<<<launch_grid(P.groups[g].rows), kThreads, 0, h->stream>>>(P, g);
    }
    if (P.ns_group >= 0 && P.groups[P.ns_group].rows > 0)
        netstim_init_kernel<<<launch_grid(P.groups[P.ns_group].rows), kThreads, 0, h->stream>>>(
            P, h->group_init[P.ns_group].digest, h->ns_logical);
    if (h->M.n > 0) macro_init_kernel<<<1, h->macro_threads, 0, h->stream>>>(h->M, h->macro_y0);
    if (h->n_sur > 0) {
        CUDA_TRY(h, cudaMemsetAsync(P.sur_drive, 0, (size_t)kSurrogateRing * h->ncells * 32 * sizeof(float), h->stream));
        CUDA_TRY(h, cudaMemsetAsync(h->sur_spikes, 0, (size_t)6 * h->n_sur * sizeof(int32_t), h->stream));
    }
    CUDA_TRY(h, cudaGetLastError());
    status = check_device_error(h);
    if (status) return status;
    h->initialized = true;
    return MIND_OK;
}

int mind_attach_macro(MindHandle *h, const MindMacroLayout *L) {
    if (!h || !L) return MIND_EARG;
    if (h->M.n > 0) return fail(h, MIND_EARG, "regions are already attached");
    // the exchange fixed a window length all ranks share; regions would change it
    if (h->ex_world) return fail(h, MIND_EARG, "a handle with a spike exchange attached takes no regions");
    const int32_t n = L->n_regions;
    if (n < 1 || n > 1024) return fail(h, MIND_ELAYOUT, "region count must be in [1, 1024]");
    if (!L->params || !L->y0 || !L->micro_gain) return fail(h, MIND_ELAYOUT, "missing region arrays");
    const double spm_f = L->dt_macro / h->dt, mpb_f = L->bin_ms / L->dt_macro;
    const int32_t spm = (int32_t)std::llround(spm_f), mpb = (int32_t)std::llround(mpb_f);
    if (spm < 1 || std::fabs(spm_f - spm) > 1e-9 * spm || mpb < 1 || std::fabs(mpb_f - mpb) > 1e-9 * mpb)
        return fail(h, MIND_ELAYOUT, "dt_macro must be a multiple of dt and bin_ms of dt_macro");
    const int32_t bin_steps = spm * mpb;
    // Region inputs are planned per window on the device, like NetStims: only cell
    // detectors and the other external inputs bound the window.
    std::vector<uint8_t> is_input(h->n_sources, 0);
    for (int64_t q = 0; q < L->n_inputs; ++q)
        if (L->input_source[q] >= 1 && L->input_source[q] <= h->n_sources) is_input[L->input_source[q] - 1] = 1;
    double min_delay = INFINITY;
    for (int64_t s = 0; s < h->n_sources; ++s)
        if (h->source_detector[s] || (h->source_external[s] && !is_input[s]))
            for (int64_t e = h->fanout[s]; e < h->fanout[s + 1]; ++e) min_delay = std::min(min_delay, h->edge_delay[e]);
    const int32_t base_window = window_for_delay(min_delay, h->dt);
    // the window: the longest multiple of the macro step within the delay bound and the bin;
    // advance() also ends a window at every bin boundary, so none straddles one (config 4:
    // windows of 16, 16 and 8 steps per 40-step bin)
    const int32_t window = std::min(base_window, bin_steps) / spm * spm;
    if (window == 0)
        return fail(h, MIND_ELAYOUT, "the shortest NetCon delay out of a cell is shorter than a macro step");
    std::vector<int32_t> order(L->n_edges), in_off(n + 1, 0), e_src, e_delay;
    std::vector<double> e_gain;
    int32_t max_delay = 1;
    for (int64_t e = 0; e < L->n_edges; ++e) {
        if (L->edge_src[e] < 1 || L->edge_src[e] > n || L->edge_dst[e] < 1 || L->edge_dst[e] > n ||
            L->edge_delay[e] < 1 || !std::isfinite(L->edge_gain[e]))
            return fail(h, MIND_ELAYOUT, "region edge out of range (delays are >= 1 macro step)");
        order[e] = (int32_t)e;
        in_off[L->edge_dst[e]]++;
        max_delay = std::max(max_delay, L->edge_delay[e]);
    }
    for (int32_t i = 0; i < n; ++i) in_off[i + 1] += in_off[i];
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return L->edge_dst[x] < L->edge_dst[y]; });
    for (int32_t e : order) {
        e_src.push_back(L->edge_src[e] - 1);
        e_gain.push_back(L->edge_gain[e]);
        e_delay.push_back(L->edge_delay[e]);
    }
    std::vector<int32_t> inp_region(L->n_inputs), inp_source(L->n_inputs);
    std::vector<double> inp_scale(L->n_inputs);
    for (int64_t q = 0; q < L->n_inputs; ++q) {
        const int64_t s = L->input_source[q];
        if (L->input_region[q] < 1 || L->input_region[q] > n || s < 1 || s > h->n_sources || !h->source_external[s - 1])
            return fail(h, MIND_ELAYOUT, "region input must name a region and an external spike input");
        if (!(L->input_scale[q] >= 0.0)) return fail(h, MIND_ELAYOUT, "region input scale must be >= 0");
        inp_region[q] = L->input_region[q] - 1;
        inp_source[q] = (int32_t)(s - 1);
        inp_scale[q] = L->input_scale[q];
    }
    std::vector<int32_t> source_region(h->n_sources, -1);
    std::vector<double> cells(n, 0.0);
    for (int64_t q = 0; q < L->n_outputs; ++q) {
        const int64_t s = L->output_source[q];
        if (L->output_region[q] < 1 || L->output_region[q] > n || s < 1 || s > h->n_sources || !h->source_detector[s - 1] ||
            source_region[s - 1] >= 0)
            return fail(h, MIND_ELAYOUT, "region output must name a region and a detector source, once");
        source_region[s - 1] = L->output_region[q] - 1;
        cells[L->output_region[q] - 1] += 1.0;
    }
    for (int32_t i = 0; i < n; ++i)
        if (L->micro_gain[i] != 0.0 && cells[i] == 0.0)
            return fail(h, MIND_ELAYOUT, "a region with a micro gain has no detector sources");
    for (int32_t i = 0; i < n; ++i)
        if (cells[i] == 0.0) cells[i] = 1.0;   // rate of an empty population: 0 / 1
    try {
        MacroParams &M = h->M;
        M.steps_per_macro = spm;
        M.macro_per_bin = mpb;
        M.hist_cap = max_delay + 2;
        M.bin_ring = 4;
        M.dt_ms = L->dt_macro;
        M.dt_s = L->dt_macro * 1e-3;
        M.bin_s = L->bin_ms * 1e-3;
        M.seed = h->P.seed;
        M.par = h->upload(std::vector<double>(L->params, L->params + (size_t)n * 9));
        M.y = h->alloc<double>((size_t)n * 6);
        h->macro_y0 = h->upload(std::vector<double>(L->y0, L->y0 + (size_t)n * 6));
        M.micro_gain = h->upload(std::vector<double>(L->micro_gain, L->micro_gain + n));
        M.cells = h->upload(cells);
        M.hist = h->alloc<double>((size_t)M.hist_cap * n);
        M.bins = h->alloc<int32_t>((size_t)M.bin_ring * n);
        M.in_off = h->upload(in_off);
        M.e_src = h->upload(e_src);
        M.e_gain = h->upload(e_gain);
        M.e_delay = h->upload(e_delay);
        M.n_inputs = L->n_inputs;
        M.inp_region = h->upload(inp_region);
        M.inp_source = h->upload(inp_source);
        M.inp_scale = h->upload(inp_scale);
        M.source_region = h->upload(source_region);
        M.trace = nullptr;
        M.n = n;
    } catch (const std::bad_alloc &) {
        h->M.n = 0;
        return fail(h, MIND_ECUDA, "device allocation failed");
    }
    h->bin_steps = bin_steps;
    h->window = window;
    h->macro_threads = ((n + 31) / 32) * 32;
    h->initialized = false;
    return MIND_OK;
}

int mind_attach_surrogate(MindHandle *h, MindMlp *mlp, const uint8_t *surrogate_cells, float drive_scale) {
    if (!h || !mlp || !surrogate_cells) return MIND_EARG;
    if (h->M.n == 0) return fail(h, MIND_EARG, "attach regions first: the surrogate predicts their rate bins");
    if (h->n_sur > 0) return fail(h, MIND_EARG, "a surrogate is already attached");
    if (mind_mlp_inputs(mlp) != 645) return fail(h, MIND_EARG, "the surrogate network must take 645 inputs");
    std::vector<uint8_t> mode(h->ncells, 0);
    std::vector<int32_t> cells, sources;
    for (int32_t c = 0; c < h->ncells; ++c)
        if (surrogate_cells[c]) {
            mode[c] = 1;
            cells.push_back(c);
            sources.push_back(h->cell_detector[c]);
        }
    if (cells.empty()) return MIND_OK;
    if (mind_mlp_reserve_device(mlp, (int64_t)cells.size())) return fail(h, MIND_ECUDA, "surrogate buffers");
    try {
        h->P.cell_mode = h->upload(mode);
        h->P.sur_drive = h->alloc<float>((size_t)kSurrogateRing * h->ncells * 32);
        h->sur_cells = h->upload(cells);
        h->sur_sources = h->upload(sources);
        h->sur_spikes = h->alloc<int32_t>((size_t)6 * cells.size());
        h->sur_x = h->alloc<float>((size_t)645 * cells.size());
        h->sur_prob = h->alloc<float>(cells.size());
        h->sur_offset = h->upload(std::vector<float>(h->ncells, 0.0f));
    } catch (const std::bad_alloc &) {
        return fail(h, MIND_ECUDA, "device allocation failed");
    }
    h->P.sur_bin_steps = h->bin_steps;
    h->sur_mlp = mlp;
    h->sur_scale = drive_scale;
    h->n_sur = (int32_t)cells.size();
    h->sur_cap = h->n_sur;
    h->sur_attached = mode;
    h->initialized = false;
    return MIND_OK;
}

int mind_set_surrogate_offsets(MindHandle *h, const float *logit_offset, int32_t n_cells) {
    if (!h || !logit_offset) return MIND_EARG;
    if (h->sur_cap == 0) return fail(h, MIND_EARG, "no surrogate is attached");
    if (n_cells != h->ncells) return fail(h, MIND_EARG, "one offset per cell of the layout");
    for (int32_t c = 0; c < n_cells; ++c)
        if (!std::isfinite(logit_offset[c])) return fail(h, MIND_EARG, "offsets must be finite");
    CUDA_TRY(h, cudaMemcpyAsync(h->sur_offset, logit_offset, (size_t)n_cells * sizeof(float), cudaMemcpyHostToDevice,
                                h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return MIND_OK;
}

int mind_set_surrogate_cells(MindHandle *h, const uint8_t *surrogate_cells) {
    if (!h || !surrogate_cells) return MIND_EARG;
    if (h->sur_cap == 0) return fail(h, MIND_EARG, "no surrogate is attached");
    for (int32_t c = 0; c < h->ncells; ++c)
        if (surrogate_cells[c] && !h->sur_attached[c])
            return fail(h, MIND_EARG, "only cells named when the surrogate was attached can be surrogate cells");
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    std::vector<int32_t> old_cells(h->n_sur), old_spikes((size_t)6 * h->n_sur);
    if (h->n_sur) {
        CUDA_TRY(h, cudaMemcpy(old_cells.data(), h->sur_cells, old_cells.size() * sizeof(int32_t),
                               cudaMemcpyDeviceToHost));
        CUDA_TRY(h, cudaMemcpy(old_spikes.data(), h->sur_spikes, old_spikes.size() * sizeof(int32_t),
                               cudaMemcpyDeviceToHost));
    }
    std::vector<int32_t> where(h->ncells, -1);
    for (int32_t i = 0; i < h->n_sur; ++i) where[old_cells[i]] = i;
    std::vector<uint8_t> mode(h->ncells, 0);
    std::vector<int32_t> cells, sources;
    for (int32_t c = 0; c < h->ncells; ++c)
        if (surrogate_cells[c]) {
            mode[c] = 1;
            cells.push_back(c);
            sources.push_back(h->cell_detector[c]);
        }
    const int32_t n = (int32_t)cells.size();
    // the last bins' own spikes (features of the next bins) follow each cell to its new slot
    std::vector<int32_t> spikes((size_t)6 * n, 0);
    for (int32_t i = 0; i < n; ++i)
        if (where[cells[i]] >= 0)
            for (int32_t k = 0; k < 6; ++k) spikes[(size_t)k * n + i] = old_spikes[(size_t)k * h->n_sur + where[cells[i]]];
    CUDA_TRY(h, cudaMemcpy(const_cast<uint8_t *>(h->P.cell_mode), mode.data(), mode.size(), cudaMemcpyHostToDevice));
    if (n) {
        CUDA_TRY(h, cudaMemcpy(h->sur_cells, cells.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(h->sur_sources, sources.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(h->sur_spikes, spikes.data(), spikes.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    }
    h->n_sur = n;
    return MIND_OK;
}

int mind_set_drive_recording(MindHandle *h, double bin_ms) {
    if (!h) return MIND_EARG;
    if (bin_ms <= 0.0) {
        h->drive_bin_steps = 0;
        return MIND_OK;
    }
    const double k = bin_ms / h->dt;
    const int32_t steps = (int32_t)std::llround(k);
    if (steps < 1 || std::fabs(k - steps) > 1e-9 * steps) return fail(h, MIND_EARG, "bin_ms must be a multiple of dt");
    h->drive_bin_steps = steps;
    return MIND_OK;
}

int mind_get_drive(const MindHandle *h, float *out, int64_t n, int64_t *bins) {
    if (!h) return MIND_EARG;
    if (bins) *bins = h->drive_bins;
    if (n == 0) return MIND_OK;
    if (n != (int64_t)h->drive.size() || !out) return MIND_EARG;
    std::memcpy(out, h->drive.data(), n * sizeof(float));
    return MIND_OK;
}

int mind_get_macro_trace(const MindHandle *h, double *out, int64_t n, int64_t *samples) {
    if (!h) return MIND_EARG;
    if (samples) *samples = h->macro_trace_samples;
    if (n == 0) return MIND_OK;
    if (n != (int64_t)h->macro_trace.size() || !out) return MIND_EARG;
    std::memcpy(out, h->macro_trace.data(), n * sizeof(double));
    return MIND_OK;
}

int mind_run(MindHandle *h, int64_t steps, const MindRecord *records, int32_t n_records, int32_t record_spikes) {
    if (!h) return MIND_EARG;
    if (!h->initialized) return fail(h, MIND_EARG, "simulation is not initialized");
    if (steps < 0 || n_records < 0 || (n_records > 0 && !records)) return fail(h, MIND_EARG, "invalid run arguments");
    int status = set_records(h, records, n_records, steps + 1);
    if (status) return status;
    status = set_macro_trace(h, steps);
    if (status) return status;
    status = set_drive(h, steps);
    if (status) return status;
    status = advance(h, steps, record_spikes != 0);
    h->M.trace = nullptr;
    h->P.drive = nullptr;
    if (status) {
        h->initialized = false;
        return status;
    }
    status = collect(h, record_spikes != 0);
    if (status) return status;
    status = collect_macro_trace(h);
    if (status) return status;
    return collect_drive(h);
}

int mind_step(MindHandle *h) {
    if (!h) return MIND_EARG;
    if (!h->initialized) return fail(h, MIND_EARG, "simulation is not initialized");
    int status = set_records(h, nullptr, 0, 2);
    if (status) return status;
    status = advance(h, 1, false);
    if (status) h->initialized = false;
    return status;
}

int mind_time(const MindHandle *h, int64_t *step, double *time) {
    if (!h) return MIND_EARG;
    if (step) *step = h->step;
    if (time) *time = (double)h->step * h->dt;
    return MIND_OK;
}

int mind_get_trace(const MindHandle *h, double *out, int64_t n) {
    if (!h) return MIND_EARG;
    if (n != h->trace_samples * (int64_t)h->trace_records || (n && !out)) return MIND_EARG;
    if (n && cudaMemcpy(out, h->trace_result, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return MIND_ECUDA;
    return MIND_OK;
}

int mind_get_trace_by_record(MindHandle *h, double *out, int64_t n) {
    if (!h) return MIND_EARG;
    const int64_t samples = h->trace_samples, records = h->trace_records;
    if (n != samples * records || (n && !out)) return MIND_EARG;
    if (n == 0) return MIND_OK;
    if ((size_t)n > h->trace_by_record_cap) {
        h->release(h->trace_by_record);
        h->trace_by_record = nullptr;
        h->trace_by_record_cap = 0;
        try {
            h->trace_by_record = h->alloc<double>((size_t)n);
        } catch (const std::bad_alloc &) {
            return fail(h, MIND_ECUDA, "device allocation failed");
        }
        h->trace_by_record_cap = (size_t)n;
    }
    const dim3 g((unsigned)((samples + 31) / 32), (unsigned)((records + 31) / 32));
    trace_transpose_kernel<<<g, dim3(32, 8), 0, h->stream>>>(h->trace_result, h->trace_by_record, samples,
                                                             (int32_t)records);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaMemcpyAsync(out, h->trace_by_record, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                                h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return MIND_OK;
}

int mind_get_spikes(const MindHandle *h, double *times, int64_t *sids, int64_t cap, int64_t *n) {
    if (!h || !n) return MIND_EARG;
    *n = (int64_t)h->spike_times.size();
    int64_t m = std::min<int64_t>(cap, *n);
    if (m > 0) {
        if (!times || !sids) return MIND_EARG;
        std::memcpy(times, h->spike_times.data(), m * sizeof(double));
        std::memcpy(sids, h->spike_sids.data(), m * sizeof(int64_t));
    }
    return MIND_OK;
}

int mind_read_voltage(const MindHandle *h, int32_t node, double *value) {
    if (!h || !value) return MIND_EARG;
    if (node < 1 || node > h->n_nodes) return MIND_EARG;
    cudaError_t e = cudaMemcpy(value, h->P.v + h->packed_of_layout[node - 1], sizeof(double), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? MIND_OK : MIND_ECUDA;
}

int mind_read_value(const MindHandle *h, const MindRecord *ref, double *value) {
    if (!h || !ref || !value) return MIND_EARG;
    MindHandle *mh = const_cast<MindHandle *>(h);   // only the error text changes
    RecordTarget target;
    int status = resolve_record(mh, *ref, target);
    if (status) return status;
    // The handle's stream is idle between calls; the device state is the completed boundary.
    cudaError_t e = cudaMemcpy(value, target.initial, sizeof(double), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? MIND_OK : cuda_fail(mh, e, "mind_read_value");
}

namespace {

/* Grows the staging buffer so that every pending injected event fits one window's batch;
 * allocation happens here, at injection, never inside a run. */
int reserve_injected(MindHandle *h) {
    if (h->injected.size() <= h->inject_cap) return MIND_OK;
    const size_t cap = std::max<size_t>(h->injected.size(), std::max<size_t>(1024, 2 * h->inject_cap));
    void *p = nullptr;
    CUDA_TRY(h, cudaMalloc(&p, cap * sizeof(InjectedEvent)));
    if (h->inject_dev) {
        cudaStreamSynchronize(h->stream);
        h->release(h->inject_dev);
    }
    h->buffers.owned.push_back(p);
    h->inject_dev = static_cast<InjectedEvent *>(p);
    h->inject_cap = cap;
    return MIND_OK;
}

/* The step whose end-of-step delivery (time <= (m + 1) dt, src/runtime/step.jl:148) reaches
 * `time`: the smallest m >= 0 with time <= (m + 1) dt.  A spike's raster entry is recorded by
 * the window of that step, as the reference records it when that delivery pops it. */
int64_t record_step(double time, double dt) {
    double estimate = std::ceil(time / dt) - 1.0;
    int64_t m = estimate < 0.0 ? 0 : (int64_t)estimate;
    for (int k = 0; k < 4 && m > 0 && time <= (double)m * dt; ++k) --m;
    for (int k = 0; k < 4 && time > (double)(m + 1) * dt; ++k) ++m;
    return m;
}

void push_injected(MindHandle *h, double time, int32_t edge, int32_t point) {
    MindHandle::Injected e;
    // a NetCon event waits for the step that delivers it; a raster entry (edge < 0) for the
    // step whose end delivery covers its time
    e.bin = edge >= 0 ? delivery_bin(time, h->dt) : record_step(time, h->dt);
    e.event.time = time;
    e.event.edge = edge;
    e.event.point = point;
    if (!h->injected.empty() && h->injected.back().bin > e.bin) h->injected_sorted = false;
    h->injected.push_back(e);
}

}  // namespace

int mind_inject_event(MindHandle *h, int64_t edge, double t) {
    if (!h) return MIND_EARG;
    if (!h->initialized) return fail(h, MIND_EARG, "simulation is not initialized");
    if (edge < 1 || edge > (int64_t)h->edge_target.size()) return fail(h, MIND_EARG, "edge index out of range");
    if (!(t >= (double)h->step * h->dt) || !std::isfinite(t)) return fail(h, MIND_EARG, "event time is in the past");
    push_injected(h, t, (int32_t)(edge - 1), h->edge_target[edge - 1]);
    return reserve_injected(h);
}

int mind_inject_spikes(MindHandle *h, int64_t n, const int64_t *sources, const double *times) {
    if (!h) return MIND_EARG;
    if (!h->initialized) return fail(h, MIND_EARG, "simulation is not initialized");
    if (n < 0 || (n > 0 && (!sources || !times))) return fail(h, MIND_EARG, "invalid spike list");
    const double now = (double)h->step * h->dt;
    for (int64_t k = 0; k < n; ++k) {
        const int64_t s = sources[k];
        if (s < 1 || s > h->n_sources || !h->source_external[s - 1])
            return fail(h, MIND_EARG, "source " + std::to_string(s) + " is not an external spike input");
        if (!std::isfinite(times[k])) return fail(h, MIND_EARG, "spike time is not finite");
        if (times[k] < now)
            for (int64_t e = h->fanout[s - 1]; e < h->fanout[s]; ++e)
                if (delivery_bin(times[k] + h->edge_delay[e], h->dt) < h->step)
                    return fail(h, MIND_EARG, "spike time precedes the current time by more than its NetCon delays");
    }
    for (int64_t k = 0; k < n; ++k) {
        const int64_t s = sources[k] - 1;
        const double t = times[k];
        if (t >= now) push_injected(h, t, -1, (int32_t)s);  // the raster entry, in the window of its time
        for (int64_t e = h->fanout[s]; e < h->fanout[s + 1]; ++e)
            push_injected(h, t + h->edge_delay[e], (int32_t)e, h->edge_target[e]);
    }
    return reserve_injected(h);
}

namespace {

/* Device time (ms) of `windows` windows from a fresh initialize, after one untimed window. */
int trial_ms(MindHandle *h, int32_t windows, double *ms) {
    int status = mind_initialize(h);
    if (status) return status;
    status = mind_run(h, h->window, nullptr, 0, 0);
    if (status) return status;
    status = mind_run(h, (int64_t)h->window * windows, nullptr, 0, 0);
    if (status) return status;
    *ms = h->last_ms;
    return MIND_OK;
}

}  // namespace

int mind_autotune(MindHandle *h, int32_t windows) {
    if (!h) return MIND_EARG;
    if (!h->initialized || h->step != 0) return fail(h, MIND_EARG, "autotune needs a handle initialized at step 0");
    if (windows < 0) return fail(h, MIND_EARG, "negative trial window count");
    if (windows == 0) windows = 4;
    double best = 0.0;
    int status = trial_ms(h, windows, &best);
    if (status) return status;
    // launch shapes: 128 threads at either register bound, 64, one warp
    const std::pair<int32_t, bool> shapes[4] = {
        {kCellThreads, false}, {kCellThreads, true}, {kCellThreads / 2, false}, {kCellThreads / 4, false}};
    for (auto &bin : h->bins) {
        if (bin.global_image || h->has_generated) continue;   // HBM images and emitted mechanisms: 128 threads
        const std::pair<int32_t, bool> keep{bin.threads, bin.tight};
        for (const auto &shape : shapes) {
            if (shape == keep || shape.first < bin.max_detectors) continue;   // one detector per thread
            const std::pair<int32_t, bool> before{bin.threads, bin.tight};
            bin.threads = shape.first;
            bin.tight = shape.second;
            double ms = 0.0;
            status = trial_ms(h, windows, &ms);
            if (status) {
                bin.threads = keep.first;
                bin.tight = keep.second;
                return status;
            }
            if (ms < 0.98 * best) {
                best = ms;
            } else {
                bin.threads = before.first;
                bin.tight = before.second;
            }
        }
    }
    return mind_initialize(h);
}

int mind_bin_threads(const MindHandle *h, int32_t *threads, int32_t cap, int32_t *n_bins) {
    if (!h || !n_bins || cap < 0 || (cap > 0 && !threads)) return MIND_EARG;
    *n_bins = (int32_t)h->bins.size();
    for (int32_t b = 0; b < cap && b < *n_bins; ++b) threads[b] = h->bins[b].threads;
    return MIND_OK;
}

int mind_set_bin_threads(MindHandle *h, const int32_t *threads, int32_t n_bins) {
    if (!h || !threads || n_bins != (int32_t)h->bins.size()) return MIND_EARG;
    for (int32_t b = 0; b < n_bins; ++b) {
        if (!valid_cell_threads(threads[b]))
            return fail(h, MIND_EARG, "a bin runs 128, 64 or 32 threads per cell");
        if (threads[b] < h->bins[b].max_detectors)
            return fail(h, MIND_EARG, "a bin's cells have more detectors than its CTA has threads");
        if ((h->bins[b].global_image || h->has_generated) && threads[b] != kCellThreads)
            return fail(h, MIND_EARG, "cells with their image in HBM, and models with emitted mechanisms, run 128 threads");
    }
    for (int32_t b = 0; b < n_bins; ++b) {
        MindHandle::Bin &bin = h->bins[b];
        bin.threads = threads[b];
        bin.tight = threads[b] == kCellThreads && !bin.global_image && tight_by_default(bin.smem_bytes);
    }
    return MIND_OK;
}

int mind_window_steps(const MindHandle *h, int32_t *steps) {
    if (!h || !steps) return MIND_EARG;
    *steps = h->window;
    return MIND_OK;
}

int mind_mechanism_count(int32_t *n) {
    if (!n) return MIND_EARG;
    GenRegistry &g = gen_registry();
    std::lock_guard<std::mutex> lock(g.mu);
    *n = (int32_t)g.entries.size();
    return MIND_OK;
}

int mind_mechanism_info(int32_t index, MindMechanismInfo *info) {
    if (!info || index < 0) return MIND_EARG;
    const GenEntry *g = gen_entry(MIND_MECH_GENERATED + index);
    if (!g) return MIND_EARG;
    info->name = g->name.c_str();
    info->kind = MIND_MECH_GENERATED + index;
    info->point = g->point;
    info->net_receive = g->net_receive;
    info->n_fields = (int32_t)g->fields.size();
    info->field_names = g->field_ptrs.data();
    info->defaults = g->defaults.data();
    info->digest = g->digest;
    info->ion_reads = g->ion_reads.c_str();
    return MIND_OK;
}

int mind_mechanism_kind(const char *name, int32_t *kind) {
    if (!name || !kind) return MIND_EARG;
    GenRegistry &g = gen_registry();
    std::lock_guard<std::mutex> lock(g.mu);
    for (size_t k = 0; k < g.entries.size(); ++k)
        if (g.entries[k]->name == name) {
            *kind = MIND_MECH_GENERATED + (int32_t)k;
            return MIND_OK;
        }
    return MIND_EARG;
}

int mind_load_mechanisms(const char *module_path, const MindMechanismInfo *mechanisms, int32_t n) {
    if (!module_path || n < 0 || (n > 0 && !mechanisms)) return MIND_EARG;
    GenRegistry &g = gen_registry();
    std::lock_guard<std::mutex> lock(g.mu);
    const size_t have = g.entries.size() - (size_t)kGeneratedCount;
    if ((size_t)n < have) {
        g_create_error = "a mechanism module must hold every mechanism registered before it";
        return MIND_EARG;
    }
    for (int32_t k = 0; k < n; ++k) {
        const MindMechanismInfo &m = mechanisms[k];
        if (!m.name || m.n_fields < 0 || (m.n_fields > 0 && (!m.field_names || !m.defaults))) {
            g_create_error = "mechanism description incomplete";
            return MIND_EARG;
        }
        if ((size_t)k < have) {
            const GenEntry &e = *g.entries[kGeneratedCount + k];
            if (e.name != m.name || e.digest != m.digest) {
                g_create_error = std::string("mechanism ") + m.name + " differs from the one registered at its index";
                return MIND_EARG;
            }
        } else {
            for (auto &e : g.entries)
                if (e->name == m.name) {
                    g_create_error = std::string("a mechanism named ") + m.name + " is already known";
                    return MIND_EARG;
                }
        }
    }
    cudaLibrary_t lib = nullptr;
    cudaError_t err = cudaLibraryLoadFromFile(&lib, module_path, nullptr, nullptr, 0, nullptr, nullptr, 0);
    cudaKernel_t k[5] = {};
    const char *names[5] = {"mind_rt_window_fp64", "mind_rt_window_fp64_hbm", "mind_rt_window_mixed",
                            "mind_rt_window_mixed_hbm", "mind_rt_generated_init"};
    for (int q = 0; err == cudaSuccess && q < 5; ++q) err = cudaLibraryGetKernel(&k[q], lib, names[q]);
    if (err != cudaSuccess) {
        g_create_error = std::string("mechanism module ") + module_path + ": " + cudaGetErrorString(err);
        return MIND_ECUDA;
    }
    for (int32_t q = (int32_t)have; q < n; ++q) {
        const MindMechanismInfo &m = mechanisms[q];
        auto e = std::make_unique<GenEntry>();
        e->name = m.name;
        e->point = m.point;
        e->net_receive = m.net_receive;
        for (int32_t f = 0; f < m.n_fields; ++f) {
            e->fields.push_back(m.field_names[f] ? m.field_names[f] : "");
            e->defaults.push_back(m.defaults[f]);
        }
        for (auto &f : e->fields) e->field_ptrs.push_back(f.c_str());
        e->digest = m.digest;
        e->ion_reads = m.ion_reads ? m.ion_reads : "";
        g.entries.push_back(std::move(e));
    }
    g.window[0][0] = k[0];
    g.window[0][1] = k[1];
    g.window[1][0] = k[2];
    g.window[1][1] = k[3];
    g.init = k[4];
    return MIND_OK;
}

const char *mind_last_error(const MindHandle *h) {
    if (!h) return g_create_error.c_str();
    return h->error.c_str();
}

int mind_last_run_ms(const MindHandle *h, double *ms) {
    if (!h || !ms) return MIND_EARG;
    *ms = h->last_ms;
    return MIND_OK;
}

int mind_run_stats(const MindHandle *h, MindRunStats *stats) {
    if (!h || !stats) return MIND_EARG;
    *stats = h->stats;
    return MIND_OK;
}

int mind_set_profiling(MindHandle *h, int32_t enable) {
    if (!h) return MIND_EARG;
    h->profiling = enable != 0;
    return MIND_OK;
}

/* ---- run! without device allocation (see include/mindgpu.h) ---- */

namespace {

// The per-run scratch of mind_run_noalloc: record maps and trace staging.
static __device__ __align__(256) unsigned char g_noalloc_scratch[MIND_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_address[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device, looked up once per device.
int noalloc_scratch(MindHandle *h, unsigned char **out) {
    int device = 0;
    CUDA_TRY(h, cudaGetDevice(&device));
    if (device < 0 || device >= kMaxDevices) return fail(h, MIND_EARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_address[device] == nullptr) {
        void *ptr = nullptr;
        CUDA_TRY(h, cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        g_noalloc_address[device] = ptr;
    }
    *out = static_cast<unsigned char *>(g_noalloc_address[device]);
    return MIND_OK;
}

}  // namespace

int mind_run_noalloc(MindHandle *h, int64_t steps, const MindRecord *records, int32_t n_records, double *trace) {
    if (!h) return MIND_EARG;
    if (!h->initialized) return fail(h, MIND_EARG, "simulation is not initialized");
    if (steps < 0 || n_records < 0 || (n_records > 0 && (!records || !trace)))
        return fail(h, MIND_EARG, "invalid run arguments");
    {
        int device = -1;
        CUDA_TRY(h, cudaGetDevice(&device));
        if (device != h->device)
            return fail(h, MIND_EARG, "mind_run_noalloc called with device " + std::to_string(device) +
                                          " current; the handle lives on device " + std::to_string(h->device));
    }
    // Scratch carve: rec_off [ncells+1] i32 | rec_node [n] i32 | rec_col [n] i32 | rec_ptr [n] ptr |
    // rec_initial [n] ptr | trace.
    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t off_bytes = align((size_t)(h->ncells + 1) * sizeof(int32_t));
    const size_t node_bytes = align((size_t)std::max(n_records, 1) * sizeof(int32_t));
    const size_t ptr_bytes = align((size_t)std::max(n_records, 1) * sizeof(const double *));
    const size_t fixed = off_bytes + 2 * node_bytes + 2 * ptr_bytes;
    // The trace holds (steps + 1) samples of n_records doubles.  The sample count is bounded
    // by division before anything is multiplied, so no product can wrap.
    const size_t room = fixed < MIND_NOALLOC_SCRATCH_BYTES ? MIND_NOALLOC_SCRATCH_BYTES - fixed : 0;
    const size_t max_samples = n_records > 0 ? room / ((size_t)n_records * sizeof(double)) : (size_t)INT64_MAX;
    if (fixed > MIND_NOALLOC_SCRATCH_BYTES || (uint64_t)steps >= (uint64_t)max_samples) {
        // Refused before any work: the simulation state is unchanged and stays usable.
        h->error = "mind_run_noalloc: " + std::to_string(steps) + " steps of " + std::to_string(n_records) +
                   " records need more scratch than its static array holds (" +
                   std::to_string((size_t)MIND_NOALLOC_SCRATCH_BYTES) + " bytes, at most " +
                   std::to_string(max_samples > 0 ? max_samples - 1 : 0) +
                   " steps per call at this record count); use fewer steps or records per call";
        return MIND_ECAPACITY;
    }
    const size_t trace_bytes = (size_t)(steps + 1) * (size_t)n_records * sizeof(double);
    // Record maps (host side), then into the scratch: every entry is written, nothing needs clearing.
    RecordTables t;
    int status = build_records(h, records, n_records, t);
    if (status) return status;
    unsigned char *scratch = nullptr;
    status = noalloc_scratch(h, &scratch);
    if (status) return status;
    int32_t *d_off = reinterpret_cast<int32_t *>(scratch);
    int32_t *d_node = reinterpret_cast<int32_t *>(scratch + off_bytes);
    int32_t *d_col = reinterpret_cast<int32_t *>(scratch + off_bytes + node_bytes);
    const double **d_ptr = reinterpret_cast<const double **>(scratch + off_bytes + 2 * node_bytes);
    const double **d_initial = reinterpret_cast<const double **>(scratch + off_bytes + 2 * node_bytes + ptr_bytes);
    double *d_trace = reinterpret_cast<double *>(scratch + off_bytes + 2 * node_bytes + 2 * ptr_bytes);
    CUDA_TRY(h, cudaMemcpyAsync(d_off, t.off.data(), t.off.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                h->stream));
    if (n_records) {
        CUDA_TRY(h, cudaMemcpyAsync(d_node, t.code.data(), t.code.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                    h->stream));
        CUDA_TRY(h, cudaMemcpyAsync(d_col, t.col.data(), t.col.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                    h->stream));
        CUDA_TRY(h, cudaMemcpyAsync(d_ptr, t.ptr.data(), t.ptr.size() * sizeof(const double *),
                                    cudaMemcpyHostToDevice, h->stream));
        CUDA_TRY(h, cudaMemcpyAsync(d_initial, t.initial.data(), t.initial.size() * sizeof(const double *),
                                    cudaMemcpyHostToDevice, h->stream));
    }
    // Point the run at the scratch for this call only; the handle's own record fields are
    // restored on every return, so no later call can record into the shared array.
    Params &P = h->P;
    const Params own = P;
    const double **own_initial = h->rec_initial_dev;
    auto restore = [&]() {
        P.rec_off = own.rec_off;
        P.rec_node = own.rec_node;
        P.rec_ptr = own.rec_ptr;
        P.rec_col = own.rec_col;
        P.nrec = own.nrec;
        P.trace = own.trace;
        P.trace_samples = own.trace_samples;
        h->rec_initial_dev = own_initial;
    };
    P.rec_off = d_off;
    P.rec_node = d_node;
    P.rec_ptr = d_ptr;
    P.rec_col = d_col;
    P.nrec = n_records;
    P.trace = d_trace;
    P.trace_samples = steps + 1;
    h->rec_initial_dev = d_initial;
    status = advance(h, steps, false);
    restore();
    if (status) {
        h->initialized = false;
        return status;
    }
    if (trace_bytes)
        CUDA_TRY(h, cudaMemcpyAsync(trace, d_trace, trace_bytes, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return MIND_OK;
}

int mind_exchange_id(uint8_t id[128]) {
    if (!id) return MIND_EARG;
    const NcclApi *api = nccl();
    if (!api) return MIND_ECUDA;
    ncclUniqueId u;
    if (api->get_unique_id(&u) != ncclSuccess) return MIND_ECUDA;
    static_assert(sizeof(u) == 128, "NCCL unique id of 128 bytes");
    std::memcpy(id, &u, sizeof u);
    return MIND_OK;
}

int mind_attach_exchange(MindHandle *h, const uint8_t *nccl_id, int32_t world, int32_t rank, int32_t window,
                         int32_t width, const int32_t *detector_sources, const int32_t *detector_sids,
                         int32_t n_detectors, const int32_t *external_sids, const int32_t *external_sources,
                         int32_t n_external) {
    if (!h || world < 1 || rank < 0 || rank >= world || window < 1 || width < 1 || n_detectors < 0 ||
        n_external < 0 || (n_detectors > 0 && (!detector_sources || !detector_sids)) ||
        (n_external > 0 && (!external_sids || !external_sources)))
        return MIND_EARG;
    if (h->ex_world) return fail(h, MIND_EARG, "an exchange is already attached");
    if (h->M.n > 0) return fail(h, MIND_EARG, "a handle with regions attached runs on one GPU");
    if ((int64_t)world * (1 + 2 * (int64_t)width) > (int64_t)1 << 31) return fail(h, MIND_EARG, "exchange too wide");
    std::vector<int32_t> sid_of_source(std::max<int64_t>(h->n_sources, 1), -1);
    for (int32_t k = 0; k < n_detectors; ++k) {
        const int32_t src = detector_sources[k];
        if (src < 0 || src >= h->n_sources || !h->source_detector[src] || detector_sids[k] < 0)
            return fail(h, MIND_EARG, "an exchanged detector must be a detector source with a sid >= 0");
        sid_of_source[src] = detector_sids[k];
    }
    std::vector<std::pair<int32_t, int32_t>> ext(n_external);
    for (int32_t k = 0; k < n_external; ++k) {
        const int32_t src = external_sources[k];
        if (src < 0 || src >= h->n_sources || !h->source_external[src])
            return fail(h, MIND_EARG, "a received sid must map to an external spike input");
        ext[k] = {external_sids[k], src};
    }
    std::sort(ext.begin(), ext.end());
    for (int32_t k = 1; k < n_external; ++k)
        if (ext[k].first == ext[k - 1].first) return fail(h, MIND_EARG, "a sid is received by one source");
    std::vector<int32_t> ext_sid(std::max(n_external, 1), -1), ext_source(std::max(n_external, 1), -1);
    for (int32_t k = 0; k < n_external; ++k) {
        ext_sid[k] = ext[k].first;
        ext_source[k] = ext[k].second;
    }
    try {
        h->ex_sid_of_source = h->upload(sid_of_source);
        h->ex_ext_sid = h->upload(ext_sid);
        h->ex_ext_source = h->upload(ext_source);
        h->ex_send = h->alloc<int64_t>(1 + 2 * (size_t)width);
        h->ex_recv = h->alloc<int64_t>((size_t)world * (1 + 2 * (size_t)width));
    } catch (const std::bad_alloc &) {
        return fail(h, MIND_ECUDA, "device allocation failed");
    }
    if (nccl_id) {
        const NcclApi *api = nccl();
        if (!api) return fail(h, MIND_ECUDA, "libnccl.so.2 could not be opened");
        ncclUniqueId u;
        std::memcpy(&u, nccl_id, sizeof u);
        const ncclResult_t r = api->comm_init_rank(&h->ex_comm, world, u, rank);
        if (r != ncclSuccess) {
            h->ex_comm = nullptr;
            return fail(h, MIND_ECUDA, std::string("ncclCommInitRank: ") + api->error_string(r));
        }
    }
    h->ex_world = world;
    h->ex_rank = rank;
    h->ex_width = width;
    h->ex_n_ext = n_external;
    h->window = std::min(h->window, window);
    return MIND_OK;
}

int mind_exchange_pack(MindHandle *h, int64_t *send) {
    if (!h || !send) return MIND_EARG;
    if (!h->ex_world) return fail(h, MIND_EARG, "no exchange is attached");
    clear_foreign_error();
    exchange_pack_kernel<<<1, 256, 0, h->stream>>>(h->P, h->ex_sid_of_source, send, h->ex_width);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return check_device_error(h);
}

int mind_exchange_inject(MindHandle *h, const int64_t *recv) {
    if (!h || !recv) return MIND_EARG;
    if (!h->ex_world) return fail(h, MIND_EARG, "no exchange is attached");
    clear_foreign_error();
    const int64_t total = (int64_t)h->ex_world * h->ex_width;
    exchange_inject_kernel<<<launch_grid(std::max<int64_t>(total, 1)), kThreads, 0, h->stream>>>(
        h->P, recv, h->ex_world, h->ex_width, h->ex_ext_sid, h->ex_ext_source, h->ex_n_ext, h->step);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return check_device_error(h);
}

int mind_destroy(MindHandle *h) {
    if (!h) return MIND_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->ex_comm && nccl()) nccl()->comm_destroy(h->ex_comm);
    for (cudaEvent_t e : h->prof_events) cudaEventDestroy(e);
    for (cudaEvent_t e : h->bin_done) cudaEventDestroy(e);
    for (cudaStream_t s : h->bin_streams) cudaStreamDestroy(s);
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->ev_start) cudaEventDestroy(h->ev_start);
    if (h->ev_stop) cudaEventDestroy(h->ev_stop);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return MIND_OK;
}

}  // extern "C"
