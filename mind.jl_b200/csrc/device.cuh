/*
 * device.cuh — device-side data layout and kernels of libmindgpu.so.
 *
 * Layout in HBM (built by mindgpu.cu from the C-ABI layout):
 *   - Nodes are packed cell by cell.  Inside a cell, nodes are grouped into
 *     chains (maximal unbranched paths: every node but the chain's top is the
 *     only child of its parent), chains sorted by level (0 = ends in a leaf,
 *     otherwise 1 + the highest level among its child chains), each chain's
 *     nodes contiguous from top to bottom.  A cell is staged in shared memory
 *     once per window of steps.
 *   - Mechanism rows are structure-of-arrays per group, sorted by
 *     (cell, owner thread = local node mod 64, local node, layout row): a cell
 *     owns one contiguous row range per group, each thread of its CTA one
 *     sub-range, and rows on one node are adjacent (a "segment").
 *   - Events live in a ring of delivery bins (bin m = the events NEURON's two
 *     half-step deliveries hand to step m's currents, i.e. event times in
 *     ((m-1) dt + dt/2, m dt + dt/2]).  Before a window, the bins of the
 *     window are moved into a per-window CSR of per-cell inboxes (count, scan,
 *     fill: any number of events per cell); the cell sorts its inbox by
 *     (bin, target, time, edge) and applies it in that order, which is the
 *     heap order of the reference (src/runtime/utils/events.jl:7-62) for every
 *     target.
 *
 * Arithmetic order in FP64 mode is the oracle's (oracle/mind_oracle.cpp):
 * group order, row order inside a segment, own axial term before children,
 * children in ascending layout index.  The file is compiled with -fmad=false
 * so that no multiply-add is fused behind the source's back; the fused
 * multiply-adds it does contain are explicit and exact (mind_div_milli).
 */
#pragma once

#include <cstdint>
#include "mind_math.h"
#include "../../include/mindgpu.h"
#ifdef MIND_RUNTIME_MECHANISMS
// a mechanism module compiled at run time: the compiled-in mechanisms and those after them
#include "runtime_mechanisms.cuh"
#else
#include "generated_mechanisms.cuh"
#endif

namespace mind {

constexpr int kMaxGroups = 16;
constexpr int kThreads = 128;      // auxiliary kernels
constexpr int kCellThreads = 128;  // window kernel: one cell per CTA of four warps
// A 128-thread window launch whose cells need little shared memory can keep more CTAs per SM
// than its registers allow at the default bound (5): the tight variant is compiled for 7.
constexpr int kTightBlocks = 7;
// CTAs per SM a launch shape is compiled for by default (its __launch_bounds__): 5 at 128
// threads per cell, 10 at 64, 16 at one warp.
constexpr int default_min_blocks(int threads) {
    return threads == kCellThreads ? 5 : threads == kCellThreads / 2 ? 10 : 16;
}
constexpr int kSurrogateRing = 21;  // drive bins kept for the surrogate: the last 20 and the current


struct RingEvent {       // an event waiting in a delivery bin
    double time;
    int32_t edge;        // 0-based edge, -1 for an injected event without weight
    int32_t point;       // 0-based point
};

struct InjectedEvent {
    double time;
    int32_t edge;   // 0-based edge, or -1 for the raster entry of an external spike input
    int32_t point;  // 0-based target point, or the 0-based source for a raster entry
};
struct InboxEvent {      // an event moved to its cell's window inbox
    double time;
    int32_t edge;
    int32_t point;
    int64_t bin;
};

struct DevGroup {
    int32_t kind;
    int32_t rows;
    const int32_t *row_off;   // [ncells+1] per-cell row ranges
    int32_t *node;            // local node per row
    int32_t *seg;             // rows in the segment starting here (0 = not a segment head)
    double *f[12];            // field arrays, meaning by kind (see mindgpu.cu)
    float *s[4];              // FP32 decay factors of the synapses (mixed mode)
    // mechanisms emitted from MOD files (kind MIND_MECH_GENERATED + gen): their fields as
    // ncols columns of `cols` (column k of row r at cols[k * rows + r]), then one column of
    // current scale (area * 0.01 for density mechanisms, 1 for point processes)
    double *cols;
    int32_t ncols;
    int32_t gen;              // index into kGenMechanisms, -1 for the hand-written kinds
};

__host__ __device__ inline bool kind_generated(int32_t kind) {
    return kind >= MIND_MECH_GENERATED && kind < MIND_MECH_GENERATED + kGeneratedCount;
}

/* Field slots per kind. */
enum { HH_GNABAR, HH_GKBAR, HH_GL, HH_EL, HH_ENA, HH_EK, HH_SCALE, HH_M, HH_H, HH_N, HH_NSLOT };
enum { PAS_G, PAS_E, PAS_SCALE, PAS_NSLOT };
enum { ES_E, ES_G, ES_TAU, ES_DECAY, ES_NSLOT };
enum { E2_E, E2_A, E2_B, E2_FACTOR, E2_TAU1, E2_TAU2, E2_DECAY1, E2_DECAY2, E2_NSLOT };
enum { IC_DEL, IC_DUR, IC_AMP, IC_NSLOT };
enum { AS_ONSET, AS_TAU, AS_GMAX, AS_E, AS_NSLOT };
enum { NS_INTERVAL, NS_NUMBER, NS_START, NS_NOISE, NS_EVENT, NS_ON, NS_ISPIKE, NS_NEXT_T,
       NS_NEXT_FLAG, NS_NSLOT };
/* FP32 parameter slots (mixed mode). */
enum { ESS_DECAY };
enum { E2S_DECAY1, E2S_DECAY2 };

/* Number of FP64 slots and FP32 (mixed-mode) parameter slots of each kind. */
__host__ __device__ inline int kind_slots(int32_t kind) {
    switch (kind) {
        case MIND_MECH_HH: return HH_NSLOT;
        case MIND_MECH_PAS: return PAS_NSLOT;
        case MIND_MECH_EXPSYN: return ES_NSLOT;
        case MIND_MECH_EXP2SYN: return E2_NSLOT;
        case MIND_MECH_ICLAMP: return IC_NSLOT;
        case MIND_MECH_ALPHASYN: return AS_NSLOT;
        case MIND_MECH_NETSTIM: return NS_NSLOT;
        default: return 0;
    }
}
/*
 * Rows whose state changes every step keep that state in shared memory for the
 * window; everything else of a row (parameters, decay factors) is streamed
 * from HBM.  hh rows are few per cell and keep all their slots on chip.
 *   staged_doubles  FP64 slots staged per row: hh all, ExpSyn g, Exp2Syn A,B.  State is
 *                   FP64 in both modes; the mixed mode computes hh's rates and the
 *                   synapses' per-step decrements in FP32 and accumulates them in FP64.
 */
__host__ __device__ inline bool kind_staged(int32_t kind) {
    return kind == MIND_MECH_HH || kind == MIND_MECH_EXPSYN || kind == MIND_MECH_EXP2SYN;
}
__host__ __device__ inline int staged_doubles(int32_t kind) {
    switch (kind) {
        case MIND_MECH_HH: return HH_NSLOT;
        case MIND_MECH_EXPSYN: return 1;
        case MIND_MECH_EXP2SYN: return 2;
        default: return 0;
    }
}

/*
 * Shared-memory image of one cell for a window (all sizes in elements):
 *   doubles  v, d, rhs, a [n each]; eliminated pivot and rhs contributions of
 *            chain tops [nch each]; event increments [inbox_cap]; staged FP64
 *            slots of the staged rows;
 *   events   the cell's inbox for the window [inbox_cap];
 *   ints     per staged row: local node; chain top, length,
 *            parent, child-chain CSR; level starts; path starts; inbox
 *            order; the threads' row ranges per group [ngroups][threads + 1];
 *   shorts   chain of every node [n].
 * Host (to size the launch) and device (to carve the buffer) use this one function.
 */
struct CellShape {
    int32_t n, nch, nkids, nlev, npath;
    int32_t rows[kMaxGroups];
};

__host__ __device__ inline size_t cell_smem_bytes(const CellShape &s, const int32_t *kinds, int32_t ngroups,
                                                  int32_t inbox_cap) {
    size_t doubles = 4 * (size_t)s.n + 2 * (size_t)s.nch + (size_t)inbox_cap;
    size_t ints = 0;
    for (int32_t g = 0; g < ngroups; ++g) {
        if (!kind_staged(kinds[g])) continue;
        doubles += (size_t)staged_doubles(kinds[g]) * s.rows[g];
        ints += (size_t)s.rows[g];
    }
    ints += 4 * (size_t)s.nch + 1 + (size_t)s.nkids + (size_t)s.nlev + 1 + (size_t)s.npath + 1 + (size_t)inbox_cap;
    ints += (size_t)ngroups * (kCellThreads + 1);
    return doubles * 8 + (size_t)inbox_cap * sizeof(InboxEvent) + ints * 4 + 2 * (size_t)s.n;
}

struct Params {
    int32_t ncells;
    int32_t ngroups;
    double dt;
    double celsius;
    double vscale;             // v += vscale * increment: 1 (secondorder 0), 2 (secondorder 1, 2)
    uint64_t seed;
    // nodes (packed, local order)
    const int64_t *node_off;   // [ncells+1]
    double *v;
    const double *a, *cdt, *ad;
    // mixed mode: C/dt + axial_diagonal + pas conductance, pas conductance, and it times e
    const double *mix_dc, *mix_gs, *mix_gse;
    const int32_t *parent;     // [packed] local parent index or -1
    const int32_t *kid_off;    // [packed+1] CSR into kids (children in ascending layout index)
    const int32_t *kids;       // local child indices
    // chains
    const int32_t *chain_off;  // [ncells+1]
    const int32_t *chain_top, *chain_len, *chain_par, *chain_kid_off, *chain_kids;  // chain_kid_off global CSR
    // paths: a chain, or a chain and the child chains it continues into, eliminated by one
    // thread in one level (chains of a path contiguous, deepest first; paths sorted by level)
    const int32_t *level_off;    // [ncells+1] into level_path
    const int32_t *level_path;   // per cell: nlevels+1 local path starts
    const int32_t *path_off;     // [ncells+1] into path_chain
    const int32_t *path_chain;   // per cell: npaths+1 local chain starts; only the sentinel for a
                                 // cell on the chain schedule (its paths are its chains)
    DevGroup groups[kMaxGroups];
    // per cell, group and thread: first row (relative to the cell's first row of the group)
    // of the thread's rows; thread t owns the local nodes i with i % kCellThreads == t
    const int32_t *part;       // [ncells][ngroups][kCellThreads + 1]
    // cells whose image exceeds a CTA's shared memory keep it in HBM: slot big_slot[c] of
    // big_image, big_stride bytes each (big_slot -1 for the others)
    unsigned char *big_image;
    const int32_t *big_slot;
    int64_t big_stride;
    // detectors
    const int32_t *det_off;    // [ncells+1]
    const int32_t *det_node;   // local node
    const int32_t *det_source; // 0-based source
    const double *det_thr;
    uint8_t *above;            // per source
    // window spikes (cell detectors)
    int32_t *win_spike_source;
    int64_t *win_spike_step;
    int32_t *win_spike_count;
    int32_t win_spike_cap;
    // recorded spikes
    int32_t *rec_spike_source;
    double *rec_spike_time;
    int32_t *rec_spike_count;
    int32_t rec_spike_cap;
    int32_t record_spikes;
    // events
    RingEvent *ring;
    int32_t *ring_count;
    int32_t ring_slots;
    int32_t ring_cap;
    // the window's events by cell, a CSR rebuilt every window: cell c's events are
    // inbox[inbox_start[c] .. inbox_start[c+1]); a cell stages up to inbox_cap of them in
    // shared memory and sorts more in place in HBM (inbox_order), so no cell has a limit
    // of its own -- only the window's total (inbox_total) and each delivery bin (ring_cap)
    InboxEvent *inbox;
    int32_t *inbox_order;          // sorted order of a cell's events when they are not staged
    int32_t *inbox_count;          // [ncells] events per cell (first pass), zeroed by the cell's window
    int32_t *inbox_fill;           // [ncells] events placed (second pass), zeroed by the cell's window
    int32_t *inbox_start;          // [ncells+1] exclusive prefix sum of inbox_count
    int32_t inbox_cap;             // events staged in shared memory per cell
    int32_t inbox_total;           // capacity of inbox and inbox_order
    const double *edge_weight;
    const double *edge_delay;
    const int32_t *edge_target;    // 0-based point
    const int64_t *fanout_off;     // [nsources+1] 0-based
    const int32_t *point_cell;     // per point
    const int32_t *point_group;    // per point, 0-based
    const int32_t *point_row;      // per point, device row
    // NetStim
    int32_t ns_group;              // -1 if none
    MindRan *ns_ran;
    const int32_t *ns_source;      // per NetStim row: 0-based source or -1
    // recording
    const int32_t *rec_off;        // [ncells+1]
    // per record of the cell: rec_ptr non-null reads that HBM value (a constant parameter);
    // else rec_node >= 0 is a local node's v and rec_node < 0 a staged field,
    // -1 - rec_node = group << 24 | staged slot << 20 | row within the cell's rows
    const int32_t *rec_node;
    const double *const *rec_ptr;
    const int32_t *rec_col;
    double *trace;
    // cells the surrogate stands in for (null: none) and their drive ring [kSurrogateRing][ncells][32]
    const uint8_t *cell_mode;
    float *sur_drive;
    int32_t sur_bin_steps;
    // surrogate training data: synaptic drive [drive_bins][ncells][32] of the run (or null)
    float *drive;
    int32_t drive_bin_steps;
    int64_t drive_bins;
    int32_t nrec;
    int64_t trace_samples;
    int64_t run_start;             // step at sample 0
    int32_t *error;
};

}  // namespace mind
