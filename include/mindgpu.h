/*
 * mindgpu.h — C-ABI of libmindgpu.so, the B200 implementation of MIND.jl's
 * per-micro-timestep simulation loop.
 *
 * The library sits where MIND.jl's runtime sits today: behind build!() the Julia
 * host owns a packed, immutable ModelLayout (src/model/build.jl:101-115) and the
 * runtime uploads it, runs INITIAL and steps it.  Every entry point below
 * replaces one runtime seam of the reference:
 *
 *   mind_create       allocate_simulation(plan::ModelLayout)   src/runtime/initialize.jl:4-250
 *   mind_initialize   initialize!(state)                       src/runtime/initialize.jl:270-429
 *   mind_run          run!(state, stop; records, ...)          src/runtime/step.jl:4-74
 *   mind_step         step!(state)                             src/runtime/step.jl:77-86
 *   mind_get_trace    SimulationResult.traces                  src/runtime/recording.jl:256-295
 *   mind_get_spikes   SimulationResult.spike_times/_sources    src/runtime/recording.jl:256-295
 *   mind_read_voltage read_value(voltage_ref)                  src/runtime/state.jl:586-659
 *   mind_inject_event inject_event!(state, connection, time)   src/runtime/state.jl:586-659
 *   mind_inject_spikes inject_spike!(state, source, time)      src/runtime/state.jl:637-659
 *   mind_destroy      release of SimulationState               src/runtime/state.jl:177-212
 *
 * Conventions follow the Julia side so that its arrays pass without copies:
 * indices are 1-based (0 = none), mechanism data is column-major
 * data[row, field] (src/model/utils/build.jl:96-101), times are ms, voltages mV,
 * point currents nA, density currents mA/cm2, weights uS.
 *
 * Ownership: every pointer in MindLayout is read during mind_create only; the
 * library copies what it needs into device memory it owns and frees at
 * mind_destroy.  Outputs go to caller-provided host buffers.  A handle is
 * not reentrant: one handle per host thread, as the reference keeps one
 * SimulationState per Julia task (src/runtime/utils/step.jl:201-211).
 *
 * Status codes keep the reference's device error word
 * (src/runtime/utils/step.jl:190-196) and add codes for conditions the
 * library reports itself.  Any non-zero status from mind_run / mind_step
 * leaves the handle uninitialized, as run! does (src/runtime/step.jl:67-70).
 */
#ifndef MINDGPU_H
#define MINDGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MIND_ABI_VERSION 2

/* Status codes. 3/5/6/8 are the reference's error-word codes. */
enum {
    MIND_OK = 0,
    MIND_ECAPACITY = 3,   /* event ring, window inbox or spike record exhausted */
    MIND_ESELFEVENT = 5,  /* invalid self-event delay or target */
    MIND_ESINGULAR = 6,   /* zero or non-finite pivot in the cable solve */
    MIND_ENONFINITE = 8,  /* non-finite voltage or mechanism state */
    MIND_ETIMEOUT = 9,    /* a device wait exceeded its iteration budget */
    MIND_ELAYOUT = 10,    /* layout rejected (unsupported mechanism, bad index, ...) */
    MIND_ECUDA = 11,      /* CUDA runtime error; see mind_last_error */
    MIND_EARG = 12        /* invalid argument or call order */
};

/* Numerical modes (mind_set_precision). */
enum {
    MIND_FP64 = 0,   /* everything in FP64; reproduces the FP64 oracle bit for bit */
    MIND_MIXED = 1   /* FP32 gating and synaptic conductances; FP64 cable, voltage, clock */
};

/* Builtin mechanism kinds understood by the device kernels (the reference mod directory). */
enum {
    MIND_MECH_HH = 1,       /* mod/hh.mod       density  */
    MIND_MECH_PAS = 2,      /* mod/pas.mod      density  */
    MIND_MECH_EXPSYN = 3,   /* mod/ExpSyn.mod   point    */
    MIND_MECH_EXP2SYN = 4,  /* mod/Exp2Syn.mod  point    */
    MIND_MECH_NETSTIM = 5,  /* mod/NetStim.mod  artificial */
    MIND_MECH_ICLAMP = 6,   /* mod/IClamp.mod   point (electrode current) */
    MIND_MECH_ALPHASYN = 7, /* mod/AlphaSynapse.mod point: g = gmax alpha((t-onset)/tau), i = g (v-e) */
    MIND_MECH_PATTERNSTIM = 8, /* mod/PatternStim.mod artificial: fires at prescribed times (MindLayout.pattern_*) */
    /* MIND_MECH_GENERATED + k: the k-th mechanism whose CUDA C was emitted from a MOD file
     * (BREAKPOINT, DERIVATIVE by cnexp, PROCEDURE by after_cvode, NET_RECEIVE, INITIAL) and
     * compiled into this library; mind_mechanism_info lists them with their fields. */
    MIND_MECH_GENERATED = 64
};

/*
 * One mechanism group: the reference's MechanismPlan (src/model/build.jl:1-60)
 * restricted to what the hot path reads.  Group order is significant: when
 * several groups write the same node, their currents are accumulated in group
 * order, and rows of one group in row order.
 */
typedef struct MindMechanism {
    int32_t kind;                      /* MIND_MECH_* */
    int32_t n_fields;                  /* columns of data */
    int64_t rows;
    const double *data;                /* column-major [rows x n_fields] initial values */
    const char *const *field_names;    /* n_fields names, the MOD's own field names */
    const int32_t *nodes;              /* [rows] 1-based node; 0 for artificial cells */
    const uint64_t *logical_ids;       /* [rows] random-stream identity (micro/model.jl:510-530) */
    uint64_t digest;                   /* first 16 hex digits of the MOD source SHA-256 */
} MindMechanism;

/*
 * The packed micro layout: a POD view of ModelLayout.micro (MicroPlan,
 * src/model/build.jl:15-60) plus the build! settings the step loop reads.
 * Nodes may come in any order that forms a forest through `parent`
 * (the reference passes its DHS permutation, src/model/micro/model.jl:989-1077);
 * where the numerical result depends on an order (siblings eliminated into
 * one parent, point processes on one node) the order is ascending index.
 */
typedef struct MindLayout {
    int32_t abi_version;               /* MIND_ABI_VERSION */
    int32_t secondorder;               /* build!(secondorder=): 0 backward Euler; 1 and 2 Crank-Nicolson
                                          (C/(dt/2) in the cable matrix, v += 2 x) */
    int64_t n_nodes;
    const int32_t *parent;             /* [n_nodes] 1-based, 0 = root */
    const double *voltage;             /* [n_nodes] initial membrane voltage (mV) */
    const double *area;                /* [n_nodes] um2 */
    const double *capacitance;         /* [n_nodes] cm*area*1e-5 */
    const double *axial;               /* [n_nodes] conductance to parent (uS) */
    const double *axial_diagonal;      /* [n_nodes] sum of own and children's axial */

    int32_t n_mechanisms;
    const MindMechanism *mechanisms;

    int64_t n_points;                  /* point processes and artificial cells */
    const int32_t *point_group;        /* [n_points] 1-based mechanism index */
    const int32_t *point_row;          /* [n_points] 1-based row in that group */

    int64_t n_sources;                 /* spike sources (micro/model.jl:590-600) */
    const int64_t *source_ids;         /* [n_sources] user-visible sid */
    const int32_t *source_nodes;       /* [n_sources] 1-based detector node, 0 if event source */
    const double *source_thresholds;   /* [n_sources] detector threshold (mV) */
    const int32_t *source_points;      /* [n_sources] 1-based point whose net_event feeds it, 0 if none */

    int64_t n_edges;                   /* NetCons, grouped by source (micro/model.jl:638-671) */
    const int64_t *fanout_offsets;     /* [n_sources+1] 1-based CSR into the edge arrays */
    const int32_t *edge_targets;       /* [n_edges] 1-based point index */
    const double *edge_delays;         /* [n_edges] ms */
    const double *edge_weights;        /* [n_edges] first NET_RECEIVE weight (uS) */

    double dt;                         /* dt_micro (ms) */
    double celsius;
    uint64_t seed;                     /* build!(seed=) : Philox key */
    int64_t event_capacity;            /* events per delivery bin (ring slot) */
    int64_t spike_capacity;            /* recorded spikes per run */

    /* PatternStim spike times (add_pointprocess!(...; spike_times), micro/model.jl:586-613),
     * sorted by time (stable): at every mind_initialize each time becomes a firing of the
     * spike sources fed by that PatternStim point (src/runtime/utils/events.jl:92-110) --
     * recorded in the raster and routed through their NetCons. */
    int64_t n_pattern;
    const double *pattern_times;       /* [n_pattern] ms, >= 0 */
    const int32_t *pattern_points;     /* [n_pattern] 1-based point (a PatternStim) */
} MindLayout;

/*
 * A recorded or read quantity: RecordSpec / VariableRef (src/model/references.jl:4-80)
 * for the :voltage and :mechanism kinds.  A mechanism reference names a layout column
 * (MindMechanism.data) of one row; the columns kept on the device are the PARAMETER and
 * STATE fields the kernels use:
 *   hh       gnabar gkbar gl el ena ek m h n
 *   pas      g e
 *   ExpSyn   tau e g
 *   Exp2Syn  tau1 tau2 e A B factor
 *   IClamp   del dur amp
 *   AlphaSynapse  onset tau gmax e
 *   NetStim  interval number start noise event on ispike   (mind_read_value only)
 * ASSIGNED fields that the reference writes during BREAKPOINT (hh ina/gna/minf/..., pas
 * i, ExpSyn i, Exp2Syn g/i, IClamp i) are not kept: referencing one returns MIND_EARG.
 * A recorded mechanism field is sampled at the same boundaries as voltages.
 */
enum { MIND_RECORD_VOLTAGE = 1, MIND_RECORD_MECHANISM = 2 };
typedef struct MindRecord {
    int32_t kind;                      /* MIND_RECORD_VOLTAGE or MIND_RECORD_MECHANISM */
    int32_t node;                      /* VOLTAGE: 1-based node */
    int32_t group;                     /* MECHANISM: 1-based mechanism group (MindLayout.mechanisms) */
    int32_t row;                       /* MECHANISM: 1-based row of that group */
    int32_t field;                     /* MECHANISM: 1-based column of the group's data */
} MindRecord;

typedef struct MindHandle MindHandle;

/* allocate_simulation: validate and pack the layout onto the current device. */
int mind_create(const MindLayout *layout, MindHandle **out);

/* initialize!: reset clocks, queues and detectors; run INITIAL blocks. */
int mind_initialize(MindHandle *h);

/* mind_set_precision: MIND_FP64 (default) or MIND_MIXED; takes effect at the next mind_initialize. */
int mind_set_precision(MindHandle *h, int32_t mode);

/*
 * run!: advance `steps` micro steps, recording `records` at the starting
 * boundary and after every step (steps+1 samples) and, when record_spikes is
 * non-zero, every spike.  Results stay in the handle until the next run.
 */
int mind_run(MindHandle *h, int64_t steps, const MindRecord *records, int32_t n_records,
             int32_t record_spikes);

/* step!: one micro step without recording. */
int mind_step(MindHandle *h);

/* Current micro step count and simulation time (step * dt). */
int mind_time(const MindHandle *h, int64_t *step, double *time);

/* Traces of the last mind_run, sample-major [samples x n_records]; n must equal that size. */
int mind_get_trace(const MindHandle *h, double *out, int64_t n);
/* The same traces record-major [n_records x samples] (one record's samples contiguous, the
 * layout of SimulationResult's per-record vectors), transposed on the device before the copy. */
int mind_get_trace_by_record(MindHandle *h, double *out, int64_t n);

/* Spikes of the last mind_run, sorted by (time, sid); *n receives the count (also when cap is short). */
int mind_get_spikes(const MindHandle *h, double *times, int64_t *sids, int64_t cap, int64_t *n);

/* read_value for a voltage reference: v at a 1-based node. */
int mind_read_voltage(const MindHandle *h, int32_t node, double *value);

/* read_value (src/runtime/state.jl:585-599): the current value of a voltage or mechanism
 * reference (MindRecord); MIND_EARG for an index out of range or a field not kept. */
int mind_read_value(const MindHandle *h, const MindRecord *ref, double *value);

/* inject_event!: deliver connection `edge` (1-based) at absolute time t (ms, >= now). */
int mind_inject_event(MindHandle *h, int64_t edge, double t);

/* inject_spike! for n spikes: each external spike input sources[k] (a 1-based source with
 * neither a detector node nor a point, created by register_spike_source!(model; sid))
 * fires at absolute time times[k] (ms).  Every outgoing NetCon delivers at times[k] + its
 * delay.  A spike at or after the current time also enters the raster of the run that
 * reaches it.  A spike before the current time (one that a cell simulated elsewhere, on
 * another GPU, fired during the last window) is accepted when each of its NetCons still
 * delivers at or after the current step; it is routed but not recorded here.  Returns
 * MIND_EARG, with nothing queued, for any other source or a delivery in the past. */
int mind_inject_spikes(MindHandle *h, int64_t n, const int64_t *sources, const double *times);

/*
 * mind_autotune: the launch shape of each cell-size bin.  A bin's cells run one per CTA of
 * 128 threads (kCellThreads), 64 threads or one warp of 32 (each thread serving 1, 2 or 4
 * owner slots, so the arithmetic and its order are the same); smaller CTAs let more cells
 * share an SM (by registers and shared memory) at the price of longer parallel phases.  The
 * 128-thread launch comes compiled for two register budgets: the default, and a tight one
 * that lets 7 CTAs share an SM, which a bin starts with when its shared memory allows more
 * than 5 (the tight variant spills a few registers to L1).  The
 * call times `windows` device windows (0: 4) from a fresh initialize for the current shapes
 * and, bin by bin, for the other shapes, keeps a change that is more than 2% faster, and
 * initializes again: the state returns to t = 0 and events injected before the call are
 * dropped, as at any mind_initialize.  It needs a handle initialized at step 0 and takes the
 * precision set for it.  No reference counterpart (the reference launches fixed shapes).
 * mind_bin_threads reports the shapes (*n_bins receives the bin count), mind_set_bin_threads
 * sets them (128, 64 or 32 per bin; at least one thread per threshold detector of a cell;
 * a bin set to 128 takes the register budget it starts with).
 */
int mind_autotune(MindHandle *h, int32_t windows);
int mind_bin_threads(const MindHandle *h, int32_t *threads, int32_t cap, int32_t *n_bins);
int mind_set_bin_threads(MindHandle *h, const int32_t *threads, int32_t n_bins);

/*
 * Spike exchange between ranks, for one network sharded by cell over GPUs (one process per
 * GPU, each with the handle of its shard; the reference runs on one device, so there is no
 * counterpart).  mind_exchange_id makes an NCCL unique id on one rank, which the host sends
 * to the others (128 bytes).  mind_attach_exchange then gives the handle a communicator of
 * `world` ranks (ncclCommInitRank, a collective call) and the maps of its shard:
 * detector_sources[k] (0-based source index of a local detector) has global sid
 * detector_sids[k]; spikes of global sid external_sids[k] enter through the local external
 * input external_sources[k] (0-based).  `window` is the steps per window every rank uses
 * (the smallest of the ranks' mind_window_steps), `width` the most spikes a rank sends per
 * window (a window with more raises status 3).  From then on mind_run, after each window,
 * packs the window's detector spikes, all-gathers the blocks of all ranks on the handle's
 * stream (ncclAllGather, no host copy) and enters the received spikes through the external
 * inputs' NetCons, the same fan-out as local spikes: the sharded run reproduces the
 * unsharded one bit for bit.  Every rank must run the same steps.  With nccl_id NULL no
 * communicator is made and the host drives the exchange: after a run of one window,
 * mind_exchange_pack writes this rank's block (device memory, 1 + 2 width int64:
 * count, then (sid, step) pairs) and mind_exchange_inject takes the gathered blocks of all
 * ranks (device memory, world blocks).  Not with regions attached.  libnccl.so.2 is opened
 * at run time (status 11 if absent).
 */
int mind_exchange_id(uint8_t id[128]);
int mind_attach_exchange(MindHandle *h, const uint8_t *nccl_id, int32_t world, int32_t rank, int32_t window,
                         int32_t width, const int32_t *detector_sources, const int32_t *detector_sids,
                         int32_t n_detectors, const int32_t *external_sids, const int32_t *external_sources,
                         int32_t n_external);
int mind_exchange_pack(MindHandle *h, int64_t *send);
int mind_exchange_inject(MindHandle *h, const int64_t *recv);

/* Steps per device window: the largest step count a run advances without routing cell
 * spikes, set by the shortest NetCon delay out of cell detectors and external inputs.
 * A host that exchanges spikes with other handles runs at most this many steps between
 * exchanges (no reference counterpart: the reference routes every step on the host). */
int mind_window_steps(const MindHandle *h, int32_t *steps);

/*
 * Cross-scale coupling (advance_macro!, src/runtime/step.jl:156-204;
 * src/runtime/cuda/macro.jl): neural-mass regions advanced every dt_macro and coupled
 * to the micro network both ways.
 *
 * Regions are Jansen-Rit second-order PSP masses, six states per region (mV, mV/s):
 *   y0' = y3   y3' = A a S(y1 - y2) - 2 a y3 - a^2 y0
 *   y1' = y4   y4' = A a (p + C2 S(C1 y0)) - 2 a y4 - a^2 y1
 *   y2' = y5   y5' = B b C4 S(C3 y0) - 2 b y5 - b^2 y2
 *   S(v) = 2 e0 / (1 + exp(r (v0 - v))),  C1..C4 = C, 0.8 C, 0.25 C, 0.25 C,
 * integrated by classical RK4 over dt_macro (time in s inside the right-hand side) with
 * the input p held over the step.  A region's output is out = S(y1 - y2) (s^-1), taken at
 * the start of each macro step k.  Its input over step k is
 *   p(k) = p0 + micro_gain * rate(bin(k) - 1) + sum over edges into it (in edge order)
 *          of gain * out_src(k - delay),
 * where rate(b) is the spike rate (Hz per cell) of the detector sources mapped to the
 * region during rate bin b (bin_ms long; bin(k) = the bin containing step k; rate 0 before
 * the first bin), and out_src(m) for m < 0 is out_src(0).  Macro to micro: every input
 * source (an external spike input of the layout) fires as a Poisson process of rate
 * scale * out(k) Hz over macro step k; its n events in step k (n by inversion of the Poisson
 * CDF, at most 3) fall at k dt_macro + dt_macro u_j, with u_0 (count) and u_1..u_3 the
 * words of Philox4x32-10 on counter (k low, k high, input index, 0x4D4D), key = seed,
 * mapped to (w + 1)/(2^32 + 1); they then follow the source's NetCons.
 * dt_macro must be a multiple of dt and bin_ms a multiple of dt_macro; the library's
 * window becomes a multiple of the macro step no longer than the bin, and every window
 * ends at the next bin boundary at the latest, so bins are complete before the regions
 * read them.
 */
typedef struct {
    int32_t n_regions;
    const double *params;         /* [n_regions][9]: A, B, a, b, e0, r, v0, C, p0 */
    const double *y0;             /* [n_regions][6] initial states */
    const double *micro_gain;     /* [n_regions] */
    int64_t n_edges;
    const int32_t *edge_src;      /* 1-based regions */
    const int32_t *edge_dst;
    const double *edge_gain;
    const int32_t *edge_delay;    /* macro steps, >= 1 */
    int64_t n_inputs;
    const int32_t *input_region;  /* 1-based region driving each input */
    const int64_t *input_source;  /* 1-based external source of the micro layout */
    const double *input_scale;    /* Hz of input rate per s^-1 of region output */
    int64_t n_outputs;
    const int32_t *output_region; /* 1-based region fed by each detector source */
    const int64_t *output_source; /* 1-based detector source of the micro layout */
    double dt_macro;              /* ms */
    double bin_ms;                /* population-rate bin, ms */
} MindMacroLayout;

/* Attach regions and coupling to a created handle (before mind_initialize; allocation
 * happens here).  Runs then advance regions, inputs and rate bins with the micro steps.
 * A handle with a spike exchange attached (mind_attach_exchange) is refused: MIND_EARG. */
int mind_attach_macro(MindHandle *h, const MindMacroLayout *macro);

/* The regions' outputs out(k) recorded by the last run for every macro step boundary it
 * covered, [samples][n_regions] sample-major; `n` is the buffer length.  samples =
 * floor(end / steps per macro step) - ceil(start / steps per macro step) + 1. */
int mind_get_macro_trace(const MindHandle *h, double *out, int64_t n, int64_t *samples);

/*
 * Spike-output surrogate (no counterpart in the reference): a multilayer perceptron
 * n_in -> hidden (SiLU) x layers -> sigmoid, the probability that a cell spikes in the
 * next 1 ms bin given its recent synaptic drive and output.  Products run in BF16 with
 * FP32 accumulation on the tensor cores, parameters and Adam state in FP32.
 * Parameters: for each linear map in order, W [out x in] row-major then b [out].
 */
/* Record, during each mind_run, every cell's synaptic drive: the summed NetCon weights
 * (uS) of the events its synapses receive, per bin of bin_ms (a multiple of dt) and per
 * synapse group (the synapse's row within its cell, mod 32) — the surrogate's training
 * inputs.  bin_ms <= 0 stops recording (no counterpart in the reference). */
int mind_set_drive_recording(MindHandle *h, double bin_ms);
/* The last run's drive, [bins][cells][32] (cells in layout order); bins = run steps / bin. */
int mind_get_drive(const MindHandle *h, float *out, int64_t n, int64_t *bins);

typedef struct MindMlp MindMlp;
typedef struct {
    int32_t n_in, hidden, layers;
    uint64_t seed;                 /* initial weights uniform(+-1/sqrt(fan_in)), zero biases */
} MindMlpConfig;

int mind_mlp_create(const MindMlpConfig *config, MindMlp **mlp);
int mind_mlp_destroy(MindMlp *mlp);
const char *mind_mlp_last_error(const MindMlp *mlp);
/* Device time (ms) of the last predict, gradients or train call's network work: from the
 * inputs on the device to the last product, without the host copies. */
int mind_mlp_last_ms(const MindMlp *mlp, float *ms);
int mind_mlp_param_count(const MindMlp *mlp, int64_t *n);
int mind_mlp_set_params(MindMlp *mlp, const float *params, int64_t n);
int mind_mlp_get_params(const MindMlp *mlp, float *params, int64_t n);
/* prob[k] for the n rows x[k][n_in] (host arrays). */
int mind_mlp_predict(MindMlp *mlp, const float *x, int64_t n, float *prob);
/* Gradient of the mean sigmoid cross-entropy over the n rows (targets y in [0, 1]). */
int mind_mlp_gradients(MindMlp *mlp, const float *x, const float *y, int64_t n, float *grad, float *loss);
/* Let a trained network stand in for the cells with surrogate_cells[c] != 0 (layout cell
 * order): their membranes are no longer simulated; at the start of every rate bin b each
 * such cell spikes with the network's probability for its inputs (drive of bins b-20..b-1
 * times drive_scale, then its own spikes in bins b-5..b-1), decided by Philox4x32-10 on
 * (b, cell) and placed uniformly in the bin; the spike is recorded, follows the cell's
 * NetCons and counts in its region's bin.  Regions must be attached first (the rate bin
 * is theirs); the handle keeps `mlp`, which must outlive it; mind_initialize follows. */
int mind_attach_surrogate(MindHandle *h, MindMlp *mlp, const uint8_t *surrogate_cells, float drive_scale);
/* Between runs, the set of cells the surrogate stands in for (a subset of the attached
 * set).  A cell leaving it is simulated again from its next step, its membrane and
 * synapses resuming from their state in HBM (that of mind_initialize when it never ran
 * detailed); a cell staying keeps its spike history.  This is how a host judge reverts a
 * population whose surrogate rate drifts from its detailed sample. */
int mind_set_surrogate_cells(MindHandle *h, const uint8_t *surrogate_cells);
/* Per-cell calibration of the surrogate (n_cells = the layout's cell count, layout order):
 * a surrogate cell spikes with probability sigmoid(logit + logit_offset[c]) instead of
 * sigmoid(logit).  All offsets are 0 after mind_attach_surrogate; a host sets them per
 * population so that the coupled run keeps each population's rate
 * (mind_b200.surrogate.calibrate).  Offsets must be finite. */
int mind_set_surrogate_offsets(MindHandle *h, const float *logit_offset, int32_t n_cells);

/* Keep a training set on the device; then `steps` Adam steps (beta 0.9/0.999, eps 1e-8) on
 * batches drawn with replacement; losses[k] = the batch loss before step k (may be NULL). */
int mind_mlp_set_data(MindMlp *mlp, const float *x, const float *y, int64_t n);
int mind_mlp_train(MindMlp *mlp, int32_t steps, int32_t batch, float lr, float *losses, float *ms);

/*
 * Mechanisms emitted from MOD files and compiled into this library (kinds
 * MIND_MECH_GENERATED + index): the seam where MIND.jl's compile_mod/load_mod/builtin
 * hand the runtime a CompiledMechanism (src/compiler/frontend.jl:15-110,
 * src/compiler/ir.jl:340-356).  Here the CUDA C a MOD file lowers to (mind_b200.nmodl) is
 * compiled with the library by nvcc, so a host selects a mechanism by name and passes its
 * kind code and fields in MindLayout.  Host-side calls: no device work.
 */
typedef struct MindMechanismInfo {
    const char *name;                  /* the MOD's SUFFIX or POINT_PROCESS name */
    int32_t kind;                      /* MIND_MECH_GENERATED + index */
    int32_t point;                     /* 1: point process, 0: density mechanism */
    int32_t net_receive;               /* NET_RECEIVE arity (0: the mechanism takes no events) */
    int32_t n_fields;
    const char *const *field_names;    /* the layout columns, in order (array fields as name[k]) */
    const double *defaults;            /* PARAMETER defaults, 0 for STATE and ASSIGNED */
    uint64_t digest;                   /* first 16 hex digits of the MOD source's SHA-256 */
    const char *ion_reads;             /* "field ion" pairs (space-separated) that USEION READ fills from
                                          the model's ion species, e.g. "ena na ek k" */
} MindMechanismInfo;
int mind_mechanism_count(int32_t *n);
int mind_mechanism_info(int32_t index, MindMechanismInfo *info);
/* The kind code of the emitted mechanism named `name`; MIND_EARG if none is known. */
int mind_mechanism_kind(const char *name, int32_t *kind);
/*
 * Mechanisms compiled at run time (the reference's compile_mod / CompiledMechanism seam for a
 * user MOD file, src/compiler/frontend.jl:85-110, src/compiler/ir.jl:340-356): `module_path`
 * is a cubin of csrc/gen_module.cu built for sm_100a with MIND_RUNTIME_MECHANISMS against a
 * runtime_mechanisms.cuh that the MOD front end emitted for `mechanisms` (after the ones
 * compiled into the library); `mechanisms` describes them in the module's order (name,
 * point, net_receive, fields, defaults, digest, ion_reads; `kind` is ignored).  They get the
 * kind codes after those already known (mind_mechanism_kind gives them) and are appended
 * to the registry for the life of the process; a later module must list the mechanisms of
 * the earlier ones first, unchanged, then its own.  Handles created afterwards whose
 * layouts use them launch that module's window kernels.  mind_b200.register_mod does all
 * of this from a MOD file.  On failure the message is mind_last_error(NULL).
 */
int mind_load_mechanisms(const char *module_path, const MindMechanismInfo *mechanisms, int32_t n);

/*
 * discretize (src/model/micro/morphology.jl:406-484): one morphology's sections into its
 * cable node tree, the build-time step that produces MindLayout's node arrays.  Sections
 * are visited parents first; a root section gets a root node (area 100 um2, no
 * capacitance or axial conductance), every section nseg segment nodes whose area, axial
 * conductance to the previous node and capacitance (cm * area * 1e-5) integrate its
 * geometry over half segments, then one zero-capacitance node at its x = 1 end.  Node ids
 * are 1-based (parent 0 = none).  Host only: no device work.  Returns MIND_ECAPACITY when
 * `capacity` is below the node count (out->node_count receives it; call again with room),
 * MIND_ELAYOUT with a message for an invalid morphology.
 */
typedef struct MindSection {
    int32_t parent;                    /* 0-based index of the parent section, -1 for a root */
    int32_t nseg;
    double parent_x;                   /* where on the parent it attaches, in [0, 1] */
    double child_x;                    /* its own attached end, 0 or 1 */
    double length, diameter;           /* um, used when there are no pt3d samples */
    double Ra, cm;                     /* ohm cm, uF/cm2 */
    int32_t n_points;                  /* pt3d samples (x, y, z, diameter), >= 2 to be used */
    const double *points;              /* [n_points][4] */
} MindSection;
typedef struct MindMorphology {
    int64_t node_count;                /* out */
    int32_t *parent;                   /* [capacity] 1-based parent node, 0 = none */
    double *area, *diameter, *axial, *capacitance, *edge_length;   /* [capacity] */
    int64_t *section_start;            /* [n_sections] node at x = 0 (may be NULL) */
    int64_t *section_end;              /* [n_sections] node at x = 1 (may be NULL) */
    int64_t *section_first;            /* [n_sections] its first segment node (may be NULL) */
} MindMorphology;
int mind_discretize(const MindSection *sections, int32_t n_sections, int64_t capacity, MindMorphology *out,
                    char *message, int32_t message_len);

/* Message for the last non-zero status of this handle (or of mind_create when h is NULL). */
const char *mind_last_error(const MindHandle *h);

/* Device-side wall time of the last mind_run, in milliseconds (CUDA events). */
int mind_last_run_ms(const MindHandle *h, double *ms);

/*
 * Launch statistics of the last mind_run (no reference counterpart: the
 * reference has no timers; this is the cudaEvent instrumentation of the run
 * loop).  window_ms is filled only while profiling is enabled, which brackets
 * every window-kernel launch with CUDA events on the library's stream.
 */
typedef struct MindRunStats {
    double run_ms;            /* device time of the whole run loop */
    double window_ms;         /* summed device time of window-kernel launches */
    int64_t launches;         /* kernels launched by the run loop */
    int64_t window_launches;  /* window-kernel launches */
    int64_t steps;            /* micro steps advanced */
    int32_t window_steps;     /* steps per window (W) */
    int32_t bins;             /* window-kernel launches per window (cell size bins) */
} MindRunStats;
int mind_run_stats(const MindHandle *h, MindRunStats *stats);
int mind_set_profiling(MindHandle *h, int32_t enable);

/*
 * run! without device allocation.  No counterpart in the reference.
 *
 * For callers that may not allocate device memory while they step a model —
 * for example a host whose device memory is owned by another allocator and is
 * sized up front, or a control loop that must not enter the CUDA allocator
 * once it is running.  mind_create still allocates the model's state once; this
 * call then advances `steps` micro steps exactly as mind_run does with voltage
 * records and no spike recording, and writes the (steps+1) x n_records trace,
 * sample-major, into the caller's host buffer `trace`.
 *
 * Its per-run scratch (record maps and the trace staging area) lives in one
 * static device array of MIND_NOALLOC_SCRATCH_BYTES (16 MiB) that every GPU
 * loading the library holds until the process exits.  Runs that need more
 * (more than about 16 MiB / (8 n_records) steps per call) return MIND_ECAPACITY
 * before any work, with a message giving the limit; the state is unchanged.
 * The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress) with the device current, so make the first call before
 * any stream capture.  The call must be made with the handle's device current
 * (the one current at mind_create), otherwise it returns MIND_EARG.  Surrogate
 * cells run too: their network's buffers are reserved by mind_attach_surrogate.  All
 * handles on a device share the array and it keeps the previous call's
 * contents: calls that overlap on the GPU (two threads, two handles) race and
 * must be serialized by the caller.
 */
#define MIND_NOALLOC_SCRATCH_BYTES (16u << 20)
int mind_run_noalloc(MindHandle *h, int64_t steps, const MindRecord *records, int32_t n_records, double *trace);

int mind_destroy(MindHandle *h);

#ifdef __cplusplus
}
#endif

#endif /* MINDGPU_H */
