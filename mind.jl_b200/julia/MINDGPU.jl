# MINDGPU.jl — ccall backend that runs MIND.jl's micro step loop in libmindgpu.so.
#
# Include this file inside the MIND module (after src/model/build.jl and
# src/runtime/state.jl) to replace the runtime seams with the B200 library:
#
#   allocate_simulation / initialize!  ->  mindgpu_initialize!(model)
#   run!(model, stop; records)         ->  mindgpu_run!(model, stop; records)
#   step!(model)                       ->  mindgpu_step!(model)
#   read_value(state, ref)             ->  mindgpu_read_value(model, ref)
#   inject_spike!(state, input, t)     ->  mindgpu_inject_spikes!(model, sources, times)
#   inject_event!(state, connection, t) -> mindgpu_inject_event!(model, connection, t)
# and, with no reference counterpart: mindgpu_autotune!(model) (launch shape per size bin),
# mindgpu_run_noalloc!(model, steps, refs, trace) (a run that allocates no device memory),
# mindgpu_last_run_ms(model), mindgpu_window_steps(model).
#
# The model builders and build! are unchanged: the library receives the
# ModelLayout.micro that build! packs (src/model/build.jl:15-60), as a POD view
# whose pointers stay valid for the duration of mind_create only.
# Julia is not available where this library was built, so this adapter is
# exercised through the identical C-ABI from Python (mind_b200/abi.py).

module MINDGPU

const libmindgpu = get(ENV, "MINDGPU_LIBRARY", joinpath(@__DIR__, "..", "lib", "libmindgpu.so"))

const MIND_ABI_VERSION = Int32(2)
const MIND_RECORD_VOLTAGE = Int32(1)
const MIND_RECORD_MECHANISM = Int32(2)
const KIND_CODES = Dict(:hh => Int32(1), :pas => Int32(2), :ExpSyn => Int32(3), :Exp2Syn => Int32(4),
                        :NetStim => Int32(5), :IClamp => Int32(6), :AlphaSynapse => Int32(7),
                        :PatternStim => Int32(8))

# Kind code of a mechanism: the hand-written device code for the builtins above, else the
# CUDA C emitted from its MOD file and compiled into the library (mind_mechanism_kind;
# SEClamp, VClamp and any MOD added with csrc/gen_mechanisms.py).
function kind_code(name::Symbol)
    haskey(KIND_CODES, name) && return KIND_CODES[name]
    kind = Ref{Int32}(0)
    status = ccall((:mind_mechanism_kind, libmindgpu), Cint, (Cstring, Ref{Int32}), String(name), kind)
    status == 0 || throw(ArgumentError("libmindgpu has no device code for mechanism $name; emit its MOD file " *
                                       "with csrc/gen_mechanisms.py and rebuild the library"))
    return kind[]
end

struct MindMechanism
    kind::Int32
    n_fields::Int32
    rows::Int64
    data::Ptr{Float64}
    field_names::Ptr{Ptr{UInt8}}
    nodes::Ptr{Int32}
    logical_ids::Ptr{UInt64}
    digest::UInt64
end

struct MindLayout
    abi_version::Int32
    secondorder::Int32
    n_nodes::Int64
    parent::Ptr{Int32}
    voltage::Ptr{Float64}
    area::Ptr{Float64}
    capacitance::Ptr{Float64}
    axial::Ptr{Float64}
    axial_diagonal::Ptr{Float64}
    n_mechanisms::Int32
    mechanisms::Ptr{MindMechanism}
    n_points::Int64
    point_group::Ptr{Int32}
    point_row::Ptr{Int32}
    n_sources::Int64
    source_ids::Ptr{Int64}
    source_nodes::Ptr{Int32}
    source_thresholds::Ptr{Float64}
    source_points::Ptr{Int32}
    n_edges::Int64
    fanout_offsets::Ptr{Int64}
    edge_targets::Ptr{Int32}
    edge_delays::Ptr{Float64}
    edge_weights::Ptr{Float64}
    dt::Float64
    celsius::Float64
    seed::UInt64
    event_capacity::Int64
    spike_capacity::Int64
    n_pattern::Int64
    pattern_times::Ptr{Float64}
    pattern_points::Ptr{Int32}
end

struct MindRecord
    kind::Int32
    node::Int32
    group::Int32
    row::Int32
    field::Int32
end

# VariableRef (src/model/references.jl) -> MindRecord: voltage refs carry the node in `row`.
function c_record(ref)
    ref.kind === :voltage && return MindRecord(MIND_RECORD_VOLTAGE, Int32(ref.row), 0, 0, 0)
    ref.kind === :mechanism &&
        return MindRecord(MIND_RECORD_MECHANISM, 0, Int32(ref.group), Int32(ref.row), Int32(ref.field))
    throw(ArgumentError("libmindgpu records :voltage and :mechanism references"))
end

mutable struct Handle
    ptr::Ptr{Cvoid}
    dt::Float64
end

function check(h::Ptr{Cvoid}, status::Cint)
    status == 0 && return nothing
    message = unsafe_string(ccall((:mind_last_error, libmindgpu), Cstring, (Ptr{Cvoid},), h))
    codes = Dict(3 => "capacity exhausted", 5 => "invalid self-event delay or target",
                 6 => "singular or non-finite cable system", 8 => "non-finite numerical state",
                 9 => "device wait timeout", 10 => "layout rejected", 11 => "CUDA runtime error",
                 12 => "invalid argument")
    throw(ErrorException("libmindgpu: $(get(codes, Int(status), "error $status")): $message"))
end

# Field columns of one mechanism group, with ion reversals (ena, ek) resolved
# from the packed ion table the way the reference loads them before BREAKPOINT
# (src/runtime/cuda/micro.jl:436-438).
function group_columns(plan, group)
    ir = group.mechanism.ir
    data = copy(group.data)
    for (field_index, field) in enumerate(ir.fields)
        for (slot, ion) in enumerate(ir.ions)
            name = Symbol(:e, ion.name)
            field.name == name && name in ion.reads || continue
            for row in axes(data, 1)
                ion_row = group.ion_rows[row, slot]
                ion_row != 0 && (data[row, field.offset] = plan.ion_data[ion_row, 1])
            end
        end
    end
    # one name per data column: an array field of extent n is named name[0] .. name[n-1]
    columns = String[]
    for f in ir.fields
        if f.extent == 0
            push!(columns, String(f.name))
        else
            append!(columns, ["$(f.name)[$k]" for k in 0:(f.extent - 1)])
        end
    end
    names = [Base.unsafe_convert(Ptr{UInt8}, c) for c in columns]
    return data, columns, names
end

"""Create the device state from a built model (allocate_simulation + initialize!)."""
function mindgpu_initialize!(model; precision::Symbol = :fp64)
    layout = model.runtime.layout
    plan = layout.micro
    keep = Any[]
    mechs = MindMechanism[]
    for group in plan.groups
        data, names_str, _ = group_columns(plan, group)
        cnames = [pointer(s) for s in names_str]
        push!(keep, data, names_str, cnames, group.nodes, group.logical_ids)
        digest = parse(UInt64, first(group.mechanism.ir.source_digest, 16); base = 16)
        push!(mechs, MindMechanism(kind_code(group.mechanism.ir.name), Int32(size(data, 2)), size(data, 1),
                                   pointer(data), pointer(cnames), pointer(group.nodes),
                                   pointer(group.logical_ids), digest))
    end
    nsrc = length(plan.source_ids)
    source_nodes = Int32[v === nothing || v.kind != :voltage ? 0 : Int32(v.row) for v in plan.source_variables]
    first_weights = plan.edge_weights[:, 1]
    # PatternStim firings, already time-sorted by build! (micro/model.jl:586-613)
    pattern_times = Vector{Float64}(plan.pattern_times)
    pattern_points = Vector{Int32}(plan.pattern_targets)
    push!(keep, mechs, source_nodes, first_weights, pattern_times, pattern_points)
    c = MindLayout(MIND_ABI_VERSION, Int32(layout.secondorder), length(plan.parent), pointer(plan.parent),
                   pointer(plan.voltage), pointer(plan.area), pointer(plan.capacitance), pointer(plan.axial),
                   pointer(plan.axial_diagonal), Int32(length(mechs)), pointer(mechs),
                   length(plan.point_group), pointer(plan.point_group), pointer(plan.point_row),
                   nsrc, pointer(plan.source_ids), pointer(source_nodes), pointer(plan.source_thresholds),
                   pointer(plan.source_targets), length(plan.edge_targets), pointer(plan.fanout_offsets),
                   pointer(plan.edge_targets), pointer(plan.edge_delays), pointer(first_weights),
                   layout.dt_micro, plan.celsius, layout.seed, Int64(0), Int64(0),
                   length(pattern_times), pointer(pattern_times), pointer(pattern_points))
    handle = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve keep c begin
        status = ccall((:mind_create, libmindgpu), Cint, (Ref{MindLayout}, Ref{Ptr{Cvoid}}), c, handle)
        check(C_NULL, status)
    end
    h = Handle(handle[], layout.dt_micro)
    finalizer(x -> ccall((:mind_destroy, libmindgpu), Cint, (Ptr{Cvoid},), x.ptr), h)
    mode = precision === :mixed ? Int32(1) : Int32(0)
    check(h.ptr, ccall((:mind_set_precision, libmindgpu), Cint, (Ptr{Cvoid}, Int32), h.ptr, mode))
    check(h.ptr, ccall((:mind_initialize, libmindgpu), Cint, (Ptr{Cvoid},), h.ptr))
    model.runtime.state = h
    return model
end

"""run!: advance to an absolute stop time; voltage and mechanism-field records."""
function mindgpu_run!(model, stop_time::Real; records = (), record_spikes::Bool = true)
    h = model.runtime.state::Handle
    step = Ref{Int64}(0)
    now = Ref{Float64}(0.0)
    ccall((:mind_time, libmindgpu), Cint, (Ptr{Cvoid}, Ref{Int64}, Ref{Float64}), h.ptr, step, now)
    count = round(Int, (Float64(stop_time) - now[]) / h.dt)
    recs = [c_record(spec.variable) for spec in records]
    check(h.ptr, ccall((:mind_run, libmindgpu), Cint, (Ptr{Cvoid}, Int64, Ptr{MindRecord}, Int32, Int32),
                       h.ptr, count, recs, Int32(length(recs)), Int32(record_spikes)))
    # samples x records, column-major: each record's samples contiguous, the record-major
    # layout mind_get_trace_by_record writes (transposed on the device)
    trace = Matrix{Float64}(undef, count + 1, length(recs))
    check(h.ptr, ccall((:mind_get_trace_by_record, libmindgpu), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64),
                       h.ptr, trace, length(trace)))
    n = Ref{Int64}(0)
    check(h.ptr, ccall((:mind_get_spikes, libmindgpu), Cint,
                       (Ptr{Cvoid}, Ptr{Float64}, Ptr{Int64}, Int64, Ref{Int64}), h.ptr, C_NULL, C_NULL, 0, n))
    times = Vector{Float64}(undef, n[])
    sids = Vector{Int64}(undef, n[])
    check(h.ptr, ccall((:mind_get_spikes, libmindgpu), Cint,
                       (Ptr{Cvoid}, Ptr{Float64}, Ptr{Int64}, Int64, Ref{Int64}), h.ptr, times, sids, n[], n))
    time = [(step[] + k) * h.dt for k in 0:count]
    traces = Dict(spec.name => trace[:, k] for (k, spec) in enumerate(records))
    return (; time, traces, spike_times = times, spike_sources = sids)
end

"""read_value: the current value of a :voltage or :mechanism reference."""
function mindgpu_read_value(model, ref)
    h = model.runtime.state::Handle
    value = Ref{Float64}(0.0)
    rec = Ref(c_record(ref))
    check(h.ptr, ccall((:mind_read_value, libmindgpu), Cint, (Ptr{Cvoid}, Ref{MindRecord}, Ref{Float64}),
                       h.ptr, rec, value))
    return value[]
end

"""inject_spike!: external spike inputs (1-based source indices) fire at absolute times."""
function mindgpu_inject_spikes!(model, sources::AbstractVector{<:Integer}, times::AbstractVector{<:Real})
    h = model.runtime.state::Handle
    src = Int64.(sources)
    t = Float64.(times)
    check(h.ptr, ccall((:mind_inject_spikes, libmindgpu), Cint, (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Float64}),
                       h.ptr, length(src), src, t))
    return model
end

mindgpu_step!(model) = (check(model.runtime.state.ptr,
                              ccall((:mind_step, libmindgpu), Cint, (Ptr{Cvoid},), model.runtime.state.ptr)); model)

"""inject_event!: deliver NetCon `connection` (1-based edge) at absolute time `time` (ms, not
before the current time), as if its source had fired (src/runtime/state.jl:623-641)."""
function mindgpu_inject_event!(model, connection::Integer, time::Real)
    h = model.runtime.state::Handle
    check(h.ptr, ccall((:mind_inject_event, libmindgpu), Cint, (Ptr{Cvoid}, Int64, Float64),
                       h.ptr, Int64(connection), Float64(time)))
    return model
end

"""Time the launch shapes of each size bin on `windows` trial windows and keep the fastest;
leaves the model initialized at t = 0 (call right after mindgpu_initialize!).  Returns
the threads per cell chosen for each bin."""
function mindgpu_autotune!(model; windows::Integer = 4)
    h = model.runtime.state::Handle
    check(h.ptr, ccall((:mind_autotune, libmindgpu), Cint, (Ptr{Cvoid}, Int32), h.ptr, Int32(windows)))
    n = Ref{Int32}(0)
    check(h.ptr, ccall((:mind_bin_threads, libmindgpu), Cint, (Ptr{Cvoid}, Ptr{Int32}, Int32, Ref{Int32}),
                       h.ptr, C_NULL, Int32(0), n))
    threads = Vector{Int32}(undef, n[])
    check(h.ptr, ccall((:mind_bin_threads, libmindgpu), Cint, (Ptr{Cvoid}, Ptr{Int32}, Int32, Ref{Int32}),
                       h.ptr, threads, n[], n))
    return threads
end

"""Advance `steps` micro steps without any device allocation (mind_run_noalloc), recording
the references `refs` into `trace`, a caller-owned Matrix{Float64} of size
(length(refs), steps + 1): column k holds sample k - 1 of every reference, the sample-major
layout the library writes.  No spikes are recorded.  The record maps and the trace are
staged in the library's static device array (MIND_NOALLOC_SCRATCH_BYTES); runs that need
more are refused with status 3, and calls that overlap on one GPU race on that array."""
function mindgpu_run_noalloc!(model, steps::Integer, refs, trace::Matrix{Float64})
    h = model.runtime.state::Handle
    recs = [c_record(ref) for ref in refs]
    size(trace) == (length(recs), steps + 1) ||
        throw(DimensionMismatch("trace must be $(length(recs)) x $(steps + 1)"))
    check(h.ptr, ccall((:mind_run_noalloc, libmindgpu), Cint, (Ptr{Cvoid}, Int64, Ptr{MindRecord}, Int32, Ptr{Float64}),
                       h.ptr, Int64(steps), recs, Int32(length(recs)), trace))
    return trace
end

"""Device time of the last run (CUDA events around its loop), in milliseconds."""
function mindgpu_last_run_ms(model)
    h = model.runtime.state::Handle
    ms = Ref{Float64}(0.0)
    check(h.ptr, ccall((:mind_last_run_ms, libmindgpu), Cint, (Ptr{Cvoid}, Ref{Float64}), h.ptr, ms))
    return ms[]
end

"""Micro steps a run advances between two routings of cell spikes (the shortest NetCon delay
out of a cell bounds it): the exchange interval for hosts that shard one network."""
function mindgpu_window_steps(model)
    h = model.runtime.state::Handle
    w = Ref{Int32}(0)
    check(h.ptr, ccall((:mind_window_steps, libmindgpu), Cint, (Ptr{Cvoid}, Ref{Int32}), h.ptr, w))
    return Int(w[])
end

end # module
