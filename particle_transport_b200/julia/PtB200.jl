# PtB200.jl -- Julia bindings of libptb200.so for the particle_transport
# pipeline.  The functions below keep the signatures of the reference
# functions they replace; the pipeline swaps its calls to them at those
# seams.  All arrays are the reference's own Julia arrays, passed by pointer
# under GC.@preserve; the library never frees them.
module PtB200

const LIB = get(ENV, "PTB200_LIB", joinpath(@__DIR__, "..", "libptb200.so"))

const PT_FIELD_REF_F64 = Cint(0)
const PT_FIELD_BRICK_F32 = Cint(1)
const PT_FIELD_BRICK_BF16 = Cint(2)
const PT_FIELD_BRICK_F64 = Cint(4)   # FP64 push, bit-identical to PT_FIELD_REF_F64
const PT_CACHE_MU = Cint(1)
const PT_CACHE_PHASE_SPACE = Cint(2)
const PT_PUSH_F64 = Cint(0)
const PT_PUSH_F32 = Cint(1)

struct PtGrid
    nx::Int64; ny::Int64; nz::Int64
    xmin::Float64; ymin::Float64; zmin::Float64
    xmax::Float64; ymax::Float64; zmax::Float64
    dx::Float64; dy::Float64; dz::Float64
end

struct PtPushParams
    dt::Float64
    nsteps::Int64
    stride::Int64
    periodic::Int32
    cache_mode::Int32
    cache_f64::Int32
    precision::Int32
    steps_per_launch::Int32
    sort_every::Int32
    kernel_variant::Int32
    cache_pitch::Int32
end

function check(rc::Cint, where::AbstractString)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:pt_last_error, LIB), Cstring, ()))
    error(where * ": " * msg)   # same exception flow as the reference (pipeline:2031-2059)
end

mutable struct Ctx
    ptr::Ptr{Cvoid}
end

function Ctx(device::Integer=0)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:pt_ctx_create, LIB), Cint, (Cint, Ref{Ptr{Cvoid}}), device, out), "pt_ctx_create")
    c = Ctx(out[])
    finalizer(x -> ccall((:pt_ctx_destroy, LIB), Cint, (Ptr{Cvoid},), x.ptr), c)
    return c
end

const _ctx = Ref{Union{Nothing, Ctx}}(nothing)
default_ctx() = (_ctx[] === nothing && (_ctx[] = Ctx(0)); _ctx[])

mutable struct Field
    ptr::Ptr{Cvoid}
end

"Upload (Bx, By, Bz, vx, vy, vz) in SI units on the node grid (x, y, z) (load_static_fields + build_uniform_coords)."
function upload_field(fields, x, y, z; storage=PT_FIELD_REF_F64, B_ref_T=0.0, ctx=default_ctx())
    Bx, By, Bz, vx, vy, vz = map(a -> convert(Array{Float64, 3}, a), fields)
    nx, ny, nz = size(Bx)
    grid = PtGrid(nx, ny, nz, x[1], y[1], z[1], x[end], y[end], z[end], x[2] - x[1], y[2] - y[1], z[2] - z[1])
    out = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve Bx By Bz vx vy vz begin
        comps = Ptr{Float64}[pointer(Bx), pointer(By), pointer(Bz), pointer(vx), pointer(vy), pointer(vz)]
        check(ccall((:pt_field_upload, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Ptr{Float64}}, Ref{PtGrid}, Cint, Float64, Ref{Ptr{Cvoid}}),
                    ctx.ptr, comps, grid, storage, B_ref_T, out), "pt_field_upload")
    end
    f = Field(out[])
    finalizer(x -> ccall((:pt_field_destroy, LIB), Cint, (Ptr{Cvoid},), x.ptr), f)
    return f
end

# ---- save sinks: the library calls back once per save row, on this thread
mutable struct MuSink
    writer::Any     # (file, mu dataset, outtype) from create_mu_cache_writer
end
mutable struct PhaseSink
    writer::Any     # from create_phase_space_writer
    n::Int
end

function _mu_cb(user::Ptr{Cvoid}, save_index::Int64, data::Ptr{Cvoid}, nbytes::Int64)::Cint
    try
        s = unsafe_pointer_to_objref(user)::MuSink
        T = s.writer.outtype
        row = unsafe_wrap(Array, Ptr{T}(data), nbytes ÷ sizeof(T))
        s.writer.mu[:, save_index + 1] = row            # write_mu_cache_step! (pipeline:1318-1321)
        return Cint(0)
    catch
        return Cint(1)
    end
end

function _phase_cb(user::Ptr{Cvoid}, save_index::Int64, data::Ptr{Cvoid}, nbytes::Int64)::Cint
    try
        s = unsafe_pointer_to_objref(user)::PhaseSink
        T = s.writer.outtype
        row = unsafe_wrap(Array, Ptr{T}(data), (s.n, 6))   # [6][n] row: positions then momenta
        for c in 1:3                                        # write_phase_space_step! (runner:413-421)
            s.writer.positions[:, c, save_index + 1] = view(row, :, c)
            s.writer.momenta[:, c, save_index + 1] = view(row, :, 3 + c)
        end
        return Cint(0)
    catch
        return Cint(1)
    end
end

"""
    push_run!(field, x1, x2, x3, p1, p2, p3, dt, nsteps, stride; periodic, cache, writer, precision)

Body of the step loop of run_gpu_ensemble (runner:561-592) and
run_mu_cache_ensemble (pipeline:1466-1500): advances the Float64 state in
place, hands every save row to the HDF5 writer, returns alive_fraction[nsteps].
"""
function push_run!(field::Field, x1, x2, x3, p1, p2, p3, dt, nsteps::Integer, stride::Integer;
                   periodic::Bool=true, cache::Symbol=:mu, writer, precision::Symbol=:f64, sort_every::Integer=0,
                   ctx=default_ctx())
    n = length(x1)
    alive = ones(UInt8, n)
    alive_count = zeros(Int64, nsteps)
    f64out = writer.outtype == Float64
    params = PtPushParams(Float64(dt), nsteps, stride, periodic, cache == :mu ? PT_CACHE_MU : PT_CACHE_PHASE_SPACE,
                          f64out, precision == :f64 ? PT_PUSH_F64 : PT_PUSH_F32, 0, sort_every, 0, 0)
    sink = cache == :mu ? MuSink(writer) : PhaseSink(writer, n)
    cb = cache == :mu ? @cfunction(_mu_cb, Cint, (Ptr{Cvoid}, Int64, Ptr{Cvoid}, Int64)) :
                        @cfunction(_phase_cb, Cint, (Ptr{Cvoid}, Int64, Ptr{Cvoid}, Int64))
    GC.@preserve x1 x2 x3 p1 p2 p3 alive alive_count sink begin
        check(ccall((:pt_push_run, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                     Ptr{Float64}, Ptr{UInt8}, Int64, Ref{PtPushParams}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Int64}),
                    ctx.ptr, field.ptr, x1, x2, x3, p1, p2, p3, alive, n, params, cb, pointer_from_objref(sink),
                    alive_count), "pt_push_run")
    end
    return Float64.(alive_count) ./ Float64(n)
end

"Drop-in for process_mu_chunk_dmumu_cpu! (src/compute_delta_mu2_dmumu_full.jl:656)."
function process_mu_chunk_dmumu_b200!(mu_chunk, lag_steps::Vector{Int}, mu_edges::Vector{Float64}, particle_counts,
                                      particle_means, particle_m2s, pair_sum_squares, pair_counts, dmumu_counts,
                                      dmumu_sum_delta, dmumu_sum_delta2, start_mode::Symbol, bin_abs::Bool;
                                      ctx=default_ctx())
    mode = start_mode == :sliding ? Cint(0) : start_mode == :injection ? Cint(1) :
           error("Unknown dmumu_start_mode: $(start_mode)")
    mu = mu_chunk isa Matrix{Float32} ? mu_chunk : Matrix{Float32}(mu_chunk)
    nsave, chunk = size(mu)
    GC.@preserve mu lag_steps mu_edges particle_counts particle_means particle_m2s pair_sum_squares pair_counts dmumu_counts dmumu_sum_delta dmumu_sum_delta2 begin
        check(ccall((:pt_dmumu_accumulate, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Float32}, Int64, Int64, Int64, Int64, Ptr{Int64}, Cint, Ptr{Float64}, Cint, Cint,
                     Cint, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}, Ptr{Int64}, Ptr{Float64}, Ptr{Float64},
                     Ptr{Float64}, Ptr{Int64}),
                    ctx.ptr, mu, chunk, nsave, nsave, 1, lag_steps, length(lag_steps), mu_edges,
                    length(mu_edges) - 1, mode, bin_abs, dmumu_counts, dmumu_sum_delta, dmumu_sum_delta2,
                    particle_counts, particle_means, particle_m2s, pair_sum_squares, pair_counts),
              "pt_dmumu_accumulate")
    end
    return nothing
end

"Drop-in for process_momenta_chunk_dpp_cpu! (src/compute_dpp_full.jl:247)."
function process_momenta_chunk_dpp_b200!(momenta, lag_steps::Vector{Int}, p0::Float64, counts, sum_delta_p,
                                         sum_delta_p2, sum_delta_p_norm, sum_delta_p_norm2; ctx=default_ctx())
    mom = momenta isa Array{Float32, 3} ? momenta : Array{Float32, 3}(momenta)
    chunk, _, nsave = size(mom)
    GC.@preserve mom lag_steps counts sum_delta_p sum_delta_p2 sum_delta_p_norm sum_delta_p_norm2 begin
        check(ccall((:pt_dpp_accumulate, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Float32}, Int64, Int64, Ptr{Int64}, Cint, Float64, Ptr{Int64}, Ptr{Float64},
                     Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                    ctx.ptr, mom, chunk, nsave, lag_steps, length(lag_steps), p0, counts, sum_delta_p, sum_delta_p2,
                    sum_delta_p_norm, sum_delta_p_norm2), "pt_dpp_accumulate")
    end
    return nothing
end

"Drop-in for fill_energy_snapshots! (src/compute_dpp_full.jl:290); snapshot_indices are 1-based."
function fill_energy_snapshots_b200!(energy_snapshots::Matrix{Float64}, momenta, snapshot_indices, particle_offset::Integer;
                                     ctx=default_ctx())
    mom = momenta isa Array{Float32, 3} ? momenta : Array{Float32, 3}(momenta)
    chunk, _, nsave = size(mom)
    snaps = Int64.(snapshot_indices) .- 1
    GC.@preserve mom snaps energy_snapshots begin
        check(ccall((:pt_energy_snapshots, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Float32}, Int64, Int64, Ptr{Int64}, Cint, Int64, Ptr{Float64}),
                    ctx.ptr, mom, chunk, nsave, snaps, length(snaps), particle_offset - 1, energy_snapshots),
              "pt_energy_snapshots")
    end
    return nothing
end

end # module
