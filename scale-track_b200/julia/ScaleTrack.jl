# ScaleTrack.jl -- Julia host binding of libscaletrack.so (include/scaletrack.h) via ccall.
#
# Julia is not available where this library is built and tested, so this file has not been
# run; it is written against the C header, and every entry point it calls is exercised by the
# Python ctypes binding (scale-track_b200/scaletrack.py) in the test suite.  It mirrors the
# reference's Julia side: evolve_cloud/allocate_array keep their names and meaning
# (asyncParallelTracking.jl:1436-1528), and the mean-source adjoint is exposed as a
# ChainRules rrule.
module ScaleTrack

using ChainRulesCore

const libscaletrack = joinpath(@__DIR__, "..", "libscaletrack.so")

const ST_OK = Cint(0)
const ST_DRAG_STOKES_IMPLICIT = Int32(0)
const ST_DRAG_SCHILLER_NAUMANN = Int32(1)
const ST_PREC_FP32 = Int32(0)
const ST_PREC_MIXED = Int32(1)
const ST_PREC_FP64 = Int32(2)

struct StMeshDesc
    n::NTuple{3,Int32}
    origin::NTuple{3,Float64}
    ending::NTuple{3,Float64}
end

mutable struct StParams
    mu_c::Float64
    rho_c::Float64
    rho_d::Float64
    drag_model::Int32
    precision::Int32
    deposit::Int32
    n_substeps::Int32
    sort_interval::Int32
    n_clouds::Int32
    block_size::Int32
    grid_blocks::Int32
    drag_multiplier::Float64
    diameter_scale::Float64
end

struct StAdjointDesc
    n_steps::Int32
    checkpoint_interval::Int32
    dt::Float64
    fluid_scale::Ptr{Float64}
end

struct ScaleTrackError <: Exception
    code::Cint
    msg::String
end

last_error() = unsafe_string(ccall((:st_last_error, libscaletrack), Cstring, ()))
check(rc::Cint) = rc == ST_OK ? nothing : throw(ScaleTrackError(rc, last_error()))

function default_params()
    p = StParams(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)
    ccall((:st_params_default, libscaletrack), Cvoid, (Ref{StParams},), p)
    return p
end

mutable struct Tracker
    h::Ptr{Cvoid}
    ncells::Int
end

function Tracker(p::StParams, m::StMeshDesc; device::Integer = 0)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:st_create, libscaletrack), Cint,
                (Ref{StParams}, Ref{StMeshDesc}, Cint, Ref{Ptr{Cvoid}}), p, m, device, h))
    t = Tracker(h[], Int(prod(m.n)))
    finalizer(t) do t
        t.h == C_NULL || ccall((:st_destroy, libscaletrack), Cint, (Ptr{Cvoid},), t.h)
        t.h = C_NULL
    end
    return t
end

# xyz, uvw: 3×n (Julia column-major matrices of size (n, 3) give the [3][n] SoA block layout)
function set_parcels!(t::Tracker, xyz::Matrix{Float64}, uvw::Matrix{Float64},
                      d::Vector{Float64}; cloud::Integer = 0)
    n = length(d)
    @assert size(xyz) == (n, 3) && size(uvw) == (n, 3)
    check(ccall((:st_set_parcels, libscaletrack), Cint,
                (Ptr{Cvoid}, Cint, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                t.h, cloud, n, xyz, uvw, d))
end

set_fluid_velocity!(t::Tracker, U::Matrix{Float32}) =  # size (3, nCells): [nCells][3] in C
    check(ccall((:st_set_fluid_velocity, libscaletrack), Cint,
                (Ptr{Cvoid}, Ptr{Float32}, Cint), t.h, U, 4))

step!(t::Tracker, dt::Real; fluid_scale::Real = 1.0) =
    check(ccall((:st_step, libscaletrack), Cint, (Ptr{Cvoid}, Cdouble, Cdouble),
                t.h, dt, fluid_scale))

function source(t::Tracker; cloud::Integer = 0)
    S = Matrix{Float64}(undef, 3, t.ncells)
    check(ccall((:st_get_source, libscaletrack), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}, Cint),
                t.h, cloud, S, 8))
    return S
end

function desc(T::Integer, C::Integer, dt::Real, fs::Union{Nothing,Vector{Float64}})
    StAdjointDesc(T, C, dt, fs === nothing ? Ptr{Float64}(C_NULL) : pointer(fs))
end

# the parcels of one cloud in st_set_parcels order: xyz, uvw as (n, 3), d as (n,)
function get_parcels(t::Tracker; cloud::Integer = 0)
    n = Int(ccall((:st_num_parcels, libscaletrack), Int64, (Ptr{Cvoid}, Cint), t.h, cloud))
    xyz = Matrix{Float64}(undef, n, 3)
    uvw = Matrix{Float64}(undef, n, 3)
    d = Vector{Float64}(undef, n)
    check(ccall((:st_get_parcels, libscaletrack), Cint,
                (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                t.h, cloud, xyz, uvw, d))
    return xyz, uvw, d
end

set_drag_parameters!(t::Tracker, drag_multiplier::Real, diameter_scale::Real) =
    check(ccall((:st_set_drag_parameters, libscaletrack), Cint, (Ptr{Cvoid}, Cdouble, Cdouble),
                t.h, drag_multiplier, diameter_scale))

"""
    mean_source(t, α, s, v0, T, C, dt; fluid_scale, cloud) -> Sbar (3 × nCells)

Time-averaged momentum source over `T` steps of one cloud, starting from its current
positions and diameters with drag multiplier `α`, diameter scale `s` and initial velocities
`v0` (n × 3, st_set_parcels order).  The tracker's positions are not advanced; `α`, `s` and
`v0` stay set on it.  Differentiable in `α`, `s` and `v0` through `rrule` (cell ownership
and wall bounces frozen at the forward pass); `t`, `T`, `C` and `dt` are not differentiated.
"""
function mean_source(t::Tracker, α::Real, s::Real, v0::Matrix{Float64}, T::Integer,
                     C::Integer, dt::Real; fluid_scale::Union{Nothing,Vector{Float64}} = nothing,
                     cloud::Integer = 0)
    set_drag_parameters!(t, α, s)
    xyz, _, d = get_parcels(t; cloud)
    @assert size(v0) == size(xyz)
    set_parcels!(t, xyz, v0, d; cloud)
    S = Matrix{Float64}(undef, 3, t.ncells)
    GC.@preserve fluid_scale begin
        check(ccall((:st_mean_source_forward, libscaletrack), Cint,
                    (Ptr{Cvoid}, Cint, Ref{StAdjointDesc}, Ptr{Float64}),
                    t.h, cloud, desc(T, C, dt, fluid_scale), S))
    end
    return S
end

function ChainRulesCore.rrule(::typeof(mean_source), t::Tracker, α::Real, s::Real,
                              v0::Matrix{Float64}, T::Integer, C::Integer, dt::Real;
                              fluid_scale = nothing, cloud::Integer = 0)
    S = mean_source(t, α, s, v0, T, C, dt; fluid_scale, cloud)
    function mean_source_pullback(Sbar)
        cot = Matrix{Float64}(unthunk(Sbar))
        dα = Ref{Float64}(0.0)
        ds = Ref{Float64}(0.0)
        dv0 = similar(v0)    # (n, 3) column-major = the [3][n] layout of the C side
        GC.@preserve fluid_scale begin
            check(ccall((:st_mean_source_pullback, libscaletrack), Cint,
                        (Ptr{Cvoid}, Cint, Ref{StAdjointDesc}, Ptr{Float64}, Ref{Float64},
                         Ref{Float64}, Ptr{Float64}),
                        t.h, cloud, desc(T, C, dt, fluid_scale), cot, dα, ds, dv0))
        end
        # one tangent per positional argument: (mean_source, t, α, s, v0, T, C, dt)
        return (NoTangent(), NoTangent(), dα[], ds[], dv0, NoTangent(), NoTangent(),
                NoTangent())
    end
    return S, mean_source_pullback
end

# ---- the reference's coupling surface ------------------------------------------------
setup(p::StParams, m::StMeshDesc) =
    check(ccall((:st_setup, libscaletrack), Cint, (Ref{StParams}, Ref{StMeshDesc}), p, m))

function allocate_array(name::String, size::Integer, ncomp::Integer, tbytes::Integer)
    p = ccall((:st_allocate_array, libscaletrack), Ptr{Cvoid}, (Cstring, Cint, Cint, Cint),
              name, size, ncomp, tbytes)
    p == C_NULL && throw(ScaleTrackError(Cint(1), last_error()))
    T = tbytes == 4 ? Float32 : Float64
    return unsafe_wrap(Array, Ptr{T}(p), (ncomp, size))
end

evolve_cloud(dt::Real) = check(ccall((:st_evolve_cloud, libscaletrack), Cint, (Cdouble,), dt))

# the reference's default, asynchronous coupling: UTrans receives the extrapolated source
evolve_cloud_async(dt::Real) =
    check(ccall((:st_evolve_cloud_async, libscaletrack), Cint, (Cdouble,), dt))

# zero-copy exchange: 0 = copies, 1 = the kernels use the pinned U / UTrans pages in place
set_exchange_mode(mode::Integer) =
    check(ccall((:st_set_exchange_mode, libscaletrack), Cint, (Cint,), mode))

# ---- initialisation, injection, output, restart ----------------------------------------
init_parcels!(t::Tracker, n::Integer, seed::Integer, dmin::Real, dmax::Real;
              cloud::Integer = 0) =
    check(ccall((:st_init_parcels, libscaletrack), Cint,
                (Ptr{Cvoid}, Cint, Int64, UInt64, Cdouble, Cdouble),
                t.h, cloud, n, seed, dmin, dmax))

function append_parcels!(t::Tracker, xyz::Matrix{Float64}, uvw::Matrix{Float64},
                         d::Vector{Float64}; cloud::Integer = 0)
    n = length(d)
    @assert size(xyz) == (n, 3) && size(uvw) == (n, 3)   # column-major: x block, y, z
    check(ccall((:st_append_parcels, libscaletrack), Cint,
                (Ptr{Cvoid}, Cint, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                t.h, cloud, n, xyz, uvw, d))
end

write_vtu(t::Tracker, path::String; cloud::Integer = 0) =
    check(ccall((:st_write_vtu, libscaletrack), Cint, (Ptr{Cvoid}, Cint, Cstring),
                t.h, cloud, path))

function write_pvd(path::String, times::Vector{Float64}, files::Vector{String})
    check(ccall((:st_write_pvd, libscaletrack), Cint,
                (Cstring, Cint, Ptr{Float64}, Ptr{Cstring}),
                path, length(times), times, files))
end

save_state(t::Tracker, path::String) =
    check(ccall((:st_save_state, libscaletrack), Cint, (Ptr{Cvoid}, Cstring), t.h, path))
load_state!(t::Tracker, path::String) =
    check(ccall((:st_load_state, libscaletrack), Cint, (Ptr{Cvoid}, Cstring), t.h, path))

end # module
