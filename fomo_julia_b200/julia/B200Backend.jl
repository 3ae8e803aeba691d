# B200Backend.jl -- `backend(:b200)` for Elastic2D (Wuheng10086/Fomo_julia).
#
# The binding a maintainer adds to the reference to run its time loop in
# libfomo_b200.so: a backend type, device-array wrappers that satisfy the
# AbstractMatrix{Float32} fields of Wavefield/Medium/HABCConfig
# (src/core/Structures.jl:18,66,94,116,127), and methods for the dispatch
# points of the time-stepping path: to_device / synchronize
# (src/backends/backend.jl:68-79), Wavefield(nx, nz, backend)
# (Structures.jl:39-55), init_medium / init_habc (src/utils/init.jl:68-203),
# run_shot! / run_shots! (src/simulation/shot_manager.jl:46-180).  One ccall
# runs a whole shot (or a K-step chunk when an on_step callback is given).
#
# Usage, after `include("src/Elastic2D.jl")`:
#     include("B200Backend.jl"); using .B200Backend
#     B = B200Backend.B200_BACKEND            # or backend(:b200), see the backend.jl hunk
#
# This file is not exercised in this repository's test suite: the image that
# builds it has no Julia.  The Python package fomo_julia_b200 makes the same
# calls through ctypes and is what the tests run.

module B200Backend

using ..Elastic2D
import ..Elastic2D: to_device, synchronize, Wavefield, Medium, HABCConfig, Source, Receivers,
                    SimParams, ShotResult, MultiShotConfig, run_shot!, run_shots!, reset!,
                    init_medium, init_habc, _pad_array, _compute_staggered_params, _coord_to_index

const LIB = get(ENV, "FOMO_B200_LIB", joinpath(@__DIR__, "..", "_lib", "libfomo_b200.so"))

struct B200 <: Elastic2D.AbstractBackend end
const B200_BACKEND = B200()

check(rc::Integer) = rc == 0 ? nothing :
    error("libfomo_b200: ", unsafe_string(ccall((:fomo_b200_last_error, LIB), Cstring, ())))

function __init__()
    check(ccall((:fomo_b200_init, LIB), Cint, (Cint,), 0))
end

# ------------------------------------------------------------------ arrays
"""Device matrix owned by the library (a raw buffer handle)."""
mutable struct B200Matrix <: AbstractMatrix{Float32}
    handle::UInt64
    dims::NTuple{2,Int}
end
Base.size(a::B200Matrix) = a.dims
Base.getindex(a::B200Matrix, i::Int, j::Int) = Array(a)[i, j]   # slow path, host copy
function Base.Array(a::B200Matrix)
    out = Matrix{Float32}(undef, a.dims)
    GC.@preserve out check(ccall((:fomo_b200_download, LIB), Cint, (UInt64, Ptr{Cvoid}, Csize_t),
                                 a.handle, out, sizeof(out)))
    out
end
Base.fill!(a::B200Matrix, v) = (check(ccall((:fomo_b200_memset, LIB), Cint, (UInt64, Cfloat), a.handle, v)); a)

function to_device(data::Array{Float32,2}, ::B200)
    h = Ref{UInt64}(0)
    check(ccall((:fomo_b200_alloc, LIB), Cint, (Csize_t, Ref{UInt64}), sizeof(data), h))
    GC.@preserve data check(ccall((:fomo_b200_upload, LIB), Cint, (UInt64, Ptr{Cvoid}, Csize_t),
                                  h[], data, sizeof(data)))
    a = B200Matrix(h[], size(data))
    finalizer(x -> ccall((:fomo_b200_free, LIB), Cint, (UInt64,), x.handle), a)
    a
end
to_device(data::Vector{Float32}, ::B200) = data          # wavelets/coefficients stay on the host
synchronize(::B200) = check(ccall((:fomo_b200_synchronize, LIB), Cint, ()))

"""One field of a library wavefield (vx=0, vz=1, txx=2, tzz=3, txz=4)."""
struct B200Field <: AbstractMatrix{Float32}
    wavefield::UInt64
    field::Int32
    dims::NTuple{2,Int}
end
Base.size(a::B200Field) = a.dims
Base.getindex(a::B200Field, i::Int, j::Int) = Array(a)[i, j]
function Base.Array(a::B200Field)
    out = Matrix{Float32}(undef, a.dims)
    GC.@preserve out check(ccall((:fomo_b200_wavefield_download, LIB), Cint, (UInt64, Int32, Ptr{Float32}),
                                 a.wavefield, a.field, out))
    out
end

function Wavefield(nx::Int, nz::Int, ::B200)
    h = Ref{UInt64}(0)
    check(ccall((:fomo_b200_wavefield_create, LIB), Cint, (Int32, Int32, Ref{UInt64}), nx, nz, h))
    f(q) = B200Field(h[], Int32(q), (nx, nz))
    # The engine keeps the step-start copy itself, so the *_old fields alias
    # the current ones (they are never read outside the library).
    Wavefield(f(0), f(1), f(2), f(3), f(4), f(0), f(1), f(2), f(3), f(4))
end
reset!(::B200, W::Wavefield{B200Field}) =
    check(ccall((:fomo_b200_wavefield_reset, LIB), Cint, (UInt64,), W.vx.wavefield))

# ------------------------------------------------------------------ medium
"""Medium field backed by a library medium handle (q = 0..4)."""
struct B200MediumField <: AbstractMatrix{Float32}
    medium::UInt64
    q::Int
    host::Matrix{Float32}      # the host copy init_medium computed
end
Base.size(a::B200MediumField) = size(a.host)
Base.getindex(a::B200MediumField, i::Int, j::Int) = a.host[i, j]

function init_medium(vp::Matrix, vs::Matrix, rho::Matrix, dx::Real, dz::Real, nbc::Int, fd_order::Int,
                     ::B200; free_surface::Bool=true)
    M = fd_order ÷ 2
    pad = nbc + M
    nx_in, nz_in = size(vp)
    nx, nz = nx_in + 2pad, nz_in + 2pad
    lam, mu_txx, mu_txz, rho_vx, rho_vz =
        _compute_staggered_params(_pad_array(vp, pad), _pad_array(vs, pad), _pad_array(rho, pad))
    h = Ref{UInt64}(0)
    GC.@preserve rho_vx rho_vz lam mu_txx mu_txz check(ccall((:fomo_b200_medium_create, LIB), Cint,
        (Int32, Int32, Int32, Int32, Int32, Cfloat, Cfloat,
         Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Ref{UInt64}),
        nx, nz, M, pad, free_surface, dx, dz, rho_vx, rho_vz, lam, mu_txx, mu_txz, h))
    f(q, a) = B200MediumField(h[], q, a)
    Medium(nx, nz, Float32(dx), Float32(dz), Float32((nx_in - 1) * dx), Float32((nz_in - 1) * dz),
           M, pad, free_surface, f(0, rho_vx), f(1, rho_vz), f(2, lam), f(3, mu_txx), f(4, mu_txz))
end

# init_habc keeps the reference's own method (weights on the host); the
# library takes the weights as tables over dist = min(i-1, nx-i, j-1, nz-j).
weight_table(w::AbstractMatrix, nbc::Int) = Float32[w[1 + d, 1 + d] for d in 0:nbc+1]

# ------------------------------------------------------------------ shots
struct FomoHabc
    nbc::Int32; qx::Cfloat; qz::Cfloat; qt_x::Cfloat; qt_z::Cfloat; qxt::Cfloat
    w_vx::Ptr{Float32}; w_vz::Ptr{Float32}; w_tau::Ptr{Float32}
end
struct FomoShot
    a::Ptr{Float32}; M::Int32; dt::Cfloat; dtx::Cfloat; dtz::Cfloat; nt::Int32
    src_i::Int32; src_j::Int32; wavelet::Ptr{Float32}; n_wavelet::Int32
    n_rec::Int32; rec_i::Ptr{Int32}; rec_j::Ptr{Int32}; rec_kind::Int32
end
rec_kind(t::Symbol) = t === :vz ? Int32(0) : t === :vx ? Int32(1) : t === :p ? Int32(2) : error("receiver type $t")

function run_shot!(::B200, W::Wavefield{B200Field}, M::Medium, H::HABCConfig, a, src::Source,
                   rec::Receivers, params::SimParams; shot_id::Int=1, progress::Bool=true,
                   on_step=nothing, step_chunk::Int=1)
    med = M.rho_vx.medium
    wf = W.vx.wavefield
    tv, tz, tt = weight_table(Array(H.w_vx), H.nbc), weight_table(Array(H.w_vz), H.nbc),
                 weight_table(Array(H.w_tau), H.nbc)
    coeffs = Vector{Float32}(a)
    wav = Vector{Float32}(src.wavelet)
    ri, rj = Int32.(collect(rec.i)), Int32.(collect(rec.j))
    gather = zeros(Float32, params.nt, length(ri))
    GC.@preserve tv tz tt coeffs wav ri rj gather begin
        h = Ref(FomoHabc(H.nbc, H.qx, H.qz, H.qt_x, H.qt_z, H.qxt, pointer(tv), pointer(tz), pointer(tt)))
        s = Ref(FomoShot(pointer(coeffs), params.M, params.dt, params.dtx, params.dtz, params.nt,
                         src.i, src.j, pointer(wav), length(wav), length(ri), pointer(ri), pointer(rj),
                         rec_kind(rec.type)))
        if on_step === nothing
            check(ccall((:fomo_b200_run_shot, LIB), Cint,
                        (UInt64, UInt64, Ref{FomoHabc}, Ref{FomoShot}, Ptr{Float32}, Ptr{Cvoid}),
                        med, wf, h, s, gather, C_NULL))
        else   # K-step chunks, the callback sees the wavefield between chunks
            sh = Ref{UInt64}(0)
            check(ccall((:fomo_b200_shot_begin, LIB), Cint,
                        (UInt64, UInt64, Ref{FomoHabc}, Ref{FomoShot}, Ref{UInt64}), med, wf, h, s, sh))
            k = Ref{Int32}(0)
            while k[] < params.nt
                check(ccall((:fomo_b200_shot_advance, LIB), Cint, (UInt64, Int32, Ref{Int32}),
                            sh[], step_chunk, k))
                on_step(W, Elastic2D.TimeStepInfo(k[], k[] * params.dt, params.nt)) === false && break
            end
            check(ccall((:fomo_b200_shot_finish, LIB), Cint, (UInt64, Ptr{Float32}, Ptr{Cvoid}),
                        sh[], gather, C_NULL))
        end
    end
    ShotResult(gather, shot_id, Int(src.i), Int(src.j), Vector{Int}(ri), Vector{Int}(rj))
end

function run_shots!(b::B200, W::Wavefield{B200Field}, M::Medium, H::HABCConfig, a, rec_template::Receivers,
                    shot_config::MultiShotConfig, params::SimParams;
                    on_shot_complete=nothing, on_step=nothing, progress::Bool=true)
    results = ShotResult[]
    for shot in shot_config.shots
        src = Source(_coord_to_index(shot.source_x, M.dx, M.pad), _coord_to_index(shot.source_z, M.dz, M.pad),
                     shot_config.wavelet)
        rec = Receivers(rec_template.i, rec_template.j, zeros(Float32, 1, length(rec_template.i)), rec_template.type)
        r = run_shot!(b, W, M, H, a, src, rec, params; shot_id=shot.shot_id, on_step=on_step)
        push!(results, r)
        on_shot_complete === nothing || on_shot_complete(r)
    end
    results
end

"""Batched form of run_shots!: every shot of `shot_config` in one
fomo_b200_run_batch call (shots side by side on the device); the gathers
equal run_shots!'s bit for bit."""
function run_shots_batched!(::B200, M::Medium, H::HABCConfig, a, rec_template::Receivers,
                            shot_config::MultiShotConfig, params::SimParams)
    med = M.rho_vx.medium
    tv, tz, tt = weight_table(Array(H.w_vx), H.nbc), weight_table(Array(H.w_vz), H.nbc),
                 weight_table(Array(H.w_tau), H.nbc)
    coeffs = Vector{Float32}(a)
    wav = Vector{Float32}(shot_config.wavelet)
    ri, rj = Int32.(collect(rec_template.i)), Int32.(collect(rec_template.j))
    srcs = [(_coord_to_index(s.source_x, M.dx, M.pad), _coord_to_index(s.source_z, M.dz, M.pad))
            for s in shot_config.shots]
    gathers = [zeros(Float32, params.nt, length(ri)) for _ in srcs]
    GC.@preserve tv tz tt coeffs wav ri rj gathers begin
        h = Ref(FomoHabc(H.nbc, H.qx, H.qz, H.qt_x, H.qt_z, H.qxt, pointer(tv), pointer(tz), pointer(tt)))
        shots = [FomoShot(pointer(coeffs), params.M, params.dt, params.dtx, params.dtz, params.nt,
                          si, sj, pointer(wav), length(wav), length(ri), pointer(ri), pointer(rj),
                          rec_kind(rec_template.type)) for (si, sj) in srcs]
        ptrs = [pointer(g) for g in gathers]
        check(ccall((:fomo_b200_run_batch, LIB), Cint,
                    (UInt64, Ref{FomoHabc}, Ptr{FomoShot}, Int32, Ptr{Ptr{Float32}}, Ptr{Cvoid}),
                    med, h, shots, length(shots), ptrs, C_NULL))
    end
    [ShotResult(gathers[k], shot_config.shots[k].shot_id, Int(srcs[k][1]), Int(srcs[k][2]),
                Vector{Int}(ri), Vector{Int}(rj)) for k in eachindex(srcs)]
end

end # module
