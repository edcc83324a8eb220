# VeronaB200.jl -- Julia binding of libverona_b200.so for Wesenheit/Verona.
#
# UNTESTED: there is no julia on the machines this library was built and
# tested on. The binding follows include/verona_b200.h field for field (the
# struct layouts below are the ones tests/test_abi.py checks against the
# header's sizeof/offsetof for the Python mirrors); a maintainer includes it
# next to the reference's modules:
#
#     include("VeronaB200.jl")          # after `using Verona` (EosTypes, Verona1D/2D/3D)
#     VeronaB200.HARM_HLL(comm, CuP, (1,1,1), (Nx,Ny,Nz), dt, dx, dy, dz, T, eos, drops, floor,
#                         out_dir, false, n_it, tol, fun_bound)
#
# The methods keep the positional signatures of the reference's drivers
# (Verona3D.HARM_HLL, src/3dim/algos.jl:203-219; Verona2D.HARM_HLL,
# src/2dim/algos.jl:192-208; Verona1D.HARM_HLL, src/1dim/algos.jl:58-68) and
# return what they return (the dump count in 2D/3D, the vector of snapshots in
# 1D). The time loop, dump schedule and HDF5 output stay in Julia; the step
# itself (fluxes, update, con2prim, limit, ghost fill) runs in the library on
# CUDA.jl's current stream. One GPU, one rank: the reference's MPI halo
# exchange is a no-op on one rank and is not replaced.
#
# The boundary: `fun_bound` (the reference's kwargs[3]) may be
#   - a vector of `Bound(face, kind, params)` (the library's built-in device
#     kinds: OUTFLOW, FIXED with an optional decay, NOZZLE), applied on the
#     device at the start of every step, or
#   - a Julia function f(P, t, idx_mpi, MPI_dims) as in the reference; it then
#     runs on the host between single steps (P is stored, f is called, P is
#     reloaded), which recomputes U from P every step -- a slow path for
#     experiments, not for parity runs.
# `turnoff3d(dt, box_X)` / `turnoff2d(dt, box_X)` give the built-in form of
# the examples' TurnOff callbacks (examples/Jet3D/HARM_jet_breakout.jl:131-158,
# examples/Jet2D/HARM_jet_breakout.jl:84-99).
module VeronaB200

using CUDA
using ..EosTypes
using ..Verona1D, ..Verona2D, ..Verona3D

const libvb = get(ENV, "VERONA_B200_LIB", joinpath(@__DIR__, "..", "verona_b200", "libverona_b200.so"))

# ---- mirrors of the header's POD structs ------------------------------------
struct VBOptions
    version::UInt32
    recon::Int32
    riemann::Int32
    rk::Int32
    precision::Int32
    guess::Int32
    n_iter::Int32
    stats::Int32
    tol::Float64
    floor_::Float64
    w_rtol::Float64
    w_max_newton::Int32
    c2p_fp32::Int32
    reserved_i::NTuple{6,Int32}
    reserved_d::NTuple{4,Float64}
end

struct VBTuning
    split_con2prim::Int32
    force_box::Int32
    learned_fused::Int32
    fp32_pairs::Int32
    tma_tiles::Int32
    fp64_contract::Int32
    reserved::NTuple{2,Int32}
end

const RECON = Dict(:minmod => 0, :ppm => 1, :wenoz => 2)
const RIEMANN = Dict(:hll => 0, :hllc => 1)
const PRECISION = Dict(:fp64 => 0, :fp32 => 1)
const GUESS = Dict(:previous => 0, :learned => 1)
const OUTFLOW, FIXED, NOZZLE = 0, 1, 2
const XLO, XHI, YLO, YHI, ZLO, ZHI = 0, 1, 2, 3, 4, 5

"""A built-in boundary of one face: kind OUTFLOW, FIXED (params: none, or
(var, t_on, t_off, factor) for a decay of variable `var` (0-based) by
`factor` per step for t_on < t < t_off) or NOZZLE (params: radius, c1, c2 in
cells and the inflow state rho, u, u1[, u2[, u3]])."""
struct Bound
    face::Int
    kind::Int
    params::Vector{Float64}
end
Bound(face, kind) = Bound(face, kind, Float64[])

"""TurnOff of examples/Jet3D/HARM_jet_breakout.jl:131-158: x-lo ghosts keep
the loaded jet state with u^x decayed by (1 - dt/T_exp) for box_X/3 < t <
box_X (T_exp = box_X/10); zero-gradient on the other faces."""
turnoff3d(dt, box_X) = [Bound(XLO, FIXED, [2.0, box_X / 3, box_X, 1 - dt / (box_X / 10)]);
                        [Bound(f, OUTFLOW) for f in (XHI, YLO, YHI, ZLO, ZHI)]]
"""TurnOff of examples/Jet2D/HARM_jet_breakout.jl:84-99 (decays P[4], u^y,
as that example does)."""
turnoff2d(dt, box_X) = [Bound(XLO, FIXED, [3.0, box_X / 3, box_X, 1 - dt / (box_X / 10)]);
                        [Bound(f, OUTFLOW) for f in (XHI, YLO, YHI)]]

function check(rc, h)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:vb_last_error, libvb), Cstring, (Ptr{Cvoid},), h))
    error("verona_b200 ($rc): $msg")
end

function options(; recon = :wenoz, riemann = :hll, rk = 2, precision = :fp64, guess = :previous, n_iter = 50,
                 tol = 1e-10, floor = 1e-7)
    o = Ref{VBOptions}()
    check(ccall((:vb_default_options, libvb), Cint, (Ref{VBOptions},), o), C_NULL)
    x = o[]
    return VBOptions(x.version, RECON[recon], RIEMANN[riemann], rk, PRECISION[precision], GUESS[guess], n_iter, 0,
                     tol, floor, x.w_rtol, x.w_max_newton, x.c2p_fp32, x.reserved_i, x.reserved_d)
end

# ---- a solver handle ------------------------------------------------------------
mutable struct Handle
    h::Ptr{Cvoid}
    function Handle(dims, nx, ny, nz, nghost, o::VBOptions, gamma, dxs)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:vb_create, libvb), Cint, (Ref{Ptr{Cvoid}}, Cint, Cint, Cint, Cint, Cint, Ref{VBOptions}),
                    r, dims, nx, ny, nz, nghost, Ref(o)), C_NULL)
        x = new(r[])
        finalizer(close!, x)
        check(ccall((:vb_set_eos, libvb), Cint, (Ptr{Cvoid}, Cdouble), x.h, gamma), x.h)
        check(ccall((:vb_set_grid, libvb), Cint, (Ptr{Cvoid}, Cdouble, Cdouble, Cdouble), x.h, dxs...), x.h)
        return x
    end
end

function close!(x::Handle)
    x.h == C_NULL && return nothing
    ccall((:vb_destroy, libvb), Cint, (Ptr{Cvoid},), x.h)
    x.h = C_NULL
    return nothing
end

set_boundary!(x::Handle, b::Bound) =
    check(ccall((:vb_set_boundary, libvb), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Cdouble}, Cint), x.h, b.face, b.kind,
                b.params, length(b.params)), x.h)
set_tuning!(x::Handle, t::VBTuning) =
    check(ccall((:vb_set_tuning, libvb), Cint, (Ptr{Cvoid}, Ref{VBTuning}), x.h, Ref(t)), x.h)
load!(x::Handle, A::CuArray{Float64}, s) =
    check(ccall((:vb_load_prims, libvb), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, Ptr{Cvoid}), x.h, pointer(A), s), x.h)
store!(x::Handle, A::CuArray{Float64}, s) =
    check(ccall((:vb_store_prims, libvb), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, Ptr{Cvoid}), x.h, pointer(A), s), x.h)
load_host!(x::Handle, A::Array{Float64}, s) =
    check(ccall((:vb_load_prims_host, libvb), Cint, (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cvoid}), x.h, A, s), x.h)
store_host!(x::Handle, A::Array{Float64}, s) =
    check(ccall((:vb_store_prims_host, libvb), Cint, (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cvoid}), x.h, A, s), x.h)
step!(x::Handle, dt, n, s) =
    check(ccall((:vb_step, libvb), Cint, (Ptr{Cvoid}, Cdouble, Cint, Ptr{Cvoid}), x.h, dt, n, s), x.h)
function failures(x::Handle, s)
    c = zeros(UInt64, 8)
    check(ccall((:vb_get_counters, libvb), Cint, (Ptr{Cvoid}, Ptr{UInt64}, Cint, Ptr{Cvoid}), x.h, c, 8, s), x.h)
    return c[1]
end

# steps of the reference's `while t < Tmax; ...; t += dt` loop until the next
# dump threshold (the same floating-point accumulation of t)
function steps_to_dump(t, dt, Tmax, thres)
    n = 0
    while t < Tmax
        t += dt
        n += 1
        t > thres && break
    end
    return n, t
end

# the shared 2D/3D time loop: dumps as the reference's (t > thres), written by
# the caller's `save(i, t)` from P.arr after vb_store_prims
function run_loop!(x::Handle, P, dt, Tmax, drops, fun_bound, dims, save)
    s = CUDA.stream().handle
    host_bound = fun_bound isa Function
    if !host_bound && fun_bound !== nothing
        for b in fun_bound
            set_boundary!(x, b)
        end
    end
    t = 0.0
    thres = drops
    i = 0
    GC.@preserve P begin
        load!(x, P.arr, s)
        save(0, t)
        while t < Tmax
            if host_bound
                # the reference's callback between single steps (slow path)
                store!(x, P.arr, s)
                CUDA.synchronize()
                fun_bound(P, t, ntuple(_ -> 0, dims), ntuple(_ -> 1, dims))
                load!(x, P.arr, s)
                step!(x, dt, 1, s)
                t += dt
            else
                n, t = steps_to_dump(t, dt, Tmax, thres)
                step!(x, dt, n, s)
            end
            if t > thres
                i += 1
                thres += drops
                store!(x, P.arr, s)
                CUDA.synchronize()
                save(i, t)
            end
        end
        store!(x, P.arr, s)
    end
    return i
end

# ---- Verona3D.HARM_HLL (src/3dim/algos.jl:203-219) -------------------------------
function HARM_HLL(comm, P::Verona3D.CuParVector3D{Float64}, MPI_dims::Tuple{Int64,Int64,Int64},
                  Size::Tuple{Int64,Int64,Int64}, dt::Float64, dx::Float64, dy::Float64, dz::Float64, Tmax::Float64,
                  eos::EOS{Float64}, drops::Float64, floor::Float64 = 1e-7, out_dir::String = ".",
                  verbose::Bool = false, n_iter = 50, tol = 1e-10, fun_bound = nothing; recon = :wenoz,
                  riemann = :hll, rk = 2, precision = :fp64, guess = :previous, tuning = nothing)
    MPI_dims == (1, 1, 1) || error("VeronaB200: one GPU, one rank")
    o = options(; recon, riemann, rk, precision, guess, n_iter, tol, floor)
    x = Handle(3, P.size_X - 6, P.size_Y - 6, P.size_Z - 6, 3, o, eos.gamma, (dx, dy, dz))
    tuning === nothing || set_tuning!(x, tuning)
    try
        save(i, t) = Verona3D.SaveHDF5Parallel(comm, P, 1, 1, 1, out_dir * "/dump" * string(i) * ".h5",
                                               Dict("T" => t, "grid" => [dx, dy, dz]))
        t0 = time()
        i = run_loop!(x, P, dt, Tmax, drops, fun_bound, 3, save)
        if verbose
            el = time() - t0
            println("zone-updates/s (interior): ", (P.size_X - 6) * (P.size_Y - 6) * (P.size_Z - 6) *
                                                   ceil(Tmax / dt) / el)
        end
        return i
    finally
        close!(x)
    end
end

# ---- Verona2D.HARM_HLL (src/2dim/algos.jl:192-208) -------------------------------
function HARM_HLL(comm, P::Verona2D.CuParVector2D{Float64}, XMPI::Int64, YMPI::Int64, SizeX::Int64, SizeY::Int64,
                  dt::Float64, dx::Float64, dy::Float64, Tmax::Float64, eos::EOS{Float64}, drops::Float64,
                  floor::Float64 = 1e-7, out_dir::String = ".", n_iter = 50, tol = 1e-10, fun_bound = nothing;
                  recon = :wenoz, riemann = :hll, rk = 2, precision = :fp64, tuning = nothing)
    (XMPI, YMPI) == (1, 1) || error("VeronaB200: one GPU, one rank")
    o = options(; recon, riemann, rk, precision, guess = :previous, n_iter, tol, floor)
    x = Handle(2, P.size_X - 6, P.size_Y - 6, 1, 3, o, eos.gamma, (dx, dy, 1.0))
    tuning === nothing || set_tuning!(x, tuning)
    try
        save(i, t) = Verona2D.SaveHDF5Gather(comm, P, 1, 1, out_dir * "/dump" * string(i) * ".h5",
                                             Dict("T" => t, "grid" => [dx, dy]))
        return run_loop!(x, P, dt, Tmax, drops, fun_bound, 2, save)
    finally
        close!(x)
    end
end

# ---- Verona1D.HARM_HLL (src/1dim/algos.jl:58-68): N cells, no ghosts -------------
function HARM_HLL(P::Verona1D.ParVector1D, N::Int64, dt::Float64, dx::Float64, T::Float64, eos::EOS, drops::Float64,
                  rec::Symbol, n_iter = 50, tol = 1e-10)
    rec in (:minmod, :ppm, :wenoz) || (println("reconstruction not supported!"); return Verona1D.ParVector1D[])
    o = options(; recon = rec, riemann = :hll, rk = 2, n_iter, tol)
    x = Handle(1, N, 1, 1, 0, o, eos.gamma, (dx, 1.0, 1.0))
    s = CUDA.stream().handle
    A = Array{Float64}(undef, 3, N)
    pull!() = (store_host!(x, A, s); P.arr1 .= A[1, :]; P.arr2 .= A[2, :]; P.arr3 .= A[3, :]; P)
    try
        A[1, :] .= P.arr1
        A[2, :] .= P.arr2
        A[3, :] .= P.arr3
        load_host!(x, A, s)
        out = [deepcopy(P)]
        t = 0.0
        thres = drops
        while t < T
            n, t = steps_to_dump(t, dt, T, thres)
            step!(x, dt, n, s)
            if t > thres
                thres += drops
                push!(out, deepcopy(pull!()))
            end
        end
        pull!()
        return out
    finally
        close!(x)
    end
end

end # module
