"""
    AcousticWaveCPML_B200

Drop-in replacement of the GPU time loop of AcousticWaveCPML.jl's
`Acoustic2D_CUDA.solve2D` and `Acoustic3D_CUDA.solve3D`
(src/shared/acoustic_2D_xPU.jl:133-445, src/shared/acoustic_3D_xPU.jl:169-545).
The host setup below is the reference's (dt, nt, CPML coefficients, source time
functions, nearest-node snapping, assertions); the time loop runs in
libawcpml.so through `awc_forward` (include/awcpml.h).

Load it next to the reference package:

    using AcousticWaveCPML
    include("AcousticWaveCPML_B200.jl")
    pend = AcousticWaveCPML_B200.solve3D(lx, ly, lz, lt, vel, srcs, recs; halo=20)

Set `ENV["AWCPML_LIB"]` to the path of libawcpml.so if it is not in the
default location (../lib/libawcpml.so relative to this file).
"""
module AcousticWaveCPML_B200

import ..AcousticWaveCPML: Sources, Receivers, calc_Kab_CPML

export solve1D, solve2D, solve3D, misfit, misfit_gradient, misfit_gradient_shots

const LIBAWCPML = get(ENV, "AWCPML_LIB", joinpath(@__DIR__, "..", "lib", "libawcpml.so"))

const AWC_F32 = Int32(1)
const AWC_F64 = Int32(2)

# awc_problem (include/awcpml.h)
struct AwcProblem
    ndim::Int32
    precision::Int32
    nx::Int64
    ny::Int64
    nz::Int64
    halo::Int32
    freetop::Int32
    dx::Float64
    dy::Float64
    dz::Float64
    dt::Float64
    nt::Int64
    nsrc::Int64
    nrec::Int64
end

const _CTX = Ref{Ptr{Cvoid}}(C_NULL)

function context(device::Integer=0)
    if _CTX[] == C_NULL
        out = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:awc_create, LIBAWCPML), Cint, (Ref{Ptr{Cvoid}}, Int32), out, Int32(device))
        check(rc, C_NULL)
        _CTX[] = out[]
        atexit(() -> ccall((:awc_destroy, LIBAWCPML), Cvoid, (Ptr{Cvoid},), _CTX[]))
    end
    return _CTX[]
end

function check(rc::Integer, ctx::Ptr{Cvoid})
    if rc != 0
        msg = unsafe_string(ccall((:awc_last_error, LIBAWCPML), Cstring, (Ptr{Cvoid},), ctx))
        rc == -1 ? throw(ArgumentError(msg)) : error("libawcpml error $rc: $msg")
    end
    return nothing
end

# CPML block of solve2D/solve3D (acoustic_3D_xPU.jl:207-230), packed per axis
# as awc_coeffs_len documents: a_l a_r bK_l bK_r a_hl a_hr bK_hl bK_hr.
function packed_coeffs(halo, dt, ds, vel_max, rcoef, f0, freetop)
    alpha_max, npower, K_max = π * f0, 2.0, 1.0
    out = Float64[]
    for (ax, d) in enumerate(ds)
        d0 = -(npower + 1) * vel_max * log(rcoef) / (2.0 * (halo * d))
        a_l, a_r, b_K_l, b_K_r = calc_Kab_CPML(halo, dt, npower, d0, alpha_max, K_max, "ongrd")
        a_hl, a_hr, b_K_hl, b_K_hr = calc_Kab_CPML(halo, dt, npower, d0, alpha_max, K_max, "halfgrd")
        if ax == 2 && freetop
            a_l .= 0.0; a_hl .= 0.0; b_K_l .= 1.0; b_K_hl .= 1.0
        end
        append!(out, a_l, a_r, b_K_l, b_K_r, a_hl, a_hr, b_K_hl, b_K_hr)
    end
    return out
end

# The do_save branch of solve3D (acoustic_3D_xPU.jl:375-379,479-498): the time
# loop as a plan run with awc_plan_run_snapshots, writing pcur and the
# reference's metadata to save_dir/{save_name}_it{it}.h5 after every step it
# with it % nsave == 0 (HDF5.jl, which the reference's package loads too).
function _run_with_snapshots(ctx, prob, vel, coeffs, possrcs, dt2srctf, posrecs, ls, halo,
                             nsave, save_name, save_dir)
    HDF5 = Base.require(Base.PkgId(Base.UUID("f67ccb44-e63f-5c2f-98bd-6dc0ccc4ba2f"), "HDF5"))
    mkpath(save_dir)
    plan = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:awc_plan_create, LIBAWCPML), Cint,
               (Ptr{Cvoid}, Ref{AwcProblem}, Ptr{Float64}, Ptr{Float64}, Ptr{Int64},
                Ptr{Float64}, Ptr{Int64}, Ref{Ptr{Cvoid}}),
               ctx, prob, vel, coeffs, possrcs, dt2srctf, posrecs, plan)
    check(rc, ctx)
    ns = prob.ndim == 3 ? (prob.nx, prob.ny, prob.nz) : (prob.nx, prob.ny)
    chunk = 8
    buf = zeros(Float64, ns..., chunk)
    got = Ref{Int64}(0)
    try
        while (step = ccall((:awc_plan_step, LIBAWCPML), Int64, (Ptr{Cvoid},), plan[])) < prob.nt
            rc = ccall((:awc_plan_run_snapshots, LIBAWCPML), Cint,
                       (Ptr{Cvoid}, Int64, Int64, Ptr{Float64}, Int64, Ref{Int64}),
                       plan[], nsave * chunk - step % nsave, nsave, buf, chunk, got)
            check(rc, ctx)
            first_it = (step ÷ nsave + 1) * nsave
            for j = 1:got[]
                it = first_it + (j - 1) * nsave
                path = joinpath(save_dir, "$(save_name)_it$(it).h5")
                isfile(path) && rm(path)
                HDF5.h5write(path, "lx", ls[1])
                HDF5.h5write(path, "ly", ls[2])
                length(ls) == 3 && HDF5.h5write(path, "lz", ls[3])
                HDF5.h5write(path, "halo", halo)
                HDF5.h5write(path, "pcur", selectdim(buf, length(ns) + 1, j) |> collect)
                HDF5.h5write(path, "possrcs", possrcs)
                HDF5.h5write(path, "posrecs", posrecs)
            end
        end
        traces = zeros(Float64, prob.nt, prob.nrec)
        pend = zeros(Float64, ns)
        check(ccall((:awc_plan_traces, LIBAWCPML), Cint, (Ptr{Cvoid}, Ptr{Float64}), plan[],
                    traces), ctx)
        check(ccall((:awc_plan_field, LIBAWCPML), Cint, (Ptr{Cvoid}, Ptr{Float64}), plan[],
                    pend), ctx)
        return traces, pend
    finally
        ccall((:awc_plan_destroy, LIBAWCPML), Cvoid, (Ptr{Cvoid},), plan[])
    end
end

function _solve(ls::NTuple{N,Real}, lt::Real, vel::Array{<:Real,N}, srcs::Sources,
                recs::Receivers; halo::Integer=20, rcoef::Real=0.0001, ppw::Real=10.0,
                freetop::Bool=true, precision::Symbol=:f64, dt=nothing, nt=nothing,
                device::Integer=0, do_save::Bool=false, nsave::Integer=5,
                save_name::String="acoustic3D_xPU",
                save_dir::String=joinpath("simulations", "tmp")) where {N}
    f0 = srcs.freqdomain
    vel_max = maximum(vel)
    ns = size(vel)
    ds = ntuple(a -> ls[a] / (ns[a] - 1), N)
    dt = dt === nothing ? sqrt(N) / (vel_max * sum(1 ./ ds)) / 2 : Float64(dt)
    nt = nt === nothing ? ceil(Int, lt / dt) : Int(nt)
    times = collect(range(0.0, step=dt, length=nt))
    @assert sqrt(sum(ds .^ 2)) <= vel_max / (ppw * f0) "Not enough points per wavelength!"
    dt2srctf = zeros(nt, srcs.n)
    for s = 1:srcs.n
        dt2srctf[:, s] .= (dt^2 / prod(ds)) .* srcs.srctfs[s].(times, srcs.t0s[s], f0)
    end
    snap(pos) = round.(Int64, pos ./ reshape(collect(ds), 1, N) .+ 1, RoundNearestTiesUp)
    possrcs, posrecs = snap(srcs.positions), snap(recs.positions)
    @assert all(all(1 .<= possrcs[:, a] .<= ns[a]) for a in 1:N) "At least one source is not inside the model!"
    @assert all(all(1 .<= posrecs[:, a] .<= ns[a]) for a in 1:N) "At least one receiver is not inside the model!"
    coeffs = packed_coeffs(halo, dt, ds, vel_max, rcoef, f0, freetop)
    prob = AwcProblem(Int32(N), precision == :f32 ? AWC_F32 : AWC_F64, ns[1],
                      N >= 2 ? ns[2] : 1, N == 3 ? ns[3] : 1, Int32(halo), Int32(freetop),
                      ds[1], N >= 2 ? ds[2] : 1.0, N == 3 ? ds[3] : 1.0, dt, nt, srcs.n, recs.n)
    ctx = context(device)
    if do_save
        traces, pend = _run_with_snapshots(ctx, prob, Array{Float64}(vel), coeffs, possrcs,
                                           dt2srctf, posrecs, ls, halo, nsave, save_name,
                                           save_dir)
        recs.seismograms = traces
        return pend
    end
    traces = zeros(Float64, nt, recs.n)
    pend = zeros(Float64, ns)
    rc = ccall((:awc_forward, LIBAWCPML), Cint,
               (Ptr{Cvoid}, Ref{AwcProblem}, Ptr{Float64}, Ptr{Float64}, Ptr{Int64},
                Ptr{Float64}, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}),
               ctx, prob, Array{Float64}(vel), coeffs, possrcs, dt2srctf, posrecs, traces, pend)
    check(rc, ctx)
    recs.seismograms = traces
    return pend
end

"""
    solve2D(lx, ly, lt, vel, srcs, recs; halo=20, rcoef=0.0001, ppw=10.0, freetop=true,
            precision=:f64, dt=nothing, nt=nothing, device=0)

`Acoustic2D_CUDA.solve2D` with the time loop on a B200. Returns the final
pressure field and fills `recs.seismograms`. `precision=:f32` selects the
production single-precision build; `dt`/`nt` fix the time step explicitly.
"""
solve2D(lx::Real, ly::Real, lt::Real, vel::Matrix{<:Real}, srcs::Sources, recs::Receivers; kw...) =
    _solve((lx, ly), lt, vel, srcs, recs; kw...)

"""
    solve1D(lx, lt, vel, srcs, recs; halo=20, rcoef=0.0001, ppw=10.0, precision=:f64,
            dt=nothing, nt=nothing, device=0)

`Acoustic1D.solve1D` (src/shared/acoustic_1D.jl:89-297) with the time loop on
a B200 (awc_forward with ndim = 1; no free top in 1D).
"""
solve1D(lx::Real, lt::Real, vel::Vector{<:Real}, srcs::Sources, recs::Receivers; kw...) =
    _solve((lx,), lt, vel, srcs, recs; freetop=false, kw...)

"""
    solve3D(lx, ly, lz, lt, vel, srcs, recs; halo=20, rcoef=0.0001, ppw=10.0, freetop=true,
            precision=:f64, dt=nothing, nt=nothing, device=0, do_save=false, nsave=5,
            save_name="acoustic3D_xPU", save_dir="simulations/tmp")

`Acoustic3D_CUDA.solve3D` with the time loop on a B200 (depth on the second
axis, free top at j = 1). `do_save` writes the reference's HDF5 snapshot
files (pcur and metadata after every nsave-th step).
"""
solve3D(lx::Real, ly::Real, lz::Real, lt::Real, vel::Array{<:Real,3}, srcs::Sources,
        recs::Receivers; kw...) = _solve((lx, ly, lz), lt, vel, srcs, recs; kw...)

"""
    misfit_gradient(ls, vel, srcs, recs, observed; dt, nt, halo=20, rcoef=0.0001,
                    freetop=true, precision=:f64, checkpoint_every=50, device=0)

Misfit J = 1/2 Σ (traces - observed)² of one shot (set up as in solve2D/solve3D,
with a fixed `dt` and `nt`) and dJ/d(c²) per node, by the discrete adjoint in
libawcpml (`awc_misfit_gradient`). No counterpart in the reference.
"""
function misfit_gradient(ls::NTuple{N,Real}, vel::Array{<:Real,N}, srcs::Sources,
                         recs::Receivers, observed::Matrix{Float64}; dt::Real, nt::Integer,
                         halo::Integer=20, rcoef::Real=0.0001, freetop::Bool=true,
                         precision::Symbol=:f64, checkpoint_every::Integer=50,
                         device::Integer=0) where {N}
    f0 = srcs.freqdomain
    vel_max = maximum(vel)
    ns = size(vel)
    ds = ntuple(a -> ls[a] / (ns[a] - 1), N)
    times = collect(range(0.0, step=dt, length=nt))
    dt2srctf = zeros(nt, srcs.n)
    for s = 1:srcs.n
        dt2srctf[:, s] .= (dt^2 / prod(ds)) .* srcs.srctfs[s].(times, srcs.t0s[s], f0)
    end
    snap(pos) = round.(Int64, pos ./ reshape(collect(ds), 1, N) .+ 1, RoundNearestTiesUp)
    possrcs, posrecs = snap(srcs.positions), snap(recs.positions)
    coeffs = packed_coeffs(halo, dt, ds, vel_max, rcoef, f0, freetop)
    prob = AwcProblem(Int32(N), precision == :f32 ? AWC_F32 : AWC_F64, ns[1], ns[2],
                      N == 3 ? ns[3] : 1, Int32(halo), Int32(freetop), ds[1], ds[2],
                      N == 3 ? ds[3] : 1.0, Float64(dt), nt, srcs.n, recs.n)
    J = Ref{Float64}(0.0)
    grad = zeros(Float64, ns)
    traces = zeros(Float64, nt, recs.n)
    ctx = context(device)
    rc = ccall((:awc_misfit_gradient, LIBAWCPML), Cint,
               (Ptr{Cvoid}, Ref{AwcProblem}, Ptr{Float64}, Ptr{Float64}, Ptr{Int64},
                Ptr{Float64}, Ptr{Int64}, Ptr{Float64}, Int32, Ref{Float64}, Ptr{Float64},
                Ptr{Float64}),
               ctx, prob, Array{Float64}(vel), coeffs, possrcs, dt2srctf, posrecs, observed,
               Int32(checkpoint_every), J, grad, traces)
    check(rc, ctx)
    recs.seismograms = traces
    return J[], grad
end

"""
    misfit_gradient_shots(ls, vel, shots, recs, observed; dt, nt, halo=20, rcoef=0.0001,
                          freetop=true, precision=:f64, checkpoint_every=50, device=0)

Σ over the shots (a vector of `Sources` with the same number of sources and
the same frequency, over one model and one receiver set; `observed[s]` is shot
s's nt x nrec data) of the misfit and dJ/d(c²): one call of
`awc_misfit_gradient_shots`, which uploads the model once and sums the
gradients on the device; equal to summing `misfit_gradient` over the shots.
No counterpart in the reference.
"""
function misfit_gradient_shots(ls::NTuple{N,Real}, vel::Array{<:Real,N}, shots::Vector{Sources},
                               recs::Receivers, observed::Vector{Matrix{Float64}}; dt::Real,
                               nt::Integer, halo::Integer=20, rcoef::Real=0.0001,
                               freetop::Bool=true, precision::Symbol=:f64,
                               checkpoint_every::Integer=50, device::Integer=0) where {N}
    nshot = length(shots)
    nshot == length(observed) || error("one observed matrix per shot")
    nsrc = shots[1].n
    all(s -> s.n == nsrc, shots) || error("every shot needs the same number of sources")
    f0 = shots[1].freqdomain
    vel_max = maximum(vel)
    ns = size(vel)
    ds = ntuple(a -> ls[a] / (ns[a] - 1), N)
    times = collect(range(0.0, step=dt, length=nt))
    snap(pos) = round.(Int64, pos ./ reshape(collect(ds), 1, N) .+ 1, RoundNearestTiesUp)
    possrcs = zeros(Int64, nsrc, N, nshot)
    dt2srctf = zeros(nt, nsrc, nshot)
    for (k, srcs) in enumerate(shots)
        possrcs[:, :, k] .= snap(srcs.positions)
        for s = 1:nsrc
            dt2srctf[:, s, k] .= (dt^2 / prod(ds)) .* srcs.srctfs[s].(times, srcs.t0s[s], f0)
        end
    end
    obs = cat(observed...; dims=3)
    coeffs = packed_coeffs(halo, dt, ds, vel_max, rcoef, f0, freetop)
    prob = AwcProblem(Int32(N), precision == :f32 ? AWC_F32 : AWC_F64, ns[1], ns[2],
                      N == 3 ? ns[3] : 1, Int32(halo), Int32(freetop), ds[1], ds[2],
                      N == 3 ? ds[3] : 1.0, Float64(dt), nt, nsrc, recs.n)
    J = Ref{Float64}(0.0)
    grad = zeros(Float64, ns)
    ctx = context(device)
    rc = ccall((:awc_misfit_gradient_shots, LIBAWCPML), Cint,
               (Ptr{Cvoid}, Ref{AwcProblem}, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Int64},
                Ptr{Float64}, Ptr{Int64}, Ptr{Float64}, Int32, Ref{Float64}, Ptr{Float64}),
               ctx, prob, Int32(nshot), Array{Float64}(vel), coeffs, possrcs, dt2srctf,
               snap(recs.positions), obs, Int32(checkpoint_every), J, grad)
    check(rc, ctx)
    return J[], grad
end

"""
    misfit(c2, ls, srcs, recs, observed; kw...)

J as a function of c² (the squared velocity). With ChainRulesCore loaded, its
rrule returns dJ/d(c²) from the adjoint, so Zygote and friends differentiate
through the solver.
"""
misfit(c2::Array{<:Real,N}, ls::NTuple{N,Real}, srcs::Sources, recs::Receivers,
       observed::Matrix{Float64}; kw...) where {N} =
    misfit_gradient(ls, sqrt.(c2), srcs, recs, observed; kw...)[1]

try
    @eval import ChainRulesCore
catch
end
if isdefined(@__MODULE__, :ChainRulesCore)
    @eval function ChainRulesCore.rrule(::typeof(misfit), c2::Array{<:Real,N}, ls::NTuple{N,Real},
                                        srcs::Sources, recs::Receivers,
                                        observed::Matrix{Float64}; kw...) where {N}
        J, g = misfit_gradient(ls, sqrt.(c2), srcs, recs, observed; kw...)
        nt = ChainRulesCore.NoTangent()
        misfit_pullback(ΔJ) = (nt, ChainRulesCore.unthunk(ΔJ) .* g, nt, nt, nt, nt)
        return J, misfit_pullback
    end
end

end # module
