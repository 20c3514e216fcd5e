"""
    TestParticleB200

Drop-in B200 ensemble algorithm for TestParticle.jl: `EnsembleB200()` routes
`TestParticle.solve(prob, Boris() | MultistepBoris{N}(; n) | AdaptiveBoris(; safety),
EnsembleB200(); dt, savestepinterval, trajectories, ...)` and
`TestParticle.solve(prob::TraceGCProblem, EnsembleB200(); alg = :rk4 | :rk45, ...)`
to libtpb200.so through `ccall`, and returns the reference's `EnsembleSolution`
(one `ODESolution` per trajectory, `LinearInterpolation`, retcodes).

It adds methods to the reference's own dispatch points
(`_solve(::EnsembleAlg, ::TraceProblem, ...)`, src/boris/boris.jl:137-318;
`_solve_adaptive(::EnsembleAlg, ...)`, src/boris/adaptive_boris.jl:40-139;
`_solve(::EnsembleAlg, ::TraceGCProblem, ...)`, src/gc/gc_solver.jl:104-161).

Fields must be the reference's `ZeroField`, a trilinear `FieldInterpolator` on
uniform axes (what `prepare(x, y, z, E, B)` and `build_interpolator(CartesianGrid,
A, x, y, z, 1, bc)` build), or one of the device-evaluable types below
(closures cannot run on the device); these are ordinary callables, so the
reference CPU solver runs on the same objects for a like-for-like comparison.
`isoutside` must be a `Terminate` predicate.
"""
module TestParticleB200

using TestParticle
import TestParticle: _solve, _solve_adaptive, TraceProblem, TraceGCProblem, Boris, MultistepBoris,
    ZeroField, Field
using SciMLBase: BasicEnsembleAlgorithm, EnsembleSolution, EnsembleContext, ReturnCode,
    LinearInterpolation, build_solution
using StaticArrays: SVector
import ChainRulesCore

export EnsembleB200, UniformField, AffineField, DipoleField, B200Grid, Terminate, boris_final_state, grid_of

const libtpb200 = get(ENV, "TPB200_LIB", joinpath(@__DIR__, "..", "..", "..", "libtpb200.so"))

# ------------------------------------------------------------------ ensemble
"""
    EnsembleB200(; device = 0, precision = :fp64, schedule = :auto)

`precision = :fp64` is the drop-in path (reference operation order);
`:fp32c` the float32 push with compensated positions and velocities.
"""
struct EnsembleB200 <: BasicEnsembleAlgorithm
    device::Int
    precision::Symbol
    schedule::Symbol
end
EnsembleB200(; device = 0, precision = :fp64, schedule = :auto) = EnsembleB200(device, precision, schedule)

# ------------------------------------------------------------------ fields
"Uniform field F(x) = v."
struct UniformField{T} <: Function
    v::SVector{3, T}
end
(f::UniformField)(x) = f.v

"Affine field F(x, t) = v + J x + rate t."
struct AffineField{T} <: Function
    v::SVector{3, T}
    J::NTuple{9, T}       # row-major
    rate::SVector{3, T}
end
function (f::AffineField)(x, t)
    J = f.J
    return f.v + SVector(J[1] * x[1] + J[2] * x[2] + J[3] * x[3],
        J[4] * x[1] + J[5] * x[2] + J[6] * x[3],
        J[7] * x[1] + J[8] * x[2] + J[9] * x[3]) + f.rate * t
end

"Point dipole B = coef (3 (m.rhat) rhat - m) / |x - c|^3."
struct DipoleField{T} <: Function
    m::SVector{3, T}
    c::SVector{3, T}
    coef::T
end
DipoleField(m; c = SVector(0.0, 0.0, 0.0), coef = TestParticle.μ₀ / (4π)) =
    DipoleField(SVector{3}(Float64.(m)), SVector{3}(Float64.(c)), Float64(coef))
function (f::DipoleField)(x)
    d = x - f.c
    r = sqrt(d[1]^2 + d[2]^2 + d[3]^2)
    rh = d / r
    return f.coef * (3 * (f.m' * rh) * rh - f.m) / r^3
end

"""
    B200Grid(A, x, y, z; bc = :fill_nan | :clamp | :periodic)

Trilinear interpolator of a (3, nx, ny, nz) Float32/Float64 array on uniform
ranges.  This callable evaluates in Float64 with the operation order of the
device's FP64 path (`u = (x - x0) * (1/dx)`, then `a + f * (b - a)` along x,
then y, then z), so the two agree bit for bit; the device's FP32C path
evaluates the same formula in Float32 arithmetic and differs in the last bits.
"""
struct B200Grid{T} <: Function
    A::Array{T, 4}
    origin::NTuple{3, Float64}
    spacing::NTuple{3, Float64}
    bc::Int32
end
function B200Grid(A::Array{T, 4}, x::AbstractRange, y::AbstractRange, z::AbstractRange; bc = :fill_nan) where {T}
    code = bc === :fill_nan ? Int32(0) : bc === :clamp ? Int32(1) : bc === :periodic ? Int32(2) :
        throw(ArgumentError("bc must be :fill_nan, :clamp or :periodic"))
    return B200Grid{T}(A, (first(x), first(y), first(z)), (step(x), step(y), step(z)), code)
end
function (g::B200Grid)(x)
    idx = ntuple(3) do a
        n = size(g.A, a + 1)
        u = (x[a] - g.origin[a]) * (1 / g.spacing[a])
        if g.bc == 2
            fl = floor(u); i = mod(Int(fl), n)
            (i, i + 1 == n ? 0 : i + 1, u - fl)
        else
            g.bc == 1 && (u = clamp(u, 0.0, n - 1.0))
            (g.bc == 0 && !(0 <= u <= n - 1)) && return nothing
            i = min(Int(floor(u)), n - 2)
            (i, i + 1, u - i)
        end
    end
    any(isnothing, idx) && return SVector(NaN, NaN, NaN)
    (i0, i1, fx), (j0, j1, fy), (k0, k1, fz) = idx
    lerp(a, b, f) = a + f * (b - a)
    c(v, i, j, k) = Float64(g.A[v, i + 1, j + 1, k + 1])
    return SVector(ntuple(v -> lerp(lerp(lerp(c(v, i0, j0, k0), c(v, i1, j0, k0), fx),
        lerp(c(v, i0, j1, k0), c(v, i1, j1, k0), fx), fy),
        lerp(lerp(c(v, i0, j0, k1), c(v, i1, j0, k1), fx),
            lerp(c(v, i0, j1, k1), c(v, i1, j1, k1), fx), fy), fz), 3))
end

# ------------------------------------------------------------------ termination
"isoutside(u, p, t) as flags: shell rmin/rmax, box lo/hi, NaN, t > tmax."
Base.@kwdef struct Terminate <: Function
    flags::Int32 = 0
    rmin::Float64 = -Inf
    rmax::Float64 = Inf
    lo::NTuple{3, Float64} = (-Inf, -Inf, -Inf)
    hi::NTuple{3, Float64} = (Inf, Inf, Inf)
    tmax::Float64 = Inf
end
function (T::Terminate)(u, p, t)
    (T.flags & 4 != 0) && any(isnan, u) && return true
    if T.flags & 1 != 0
        r = sqrt(u[1]^2 + u[2]^2 + u[3]^2)
        (r < T.rmin || r > T.rmax) && return true
    end
    (T.flags & 2 != 0) && any(c -> u[c] < T.lo[c] || u[c] > T.hi[c], 1:3) && return true
    (T.flags & 8 != 0) && t > T.tmax && return true
    return false
end

# ------------------------------------------------------------------ C descriptors (include/tp_abi.h)
struct TpFieldDesc
    kind::Int32; bc::Int32; dtype::Int32; reserved::Int32
    value::NTuple{3, Float64}; jac::NTuple{9, Float64}; rate::NTuple{3, Float64}
    moment::NTuple{3, Float64}; center::NTuple{3, Float64}; coef::Float64
    n::NTuple{3, Int64}; origin::NTuple{3, Float64}; spacing::NTuple{3, Float64}
    data::Ptr{Cvoid}
    # grid tail: order, geometry, ndim, dir, per-axis node coordinates (all
    # zero: trilinear on a uniform Cartesian 3-D grid)
    order::Int32; geometry::Int32; ndim::Int32; dir::Int32
    axis::NTuple{3, Ptr{Float64}}
    quad::NTuple{27, Float64}   # QUADRATIC: quad_ijk at 9i + 3j + k (0-based)
    nseries::Int64              # SERIES: snapshots, their times and descriptors
    series_times::Ptr{Float64}
    series::Ptr{Cvoid}
end
TpFieldDesc(kind, bc, dtype, reserved, value, jac, rate, moment, center, coef, n, origin, spacing, data) =
    TpFieldDesc(kind, bc, dtype, reserved, value, jac, rate, moment, center, coef, n, origin, spacing, data,
        0, 0, 0, 0, (Ptr{Float64}(C_NULL), Ptr{Float64}(C_NULL), Ptr{Float64}(C_NULL)), ntuple(_ -> 0.0, 27),
        0, Ptr{Float64}(C_NULL), C_NULL)
struct TpTermDesc
    flags::Int32; reserved::Int32; rmin::Float64; rmax::Float64
    lo::NTuple{3, Float64}; hi::NTuple{3, Float64}; tmax::Float64
end
struct TpRunDesc
    alg::Int32; order::Int32; nsub::Int32; precision::Int32
    safety::Float64; t0::Float64; t1::Float64; dt::Float64; q2m::Float64; m::Float64
    savestepinterval::Int64; maxiters::Int64
    save_start::Int32; save_end::Int32; save_everystep::Int32; save_fields::Int32
    term::TpTermDesc; step_cap::Int64; schedule::Int32; block::Int32; budget_s::Float64
    save_work::Int32; particles_per_thread::Int32
end
struct TpGCDesc
    alg::Int32; precision::Int32; t0::Float64; t1::Float64; dt::Float64
    dt_given::Int32; reserved::Int32; q::Float64; q2m::Float64; mu::Float64
    abstol::Float64; reltol::Float64; savestepinterval::Int64; maxiters::Int64
    save_start::Int32; save_end::Int32; save_everystep::Int32; save_fields::Int32
    term::TpTermDesc; block::Int32; reserved2::Int32; budget_s::Float64
    save_work::Int32; reserved3::Int32
end

const Z3 = (0.0, 0.0, 0.0)
const Z9 = ntuple(_ -> 0.0, 9)
unwrap(f::Field) = f.field_function
unwrap(f) = f
fdesc(::ZeroField) = TpFieldDesc(0, 0, 0, 0, Z3, Z9, Z3, Z3, Z3, 0.0, (0, 0, 0), Z3, Z3, C_NULL)
fdesc(f::UniformField) = TpFieldDesc(1, 0, 0, 0, Tuple(Float64.(f.v)), Z9, Z3, Z3, Z3, 0.0, (0, 0, 0), Z3, Z3, C_NULL)
fdesc(f::AffineField) = TpFieldDesc(2, 0, 0, 0, Tuple(Float64.(f.v)), Float64.(f.J), Tuple(Float64.(f.rate)),
    Z3, Z3, 0.0, (0, 0, 0), Z3, Z3, C_NULL)
fdesc(f::DipoleField) = TpFieldDesc(3, 0, 0, 0, Z3, Z9, Z3, Tuple(f.m), Tuple(f.c), f.coef, (0, 0, 0), Z3, Z3, C_NULL)
fdesc(g::B200Grid{T}) where {T} = TpFieldDesc(4, g.bc, T === Float32 ? 0 : 1, 0, Z3, Z9, Z3, Z3, Z3, 0.0,
    Int64.(size(g.A)[2:4]), g.origin, g.spacing, pointer(g.A))
fdesc(f) = throw(ArgumentError("field not supported by EnsembleB200: $(typeof(f)); use ZeroField, " *
    "UniformField, AffineField, DipoleField, B200Grid or a trilinear FieldInterpolator"))

# ------------------------------------------------------------------ the reference's gridded field
# A user's gridded problem holds `Field(FieldInterpolator(itp))` with `itp` the
# FastInterpolations interpolant that build_interpolator(CartesianGrid, A, x, y, z,
# 1, bc) made (src/utility/interpolation.jl:15-36,119-148,217-235).  The device
# needs its node array, uniform axes and boundary condition.  They are found by
# type among the interpolant's properties (FastInterpolations is a dependency of
# the reference, so its field names are not relied on): the axes are a tuple of
# three vectors, the nodes an array of SVector{3} (the reinterpreted (3, nx, ny,
# nz) array, whose parent is used when it is one), and the boundary condition a
# PeriodicBC / WrapExtrap / ClampExtrap / FillExtrap(NaN) value.  The result is
# then checked against the interpolant itself at a few interior points, so a
# cubic or nearest-node interpolant, or a non-uniform axis, is an ArgumentError
# rather than a silently different field.
function _walk(f, x, depth)
    f(x) && return x
    depth == 0 && return nothing
    isstructtype(typeof(x)) || return nothing
    for name in propertynames(x)
        v = try
            getproperty(x, name)
        catch
            continue
        end
        r = _walk(f, v, depth - 1)
        isnothing(r) || return r
    end
    if x isa Tuple
        for v in x
            r = _walk(f, v, depth - 1)
            isnothing(r) || return r
        end
    end
    return nothing
end

_is_axes(v) = v isa Tuple && length(v) == 3 && all(a -> a isa AbstractVector{<:Real} && length(a) >= 2, v)
_is_nodes(v) = v isa AbstractArray{<:SVector{3, <:AbstractFloat}, 3}
_is_bc(v) = v isa TestParticle.PeriodicBC || v isa TestParticle.WrapExtrap || v isa TestParticle.ClampExtrap ||
    v isa TestParticle.FillExtrap

function _uniform_axis(a::AbstractVector{<:Real})
    a isa AbstractRange && return Float64(first(a)), Float64(step(a))
    n = length(a)
    x0 = Float64(a[1])
    h = (Float64(a[end]) - x0) / (n - 1)
    for k in 1:n
        abs(Float64(a[k]) - (x0 + (k - 1) * h)) <= 1e-12 * abs(h) ||
            throw(ArgumentError("EnsembleB200: grid axis is not uniform (node $k); only uniform CartesianGrid " *
                "axes are supported on the device"))
    end
    return x0, h
end

function _bc_code(bc)
    if bc isa TestParticle.WrapExtrap
        return Int32(2)
    elseif bc isa TestParticle.PeriodicBC
        ep = hasproperty(bc, :endpoint) ? getproperty(bc, :endpoint) : :exclusive
        return ep === :inclusive ? Int32(3) : Int32(2)
    elseif bc isa TestParticle.ClampExtrap
        return Int32(1)
    else  # FillExtrap: the device fills with NaN only
        fv = hasproperty(bc, :fill_value) ? getproperty(bc, :fill_value) : NaN
        all(isnan, fv) || throw(ArgumentError("EnsembleB200: FillExtrap supports NaN fill values only"))
        return Int32(0)
    end
end

"""
    grid_of(fi::TestParticle.FieldInterpolator) -> B200Grid

The device form of the reference's trilinear `FieldInterpolator`, sharing its
node memory (no copy when the interpolant keeps the caller's array or an
`Array{SVector{3}}`).  Used by `EnsembleB200` for every `FieldInterpolator` it
meets; throws `ArgumentError` for interpolants the device cannot reproduce.
"""
function grid_of(fi::TestParticle.FieldInterpolator)
    itp = fi.itp
    axes = _walk(_is_axes, itp, 3)
    V = _walk(_is_nodes, itp, 3)
    bc = _walk(_is_bc, itp, 3)
    (isnothing(axes) || isnothing(V)) &&
        throw(ArgumentError("EnsembleB200: cannot find the axes and node array of $(typeof(itp))"))
    isnothing(bc) && throw(ArgumentError("EnsembleB200: boundary condition of $(typeof(itp)) is not one of " *
        "PeriodicBC, WrapExtrap, ClampExtrap or FillExtrap(NaN)"))
    T = eltype(eltype(V))
    nx, ny, nz = size(V)
    P = parent(V)
    A = if P isa Array{T, 4} && size(P) == (3, nx, ny, nz)
        P                                    # the (3, nx, ny, nz) array itself
    elseif V isa Array
        unsafe_wrap(Array, Ptr{T}(pointer(V)), (3, nx, ny, nz))  # same bytes, V kept alive by fi
    else
        reshape(collect(reinterpret(T, vec(collect(V)))), 3, nx, ny, nz)
    end
    (x0, hx), (y0, hy), (z0, hz) = map(_uniform_axis, axes)
    code = _bc_code(bc)
    code == 3 && throw(ArgumentError("EnsembleB200: PeriodicBC(endpoint = :inclusive) needs the general-grid " *
        "descriptor; use endpoint = :exclusive"))
    g = B200Grid{T}(A, (x0, y0, z0), (hx, hy, hz), code)
    # the interpolant itself is the reference: it must agree with the trilinear form
    for (a, b, c) in ((0.37, 0.61, 0.23), (0.5, 0.5, 0.5), (0.91, 0.13, 0.77))
        x = SVector(x0 + (a * (nx - 1)) * hx, y0 + (b * (ny - 1)) * hy, z0 + (c * (nz - 1)) * hz)
        ref = fi(x)
        dev = g(x)
        tol = 64 * eps(float(promote_type(T, eltype(ref)))) * (1 + maximum(abs, ref))
        maximum(abs, ref - dev) <= tol || throw(ArgumentError("EnsembleB200: $(typeof(itp)) is not a trilinear " *
            "interpolant on uniform axes (order 1); the device supports order 1 here"))
    end
    return g
end

fdesc(fi::TestParticle.FieldInterpolator) = fdesc(grid_of(fi))
device_view(f) = f
device_view(fi::TestParticle.FieldInterpolator) = grid_of(fi)

termdesc(::typeof(TestParticle.ODE_DEFAULT_ISOUTOFDOMAIN)) = TpTermDesc(0, 0, -Inf, Inf, (-Inf, -Inf, -Inf), (Inf, Inf, Inf), Inf)
termdesc(T::Terminate) = TpTermDesc(T.flags, 0, T.rmin, T.rmax, T.lo, T.hi, T.tmax)
termdesc(f) = throw(ArgumentError("isoutside must be a TestParticleB200.Terminate predicate on the B200"))

# ------------------------------------------------------------------ library calls
const CTX = Dict{Int, Ptr{Cvoid}}()
function context(dev::Int)
    get!(CTX, dev) do
        r = Ref{Ptr{Cvoid}}(C_NULL)
        st = ccall((:tp_ctx_create, libtpb200), Cint, (Cint, Ref{Ptr{Cvoid}}), dev, r)
        st == 0 || error("tp_ctx_create failed ($st)")
        r[]
    end
end
function check(ctx, st, what)
    st == 0 && return
    msg = unsafe_string(ccall((:tp_last_error, libtpb200), Cstring, (Ptr{Cvoid},), ctx))
    st == -1 ? throw(ArgumentError("$what: $msg")) : error("$what: $msg (status $st)")
end
function field_handle(ctx, f)
    g = device_view(f)   # grids are copied to the device inside tp_field_create
    d = Ref(fdesc(g))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve f g check(ctx, ccall((:tp_field_create, libtpb200), Cint,
        (Ptr{Cvoid}, Ref{TpFieldDesc}, Ref{Ptr{Cvoid}}), ctx, d, h), "tp_field_create")
    return h[]
end
free_field(h) = ccall((:tp_field_destroy, libtpb200), Cvoid, (Ptr{Cvoid},), h)

# the (6, N) initial-state table: prob_func applied on the host (boris_kernel.jl:290-294)
function initial_table(prob, trajectories, seed)
    U = Matrix{Float64}(undef, length(prob.u0), trajectories)
    for i in 1:trajectories
        rng = isnothing(seed) ? TestParticle.default_rng() : TestParticle.Xoshiro(TestParticle._rng_seed(seed, i))
        U[:, i] .= prob.prob_func(prob, EnsembleContext(i, 1, 0, nothing, rng, seed)).u0
    end
    return U
end

const RETCODES = Dict(1 => ReturnCode.Success, 2 => ReturnCode.Terminated, 3 => ReturnCode.MaxIters,
    0 => ReturnCode.Default)

function collect_result(ctx, res, prob, alg_name, T)
    n = Ref{Int64}(0); w = Ref{Int32}(0); tot = Ref{Int64}(0)
    ccall((:tp_result_info, libtpb200), Cint, (Ptr{Cvoid}, Ref{Int64}, Ref{Int32}, Ref{Int64}), res, n, w, tot)
    ns = Vector{Int32}(undef, n[]); rc = Vector{Int8}(undef, n[]); st = Vector{Int64}(undef, n[])
    t = Vector{Float64}(undef, tot[]); u = Matrix{Float64}(undef, w[], tot[])
    ccall((:tp_result_copy, libtpb200), Cint, (Ptr{Cvoid}, Ptr{Int32}, Ptr{Int8}, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}),
        res, ns, rc, st, t, u)
    ms = Ref{Float64}(0.0)
    ccall((:tp_result_elapsed_ms, libtpb200), Cint, (Ptr{Cvoid}, Ref{Float64}), res, ms)
    ccall((:tp_result_destroy, libtpb200), Cvoid, (Ptr{Cvoid},), res)
    W = Int(w[])
    sols = Vector{Any}(undef, n[])
    off = 0
    for i in 1:n[]
        r = (off + 1):(off + ns[i])
        ti = t[r]
        ui = [SVector{W, T}(view(u, :, k)) for k in r]
        sols[i] = build_solution(prob, alg_name, ti, ui; interp = LinearInterpolation(ti, ui),
            retcode = RETCODES[Int(rc[i])], stats = nothing)
        off += ns[i]
    end
    return EnsembleSolution([s for s in sols], ms[] * 1e-3, true)
end

function boris_run(ens::EnsembleB200, prob::TraceProblem, alg, adaptive, trajectories, dt, savestepinterval,
        isoutside, save_start, save_end, save_everystep, save_fields, save_work, maxiters, seed, alg_name)
    ctx = context(ens.device)
    q2m, m, E, B, _ = prob.p
    hE = field_handle(ctx, unwrap(E)); hB = field_handle(ctx, unwrap(B))
    try
        multi = alg isa MultistepBoris
        N = multi ? typeof(alg).parameters[1] : 2
        desc = Ref(TpRunDesc(adaptive ? (multi ? 3 : 2) : (multi ? 1 : 0), N, multi ? alg.n : 1,
            ens.precision === :fp32c ? 1 : 0, alg.safety, prob.tspan[1], prob.tspan[2],
            isnothing(dt) ? 0.0 : dt, q2m, m, savestepinterval, maxiters,
            save_start, save_end, save_everystep, save_fields, termdesc(isoutside), 0,
            ens.schedule === :static ? 1 : ens.schedule === :queue ? 2 : 0, 0, 0.0, save_work, 0))
        U = initial_table(prob, trajectories, seed)
        res = Ref{Ptr{Cvoid}}(C_NULL)
        st = ccall((:tp_boris_run, libtpb200), Cint,
            (Ptr{Cvoid}, Ref{TpRunDesc}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64,
                Ref{Ptr{Cvoid}}), ctx, desc, hE, hB, U, C_NULL, C_NULL, trajectories, res)
        check(ctx, st, "tp_boris_run")
        return collect_result(ctx, res[], prob, alg_name, eltype(prob.u0))
    finally
        free_field(hE); free_field(hB)
    end
end

# ------------------------------------------------------------------ drop-in methods
function _solve(ens::EnsembleB200, prob::TraceProblem, alg::TestParticle.AbstractBoris, trajectories, dt,
        savestepinterval, isoutside, save_start, save_end, save_everystep,
        ::Val{SaveFields}, ::Val{SaveWork}, maxiters, batch_size, seed) where {SaveFields, SaveWork}
    name = alg isa MultistepBoris ? :multistep_boris : :boris
    return boris_run(ens, prob, alg, false, trajectories, dt, savestepinterval, isoutside, save_start,
        save_end, save_everystep, SaveFields, SaveWork, maxiters, seed, name)
end

function _solve_adaptive(ens::EnsembleB200, prob, trajectories, alg::TestParticle.AbstractBoris, savestepinterval,
        isoutside, save_start, save_end, save_everystep, ::Val{SaveFields}, ::Val{SaveWork},
        batch_size) where {SaveFields, SaveWork}
    name = alg isa Boris ? :adaptive_boris : :adaptive_multistep_boris
    return boris_run(ens, prob, alg, true, trajectories, nothing, savestepinterval, isoutside, save_start,
        save_end, save_everystep, SaveFields, SaveWork, typemax(Int64), nothing, name)
end

function _solve(ens::EnsembleB200, prob::TraceGCProblem, trajectories, dt, savestepinterval, isoutside,
        save_start, save_end, save_everystep, alg, abstol, reltol, maxiters,
        ::Val{SaveFields}, ::Val{SaveWork}, seed) where {SaveFields, SaveWork}
    ctx = context(ens.device)
    q, q2m, μ, E, B = prob.p
    hE = field_handle(ctx, unwrap(E)); hB = field_handle(ctx, unwrap(B))
    try
        desc = Ref(TpGCDesc(alg == :rk45 ? 1 : 0, ens.precision === :fp64 ? 0 : 1, prob.tspan[1], prob.tspan[2],
            isnothing(dt) ? 0.0 : dt, isnothing(dt) ? 0 : 1, 0, q, q2m, μ, abstol, reltol, savestepinterval,
            maxiters, save_start, save_end, save_everystep, SaveFields, termdesc(isoutside), 0, 0, 0.0,
            SaveWork, 0))
        Y = initial_table(prob, trajectories, seed)
        res = Ref{Ptr{Cvoid}}(C_NULL)
        st = ccall((:tp_gc_run, libtpb200), Cint,
            (Ptr{Cvoid}, Ref{TpGCDesc}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Ref{Ptr{Cvoid}}),
            ctx, desc, hE, hB, Y, C_NULL, C_NULL, C_NULL, C_NULL, C_NULL, trajectories, res)
        check(ctx, st, "tp_gc_run")
        return collect_result(ctx, res[], prob, alg == :rk45 ? :rk45 : :rk4, eltype(prob.u0))
    finally
        free_field(hE); free_field(hB)
    end
end

# ------------------------------------------------------------------ adjoint (tp_adjoint_*)
# Final save (x_N, v_N) of the fixed-step Boris solve as a differentiable
# function of the initial states and of the fields: forward
# tp_adjoint_forward (FP32C push, checkpoints every K steps), pullback
# tp_adjoint_backward.  Field cotangents are Tangent{B200Grid}(A = dA) for
# grids, Tangent{UniformField}(v = ...) and Tangent{DipoleField}(m = ...).
struct TpAdjDesc
    run::TpRunDesc
    checkpoint_every::Int64
end

function adj_desc(q2m, m, dt, tspan, K)
    nt = round(Int, abs((tspan[2] - tspan[1]) / dt))
    TpAdjDesc(TpRunDesc(0, 2, 1, 1, 0.0, tspan[1], tspan[2], dt, q2m, m, 1, max(1_000_000, nt),
        0, 1, 0, 0, termdesc(TestParticle.ODE_DEFAULT_ISOUTOFDOMAIN), 0, 0, 0, 0.0, 0, 0), K)
end

# tape and field handles of one recorded forward pass, released by the GC
mutable struct AdjointTape
    ctx::Ptr{Cvoid}; tape::Ptr{Cvoid}; hE::Ptr{Cvoid}; hB::Ptr{Cvoid}; n::Int
    function AdjointTape(ctx, tape, hE, hB, n)
        t = new(ctx, tape, hE, hB, n)
        finalizer(release!, t)
    end
end
function release!(t::AdjointTape)
    t.tape != C_NULL && ccall((:tp_tape_destroy, libtpb200), Cvoid, (Ptr{Cvoid},), t.tape)
    t.hE != C_NULL && free_field(t.hE)
    t.hB != C_NULL && free_field(t.hB)
    t.tape = t.hE = t.hB = C_NULL
    return nothing
end

function adjoint_forward(U0::Matrix{Float64}, E, B; q2m, m = 1.0, dt, tspan, checkpoint_every = 0, device = 0)
    size(U0, 1) == 6 || throw(ArgumentError("U0 must be a (6, N) matrix"))
    ctx = context(device)
    hE = field_handle(ctx, unwrap(E)); hB = field_handle(ctx, unwrap(B))
    n = size(U0, 2)
    UN = Matrix{Float64}(undef, 6, n)
    tape = Ref{Ptr{Cvoid}}(C_NULL)
    d = Ref(adj_desc(q2m, m, dt, tspan, checkpoint_every))
    st = ccall((:tp_adjoint_forward, libtpb200), Cint,
        (Ptr{Cvoid}, Ref{TpAdjDesc}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{Float64}, Ref{Ptr{Cvoid}}),
        ctx, d, hE, hB, U0, n, UN, tape)
    t = AdjointTape(ctx, tape[], hE, hB, n)
    if st != 0
        release!(t)
        check(ctx, st, "tp_adjoint_forward")
    end
    return UN, t
end

"""
    boris_final_state(U0, E, B; q2m, m, dt, tspan, checkpoint_every = 0, device = 0)

(6, N) final saves of `solve(TraceProblem(u0, tspan, (q2m, m, E, B, ...)), Boris(); dt)` for the
columns of `U0`, in the FP32C arithmetic of `EnsembleB200(; precision = :fp32c)`.  Differentiable
through its `ChainRulesCore.rrule` (discrete adjoint on the B200).
"""
function boris_final_state(U0::Matrix{Float64}, E, B; kw...)
    UN, t = adjoint_forward(U0, E, B; kw...)
    release!(t)
    return UN
end

field_cotangent(f::B200Grid, g, _) = ChainRulesCore.Tangent{typeof(f)}(; A = g)
# the reference's FieldInterpolator: the node gradient, shaped like the (3, nx, ny, nz) array
field_cotangent(f::TestParticle.FieldInterpolator, g, _) = g
field_cotangent(f::UniformField, _, p) = ChainRulesCore.Tangent{typeof(f)}(; v = SVector{3}(p))
field_cotangent(f::DipoleField, _, p) = ChainRulesCore.Tangent{typeof(f)}(; m = SVector{3}(p))
field_cotangent(f, _, _) = ChainRulesCore.NoTangent()

function ChainRulesCore.rrule(::typeof(boris_final_state), U0::Matrix{Float64}, E, B; kw...)
    UN, t = adjoint_forward(U0, E, B; kw...)
    function boris_final_state_pullback(dUN)
        G = Matrix{Float64}(ChainRulesCore.unthunk(dUN))
        dU0 = Matrix{Float64}(undef, 6, t.n)
        vE, vB = device_view(unwrap(E)), device_view(unwrap(B))
        gE = vE isa B200Grid ? Array{Float64}(undef, size(vE.A)) : nothing
        gB = vB isa B200Grid ? Array{Float64}(undef, size(vB.A)) : nothing
        gp = Vector{Float64}(undef, 6)
        st = ccall((:tp_adjoint_backward, libtpb200), Cint,
            (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
            t.tape, G, dU0, isnothing(gE) ? C_NULL : gE, isnothing(gB) ? C_NULL : gB, gp)
        check(t.ctx, st, "tp_adjoint_backward")
        return (ChainRulesCore.NoTangent(), dU0, field_cotangent(unwrap(E), gE, gp[1:3]),
            field_cotangent(unwrap(B), gB, gp[4:6]))
    end
    return UN, boris_final_state_pullback
end

end # module
