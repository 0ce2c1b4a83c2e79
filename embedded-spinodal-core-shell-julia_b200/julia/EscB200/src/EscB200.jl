"""
    EscB200

Julia front end of `libesc.so`, the B200 stepper for the time loop of
`run_simulation` (core_shell.jl:84-103).

`run_simulation_gpu` keeps the keyword arguments and the return value of
`run_simulation` (core_shell.jl:84-85, 103): `(c, history)`, `history` the
(steps+1)×6 matrix `[s*dt, mean c, energy, min c, max c, dissipation]` recorded
before each step.  A non-finite field raises
`error("Non-finite composition at step \$s")`, as core_shell.jl:93 does, and
`directory` writes the same three CSV files (core_shell.jl:96-101).

Arrays cross the C ABI (include/esc.h) as they are: a Julia `Matrix{Float64}`
is column-major with x (the index `kx` varies along, core_shell.jl:21)
contiguous, which is the layout the library expects.

The library path is `ENV["ESC_LIBRARY"]` at precompile time, else the library
built next to this package (`../../esc/libesc.so`).
"""
module EscB200

export EscParams, default_params, run_simulation_gpu, run_batch_gpu, esc_adjoint_call, calibration_loss,
       loss_and_gradients, supported_size, ESC_FP64, ESC_MIXED

const libesc = get(ENV, "ESC_LIBRARY", normpath(joinpath(@__DIR__, "..", "..", "..", "esc", "libesc.so")))

# esc_status (include/esc.h)
const ESC_OK = Cint(0)
const ESC_EINVAL = Cint(1)
const ESC_ECUDA = Cint(2)
const ESC_ENONFINITE = Cint(3)
const ESC_ETIMEOUT = Cint(4)
const ESC_ENOMEM = Cint(5)
# esc_precision: FP64 drop-in, or FP64 state with FP32 flux transforms
const ESC_FP64 = Cint(0)
const ESC_MIXED = Cint(1)

"""
The ten model constants in the field order of `Parameters` (core_shell.jl:4-15)
and of the C struct `esc_params`.
"""
struct EscParams
    A::Float64
    B::Float64
    chi::Float64
    P::Float64
    ca::Float64
    cb::Float64
    cc::Float64
    kappa::Float64
    mobility::Float64
    Q::Float64
end

"""Copies any object with the fields of `Parameters` (core_shell.jl:4-15), e.g. a `Parameters()`."""
EscParams(p) = EscParams(p.A, p.B, p.chi, p.P, p.ca, p.cb, p.cc, p.kappa, p.mobility, p.Q)

"""The defaults of `Parameters()` (core_shell.jl:5-14), as the library holds them."""
function default_params()
    r = Ref{EscParams}()
    ccall((:esc_default_params, libesc), Cvoid, (Ref{EscParams},), r)
    return r[]
end

"""True when the library has kernels for n×n grids."""
supported_size(n::Integer) = ccall((:esc_supported_size, libesc), Cint, (Cint,), n) == 1

"""Version string of the loaded library."""
version() = unsafe_string(ccall((:esc_version, libesc), Cstring, ()))

ctx_error(ctx::Ptr{Cvoid}) = unsafe_string(ccall((:esc_last_error, libesc), Cstring, (Ptr{Cvoid},), ctx))
batch_error(b::Ptr{Cvoid}) = unsafe_string(ccall((:esc_batch_last_error, libesc), Cstring, (Ptr{Cvoid},), b))
destroy(ctx::Ptr{Cvoid}) = ccall((:esc_destroy, libesc), Cvoid, (Ptr{Cvoid},), ctx)
destroy_batch(b::Ptr{Cvoid}) = ccall((:esc_batch_destroy, libesc), Cvoid, (Ptr{Cvoid},), b)

function create_context(phi::AbstractMatrix, p::EscParams, spacing::Real, precision::Integer)
    n = size(phi, 1)
    size(phi) == (n, n) || throw(DimensionMismatch("phi must be square"))
    phi64 = Matrix{Float64}(phi)
    ctx = Ref{Ptr{Cvoid}}(C_NULL)
    pp = Ref(p)
    st = GC.@preserve phi64 ccall((:esc_create, libesc), Cint,
        (Ref{Ptr{Cvoid}}, Cint, Cdouble, Ptr{Float64}, Ref{EscParams}, Cint),
        ctx, n, spacing, phi64, pp, precision)
    st == ESC_OK || error("libesc: ", ctx_error(C_NULL))
    return ctx[]
end

# The reference writes its result files with writedlm(path, a, ','): one matrix
# row per line, values printed in Julia's shortest round-trip form.
function write_csv(path::AbstractString, a::AbstractMatrix)
    open(path, "w") do io
        for i in axes(a, 1)
            join(io, (string(x) for x in view(a, i, :)), ',')
            write(io, '\n')
        end
    end
end

"""
    run_simulation_gpu(c0, phi; dt=0.01, steps=1000, spacing=1.0, p=nothing, directory=nothing,
                       precision=ESC_FP64) -> (c, history)

The loop of `run_simulation` (core_shell.jl:84-103) on the GPU.  `p` is a
`Parameters` (or `EscParams`); `nothing` means the defaults.  With
`precision=ESC_FP64` the results agree with the reference loop to rounding
(1e-12 relative); `ESC_MIXED` computes the flux transforms in FP32.
"""
function run_simulation_gpu(c0, phi; dt=0.01, steps=1000, spacing=1.0, p=nothing, directory=nothing,
                            precision=ESC_FP64)
    n = size(c0, 1)
    size(c0) == (n, n) == size(phi) || throw(DimensionMismatch("c0 and phi must be n×n of one size"))
    params = p === nothing ? default_params() : EscParams(p)
    ctx = create_context(phi, params, spacing, precision)
    c = copyto!(Matrix{Float64}(undef, n, n), c0)
    history = zeros(steps + 1, 6)
    bad = Ref{Int64}(-1)
    try
        st = GC.@preserve c history ccall((:esc_run, libesc), Cint,
            (Ptr{Cvoid}, Ptr{Float64}, Cint, Cdouble, Ptr{Float64}, Ref{Int64}),
            ctx, c, steps, dt, history, bad)
        st == ESC_ENONFINITE && error("Non-finite composition at step $(bad[])")   # core_shell.jl:93
        st == ESC_OK || error("libesc: ", ctx_error(ctx))
    finally
        destroy(ctx)
    end
    if directory !== nothing                                                        # core_shell.jl:96-101
        mkpath(directory)
        write_csv(joinpath(directory, "history.csv"), history)
        write_csv(joinpath(directory, "composition.csv"), c)
        write_csv(joinpath(directory, "particle.csv"), phi)
    end
    return c, history
end

"""
    run_batch_gpu(c0s, phis; dt=0.01, steps=1000, spacing=1.0, p=nothing, precision=ESC_MIXED)
        -> (cs, histories, bad_steps)

Many independent particles advanced together (grid sizes may differ).
`spacing` and `p` may be one value for all or one per particle.
`bad_steps[i]` is -1, or the step at which particle i became non-finite; such
a particle's field is returned unchanged and its history rows before that step
are valid, while the other particles run to the end.
"""
function run_batch_gpu(c0s::AbstractVector, phis::AbstractVector; dt=0.01, steps=1000, spacing=1.0, p=nothing,
                       precision=ESC_MIXED)
    count = length(c0s)
    count == length(phis) || throw(DimensionMismatch("one phi per particle"))
    for (c0, phi) in zip(c0s, phis)
        n = size(phi, 1)
        size(c0) == (n, n) == size(phi) || throw(DimensionMismatch("c0 and phi must be n×n of one size"))
    end
    ns = Cint[size(phi, 1) for phi in phis]
    dxs = spacing isa AbstractVector ? Float64.(spacing) : fill(Float64(spacing), count)
    ps = p === nothing ? fill(default_params(), count) :
         p isa AbstractVector ? EscParams[EscParams(x) for x in p] : fill(EscParams(p), count)
    length(dxs) == count == length(ps) || throw(DimensionMismatch("one spacing and one Parameters per particle"))
    phi64 = [Matrix{Float64}(phi) for phi in phis]
    cs = [copyto!(Matrix{Float64}(undef, size(c0)), c0) for c0 in c0s]
    hs = [zeros(steps + 1, 6) for _ in 1:count]
    bad = fill(Int64(-1), count)
    b = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve phi64 cs hs begin
        phiptrs = Ptr{Float64}[pointer(x) for x in phi64]
        st = ccall((:esc_batch_create, libesc), Cint,
            (Ref{Ptr{Cvoid}}, Cint, Ptr{Cint}, Ptr{Float64}, Ptr{Ptr{Float64}}, Ptr{EscParams}, Cint),
            b, count, ns, dxs, phiptrs, ps, precision)
        st == ESC_OK || error("libesc: ", batch_error(C_NULL))
        try
            cptrs = Ptr{Float64}[pointer(x) for x in cs]
            hptrs = Ptr{Float64}[pointer(x) for x in hs]
            st = ccall((:esc_batch_run, libesc), Cint,
                (Ptr{Cvoid}, Ptr{Ptr{Float64}}, Cint, Cdouble, Ptr{Ptr{Float64}}, Ptr{Int64}),
                b[], cptrs, steps, dt, hptrs, bad)
            (st == ESC_OK || st == ESC_ENONFINITE) || error("libesc: ", batch_error(b[]))
        finally
            destroy_batch(b[])
        end
    end
    return cs, hs, bad
end

"""
    esc_adjoint_call(c0, phi, c_target; p=nothing, dt=0.01, steps=2000, lambdaF=1e-3, ckpt=0,
                     spacing=1.0, precision=ESC_MIXED) -> (L, dL_dc0, dL_dtheta)

L = ½‖c_T − c_target‖² + lambdaF·F[c_T] (F the energy of core_shell.jl:78-82),
with its gradient with respect to c0 and to θ = (P, χ, κ, M0), from the
library's FP64 adjoint with checkpoints every `ckpt` steps (≤ 0: ⌈√steps⌉).
The forward and recomputed passes run in `precision`.  The reference has no
gradients; this serves parameter calibration.
"""
function esc_adjoint_call(c0, phi, c_target; p=nothing, dt=0.01, steps=2000, lambdaF=1e-3, ckpt=0, spacing=1.0,
                          precision=ESC_MIXED)
    n = size(c0, 1)
    size(c0) == (n, n) == size(phi) == size(c_target) ||
        throw(DimensionMismatch("c0, phi and c_target must be n×n of one size"))
    params = p === nothing ? default_params() : EscParams(p)
    ctx = create_context(phi, params, spacing, precision)
    c0m = Matrix{Float64}(c0)
    ct = Matrix{Float64}(c_target)
    dc0 = zeros(n, n)
    dtheta = zeros(4)
    L = Ref(0.0)
    try
        st = GC.@preserve c0m ct dc0 dtheta ccall((:esc_adjoint, libesc), Cint,
            (Ptr{Cvoid}, Ptr{Float64}, Cint, Cdouble, Ptr{Float64}, Cdouble, Cint, Ptr{Float64}, Ptr{Float64},
             Ref{Float64}),
            ctx, c0m, steps, dt, ct, lambdaF, ckpt, dc0, dtheta, L)
        st == ESC_OK || error("libesc: ", ctx_error(ctx))
    finally
        destroy(ctx)
    end
    return L[], dc0, dtheta
end

"""Parameters with θ = (P, χ, κ, M0) replaced, the rest taken from `base` (defaults if `nothing`)."""
function theta_params(theta, base)
    b = base === nothing ? default_params() : EscParams(base)
    return EscParams(b.A, b.B, theta[2], theta[1], b.ca, b.cb, b.cc, theta[3], theta[4], b.Q)
end

"""(L, dL/dc0, dL/dθ) of `calibration_loss` in one library call."""
function loss_and_gradients(c0, theta, phi, c_target; base=nothing, kw...)
    return esc_adjoint_call(c0, phi, c_target; p=theta_params(theta, base), kw...)
end

"""
    calibration_loss(c0, theta, phi, c_target; base=nothing, dt, steps, lambdaF, ckpt, spacing, precision)

The loss of `esc_adjoint_call` as a function of the initial field and of
θ = (P, χ, κ, M0).  With ChainRulesCore loaded, its `rrule` returns the
library's adjoint gradients (package extension EscB200ChainRulesCoreExt).
"""
calibration_loss(c0, theta, phi, c_target; kw...) = first(loss_and_gradients(c0, theta, phi, c_target; kw...))

end # module
