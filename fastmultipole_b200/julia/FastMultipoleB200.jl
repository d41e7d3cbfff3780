"""
    FastMultipoleB200

Julia binding of libfmmb200.so (C ABI in include/fmm_b200.h) that keeps
FastMultipole.jl's user API for the evaluation hot path: a user system overloads
the same interface functions (`source_system_to_buffer!`, `data_per_body`,
`get_position`, `strength_dims`, `get_n_bodies`, `body_to_multipole!`,
`buffer_to_target_system!`, `has_vector_potential`) and calls `fmm!` / `direct!`
with the reference's keyword arguments.  Gathering and scattering happen in
Julia through those overloads; everything in between runs on the B200.

Load it next to FastMultipole.jl (it reuses the reference's interface function
names so existing overloads apply unchanged):

    using FastMultipole
    include("FastMultipoleB200.jl"); using .FastMultipoleB200
    FastMultipoleB200.fmm!(system; expansion_order=10, leaf_size=64, multipole_acceptance=0.5)
"""
module FastMultipoleB200

import FastMultipole
import ChainRulesCore
import FastMultipole: source_system_to_buffer!, data_per_body, get_position, strength_dims, get_n_bodies,
                      buffer_to_target_system!, has_vector_potential, DerivativesSwitch, Point, Source, Vortex,
                      PowerAbsoluteGradient, PowerRelativeGradient, RotatedCoefficientsAbsoluteGradient,
                      RotatedCoefficientsRelativeGradient, SelfTuningTreeStop, SelfTuning, Barba

const libfmm = joinpath(@__DIR__, "..", "libfmmb200.so")

# ---- C structs (field order and types of include/fmm_b200.h) ----
struct FmmSourceSystem
    kind::Cint
    n_bodies::Int64
    data_per_body::Cint
    buffer::Ptr{Cdouble}
    memory::Cint
end

struct FmmTargetSystem
    n_bodies::Int64
    positions::Ptr{Cdouble}
    stride::Int64
    out::Ptr{Cdouble}
    memory::Cint
end

mutable struct FmmOptions
    expansion_order::Cint
    leaf_size_source::Cint
    leaf_size_target::Cint
    multipole_acceptance::Cdouble
    error_method::Cint
    error_tolerance::Cdouble
    bonus_expansion::Cint
    shrink_recenter::Cint
    list_method::Cint
    farfield::Cint
    nearfield::Cint
    self_induced::Cint
    upward_pass::Cint
    horizontal_pass::Cint
    downward_pass::Cint
    scalar_potential::Cint
    gradient::Cint
    hessian::Cint
    precision::Cint
end

mutable struct FmmResult
    p_max::Cint
    error_success::Cint
    n_target_branches::Int64
    n_source_branches::Int64
    n_target_leaves::Int64
    n_source_leaves::Int64
    n_m2l::Int64
    n_direct::Int64
    n_p2p_pairs::Int64
    m2l_flops::Int64
    t_total_ms::Cdouble
    t_tree_ms::Cdouble
    t_lists_ms::Cdouble
    t_nearfield_ms::Cdouble
    t_upward_ms::Cdouble
    t_horizontal_ms::Cdouble
    t_downward_ms::Cdouble
    n_kernel_launches::Int64
    t_influence_ms::Cdouble
end
FmmResult() = FmmResult(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)

const CTX = Ref{Ptr{Cvoid}}(C_NULL)

function context()
    if CTX[] == C_NULL
        h = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:fmm_ctx_create, libfmm), Cint, (Ref{Ptr{Cvoid}}, Cint), h, 0)
        rc == 0 || error("fmm_ctx_create failed with status $rc (no sm_100 GPU?)")
        CTX[] = h[]
    end
    return CTX[]
end

function check(rc)
    if rc != 0
        msg = unsafe_string(ccall((:fmm_ctx_last_error, libfmm), Cstring, (Ptr{Cvoid},), context()))
        error("libfmmb200 status $rc: $msg")
    end
end

kernel_kind(system) = has_vector_potential(system) ? Cint(3) : Cint(1)

error_code(::Nothing) = (Cint(0), 0.0, Cint(1))
error_code(::PowerAbsoluteGradient{E,BE}) where {E,BE} = (Cint(1), Float64(E), Cint(BE))
error_code(::PowerRelativeGradient{E,BE}) where {E,BE} = (Cint(2), Float64(E), Cint(BE))
error_code(::RotatedCoefficientsAbsoluteGradient{E,BE}) where {E,BE} = (Cint(3), Float64(E), Cint(BE))
error_code(::RotatedCoefficientsRelativeGradient{E,BE}) where {E,BE} = (Cint(4), Float64(E), Cint(BE))
error_code(::FastMultipole.PowerAbsolutePotential{E,BE}) where {E,BE} = (Cint(5), Float64(E), Cint(BE))
error_code(::FastMultipole.PowerRelativePotential{E,BE}) where {E,BE} = (Cint(6), Float64(E), Cint(BE))

list_code(::SelfTuningTreeStop) = Cint(0)
list_code(::Barba) = Cint(1)
list_code(::SelfTuning) = Cint(2)

# gather: source_system_to_buffer! in body order (src/compatibility.jl:377-387)
function source_buffer(system)
    n = get_n_bodies(system)
    buf = zeros(Float64, data_per_body(system), n)
    for i in 1:n
        source_system_to_buffer!(buf, i, system, i)
    end
    return buf
end

# scatter: buffer_to_target_system! (src/compatibility.jl:324-338)
function scatter!(system, out, switch)
    for i in 1:get_n_bodies(system)
        buffer_to_target_system!(system, i, switch, out, i)
    end
end

"""
    fmm!(target_system, source_system; kwargs...)
    fmm!(system; leaf_size=20, kwargs...)

FastMultipole.fmm! (src/fmm.jl:807-1176) on the B200.  Keyword arguments as the
reference's; `precision=:mixed` selects the FP32 evaluation path.
"""
function fmm!(target_system, source_system; expansion_order=5, leaf_size_source=20, leaf_size_target=nothing,
              multipole_acceptance=0.4, error_tolerance=nothing, shrink_recenter=true,
              interaction_list_method=SelfTuningTreeStop(), scalar_potential=false, gradient=true, hessian=false,
              farfield=true, nearfield=true, self_induced=true, upward_pass=true, horizontal_pass=true,
              downward_pass=true, precision=:f64)
    self_eval = target_system === source_system
    buf = source_buffer(source_system)
    n_s = size(buf, 2)
    n_t = self_eval ? n_s : get_n_bodies(target_system)
    pos = self_eval ? buf : reduce(hcat, [Vector{Float64}(get_position(target_system, i)) for i in 1:n_t])
    out = zeros(Float64, 16, n_t)
    em, eps, be = error_code(error_tolerance)
    opt = FmmOptions(expansion_order, leaf_size_source, something(leaf_size_target, 0), multipole_acceptance,
                     em, eps, be, shrink_recenter, list_code(interaction_list_method), farfield, nearfield,
                     self_induced, upward_pass, horizontal_pass, downward_pass, scalar_potential, gradient, hessian,
                     precision == :mixed ? 1 : 0)
    res = FmmResult()
    GC.@preserve buf pos out begin
        src = FmmSourceSystem(kernel_kind(source_system), n_s, size(buf, 1), pointer(buf), 0)
        tgt = FmmTargetSystem(n_t, self_eval ? Ptr{Cdouble}(C_NULL) : pointer(pos), 3, pointer(out), 0)
        check(ccall((:fmm_solve, libfmm), Cint,
                    (Ptr{Cvoid}, Ref{FmmTargetSystem}, Ref{FmmSourceSystem}, Ref{FmmOptions}, Ref{FmmResult}),
                    context(), tgt, src, opt, res))
    end
    switch = DerivativesSwitch(scalar_potential, gradient, hessian)
    scatter!(target_system, out, switch)
    optimized_args = (leaf_size_source=leaf_size_source, expansion_order=max(expansion_order, 1),
                      multipole_acceptance=multipole_acceptance)
    return optimized_args, res, res.error_success != 0
end

fmm!(system; leaf_size=20, kwargs...) = fmm!(system, system; leaf_size_source=leaf_size, kwargs...)

"""
    fmm!(target_system, source_systems::Tuple; kwargs...)

A tuple of source systems (point sources and vortex particles mixed): one octree over
the bodies of all of them, as `Tree(systems::Tuple, ...)` builds it (src/tree.jl:3-122),
through `fmm_solve_multi`.  The target system gets the summed field.
"""
function fmm!(target_system, source_systems::Tuple; expansion_order=5, leaf_size_source=20, leaf_size_target=nothing,
              multipole_acceptance=0.4, error_tolerance=nothing, shrink_recenter=true,
              interaction_list_method=SelfTuningTreeStop(), scalar_potential=false, gradient=true, hessian=false,
              farfield=true, nearfield=true, self_induced=true, upward_pass=true, horizontal_pass=true,
              downward_pass=true, precision=:f64)
    length(source_systems) == 1 && return fmm!(target_system, source_systems[1]; expansion_order, leaf_size_source,
        leaf_size_target, multipole_acceptance, error_tolerance, shrink_recenter, interaction_list_method,
        scalar_potential, gradient, hessian, farfield, nearfield, self_induced, upward_pass, horizontal_pass,
        downward_pass, precision)
    bufs = [source_buffer(s) for s in source_systems]
    n_t = get_n_bodies(target_system)
    pos = reduce(hcat, [Vector{Float64}(get_position(target_system, i)) for i in 1:n_t])
    out = zeros(Float64, 16, n_t)
    em, eps, be = error_code(error_tolerance)
    opt = FmmOptions(expansion_order, leaf_size_source, something(leaf_size_target, 0), multipole_acceptance,
                     em, eps, be, shrink_recenter, list_code(interaction_list_method), farfield, nearfield,
                     self_induced, upward_pass, horizontal_pass, downward_pass, scalar_potential, gradient, hessian,
                     precision == :mixed ? 1 : 0)
    res = FmmResult()
    GC.@preserve bufs pos out begin
        srcs = [FmmSourceSystem(kernel_kind(s), size(b, 2), size(b, 1), pointer(b), 0)
                for (s, b) in zip(source_systems, bufs)]
        tgt = FmmTargetSystem(n_t, pointer(pos), 3, pointer(out), 0)
        check(ccall((:fmm_solve_multi, libfmm), Cint,
                    (Ptr{Cvoid}, Ref{FmmTargetSystem}, Ptr{FmmSourceSystem}, Cint, Ref{FmmOptions}, Ref{FmmResult}),
                    context(), tgt, srcs, length(srcs), opt, res))
    end
    scatter!(target_system, out, DerivativesSwitch(scalar_potential, gradient, hessian))
    optimized_args = (leaf_size_source=leaf_size_source, expansion_order=max(expansion_order, 1),
                      multipole_acceptance=multipole_acceptance)
    return optimized_args, res, res.error_success != 0
end

"""
    direct!(target_system, source_system; scalar_potential=false, gradient=true, hessian=false)

FastMultipole.direct! (src/direct.jl:20-75) on the B200, all pairs.
"""
function direct!(target_system, source_system; scalar_potential=false, gradient=true, hessian=false,
                 precision=:f64)
    buf = source_buffer(source_system)
    n_t = get_n_bodies(target_system)
    pos = reduce(hcat, [Vector{Float64}(get_position(target_system, i)) for i in 1:n_t])
    out = zeros(Float64, 16, n_t)
    GC.@preserve buf pos out begin
        src = FmmSourceSystem(kernel_kind(source_system), size(buf, 2), size(buf, 1), pointer(buf), 0)
        tgt = FmmTargetSystem(n_t, pointer(pos), 3, pointer(out), 0)
        check(ccall((:fmm_direct, libfmm), Cint,
                    (Ptr{Cvoid}, Ref{FmmTargetSystem}, Ref{FmmSourceSystem}, Cint, Cint, Cint, Cint),
                    context(), tgt, src, scalar_potential, gradient, hessian, precision == :mixed ? 1 : 0))
    end
    scatter!(target_system, out, DerivativesSwitch(scalar_potential, gradient, hessian))
    return nothing
end

direct!(system; kwargs...) = direct!(system, system; kwargs...)

"""
    vjp(system, cotangent; targets=nothing, kwargs...)

Gradient of a scalar loss through `fmm!` (the adjoint FMM; the reference obtains it
by differentiating `fmm!` with ReverseDiff, README.md:19).  `cotangent` is dL/dphi per
target (point sources) or dL/du (3 x n_t, vortex particles).  Returns
`(d_strength, d_position, d_target_position)`; the last is `nothing` when the sources
are the targets.  Keyword arguments as `fmm!`.
"""
function vjp(system, cotangent; targets=nothing, expansion_order=5, leaf_size=20, multipole_acceptance=0.4,
             error_tolerance=nothing, shrink_recenter=true, interaction_list_method=SelfTuningTreeStop(),
             precision=:f64)
    buf = source_buffer(system)
    n_s = size(buf, 2)
    vortex = has_vector_potential(system)
    self_eval = targets === nothing
    n_t = self_eval ? n_s : get_n_bodies(targets)
    pos = self_eval ? buf : reduce(hcat, [Vector{Float64}(get_position(targets, i)) for i in 1:n_t])
    d_out = zeros(Float64, 16, n_t)
    if vortex
        d_out[5:7, :] .= reshape(cotangent, 3, n_t)
    else
        d_out[4, :] .= vec(cotangent)
    end
    out = zeros(Float64, 16, n_t)
    d_str = zeros(Float64, vortex ? 3 : 1, n_s)
    d_pos = zeros(Float64, 3, n_s)
    d_tpos = self_eval ? zeros(Float64, 3, 0) : zeros(Float64, 3, n_t)
    em, eps, be = error_code(error_tolerance)
    opt = FmmOptions(expansion_order, leaf_size, 0, multipole_acceptance, em, eps, be, shrink_recenter,
                     list_code(interaction_list_method), 1, 1, 1, 1, 1, 1, 1, 1, 0, precision == :mixed ? 1 : 0)
    res = FmmResult()
    GC.@preserve buf pos out d_out d_str d_pos d_tpos begin
        src = FmmSourceSystem(kernel_kind(system), n_s, size(buf, 1), pointer(buf), 0)
        tgt = FmmTargetSystem(n_t, self_eval ? Ptr{Cdouble}(C_NULL) : pointer(pos), 3, pointer(out), 0)
        check(ccall((:fmm_vjp, libfmm), Cint,
                    (Ptr{Cvoid}, Ref{FmmTargetSystem}, Ref{FmmSourceSystem}, Ref{FmmOptions}, Ptr{Cdouble},
                     Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ref{FmmResult}),
                    context(), tgt, src, opt, pointer(d_out), pointer(d_str), pointer(d_pos),
                    self_eval ? Ptr{Cdouble}(C_NULL) : pointer(d_tpos), res))
    end
    return vortex ? d_str : vec(d_str), d_pos, self_eval ? nothing : d_tpos
end

# ---- differentiable form (the reference is differentiated with ForwardDiff/ReverseDiff
# through its Julia code, README.md:19; here the gradient is the adjoint FMM) ----

function _options(; expansion_order=5, leaf_size_source=20, multipole_acceptance=0.4, error_tolerance=nothing,
                  shrink_recenter=true, interaction_list_method=SelfTuningTreeStop(), scalar_potential=true,
                  gradient=true, hessian=false, precision=:f64)
    em, eps, be = error_code(error_tolerance)
    return FmmOptions(expansion_order, leaf_size_source, 0, multipole_acceptance, em, eps, be, shrink_recenter,
                      list_code(interaction_list_method), 1, 1, 1, 1, 1, 1, scalar_potential, gradient, hessian,
                      precision == :mixed ? 1 : 0)
end

"""
    fmm_buffer(source_buffer, target_positions, kind; kwargs...) -> 16 x n_t matrix

`fmm!` as a pure function of arrays: `source_buffer` is the d x n_s buffer that
`source_system_to_buffer!` fills (rows 1:3 position, 4 radius, 5:d strength),
`target_positions` a 3 x n_t matrix or `nothing` (the sources are the targets),
`kind` `:source` (Laplace point sources) or `:vortex`.  Returns the target buffer
(rows 1:3 positions, 4 potential, 5:7 gradient / velocity, 8:16 Hessian / velocity
gradient).  Keyword arguments as `fmm!`.  Differentiable through the
`ChainRulesCore.rrule` below (and so with any ChainRules-aware AD, or ReverseDiff
via `ReverseDiff.@grad_from_chainrules fmm_buffer(x::TrackedArray, y, k; kw...)`).
"""
function fmm_buffer(source_buffer::AbstractMatrix, target_positions, kind::Symbol; kwargs...)
    buf = Matrix{Float64}(source_buffer)
    n_s = size(buf, 2)
    self_eval = target_positions === nothing
    pos = self_eval ? buf : Matrix{Float64}(target_positions)
    n_t = self_eval ? n_s : size(pos, 2)
    out = zeros(Float64, 16, n_t)
    opt = _options(; kwargs...)
    res = FmmResult()
    GC.@preserve buf pos out begin
        src = FmmSourceSystem(kind === :vortex ? Cint(3) : Cint(1), n_s, size(buf, 1), pointer(buf), 0)
        tgt = FmmTargetSystem(n_t, self_eval ? Ptr{Cdouble}(C_NULL) : pointer(pos), self_eval ? 0 : size(pos, 1),
                              pointer(out), 0)
        check(ccall((:fmm_solve, libfmm), Cint,
                    (Ptr{Cvoid}, Ref{FmmTargetSystem}, Ref{FmmSourceSystem}, Ref{FmmOptions}, Ref{FmmResult}),
                    context(), tgt, src, opt, res))
    end
    return out
end

"""
ChainRulesCore.rrule of `fmm_buffer`: the pullback runs `fmm_vjp` (forward solve plus
the adjoint solve whose sources sit at the targets with the cotangents as strengths).
Cotangents are read from rows 1:3 (positions) and 4 (potential) for point sources,
rows 1:3 and 5:7 (velocity) for vortex particles; a non-zero cotangent on another
row is an error (libfmmb200 status 1).  Tangents: the source buffer (positions and
strengths; the radius row gets zero) and the target positions; none for `kind`.
Not executed in this repository: Julia is not installed on the build image, so the
adjoint it calls is tested through the same C ABI from Python.
"""
function ChainRulesCore.rrule(::typeof(fmm_buffer), source_buffer::AbstractMatrix, target_positions, kind::Symbol;
                              kwargs...)
    out = fmm_buffer(source_buffer, target_positions, kind; kwargs...)
    function fmm_buffer_pullback(Δout)
        Δ = Matrix{Float64}(ChainRulesCore.unthunk(Δout))
        buf = Matrix{Float64}(source_buffer)
        n_s = size(buf, 2)
        self_eval = target_positions === nothing
        pos = self_eval ? buf : Matrix{Float64}(target_positions)
        n_t = self_eval ? n_s : size(pos, 2)
        sdim = kind === :vortex ? 3 : 1
        d_str = zeros(Float64, sdim, n_s)
        d_pos = zeros(Float64, 3, n_s)
        d_tpos = zeros(Float64, 3, self_eval ? 0 : n_t)
        fwd = zeros(Float64, 16, n_t)
        opt = _options(; kwargs...)
        res = FmmResult()
        GC.@preserve buf pos fwd Δ d_str d_pos d_tpos begin
            src = FmmSourceSystem(kind === :vortex ? Cint(3) : Cint(1), n_s, size(buf, 1), pointer(buf), 0)
            tgt = FmmTargetSystem(n_t, self_eval ? Ptr{Cdouble}(C_NULL) : pointer(pos),
                                  self_eval ? 0 : size(pos, 1), pointer(fwd), 0)
            check(ccall((:fmm_vjp, libfmm), Cint,
                        (Ptr{Cvoid}, Ref{FmmTargetSystem}, Ref{FmmSourceSystem}, Ref{FmmOptions}, Ptr{Cdouble},
                         Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ref{FmmResult}),
                        context(), tgt, src, opt, pointer(Δ), pointer(d_str), pointer(d_pos),
                        self_eval ? Ptr{Cdouble}(C_NULL) : pointer(d_tpos), res))
        end
        Δbuf = zeros(Float64, size(buf))
        Δbuf[1:3, :] .= d_pos
        Δbuf[5:4+sdim, :] .= d_str
        Δtargets = self_eval ? ChainRulesCore.NoTangent() : d_tpos
        return ChainRulesCore.NoTangent(), Δbuf, Δtargets, ChainRulesCore.NoTangent()
    end
    return out, fmm_buffer_pullback
end

end # module
