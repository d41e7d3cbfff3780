"""Host-side mirror of FastMultipole.jl's user API for the evaluation hot path.

The reference lets a user overload, per system type, a handful of interface
functions (src/compatibility.jl) and then call ``fmm!`` / ``direct!``
(src/fmm.jl:807-1176, src/direct.jl:20-75).  This module keeps that shape:

* a system is any object providing the interface methods below (the names are
  the reference's, without the ``!``); :class:`System` documents them and
  :class:`PointSources` / :class:`VortexParticles` are ready-made systems
  equivalent to the reference test suite's ``Gravitational`` and
  ``VortexParticles`` (test/gravitational.jl, test/vortex.jl);
* :func:`fmm` and :func:`direct` take the reference's keyword arguments and
  return the reference's 8-tuple / nothing, writing results back through
  ``buffer_to_target_system``.

Between gather and scatter all work happens on the GPU through the C ABI
(libfmmb200.so); there is no CPU path.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


# ---------------------------------------------------------------------------
# interaction list methods and error tolerances (src/containers.jl:84-123)
class InteractionListMethod:
    code = L.FMM_LIST_SELF_TUNING_TREE_STOP


class SelfTuningTreeStop(InteractionListMethod):
    code = L.FMM_LIST_SELF_TUNING_TREE_STOP


class Barba(InteractionListMethod):
    code = L.FMM_LIST_BARBA


class SelfTuning(InteractionListMethod):
    code = L.FMM_LIST_SELF_TUNING


@dataclass(frozen=True)
class ErrorMethod:
    eps: float
    BE: bool = True
    code: int = 0


def PowerAbsoluteGradient(eps, BE=True):
    return ErrorMethod(float(eps), bool(BE), L.FMM_POWER_ABSOLUTE_GRADIENT)


def PowerRelativeGradient(eps, BE=True):
    return ErrorMethod(float(eps), bool(BE), L.FMM_POWER_RELATIVE_GRADIENT)


def RotatedCoefficientsAbsoluteGradient(eps, BE=True):
    return ErrorMethod(float(eps), bool(BE), L.FMM_ROTATED_COEFFICIENTS_ABSOLUTE_GRADIENT)


def RotatedCoefficientsRelativeGradient(eps, BE=True):
    return ErrorMethod(float(eps), bool(BE), L.FMM_ROTATED_COEFFICIENTS_RELATIVE_GRADIENT)


def PowerAbsolutePotential(eps, BE=True):
    return ErrorMethod(float(eps), bool(BE), L.FMM_POWER_ABSOLUTE_POTENTIAL)


def PowerRelativePotential(eps, BE=True):
    return ErrorMethod(float(eps), bool(BE), L.FMM_POWER_RELATIVE_POTENTIAL)


@dataclass(frozen=True)
class DerivativesSwitch:
    """DerivativesSwitch{PS,GS,HS} (src/containers.jl:50)."""
    scalar_potential: bool = True
    gradient: bool = True
    hessian: bool = True


# ---------------------------------------------------------------------------
class System:
    """Interface a user system implements (src/compatibility.jl:21-286).

    Vectorised forms of the reference's per-body functions:

    ``get_n_bodies()``                -> int
    ``kernel``                        -> "source" | "vortex"  (body_to_multipole!(Point{Source|Vortex}, ...))
    ``data_per_body()``               -> int   (>= 5 for sources, >= 7 for vortices)
    ``strength_dims()``               -> 1 | 3
    ``positions()``                   -> (N, 3) float64, get_position for every body
    ``source_system_to_buffer(buf)``  fills buf (N, data_per_body): x y z radius strength...
    ``buffer_to_target_system(buf, switch)``  reads buf (N, 16): x y z phi grad(3) hessian(9)
    ``has_vector_potential()``        -> bool
    """

    kernel = "source"

    def get_n_bodies(self):
        raise NotImplementedError("get_n_bodies not overloaded for " + type(self).__name__)

    def data_per_body(self):
        raise NotImplementedError("data_per_body not overloaded for " + type(self).__name__)

    def strength_dims(self):
        raise NotImplementedError("strength_dims not overloaded for " + type(self).__name__)

    def positions(self):
        raise NotImplementedError("get_position not overloaded for " + type(self).__name__)

    def source_system_to_buffer(self, buffer):
        raise NotImplementedError("source_system_to_buffer! not overloaded for " + type(self).__name__)

    def buffer_to_target_system(self, buffer, switch):
        raise NotImplementedError("buffer_to_target_system! not overloaded for " + type(self).__name__)

    def has_vector_potential(self):
        raise NotImplementedError("has_vector_potential not overloaded for " + type(self).__name__)


class PointSources(System):
    """Laplace point sources (the reference test suite's ``Gravitational``).

    ``potential`` is (N, 16) like the reference's: row 0 phi, 4..6 gradient, 7..15 hessian.
    """

    kernel = "source"

    def __init__(self, position, strength, radius=None):
        self.position = np.ascontiguousarray(position, dtype=np.float64).reshape(-1, 3)
        n = len(self.position)
        self.strength = np.ascontiguousarray(strength, dtype=np.float64).reshape(n)
        self.radius = np.zeros(n) if radius is None else np.ascontiguousarray(radius, np.float64).reshape(n)
        self.potential = np.zeros((n, 16))

    def get_n_bodies(self):
        return len(self.position)

    def data_per_body(self):
        return 5

    def strength_dims(self):
        return 1

    def positions(self):
        return self.position

    def has_vector_potential(self):
        return False

    def source_system_to_buffer(self, buffer):
        buffer[:, 0:3] = self.position
        buffer[:, 3] = self.radius
        buffer[:, 4] = self.strength

    def buffer_to_target_system(self, buffer, switch):
        # test/gravitational.jl:106-119: assignment of the requested quantities
        self.potential[:, 0] = buffer[:, 3] if switch.scalar_potential else 0.0
        self.potential[:, 4:7] = buffer[:, 4:7] if switch.gradient else 0.0
        self.potential[:, 7:16] = buffer[:, 7:16] if switch.hessian else 0.0


class VortexParticles(System):
    """Vortex particles (the reference test suite's ``VortexParticles``).

    ``gradient_stretching[:, 0:3]`` accumulates the velocity, ``potential[:, 4:13]``
    the velocity gradient (test/vortex.jl:130-146).
    """

    kernel = "vortex"

    def __init__(self, position, strength, sigma=None):
        self.position = np.ascontiguousarray(position, dtype=np.float64).reshape(-1, 3)
        n = len(self.position)
        self.strength = np.ascontiguousarray(strength, dtype=np.float64).reshape(n, 3)
        self.sigma = np.zeros(n) if sigma is None else np.ascontiguousarray(sigma, np.float64).reshape(n)
        self.potential = np.zeros((n, 13))
        self.gradient_stretching = np.zeros((n, 6))

    def get_n_bodies(self):
        return len(self.position)

    def data_per_body(self):
        return 7

    def strength_dims(self):
        return 3

    def positions(self):
        return self.position

    def has_vector_potential(self):
        return True

    def source_system_to_buffer(self, buffer):
        buffer[:, 0:3] = self.position
        buffer[:, 3] = self.sigma
        buffer[:, 4:7] = self.strength

    def buffer_to_target_system(self, buffer, switch):
        if switch.gradient:
            self.gradient_stretching[:, 0:3] += buffer[:, 4:7]
        if switch.hessian:
            self.potential[:, 4:13] += buffer[:, 7:16]


class ProbeSystem(System):
    """Target-only evaluation points (src/probes.jl:1-60)."""

    def __init__(self, position):
        self.position = np.ascontiguousarray(position, dtype=np.float64).reshape(-1, 3)
        n = len(self.position)
        self.scalar_potential = np.zeros(n)
        self.gradient = np.zeros((n, 3))
        self.hessian = np.zeros((n, 9))

    def get_n_bodies(self):
        return len(self.position)

    def positions(self):
        return self.position

    def buffer_to_target_system(self, buffer, switch):
        if switch.scalar_potential:
            self.scalar_potential += buffer[:, 3]
        if switch.gradient:
            self.gradient += buffer[:, 4:7]
        if switch.hessian:
            self.hessian += buffer[:, 7:16]


# ---------------------------------------------------------------------------
_default_ctx = None


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = L.Context(0)
    return _default_ctx


def _tuple(x):
    return tuple(x) if isinstance(x, (tuple, list)) else (x,)


def _kind(systems):
    kinds = {s.kernel for s in systems}
    if len(kinds) != 1:
        raise NotImplementedError("source systems of mixed kernels in one call are not supported yet")
    k = kinds.pop()
    if k not in ("source", "vortex"):
        raise ValueError(f"unknown kernel {k!r}")
    return L.FMM_POINT_SOURCE if k == "source" else L.FMM_POINT_VORTEX


def _source_buffer(systems, kind):
    d = 5 if kind == L.FMM_POINT_SOURCE else 7
    n = sum(s.get_n_bodies() for s in systems)
    buf = np.zeros((n, d))
    o = 0
    for s in systems:
        m = s.get_n_bodies()
        tmp = np.zeros((m, s.data_per_body()))
        s.source_system_to_buffer(tmp)
        buf[o:o + m] = tmp[:, :d]
        o += m
    return buf


def _positions(systems):
    return np.ascontiguousarray(np.concatenate([np.asarray(s.positions(), np.float64).reshape(-1, 3)
                                                for s in systems]), dtype=np.float64)


def _scatter(systems, out, switch):
    o = 0
    for s in systems:
        m = s.get_n_bodies()
        s.buffer_to_target_system(out[o:o + m], switch)
        o += m


def make_options(expansion_order=5, leaf_size_source=20, leaf_size_target=None, multipole_acceptance=0.4,
                 error_tolerance=None, shrink_recenter=True, interaction_list_method=None, farfield=True,
                 nearfield=True, self_induced=True, upward_pass=True, horizontal_pass=True, downward_pass=True,
                 scalar_potential=False, gradient=True, hessian=False, precision="f64"):
    o = L.default_options()
    o.expansion_order = int(expansion_order)
    o.leaf_size_source = int(leaf_size_source)
    o.leaf_size_target = int(leaf_size_target) if leaf_size_target else 0
    o.multipole_acceptance = float(multipole_acceptance)
    if error_tolerance is not None:
        o.error_method = error_tolerance.code
        o.error_tolerance = error_tolerance.eps
        o.bonus_expansion = 1 if error_tolerance.BE else 0
    o.shrink_recenter = 1 if shrink_recenter else 0
    o.list_method = (interaction_list_method or SelfTuningTreeStop()).code
    o.farfield, o.nearfield, o.self_induced = int(farfield), int(nearfield), int(self_induced)
    o.upward_pass, o.horizontal_pass, o.downward_pass = int(upward_pass), int(horizontal_pass), int(downward_pass)
    o.scalar_potential, o.gradient, o.hessian = int(scalar_potential), int(gradient), int(hessian)
    o.precision = {"f64": L.FMM_PRECISION_F64, "mixed": L.FMM_PRECISION_MIXED}[precision]
    return o


class TreeHandle:
    """The exported Tree of the context's last solve (src/containers.jl:182-195), fetched on demand."""

    def __init__(self, ctx, which):
        self.ctx, self.which = ctx, which

    def fetch(self):
        return get_tree(self.ctx, self.which)


def get_tree(ctx, which):
    v = L.TreeView()
    ctx.check(L.lib().fmm_get_tree(ctx.handle, which, C.byref(v)))
    nb, nl, nlv, n = v.n_branches, v.n_levels, v.n_leaves, v.n_bodies
    i64 = {k: np.zeros(nb, np.int64) for k in ("body_start", "body_count", "child_start", "n_children", "parent",
                                                 "i_leaf")}
    f3 = {k: np.zeros((nb, 3)) for k in ("target_center", "source_center", "target_box", "source_box")}
    f1 = {k: np.zeros(nb) for k in ("target_radius", "source_radius", "max_influence")}
    extra = dict(sort_index=np.zeros(n, np.int64), levels_start=np.zeros(nl, np.int64),
                 levels_end=np.zeros(nl, np.int64), leaf_index=np.zeros(nlv, np.int64))
    for k, a in list(i64.items()) + list(extra.items()):
        setattr(v, k, a.ctypes.data_as(L._i64p))
    for k, a in list(f3.items()) + list(f1.items()):
        setattr(v, k, a.ctypes.data_as(L._dp))
    ctx.check(L.lib().fmm_get_tree(ctx.handle, which, C.byref(v)))
    d = dict(n_branches=nb, n_levels=nl, n_leaves=nlv, n_bodies=n)
    d.update(i64)
    d.update(f3)
    d.update(f1)
    d.update(extra)
    return d


def get_lists(ctx):
    nm, nd = C.c_int64(), C.c_int64()
    ctx.check(L.lib().fmm_get_lists(ctx.handle, None, C.byref(nm), None, C.byref(nd)))
    m2l = np.zeros((nm.value, 2), np.int32)
    dl = np.zeros((nd.value, 2), np.int32)
    ctx.check(L.lib().fmm_get_lists(ctx.handle, m2l.ctypes.data_as(L._i32p), C.byref(nm),
                                    dl.ctypes.data_as(L._i32p), C.byref(nd)))
    return m2l, dl


def solve_buffers(source_buf, kind, opt, target_pos=None, ctx=None, timing=False):
    """fmm! on raw buffers: source_buf (N, d), target_pos (Nt, 3) or None (targets = sources).

    Returns (out (Nt, 16), fmm_result)."""
    ctx = ctx or default_context()
    sb = np.ascontiguousarray(source_buf, dtype=np.float64)
    n_s, d = sb.shape
    src = L.SourceSystem(kind, n_s, d, sb.ctypes.data, L.FMM_MEMORY_HOST)
    if target_pos is None:
        out = np.zeros((n_s, 16))
        tgt = L.TargetSystem(n_s, None, 0, out.ctypes.data, L.FMM_MEMORY_HOST)
    else:
        tp = np.ascontiguousarray(target_pos, dtype=np.float64)
        out = np.zeros((len(tp), 16))
        tgt = L.TargetSystem(len(tp), tp.ctypes.data, 3, out.ctypes.data, L.FMM_MEMORY_HOST)
    res = L.Result()
    ctx.set_timing(timing)
    ctx.check(L.lib().fmm_solve(ctx.handle, C.byref(tgt), C.byref(src), C.byref(opt), C.byref(res)))
    return out, res


def solve_multi_buffers(sources, opt, target_pos, ctx=None):
    """fmm! of a tuple of source systems on raw buffers: ``sources`` is a list of
    (buffer (N_k, d_k), kind) in tuple order; one octree over all of their bodies
    (fmm_solve_multi).  Returns (out (Nt, 16), fmm_result)."""
    ctx = ctx or default_context()
    bufs = [np.ascontiguousarray(b, dtype=np.float64) for b, _ in sources]
    arr = (L.SourceSystem * len(bufs))(*[L.SourceSystem(k, b.shape[0], b.shape[1], b.ctypes.data, L.FMM_MEMORY_HOST)
                                         for b, (_, k) in zip(bufs, sources)])
    tp = np.ascontiguousarray(target_pos, dtype=np.float64)
    out = np.zeros((len(tp), 16))
    tgt = L.TargetSystem(len(tp), tp.ctypes.data, 3, out.ctypes.data, L.FMM_MEMORY_HOST)
    res = L.Result()
    ctx.check(L.lib().fmm_solve_multi(ctx.handle, C.byref(tgt), arr, len(bufs), C.byref(opt), C.byref(res)))
    return out, res


def vjp_buffers(source_buf, kind, opt, d_out, target_pos=None, ctx=None):
    """Gradients of a loss through fmm! on raw buffers (fmm_vjp).

    ``d_out`` (Nt, 16) holds dL/d(target buffer): columns 0..2 (the echoed target
    positions) and column 3 (phi) for point sources, columns 0..2 and 4..6 (velocity) for
    vortex particles; a non-zero value in any other column is rejected.  Returns ``(out, d_strength,
    d_source_position, d_target_position, fmm_result)``: the forward target buffer,
    dL/dstrength (N,) or (N, 3), dL/dx (N, 3) and, for separate targets, dL/dy
    (Nt, 3) (None when the sources are the targets)."""
    ctx = ctx or default_context()
    sb = np.ascontiguousarray(source_buf, dtype=np.float64)
    n_s, d = sb.shape
    src = L.SourceSystem(kind, n_s, d, sb.ctypes.data, L.FMM_MEMORY_HOST)
    sdim = 1 if kind == L.FMM_POINT_SOURCE else 3
    if target_pos is None:
        nt = n_s
        out = np.zeros((nt, 16))
        tgt = L.TargetSystem(nt, None, 0, out.ctypes.data, L.FMM_MEMORY_HOST)
        dtp = None
    else:
        tp = np.ascontiguousarray(target_pos, dtype=np.float64)
        nt = len(tp)
        out = np.zeros((nt, 16))
        tgt = L.TargetSystem(nt, tp.ctypes.data, 3, out.ctypes.data, L.FMM_MEMORY_HOST)
        dtp = np.zeros((nt, 3))
    dd = np.ascontiguousarray(d_out, dtype=np.float64).reshape(nt, 16)
    dstr = np.zeros((n_s, sdim))
    dpos = np.zeros((n_s, 3))
    res = L.Result()
    ctx.check(L.lib().fmm_vjp(ctx.handle, C.byref(tgt), C.byref(src), C.byref(opt), dd.ctypes.data_as(L._dp),
                              dstr.ctypes.data_as(L._dp), dpos.ctypes.data_as(L._dp),
                              None if dtp is None else dtp.ctypes.data_as(L._dp), C.byref(res)))
    return out, (dstr[:, 0] if sdim == 1 else dstr), dpos, dtp, res


def vjp(system, d_potential=None, d_velocity=None, targets=None, *, leaf_size=20, expansion_order=5,
        multipole_acceptance=0.4, error_tolerance=None, precision="f64", context=None):
    """Gradient of L = sum_t d_potential_t phi_t (point sources) or sum_t d_velocity_t . u_t
    (vortex particles) with respect to the source strengths and positions, and the
    target positions when ``targets`` (a ProbeSystem or positions) is given.

    The reference differentiates fmm! with ReverseDiff (README.md:19); this is the
    adjoint FMM of the same problem.  Returns a dict with ``d_strength``,
    ``d_position`` and (separate targets) ``d_target_position``."""
    kind = _kind((system,))
    buf = _source_buffer((system,), kind)
    tpos = None
    if targets is not None:
        tpos = targets.positions() if hasattr(targets, "positions") else np.asarray(targets, dtype=np.float64)
    nt = len(buf) if tpos is None else len(tpos)
    d_out = np.zeros((nt, 16))
    if kind == L.FMM_POINT_SOURCE:
        d_out[:, 3] = np.asarray(d_potential, dtype=np.float64).reshape(nt)
    else:
        d_out[:, 4:7] = np.asarray(d_velocity, dtype=np.float64).reshape(nt, 3)
    opt = make_options(expansion_order, leaf_size, None, multipole_acceptance, error_tolerance,
                       scalar_potential=True, gradient=True, precision=precision)
    out, dstr, dpos, dtp, res = vjp_buffers(buf, kind, opt, d_out, tpos, context)
    r = {"d_strength": dstr, "d_position": dpos, "out": out, "error_success": bool(res.error_success)}
    if dtp is not None:
        r["d_target_position"] = dtp
    return r


def request_footprint(source_buf, kind, opt, target_pos=None):
    """Device bytes the serving account reserves for one request (fmm_request_footprint)."""
    sb = np.ascontiguousarray(source_buf, dtype=np.float64)
    n_s, d = sb.shape
    if target_pos is None:
        tgt = L.TargetSystem(n_s, None, 0, None, L.FMM_MEMORY_HOST)
    else:
        tp = np.ascontiguousarray(target_pos, dtype=np.float64)
        tgt = L.TargetSystem(len(tp), tp.ctypes.data, 3, None, L.FMM_MEMORY_HOST)
    req = L.Request(tgt, L.SourceSystem(kind, n_s, d, sb.ctypes.data, L.FMM_MEMORY_HOST), opt)
    return int(L.lib().fmm_request_footprint(C.byref(req)))


class Server:
    """Concurrent fmm! requests on one device (fmm_serve_*): ``n_workers`` solver
    contexts run queued requests (oldest first) as soon as one finishes, and
    ``n_workers // 2`` (at least one) express contexts on highest-priority streams run
    requests of at most 65,536 source plus target bodies.  ``hbm_budget`` (bytes, 0:
    unlimited) is one account shared by all workers: a request that fits it waits for
    memory in arrival order; only a request larger than the whole budget fails with
    FMM_ERR_MEMORY."""

    def __init__(self, n_workers=4, hbm_budget=0, ctx=None):
        self.ctx = ctx or default_context()
        self.ctx.check(L.lib().fmm_serve_start(self.ctx.handle, int(n_workers), int(hbm_budget)))
        self._live = {}

    def submit(self, source_buf, kind, opt, target_pos=None):
        """Queue one fmm! on raw buffers; returns the request id."""
        sb = np.ascontiguousarray(source_buf, dtype=np.float64)
        n_s, d = sb.shape
        if target_pos is None:
            tp = None
            out = np.zeros((n_s, 16))
            tgt = L.TargetSystem(n_s, None, 0, out.ctypes.data, L.FMM_MEMORY_HOST)
        else:
            tp = np.ascontiguousarray(target_pos, dtype=np.float64)
            out = np.zeros((len(tp), 16))
            tgt = L.TargetSystem(len(tp), tp.ctypes.data, 3, out.ctypes.data, L.FMM_MEMORY_HOST)
        req = L.Request(tgt, L.SourceSystem(kind, n_s, d, sb.ctypes.data, L.FMM_MEMORY_HOST), opt)
        rid = C.c_uint64(0)
        self.ctx.check(L.lib().fmm_serve_submit(self.ctx.handle, C.byref(req), C.byref(rid)))
        self._live[rid.value] = (sb, tp, out, req)  # the buffers stay alive until the request is polled
        return rid.value

    def poll(self, rid, timeout_ms=-1):
        """Returns (status, out, fmm_result); status FMM_PENDING if not finished."""
        res = L.Result()
        rc = L.lib().fmm_serve_poll(self.ctx.handle, C.c_uint64(rid), C.byref(res), int(timeout_ms))
        if rc == L.FMM_PENDING:
            return rc, None, None
        _, _, out, _ = self._live.pop(rid)
        return rc, out, res

    def stop(self):
        self.ctx.check(L.lib().fmm_serve_stop(self.ctx.handle))


def fmm(target_systems, source_systems=None, *, leaf_size=None, leaf_size_source=None, leaf_size_target=None,
        expansion_order=5, multipole_acceptance=0.4, error_tolerance=None, shrink_recenter=True,
        interaction_list_method=None, scalar_potential=False, gradient=True, hessian=False, farfield=True,
        nearfield=True, self_induced=True, upward_pass=True, horizontal_pass=True, downward_pass=True,
        precision="f64", context=None):
    """fmm!(target_systems, source_systems; kwargs...) (src/fmm.jl:807-1176).

    ``fmm(system)`` evaluates a system on itself (default leaf_size 20).  Returns
    ``(optimized_args, cache, target_tree, source_tree, m2l_list, direct_list,
    derivatives_switches, error_success)`` like the reference; the trees are
    handles whose ``fetch()`` exports the device octree, the lists are arrays of
    (target, source) branch pairs sorted by target (0-based).
    """
    ctx = context or default_context()
    self_eval = source_systems is None
    targets = _tuple(target_systems)
    sources = targets if self_eval else _tuple(source_systems)
    ls_s = leaf_size_source or leaf_size or 20
    opt = make_options(expansion_order, ls_s, leaf_size_target or (leaf_size if self_eval else None),
                       multipole_acceptance, error_tolerance, shrink_recenter, interaction_list_method, farfield,
                       nearfield, self_induced, upward_pass, horizontal_pass, downward_pass, scalar_potential,
                       gradient, hessian, precision)
    if len({s.kernel for s in sources}) > 1:
        # systems of different kernels: one octree over all of them (Tree(systems::Tuple),
        # src/tree.jl:3-122), the systems in tuple order
        out, res = solve_multi_buffers([(_source_buffer((s,), _kind((s,))), _kind((s,))) for s in sources], opt,
                                       _positions(targets), ctx)
        switch = DerivativesSwitch(bool(scalar_potential), bool(gradient), bool(hessian))
        _scatter(targets, out, switch)
        m2l, dl = get_lists(ctx)
        optimized = dict(leaf_size_source=ls_s, expansion_order=max(expansion_order, 1),
                         multipole_acceptance=multipole_acceptance)
        return (optimized, ctx, TreeHandle(ctx, 0), TreeHandle(ctx, 1), m2l, dl, tuple(switch for _ in targets),
                bool(res.error_success))
    kind = _kind(sources)
    buf = _source_buffer(sources, kind)
    same = self_eval or all(a is b for a, b in zip(targets, sources)) and len(targets) == len(sources)
    tpos = None if same else _positions(targets)
    out, res = solve_buffers(buf, kind, opt, tpos, ctx)
    switch = DerivativesSwitch(bool(scalar_potential), bool(gradient), bool(hessian))
    _scatter(targets, out, switch)
    m2l, dl = get_lists(ctx)
    optimized = dict(leaf_size_source=ls_s, expansion_order=max(expansion_order, 1),
                     multipole_acceptance=multipole_acceptance)
    return (optimized, ctx, TreeHandle(ctx, 0), TreeHandle(ctx, 1), m2l, dl,
            tuple(switch for _ in targets), bool(res.error_success))


def direct(target_systems, source_systems=None, *, scalar_potential=False, gradient=True, hessian=False,
           precision="f64", context=None):
    """direct!(targets, sources; scalar_potential, gradient, hessian) (src/direct.jl:20-75)."""
    ctx = context or default_context()
    targets = _tuple(target_systems)
    sources = targets if source_systems is None else _tuple(source_systems)
    kind = _kind(sources)
    buf = _source_buffer(sources, kind)
    tp = _positions(targets)
    out = np.zeros((len(tp), 16))
    src = L.SourceSystem(kind, len(buf), buf.shape[1], buf.ctypes.data, L.FMM_MEMORY_HOST)
    tgt = L.TargetSystem(len(tp), tp.ctypes.data, 3, out.ctypes.data, L.FMM_MEMORY_HOST)
    prec = {"f64": L.FMM_PRECISION_F64, "mixed": L.FMM_PRECISION_MIXED}[precision]
    ctx.check(L.lib().fmm_direct(ctx.handle, C.byref(tgt), C.byref(src), int(scalar_potential), int(gradient),
                                 int(hessian), prec))
    _scatter(targets, out, DerivativesSwitch(bool(scalar_potential), bool(gradient), bool(hessian)))
