"""ctypes binding of the FP64 oracle (oracle/liboracle.so) for the test suite.

Test infrastructure only: the oracle is the checker, never the thing measured.
Builds the library with `make -C oracle` when it is missing.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "liboracle.so")

POINT_SOURCE, POINT_VORTEX = 1, 3
LIST_TREE_STOP, LIST_BARBA, LIST_SELF_TUNING = 0, 1, 2
ERR_NONE, ERR_POWER_ABS_GRAD, ERR_POWER_REL_GRAD, ERR_ROT_ABS_GRAD, ERR_ROT_REL_GRAD = 0, 1, 2, 3, 4
ERR_POWER_ABS_POT, ERR_POWER_REL_POT = 5, 6

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)


class Options(C.Structure):
    _fields_ = [("expansion_order", C.c_int), ("leaf_size_source", C.c_int), ("leaf_size_target", C.c_int),
                ("multipole_acceptance", C.c_double), ("error_method", C.c_int), ("error_tolerance", C.c_double),
                ("bonus_expansion", C.c_int), ("shrink_recenter", C.c_int), ("list_method", C.c_int),
                ("farfield", C.c_int), ("nearfield", C.c_int), ("self_induced", C.c_int),
                ("upward_pass", C.c_int), ("horizontal_pass", C.c_int), ("downward_pass", C.c_int),
                ("scalar_potential", C.c_int), ("gradient", C.c_int), ("hessian", C.c_int),
                ("n_threads", C.c_int)]


class TreeView(C.Structure):
    _fields_ = [("n_branches", C.c_int64), ("n_levels", C.c_int64), ("n_leaves", C.c_int64),
                ("n_bodies", C.c_int64)] + \
               [(n, _i64p) for n in ("body_start", "body_count", "child_start", "n_children", "parent", "i_leaf")] + \
               [(n, _dp) for n in ("target_center", "source_center", "target_radius", "source_radius",
                                   "target_box", "source_box", "max_influence")] + \
               [(n, _i64p) for n in ("sort_index", "levels_start", "levels_end", "leaf_index")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
        L = C.CDLL(LIB_PATH)
        L.oracle_fmm_run.restype = C.c_void_p
        L.oracle_fmm_run.argtypes = [_dp, C.c_int64, _dp, C.c_int, C.c_int, C.c_int64, C.POINTER(Options)]
        for n in ("oracle_run_output", "oracle_run_target_tree", "oracle_run_source_tree", "oracle_run_lists",
                  "oracle_run_pmax", "oracle_run_times"):
            getattr(L, n).restype = C.c_int
        L.oracle_run_output.argtypes = [C.c_void_p, _dp]
        L.oracle_run_target_tree.argtypes = [C.c_void_p, C.POINTER(TreeView)]
        L.oracle_run_source_tree.argtypes = [C.c_void_p, C.POINTER(TreeView)]
        L.oracle_run_n_m2l.restype = C.c_int64
        L.oracle_run_n_m2l.argtypes = [C.c_void_p]
        L.oracle_run_n_direct.restype = C.c_int64
        L.oracle_run_n_direct.argtypes = [C.c_void_p]
        L.oracle_run_lists.argtypes = [C.c_void_p, _i32p, _i32p]
        L.oracle_run_pmax.argtypes = [C.c_void_p, _ip, _ip]
        L.oracle_run_times.argtypes = [C.c_void_p, _dp]
        L.oracle_run_free.restype = None
        L.oracle_run_free.argtypes = [C.c_void_p]
        L.oracle_direct.argtypes = [_dp, C.c_int64, _dp, C.c_int, C.c_int, C.c_int64, C.c_int, C.c_int, C.c_int,
                                    C.c_int, _dp]
        L.oracle_direct_subset.argtypes = [_dp, C.c_int64, _i64p, C.c_int64, _dp, C.c_int, C.c_int, C.c_int64,
                                           C.c_int, _dp]
        L.oracle_tables.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.oracle_length_Hs.restype = C.c_int64
        L.oracle_length_Ts.restype = C.c_int64
        L.oracle_update_Ts.argtypes = [C.c_int, C.c_double, _dp]
        L.oracle_compute_Pnms.argtypes = [C.c_int, C.c_double, C.c_double, _dp]
        L.oracle_regular_harmonics.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, _dp]
        L.oracle_irregular_harmonics.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, _dp]
        for n in ("oracle_translate_multipole_z", "oracle_translate_multipole_to_local_z", "oracle_translate_local_z"):
            getattr(L, n).argtypes = [_dp, C.c_double, C.c_int, C.c_int, _dp]
        L.oracle_m2m.argtypes = [_dp, _dp, _dp, _dp, C.c_int, C.c_int]
        L.oracle_l2l.argtypes = [_dp, _dp, _dp, _dp, C.c_int, C.c_int]
        L.oracle_m2l.argtypes = [_dp, _dp, _dp, C.c_double, C.c_double, _dp, _dp, C.c_int, C.c_int, C.c_int,
                                 C.c_double, C.c_int, _ip, _ip]
        L.oracle_l2p.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
        L.oracle_p2m.argtypes = [C.c_int, _dp, C.c_int, C.c_int64, _dp, C.c_int, _dp]
        L.oracle_cartesian_to_spherical.argtypes = [C.c_double, C.c_double, C.c_double, _dp]
        _lib = L
    return _lib


def dptr(a):
    return a.ctypes.data_as(_dp)


def nh(p):
    return (p + 1) * (p + 2) // 2


def options(**kw):
    o = Options(expansion_order=5, leaf_size_source=20, leaf_size_target=0, multipole_acceptance=0.4,
                error_method=ERR_NONE, error_tolerance=0.0, bonus_expansion=1, shrink_recenter=1,
                list_method=LIST_TREE_STOP, farfield=1, nearfield=1, self_induced=1, upward_pass=1,
                horizontal_pass=1, downward_pass=1, scalar_potential=0, gradient=1, hessian=0, n_threads=0)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _tree_to_dict(v):
    nb = v.n_branches

    def a(ptr, n, dt=np.int64):
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n > 0 else np.zeros(0, dt)

    return dict(
        n_branches=nb, n_leaves=v.n_leaves,
        body_start=a(v.body_start, nb), body_count=a(v.body_count, nb), child_start=a(v.child_start, nb),
        n_children=a(v.n_children, nb), parent=a(v.parent, nb), i_leaf=a(v.i_leaf, nb),
        target_center=a(v.target_center, 3 * nb, np.float64).reshape(nb, 3),
        source_center=a(v.source_center, 3 * nb, np.float64).reshape(nb, 3),
        target_radius=a(v.target_radius, nb, np.float64), source_radius=a(v.source_radius, nb, np.float64),
        target_box=a(v.target_box, 3 * nb, np.float64).reshape(nb, 3),
        source_box=a(v.source_box, 3 * nb, np.float64).reshape(nb, 3),
        max_influence=a(v.max_influence, nb, np.float64),
        sort_index=a(v.sort_index, v.n_bodies),
        levels_start=a(v.levels_start, v.n_levels), levels_end=a(v.levels_end, v.n_levels),
        leaf_index=a(v.leaf_index, v.n_leaves))


def fmm(source_buf, kind, opt, target_pos=None, want_tree=False):
    """Run the oracle fmm!. source_buf: (N, d) float64; target_pos: (Nt, 3) or None for fmm!(system)."""
    L = lib()
    sb = np.ascontiguousarray(source_buf, dtype=np.float64)
    n_s, d = sb.shape
    if target_pos is None:
        tp, n_t = None, n_s
    else:
        tp = np.ascontiguousarray(target_pos, dtype=np.float64)
        n_t = tp.shape[0]
    run = L.oracle_fmm_run(dptr(tp) if tp is not None else None, n_t, dptr(sb), d, kind, n_s, C.byref(opt))
    if not run:
        raise RuntimeError("oracle_fmm_run failed")
    try:
        out = np.zeros((n_t, 16))
        L.oracle_run_output(run, dptr(out))
        res = dict(out=out)
        pm, ok = C.c_int(), C.c_int()
        L.oracle_run_pmax(run, C.byref(pm), C.byref(ok))
        res["pmax"], res["error_success"] = pm.value, bool(ok.value)
        t6 = np.zeros(6)
        L.oracle_run_times(run, dptr(t6))
        res["times"] = t6
        if want_tree:
            nm, nd = L.oracle_run_n_m2l(run), L.oracle_run_n_direct(run)
            m2l = np.zeros((nm, 2), np.int32)
            dl = np.zeros((nd, 2), np.int32)
            L.oracle_run_lists(run, m2l.ctypes.data_as(_i32p), dl.ctypes.data_as(_i32p))
            res["m2l"], res["direct"] = m2l, dl
            v = TreeView()
            L.oracle_run_target_tree(run, C.byref(v))
            res["target_tree"] = _tree_to_dict(v)
            v = TreeView()
            L.oracle_run_source_tree(run, C.byref(v))
            res["source_tree"] = _tree_to_dict(v)
        return res
    finally:
        L.oracle_run_free(run)


KIND_PER_BODY = -1


def concat_systems(systems):
    """A tuple of systems [(buf, kind), ...] as one (N, 8) buffer of rows
    (x, y, z, radius, s0, s1, s2, kind), in tuple order (the oracle's tuple mode)."""
    parts = []
    for buf, kind in systems:
        b = np.asarray(buf, dtype=np.float64)
        c = np.zeros((len(b), 8))
        c[:, :4] = b[:, :4]
        ns = 1 if kind == POINT_SOURCE else 3
        c[:, 4:4 + ns] = b[:, 4:4 + ns]
        c[:, 7] = kind
        parts.append(c)
    return np.concatenate(parts, axis=0)


def fmm_multi(systems, opt, target_pos, want_tree=False):
    """The oracle fmm! on a tuple of source systems [(buf, kind), ...]: one octree over all
    of them (Tree(systems::Tuple, ...), src/tree.jl:3-122)."""
    return fmm(concat_systems(systems), KIND_PER_BODY, opt, target_pos=target_pos, want_tree=want_tree)


def direct(source_buf, kind, target_pos=None, ps=1, gs=1, hs=0, n_threads=0):
    L = lib()
    sb = np.ascontiguousarray(source_buf, dtype=np.float64)
    n_s, d = sb.shape
    tp = None if target_pos is None else np.ascontiguousarray(target_pos, dtype=np.float64)
    n_t = n_s if tp is None else tp.shape[0]
    out = np.zeros((n_t, 16))
    rc = L.oracle_direct(dptr(tp) if tp is not None else None, n_t, dptr(sb), d, kind, n_s, ps, gs, hs, n_threads,
                         dptr(out))
    assert rc == 0
    return out


def direct_subset(source_buf, kind, ids, target_pos=None, n_threads=0):
    L = lib()
    sb = np.ascontiguousarray(source_buf, dtype=np.float64)
    n_s, d = sb.shape
    tp = None if target_pos is None else np.ascontiguousarray(target_pos, dtype=np.float64)
    n_t = n_s if tp is None else tp.shape[0]
    ids = np.ascontiguousarray(ids, dtype=np.int64)
    out = np.zeros((len(ids), 16))
    rc = L.oracle_direct_subset(dptr(tp) if tp is not None else None, n_t, ids.ctypes.data_as(_i64p), len(ids),
                                dptr(sb), d, kind, n_s, n_threads, dptr(out))
    assert rc == 0
    return out


# ---- expansion helpers (layout e[4*i + 2*set + reim]) ----
def expansion(p):
    return np.zeros(4 * nh(p))


def full_to_expansion(vec, p, set_=0, e=None):
    """Reference test layout (n, m=-n..n) -> compressed m>=0 expansion."""
    e = expansion(p) if e is None else e
    i = ic = 0
    for n in range(p + 1):
        for m in range(-n, n + 1):
            if m >= 0:
                e[4 * ic + 2 * set_] = vec[i][0]
                e[4 * ic + 2 * set_ + 1] = vec[i][1]
                ic += 1
            i += 1
    return e


def full_compressed(vec, p):
    """(n, m=-n..n) list -> array (nh, 2) of the m >= 0 entries."""
    out = []
    i = 0
    for n in range(p + 1):
        for m in range(-n, n + 1):
            if m >= 0:
                out.append(vec[i])
            i += 1
    return np.array(out)
