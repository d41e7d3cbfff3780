"""ctypes binding of libfmmb200.so (the C ABI declared in include/fmm_b200.h).

The product has no CPU fallback: importing the binding without the built
library, or creating a context without an sm_100 GPU, raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfmmb200.so")

(FMM_OK, FMM_ERR_ARGUMENT, FMM_ERR_CUDA, FMM_ERR_NO_DEVICE, FMM_ERR_TREE_DEPTH, FMM_ERR_MEMORY, FMM_ERR_STATE,
 FMM_PENDING) = range(8)
FMM_POINT_SOURCE, FMM_POINT_VORTEX = 1, 3
FMM_LIST_SELF_TUNING_TREE_STOP, FMM_LIST_BARBA, FMM_LIST_SELF_TUNING = 0, 1, 2
FMM_ERROR_NONE = 0
FMM_POWER_ABSOLUTE_GRADIENT = 1
FMM_POWER_RELATIVE_GRADIENT = 2
FMM_ROTATED_COEFFICIENTS_ABSOLUTE_GRADIENT = 3
FMM_ROTATED_COEFFICIENTS_RELATIVE_GRADIENT = 4
FMM_POWER_ABSOLUTE_POTENTIAL = 5
FMM_POWER_RELATIVE_POTENTIAL = 6
FMM_PRECISION_F64, FMM_PRECISION_MIXED = 0, 1
FMM_MEMORY_HOST, FMM_MEMORY_DEVICE = 0, 1

STATUS_NAMES = {0: "FMM_OK", 1: "FMM_ERR_ARGUMENT", 2: "FMM_ERR_CUDA", 3: "FMM_ERR_NO_DEVICE",
                4: "FMM_ERR_TREE_DEPTH", 5: "FMM_ERR_MEMORY", 6: "FMM_ERR_STATE", 7: "FMM_PENDING"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


class SourceSystem(C.Structure):
    _fields_ = [("kind", C.c_int), ("n_bodies", C.c_int64), ("data_per_body", C.c_int),
                ("buffer", C.c_void_p), ("memory", C.c_int)]


class TargetSystem(C.Structure):
    _fields_ = [("n_bodies", C.c_int64), ("positions", C.c_void_p), ("stride", C.c_int64),
                ("out", C.c_void_p), ("memory", C.c_int)]


class Options(C.Structure):
    _fields_ = [("expansion_order", C.c_int), ("leaf_size_source", C.c_int), ("leaf_size_target", C.c_int),
                ("multipole_acceptance", C.c_double), ("error_method", C.c_int), ("error_tolerance", C.c_double),
                ("bonus_expansion", C.c_int), ("shrink_recenter", C.c_int), ("list_method", C.c_int),
                ("farfield", C.c_int), ("nearfield", C.c_int), ("self_induced", C.c_int),
                ("upward_pass", C.c_int), ("horizontal_pass", C.c_int), ("downward_pass", C.c_int),
                ("scalar_potential", C.c_int), ("gradient", C.c_int), ("hessian", C.c_int),
                ("precision", C.c_int)]


class Result(C.Structure):
    _fields_ = [("p_max", C.c_int), ("error_success", C.c_int),
                ("n_target_branches", C.c_int64), ("n_source_branches", C.c_int64),
                ("n_target_leaves", C.c_int64), ("n_source_leaves", C.c_int64),
                ("n_m2l", C.c_int64), ("n_direct", C.c_int64), ("n_p2p_pairs", C.c_int64),
                ("m2l_flops", C.c_int64),
                ("t_total_ms", C.c_double), ("t_tree_ms", C.c_double), ("t_lists_ms", C.c_double),
                ("t_nearfield_ms", C.c_double), ("t_upward_ms", C.c_double), ("t_horizontal_ms", C.c_double),
                ("t_downward_ms", C.c_double), ("n_kernel_launches", C.c_int64),
                ("t_influence_ms", C.c_double)]


class TreeView(C.Structure):
    _fields_ = [("n_branches", C.c_int64), ("n_levels", C.c_int64), ("n_leaves", C.c_int64),
                ("n_bodies", C.c_int64)] + \
               [(n, _i64p) for n in ("body_start", "body_count", "child_start", "n_children", "parent", "i_leaf")] + \
               [(n, _dp) for n in ("target_center", "source_center", "target_radius", "source_radius",
                                   "target_box", "source_box", "max_influence")] + \
               [(n, _i64p) for n in ("sort_index", "levels_start", "levels_end", "leaf_index")]


class Request(C.Structure):
    _fields_ = [("target", TargetSystem), ("source", SourceSystem), ("options", Options)]


# every entry point of include/fmm_b200.h with its ctypes signature
SIGNATURES = {
    "fmm_ctx_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    "fmm_ctx_destroy": (C.c_int, [C.c_void_p]),
    "fmm_ctx_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "fmm_ctx_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "fmm_ctx_set_hbm_budget": (C.c_int, [C.c_void_p, C.c_size_t]),
    "fmm_ctx_device_bytes": (C.c_size_t, [C.c_void_p]),
    "fmm_ctx_last_error": (C.c_char_p, [C.c_void_p]),
    "fmm_default_options": (None, [C.POINTER(Options)]),
    "fmm_solve": (C.c_int, [C.c_void_p, C.POINTER(TargetSystem), C.POINTER(SourceSystem), C.POINTER(Options),
                            C.POINTER(Result)]),
    "fmm_direct": (C.c_int, [C.c_void_p, C.POINTER(TargetSystem), C.POINTER(SourceSystem), C.c_int, C.c_int,
                             C.c_int, C.c_int]),
    "fmm_solve_multi": (C.c_int, [C.c_void_p, C.POINTER(TargetSystem), C.POINTER(SourceSystem), C.c_int,
                                  C.POINTER(Options), C.POINTER(Result)]),
    "fmm_vjp": (C.c_int, [C.c_void_p, C.POINTER(TargetSystem), C.POINTER(SourceSystem), C.POINTER(Options), _dp, _dp,
                          _dp, _dp, C.POINTER(Result)]),
    "fmm_serve_start": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t]),
    "fmm_serve_submit": (C.c_int, [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_uint64)]),
    "fmm_serve_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Result), C.c_int]),
    "fmm_serve_stop": (C.c_int, [C.c_void_p]),
    "fmm_request_footprint": (C.c_size_t, [C.POINTER(Request)]),
    "fmm_measure_fp32_peak": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "fmm_direct_noalloc": (C.c_int, [C.c_int, C.c_void_p, C.POINTER(TargetSystem), C.POINTER(SourceSystem), C.c_int,
                                     C.c_int, C.c_int, C.c_int]),
    "fmm_get_tree": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(TreeView)]),
    "fmm_get_lists": (C.c_int, [C.c_void_p, _i32p, _i64p, _i32p, _i64p]),
    "fmm_get_expansions": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int64]),
    "fmm_op_p2m": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int, C.c_int64, _dp, C.c_int, _dp]),
    "fmm_op_m2m": (C.c_int, [C.c_void_p, C.c_int64, _dp, _dp, _dp, _dp, C.c_int, C.c_int]),
    "fmm_op_m2l": (C.c_int, [C.c_void_p, C.c_int64, _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, C.c_int, C.c_int,
                             C.c_double, C.c_int, _ip]),
    "fmm_op_l2l": (C.c_int, [C.c_void_p, C.c_int64, _dp, _dp, _dp, _dp, C.c_int, C.c_int]),
    "fmm_op_l2p": (C.c_int, [C.c_void_p, C.c_int64, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp]),
}

_lib = None


class FMMError(RuntimeError):
    def __init__(self, status, msg=""):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib():
    """The loaded library; raises if it has not been built (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m fastmultipole_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def dptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


class Context:
    """One fmm_ctx (device resources, stream, last solve for the parity exports)."""

    def __init__(self, device=0):
        self._h = C.c_void_p()
        rc = lib().fmm_ctx_create(C.byref(self._h), device)
        if rc != FMM_OK:
            raise FMMError(rc, f"no usable sm_100 device {device}")

    @property
    def handle(self):
        return self._h

    def check(self, rc):
        if rc != FMM_OK:
            raise FMMError(rc, lib().fmm_ctx_last_error(self._h).decode())

    def set_stream(self, stream_ptr):
        self.check(lib().fmm_ctx_set_stream(self._h, C.c_void_p(stream_ptr)))

    def set_timing(self, on):
        self.check(lib().fmm_ctx_set_timing(self._h, 1 if on else 0))

    def set_hbm_budget(self, nbytes):
        self.check(lib().fmm_ctx_set_hbm_budget(self._h, int(nbytes)))

    def device_bytes(self):
        return lib().fmm_ctx_device_bytes(self._h)

    def close(self):
        if self._h:
            lib().fmm_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_options():
    o = Options()
    lib().fmm_default_options(C.byref(o))
    return o
