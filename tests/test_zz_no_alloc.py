"""fmm_direct_noalloc: the allocation-free all-pairs direct! for callers that cannot
call cudaMalloc (graph-capture code, fixed device arenas, real-time loops).

Each case runs two calls in a row through the C ABI (the second call reuses the
static scratch left by the first, so it also checks that the accumulators are
cleared):
* FP64 against the existing fmm_direct entry point (itself pinned to the oracle) at
  1e-12 of the largest value;
* MIXED against the oracle's FP64 all-pairs direct sum, relative L2 error below 1e-5
  (the bound the mixed paths are held to elsewhere);
* explicit target positions and the self-target form (target->positions == NULL).

This file is named so that pytest collects it last.  To run it alone in a fresh
process: python -m pytest tests/test_zz_no_alloc.py -m gpu
"""
import ctypes as C

import numpy as np
import pytest

import fastmultipole_b200 as fm
from fastmultipole_b200 import _lib as L
import oracle_lib as O

pytestmark = pytest.mark.gpu


def bodies(n, kind, seed):
    rng = np.random.default_rng(seed)
    d = 5 if kind == L.FMM_POINT_SOURCE else 7
    b = np.zeros((n, d))
    b[:, :3] = rng.random((n, 3))
    b[:, 4:] = rng.standard_normal((n, d - 4)) / n
    return b


def reference_direct(ctx, buf, kind, tpos):
    n_t = len(buf) if tpos is None else len(tpos)
    out = np.zeros((n_t, 16))
    src = L.SourceSystem(kind, len(buf), buf.shape[1], buf.ctypes.data, L.FMM_MEMORY_HOST)
    tgt = L.TargetSystem(n_t, None if tpos is None else tpos.ctypes.data, 3, out.ctypes.data, L.FMM_MEMORY_HOST)
    ctx.check(L.lib().fmm_direct(ctx.handle, C.byref(tgt), C.byref(src), 1, 1, 1, L.FMM_PRECISION_F64))
    return out


def rows_of(kind):
    return slice(3, 7) if kind == L.FMM_POINT_SOURCE else slice(4, 16)


@pytest.mark.parametrize("self_target", [False, True])
@pytest.mark.parametrize("precision", [L.FMM_PRECISION_F64, L.FMM_PRECISION_MIXED])
@pytest.mark.parametrize("kind", [L.FMM_POINT_SOURCE, L.FMM_POINT_VORTEX])
def test_noalloc_direct_matches_direct_twice(kind, precision, self_target):
    import torch
    ctx = fm.Context(0)
    stream = torch.cuda.current_stream()
    rows = rows_of(kind)
    try:
        for call, (ns, nt) in enumerate([(3000, 2000), (1500, 2500)]):
            buf = bodies(ns, kind, 10 + call)
            tpos = None if self_target else np.ascontiguousarray(np.random.default_rng(20 + call).random((nt, 3)))
            nt = ns if self_target else nt
            d_buf = torch.from_numpy(buf).cuda()
            d_pos = None if self_target else torch.from_numpy(tpos).cuda()
            d_out = torch.full((nt, 16), float("nan"), dtype=torch.float64, device="cuda")
            src = L.SourceSystem(kind, ns, buf.shape[1], d_buf.data_ptr(), L.FMM_MEMORY_DEVICE)
            tgt = L.TargetSystem(nt, None if self_target else d_pos.data_ptr(), 3, d_out.data_ptr(),
                                 L.FMM_MEMORY_DEVICE)
            rc = L.lib().fmm_direct_noalloc(0, C.c_void_p(stream.cuda_stream), C.byref(tgt), C.byref(src), 1, 1, 1,
                                            precision)
            assert rc == L.FMM_OK
            stream.synchronize()
            got = d_out.cpu().numpy()
            np.testing.assert_array_equal(got[:, :3], buf[:, :3] if self_target else tpos)
            if precision == L.FMM_PRECISION_F64:
                ref = reference_direct(ctx, buf, kind, tpos)
                scale = np.abs(ref[:, rows]).max()
                np.testing.assert_allclose(got[:, rows], ref[:, rows], rtol=0, atol=1e-12 * scale)
            else:
                ref = O.direct(buf, kind, target_pos=tpos, ps=1, gs=1, hs=1)
                err = np.linalg.norm(got[:, rows] - ref[:, rows]) / np.linalg.norm(ref[:, rows])
                assert err < 1e-5, err
    finally:
        ctx.close()


def test_noalloc_rejects_oversize_negative_and_host_memory():
    import torch
    n = 32769
    buf = bodies(8, L.FMM_POINT_SOURCE, 1)
    d_buf = torch.from_numpy(buf).cuda()
    d_out = torch.zeros((8, 16), dtype=torch.float64, device="cuda")
    big = L.SourceSystem(L.FMM_POINT_SOURCE, n, 5, d_buf.data_ptr(), L.FMM_MEMORY_DEVICE)
    tgt = L.TargetSystem(8, d_buf.data_ptr(), 5, d_out.data_ptr(), L.FMM_MEMORY_DEVICE)
    assert L.lib().fmm_direct_noalloc(0, None, C.byref(tgt), C.byref(big), 1, 1, 0, 0) == L.FMM_ERR_MEMORY
    host = L.SourceSystem(L.FMM_POINT_SOURCE, 8, 5, buf.ctypes.data, L.FMM_MEMORY_HOST)
    assert L.lib().fmm_direct_noalloc(0, None, C.byref(tgt), C.byref(host), 1, 1, 0, 0) == L.FMM_ERR_ARGUMENT
    ok = L.SourceSystem(L.FMM_POINT_SOURCE, 8, 5, d_buf.data_ptr(), L.FMM_MEMORY_DEVICE)
    neg = L.TargetSystem(-5, d_buf.data_ptr(), 5, d_out.data_ptr(), L.FMM_MEMORY_DEVICE)
    assert L.lib().fmm_direct_noalloc(0, None, C.byref(neg), C.byref(ok), 1, 1, 0, 0) == L.FMM_ERR_ARGUMENT
