"""fmm_direct_noalloc: the allocation-free all-pairs direct! for callers that cannot
call cudaMalloc (graph-capture code, fixed device arenas, real-time loops).

It is checked through the C ABI against the existing fmm_direct entry point on two
calls in a row (the second call reuses the static scratch left by the first, so it
also checks that the accumulators are cleared).  This file is named so that pytest
collects it last; it also runs alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import fastmultipole_b200 as fm
from fastmultipole_b200 import _lib as L

pytestmark = pytest.mark.gpu


def bodies(n, kind, seed):
    rng = np.random.default_rng(seed)
    d = 5 if kind == L.FMM_POINT_SOURCE else 7
    b = np.zeros((n, d))
    b[:, :3] = rng.random((n, 3))
    b[:, 4:] = rng.standard_normal((n, d - 4)) / n
    return b


def reference_direct(ctx, buf, kind, tpos):
    out = np.zeros((len(tpos), 16))
    src = L.SourceSystem(kind, len(buf), buf.shape[1], buf.ctypes.data, L.FMM_MEMORY_HOST)
    tgt = L.TargetSystem(len(tpos), tpos.ctypes.data, 3, out.ctypes.data, L.FMM_MEMORY_HOST)
    ctx.check(L.lib().fmm_direct(ctx.handle, C.byref(tgt), C.byref(src), 1, 1, 1, L.FMM_PRECISION_F64))
    return out


@pytest.mark.parametrize("kind", [L.FMM_POINT_SOURCE, L.FMM_POINT_VORTEX])
def test_noalloc_direct_matches_fmm_direct_twice(kind):
    import torch
    ctx = fm.Context(0)
    stream = torch.cuda.current_stream()
    try:
        for call, (ns, nt) in enumerate([(3000, 2000), (1500, 2500)]):
            buf = bodies(ns, kind, 10 + call)
            tpos = np.ascontiguousarray(np.random.default_rng(20 + call).random((nt, 3)))
            ref = reference_direct(ctx, buf, kind, tpos)
            d_buf = torch.from_numpy(buf).cuda()
            d_pos = torch.from_numpy(tpos).cuda()
            d_out = torch.full((nt, 16), float("nan"), dtype=torch.float64, device="cuda")
            src = L.SourceSystem(kind, ns, buf.shape[1], d_buf.data_ptr(), L.FMM_MEMORY_DEVICE)
            tgt = L.TargetSystem(nt, d_pos.data_ptr(), 3, d_out.data_ptr(), L.FMM_MEMORY_DEVICE)
            rc = L.lib().fmm_direct_noalloc(0, C.c_void_p(stream.cuda_stream), C.byref(tgt), C.byref(src), 1, 1, 1,
                                            L.FMM_PRECISION_F64)
            assert rc == L.FMM_OK
            stream.synchronize()
            got = d_out.cpu().numpy()
            rows = slice(3, 7) if kind == L.FMM_POINT_SOURCE else slice(4, 16)
            scale = np.abs(ref[:, rows]).max()
            np.testing.assert_allclose(got[:, rows], ref[:, rows], rtol=0, atol=1e-12 * scale)
            np.testing.assert_array_equal(got[:, :3], tpos)
    finally:
        ctx.close()


def test_noalloc_rejects_oversize_and_host_memory():
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
