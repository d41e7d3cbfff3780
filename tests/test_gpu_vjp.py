"""fmm_vjp: gradients of a loss through fmm! against central finite differences.

The loss is L = sum_t w_t phi_t (point sources) or L = sum_t w_t . u_t (vortex
particles) with fixed random cotangents w.  The finite differences use the
all-pairs direct sum in FP64 (fmm_direct), so they carry no FMM error; the FMM
adjoint is compared at the accuracy of the expansion order (relative to the
largest gradient entry).  Strength derivatives are exact for a linear loss, so
their finite differences only carry rounding.
"""
import ctypes as C

import numpy as np
import pytest

import fastmultipole_b200 as fm
from fastmultipole_b200 import _lib as L

pytestmark = pytest.mark.gpu

H = 1e-6  # finite-difference step on positions (unit-cube scale)


@pytest.fixture(scope="module")
def ctx():
    c = fm.Context(0)
    yield c
    c.close()


def bodies(n, kind, seed):
    rng = np.random.default_rng(seed)
    d = 5 if kind == L.FMM_POINT_SOURCE else 7
    b = np.zeros((n, d))
    b[:, :3] = rng.random((n, 3))
    if kind == L.FMM_POINT_SOURCE:
        b[:, 4] = rng.random(n) - 0.3
    else:
        b[:, 4:7] = (2 * rng.random((n, 3)) - 1) / n
    return b


def direct_out(ctx, buf, kind, tpos=None):
    n = len(buf)
    nt = n if tpos is None else len(tpos)
    out = np.zeros((nt, 16))
    src = L.SourceSystem(kind, n, buf.shape[1], buf.ctypes.data, L.FMM_MEMORY_HOST)
    if tpos is None:
        tgt = L.TargetSystem(nt, None, 0, out.ctypes.data, L.FMM_MEMORY_HOST)
    else:
        tgt = L.TargetSystem(nt, tpos.ctypes.data, 3, out.ctypes.data, L.FMM_MEMORY_HOST)
    ctx.check(L.lib().fmm_direct(ctx.handle, C.byref(tgt), C.byref(src), 1, 1, 0, L.FMM_PRECISION_F64))
    return out


def loss(ctx, buf, kind, w, tpos=None):
    out = direct_out(ctx, np.ascontiguousarray(buf), kind, None if tpos is None else np.ascontiguousarray(tpos))
    if kind == L.FMM_POINT_SOURCE:
        return float(np.dot(w, out[:, 3]))
    return float(np.sum(w * out[:, 4:7]))


def check(ctx, kind, tpos, seed):
    n = 2500
    buf = bodies(n, kind, seed)
    rng = np.random.default_rng(seed + 100)
    nt = n if tpos is None else len(tpos)
    d_out = np.zeros((nt, 16))
    w = rng.standard_normal(nt) if kind == L.FMM_POINT_SOURCE else rng.standard_normal((nt, 3))
    if kind == L.FMM_POINT_SOURCE:
        d_out[:, 3] = w
    else:
        d_out[:, 4:7] = w
    opt = fm.make_options(expansion_order=14, leaf_size_source=40, multipole_acceptance=0.4, scalar_potential=True)
    out, dstr, dpos, dtp, res = fm.vjp_buffers(buf, kind, opt, d_out, tpos, ctx)
    # the forward buffer is the fmm! result
    ref = direct_out(ctx, buf, kind, tpos)
    rows = slice(3, 7) if kind == L.FMM_POINT_SOURCE else slice(4, 7)
    np.testing.assert_allclose(out[:, rows], ref[:, rows], rtol=0, atol=1e-8 * np.abs(ref[:, rows]).max())
    idx = rng.choice(n, 10, replace=False)
    # strengths (linear loss: central differences are exact up to rounding)
    sc = np.abs(dstr).max()
    for i in idx:
        for c in range(1 if kind == L.FMM_POINT_SOURCE else 3):
            hq = 1e-3 * max(abs(buf[i, 4 + c]), 1e-3 / n)
            bp, bm = buf.copy(), buf.copy()
            bp[i, 4 + c] += hq
            bm[i, 4 + c] -= hq
            fd = (loss(ctx, bp, kind, w, tpos) - loss(ctx, bm, kind, w, tpos)) / (2 * hq)
            got = dstr[i] if kind == L.FMM_POINT_SOURCE else dstr[i, c]
            assert abs(got - fd) <= 1e-7 * sc, (i, c, got, fd)
    # source positions
    sp = np.abs(dpos).max()
    for i in idx:
        for k in range(3):
            bp, bm = buf.copy(), buf.copy()
            bp[i, k] += H
            bm[i, k] -= H
            fd = (loss(ctx, bp, kind, w, tpos) - loss(ctx, bm, kind, w, tpos)) / (2 * H)
            assert abs(dpos[i, k] - fd) <= 2e-6 * sp, (i, k, dpos[i, k], fd)
    # target positions
    if tpos is not None:
        st = np.abs(dtp).max()
        for i in rng.choice(nt, 8, replace=False):
            for k in range(3):
                tp, tm = tpos.copy(), tpos.copy()
                tp[i, k] += H
                tm[i, k] -= H
                fd = (loss(ctx, buf, kind, w, tp) - loss(ctx, buf, kind, w, tm)) / (2 * H)
                assert abs(dtp[i, k] - fd) <= 2e-6 * st, (i, k, dtp[i, k], fd)


@pytest.mark.parametrize("kind", [L.FMM_POINT_SOURCE, L.FMM_POINT_VORTEX], ids=["source", "vortex"])
def test_vjp_self_matches_finite_differences(ctx, kind):
    check(ctx, kind, None, 31 + kind)


@pytest.mark.parametrize("kind", [L.FMM_POINT_SOURCE, L.FMM_POINT_VORTEX], ids=["source", "vortex"])
def test_vjp_probes_matches_finite_differences(ctx, kind):
    rng = np.random.default_rng(77 + kind)
    tpos = np.ascontiguousarray(-0.25 + 1.5 * rng.random((1500, 3)))
    check(ctx, kind, tpos, 41 + kind)


def test_vjp_python_api(ctx):
    rng = np.random.default_rng(5)
    n = 1200
    sys = fm.PointSources(rng.random((n, 3)), rng.random(n))
    w = rng.standard_normal(n)
    r = fm.vjp(sys, d_potential=w, leaf_size=30, expansion_order=12, context=ctx)
    assert r["d_strength"].shape == (n,) and r["d_position"].shape == (n, 3)
    # dL/dq is the potential of the adjoint sources: compare with the direct sum
    buf = np.zeros((n, 5))
    buf[:, :3] = sys.position
    buf[:, 4] = w
    psi = direct_out(ctx, buf, L.FMM_POINT_SOURCE)[:, 3]
    np.testing.assert_allclose(r["d_strength"], psi, rtol=0, atol=1e-8 * np.abs(psi).max())
