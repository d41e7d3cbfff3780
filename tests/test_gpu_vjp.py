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


def loss(ctx, buf, kind, w, tpos=None, wpos=None):
    out = direct_out(ctx, np.ascontiguousarray(buf), kind, None if tpos is None else np.ascontiguousarray(tpos))
    extra = 0.0 if wpos is None else float(np.sum(wpos * out[:, 0:3]))  # rows 1..3 echo the target positions
    if kind == L.FMM_POINT_SOURCE:
        return float(np.dot(w, out[:, 3])) + extra
    return float(np.sum(w * out[:, 4:7])) + extra


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
    # cotangents on the echoed target positions (rows 1..3) pass straight through
    wpos = 0.1 * rng.standard_normal((nt, 3))
    d_out[:, 0:3] = wpos
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
            fd = (loss(ctx, bp, kind, w, tpos, wpos) - loss(ctx, bm, kind, w, tpos, wpos)) / (2 * hq)
            got = dstr[i] if kind == L.FMM_POINT_SOURCE else dstr[i, c]
            assert abs(got - fd) <= 1e-7 * sc, (i, c, got, fd)
    # source positions
    sp = np.abs(dpos).max()
    for i in idx:
        for k in range(3):
            bp, bm = buf.copy(), buf.copy()
            bp[i, k] += H
            bm[i, k] -= H
            fd = (loss(ctx, bp, kind, w, tpos, wpos) - loss(ctx, bm, kind, w, tpos, wpos)) / (2 * H)
            assert abs(dpos[i, k] - fd) <= 2e-6 * sp, (i, k, dpos[i, k], fd)
    # target positions
    if tpos is not None:
        st = np.abs(dtp).max()
        for i in rng.choice(nt, 8, replace=False):
            for k in range(3):
                tp, tm = tpos.copy(), tpos.copy()
                tp[i, k] += H
                tm[i, k] -= H
                fd = (loss(ctx, buf, kind, w, tp, wpos) - loss(ctx, buf, kind, w, tm, wpos)) / (2 * H)
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


@pytest.mark.parametrize("kind", [L.FMM_POINT_SOURCE, L.FMM_POINT_VORTEX], ids=["source", "vortex"])
def test_vjp_rejects_cotangents_it_cannot_propagate(ctx, kind):
    # gradient rows of point sources (dipole sources would be needed), the velocity gradient
    # of vortex particles: an error, not a silently wrong gradient
    buf = bodies(300, kind, 3)
    opt = fm.make_options(expansion_order=6, leaf_size_source=30, multipole_acceptance=0.5, scalar_potential=True)
    d_out = np.zeros((300, 16))
    d_out[7, 5 if kind == L.FMM_POINT_SOURCE else 9] = 1.0
    with pytest.raises(L.FMMError) as e:
        fm.vjp_buffers(buf, kind, opt, d_out, None, ctx)
    assert e.value.status == L.FMM_ERR_ARGUMENT


def test_vjp_mixed_precision_matches_f64(ctx):
    # the mixed-precision forward and adjoint solves against the FP64 ones
    n = 20000
    buf = bodies(n, L.FMM_POINT_SOURCE, 12)
    rng = np.random.default_rng(13)
    tpos = np.ascontiguousarray(-0.5 + 2.0 * rng.random((4000, 3)))
    d_out = np.zeros((4000, 16))
    d_out[:, 3] = rng.standard_normal(4000)
    r = {}
    for prec in ("f64", "mixed"):
        opt = fm.make_options(expansion_order=8, leaf_size_source=50, multipole_acceptance=0.5,
                              scalar_potential=True, precision=prec)
        r[prec] = fm.vjp_buffers(buf, L.FMM_POINT_SOURCE, opt, d_out, tpos, ctx)
    for k in (1, 2, 3):
        a, b = r["mixed"][k], r["f64"][k]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5, k


def test_vjp_adjoint_workload_shape_finite_differences(ctx):
    # 200k sources U[0,1]^3, 10k probes U[-0.5,1.5]^3, p = 8, L = sum phi^2 (dL/dphi = 2 phi);
    # central differences of the exact loss (FP64 all-pairs) on 64 coordinates, h = 1e-6
    rng = np.random.default_rng(4)
    n, npr = 200_000, 10_000
    buf = np.zeros((n, 5))
    buf[:, :3] = rng.random((n, 3))
    buf[:, 4] = rng.random(n)
    probes = np.ascontiguousarray(-0.5 + 2.0 * rng.random((npr, 3)))
    opt = fm.make_options(expansion_order=8, leaf_size_source=50, multipole_acceptance=0.5, scalar_potential=True)
    out, _ = fm.solve_buffers(buf, L.FMM_POINT_SOURCE, opt, target_pos=probes, ctx=ctx)
    d_out = np.zeros((npr, 16))
    d_out[:, 3] = 2.0 * out[:, 3]
    _, dq, dx, dy, _ = fm.vjp_buffers(buf, L.FMM_POINT_SOURCE, opt, d_out, probes, ctx)

    def lossq(b, pr):
        o = direct_out(ctx, np.ascontiguousarray(b), L.FMM_POINT_SOURCE, np.ascontiguousarray(pr))
        return float(np.sum(o[:, 3] ** 2))

    h = 1e-6
    devs = []
    for j in range(64):
        which = j % 3
        if which == 0:
            i = rng.integers(0, n)
            bp, bm = buf.copy(), buf.copy()
            hq = 1e-3 * buf[i, 4]
            bp[i, 4] += hq
            bm[i, 4] -= hq
            fd = (lossq(bp, probes) - lossq(bm, probes)) / (2 * hq)
            devs.append(abs(dq[i] - fd) / np.abs(dq).max())
        elif which == 1:
            i, k = rng.integers(0, n), rng.integers(0, 3)
            bp, bm = buf.copy(), buf.copy()
            bp[i, k] += h
            bm[i, k] -= h
            fd = (lossq(bp, probes) - lossq(bm, probes)) / (2 * h)
            devs.append(abs(dx[i, k] - fd) / np.abs(dx).max())
        else:
            i, k = rng.integers(0, npr), rng.integers(0, 3)
            pp, pm = probes.copy(), probes.copy()
            pp[i, k] += h
            pm[i, k] -= h
            fd = (lossq(buf, pp) - lossq(buf, pm)) / (2 * h)
            devs.append(abs(dy[i, k] - fd) / np.abs(dy).max())
    assert max(devs) <= 1e-5, max(devs)


def test_vjp_gap_to_the_discrete_gradient(ctx):
    # fmm_vjp is the continuous adjoint (a second FMM with the cotangents as strengths); the
    # gradient ReverseDiff takes through the reference is the discrete one, the derivative of
    # the FMM's own output.  Measured here against central differences of the FMM loss itself
    # (FP64, same options; the loss is linear in the strengths, so those differences are exact
    # up to rounding).  The exact gradient dL/dq_i = sum_t w_t / (4 pi r_ti) is the direct
    # potential of sources of strength w.  The gap between the two FMM gradients is real (well
    # above rounding) and no larger than the truncation error of the adjoint solve itself.
    n = 3000
    buf = bodies(n, L.FMM_POINT_SOURCE, 91)
    rng = np.random.default_rng(92)
    w = rng.standard_normal(n)
    d_out = np.zeros((n, 16))
    d_out[:, 3] = w
    opt = fm.make_options(expansion_order=4, leaf_size_source=10, multipole_acceptance=0.6, scalar_potential=True)
    _, dstr, _, _, _ = fm.vjp_buffers(buf, L.FMM_POINT_SOURCE, opt, d_out, None, ctx)
    wbuf = buf.copy()
    wbuf[:, 4] = w
    exact = direct_out(ctx, wbuf, L.FMM_POINT_SOURCE)[:, 3]
    sc = np.abs(exact).max()
    adj_err = np.abs(dstr - exact).max() / sc
    assert 1e-7 < adj_err < 1e-2, adj_err  # a visible truncation error at p = 4

    def loss_fmm(b):
        o, _ = fm.solve_buffers(b, L.FMM_POINT_SOURCE, opt, None, ctx)
        return float(np.dot(w, o[:, 3]))

    gaps, disc_err = [], []
    for i in rng.choice(n, 12, replace=False):
        hq = 1e-3 * max(abs(buf[i, 4]), 1e-3)
        bp, bm = buf.copy(), buf.copy()
        bp[i, 4] += hq
        bm[i, 4] -= hq
        disc = (loss_fmm(bp) - loss_fmm(bm)) / (2 * hq)
        gaps.append(abs(dstr[i] - disc) / sc)
        disc_err.append(abs(disc - exact[i]) / sc)
    gap = max(gaps)
    assert 1e-12 < gap <= 2 * adj_err, (gap, adj_err)
    assert max(disc_err) <= 2 * adj_err, (max(disc_err), adj_err)
    print(f"continuous adjoint vs discrete gradient: {gap:.2e}; adjoint vs exact (all bodies): {adj_err:.2e}; "
          f"discrete vs exact (sampled): {max(disc_err):.2e}")
