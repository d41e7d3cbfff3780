"""GPU single-operator parity: the reference test suite's golden vectors through the
C ABI's fmm_op_* entry points (device kernels), plus agreement with the FP64 oracle
on random inputs at the orders the configurations use."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import fastmultipole_b200 as fm
from fastmultipole_b200 import _lib as L
import oracle_lib as O

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))["cases"]


@pytest.fixture(scope="module")
def ctx():
    c = fm.Context(0)
    yield c
    c.close()


def comp(e, p, set_=0):
    n = O.nh(p)
    return np.stack([e[2 * set_: 4 * n: 4], e[2 * set_ + 1: 4 * n: 4]], axis=1)


def d(a):
    return a.ctypes.data_as(L._dp)


def gpu_m2l(ctx, tgt, tc, src, sc, p, lh, em=0, eps=0.0, tbox=None, trad=None, maxinf=None, be=1):
    n = 1 if tgt.ndim == 1 else tgt.shape[0]
    pu = np.zeros(n, np.int32)
    ctx.check(L.lib().fmm_op_m2l(ctx.handle, n, d(tgt), d(np.ascontiguousarray(tc, float)),
                                 None if tbox is None else d(tbox), None if trad is None else d(trad),
                                 None if maxinf is None else d(maxinf), d(src), d(np.ascontiguousarray(sc, float)),
                                 p, lh, em, eps, be, pu.ctypes.data_as(C.POINTER(C.c_int))))
    return pu


def test_golden_m2l_point_and_shoot(ctx):
    c = GOLD["m2l_point_and_shoot"]
    p = c["p"]
    src = O.full_to_expansion(c["src"], p)
    out = O.expansion(p)
    gpu_m2l(ctx, out, np.array(c["target_center"]), src, np.array(c["source_center"]), p, 0)
    np.testing.assert_allclose(comp(out, p), O.full_compressed(c["expected"], p), rtol=0, atol=c["atol"])


def test_golden_m2m_and_p2m(ctx):
    c = GOLD["m2m_point_and_shoot"]
    p = c["p"]
    x = np.array(c["x"])
    xs = x + np.array(c["offset"])
    buf = np.array([[*xs, 0.0, c["mass"]]])
    M = O.expansion(p)
    ctx.check(L.lib().fmm_op_p2m(ctx.handle, L.FMM_POINT_SOURCE, d(buf), 5, 1, d(x), p, d(M)))
    M2 = O.expansion(p)
    x2 = x + np.array(c["shift"])
    ctx.check(L.lib().fmm_op_m2m(ctx.handle, 1, d(M2), d(x2), d(M), d(x), p, 0))
    exp = O.full_compressed(c["expected"], 10)[: O.nh(p)]
    np.testing.assert_allclose(comp(M2, p), exp, rtol=0, atol=c["atol"])


def test_golden_l2l(ctx):
    c = GOLD["l2l_point_and_shoot"]
    p = c["p"]
    src = O.full_to_expansion(c["src"], p)
    out = O.expansion(p)
    ctx.check(L.lib().fmm_op_l2l(ctx.handle, 1, d(out), d(np.array(c["target_center"])), d(src),
                                 d(np.array(c["source_center"])), p, 0))
    np.testing.assert_allclose(comp(out, p), O.full_compressed(c["expected"], p), rtol=0, atol=c["atol"])


def test_golden_l2p(ctx):
    c = GOLD["l2p_point_mass"]
    p = c["p"]
    Lx = O.full_to_expansion(c["local"], p)
    xt, ctr, xs, mass = map(np.array, (c["x_target"], c["center"], c["source"], c["mass"]))
    dx = (xt - ctr).reshape(1, 3)
    out = np.zeros((1, 13))
    ctx.check(L.lib().fmm_op_l2p(ctx.handle, 1, d(dx), d(Lx), p, 0, 1, 1, 1, d(out)))
    dd = xt - xs
    r = np.linalg.norm(dd)
    np.testing.assert_allclose(out[0, 0], mass / r / 4 / np.pi, atol=c["atol_phi"], rtol=0)
    np.testing.assert_allclose(out[0, 1:4], dd / r**3 * mass / 4 / np.pi, atol=c["atol_grad"], rtol=0)
    ref_phi, ref_g, ref_h = np.zeros(1), np.zeros(3), np.zeros(9)
    O.lib().oracle_l2p(O.dptr(dx[0].copy()), O.dptr(Lx), p, 0, 1, 1, 1, O.dptr(ref_phi), O.dptr(ref_g),
                       O.dptr(ref_h))
    np.testing.assert_allclose(out[0, 4:], ref_h, rtol=1e-10, atol=1e-14)


@pytest.mark.parametrize("name", ["lh_m2m", "lh_m2l", "lh_l2l"])
def test_golden_lamb_helmholtz(ctx, name):
    c = GOLD[name]
    p = c["p"]
    src = O.full_to_expansion(c["phi"], p)
    O.full_to_expansion(c["chi"], p, 1, src)
    out = O.expansion(p)
    tc, sc = np.array(c["target_center"]), np.array(c["source_center"])
    if name == "lh_m2m":
        ctx.check(L.lib().fmm_op_m2m(ctx.handle, 1, d(out), d(tc), d(src), d(sc), p, 1))
    elif name == "lh_l2l":
        ctx.check(L.lib().fmm_op_l2l(ctx.handle, 1, d(out), d(tc), d(src), d(sc), p, 1))
    else:
        gpu_m2l(ctx, out, tc, src, sc, p, 1)
    k = O.nh(c["n_check"])
    for s, key in ((0, "expected_phi"), (1, "expected_chi")):
        np.testing.assert_allclose(comp(out, p, s)[:k], O.full_compressed(c[key], p)[:k], rtol=c.get("rtol", 0),
                                   atol=c["atol"])


def test_golden_vorton_p2m_m2l_l2p(ctx):
    c = GOLD["lh_vorton"]
    p = c["p"]
    M = O.full_to_expansion(c["phi"], p)
    O.full_to_expansion(c["chi"], p, 1, M)
    xs, G, sc = map(np.array, (c["x_source"], c["gamma"], c["source_center"]))
    Mp = O.expansion(p)
    buf = np.array([[*xs, 0.0, *G]])
    ctx.check(L.lib().fmm_op_p2m(ctx.handle, L.FMM_POINT_VORTEX, d(buf), 7, 1, d(sc), p, d(Mp)))
    np.testing.assert_allclose(Mp, M, rtol=0, atol=1e-12)
    Lx = O.expansion(p)
    tc = np.array(c["target_center"])
    gpu_m2l(ctx, Lx, tc, M, sc, p, 1)
    xt = np.array(c["x_target"])
    dx = (xt - tc).reshape(1, 3)
    out = np.zeros((1, 13))
    ctx.check(L.lib().fmm_op_l2p(ctx.handle, 1, d(dx), d(Lx), p, 1, 0, 1, 1, d(out)))
    dd = xt - xs
    r = np.linalg.norm(dd)
    np.testing.assert_allclose(out[0, 1:4], -np.cross(dd, G) / r**3 / (4 * np.pi), atol=c["atol_grad"], rtol=0)


@pytest.mark.parametrize("p,lh,em", [(6, 0, 0), (10, 0, 0), (12, 1, 0), (16, 0, 0), (10, 0, 1), (10, 0, 2),
                                     (10, 1, 2), (10, 0, 3), (12, 1, 4), (20, 0, 0), (10, 0, 5), (10, 1, 6),
                                     (14, 0, 6)])
def test_m2l_batch_matches_oracle(ctx, p, lh, em):
    rng = np.random.default_rng(100 * p + 10 * lh + em)
    n = 64
    nh4 = 4 * O.nh(p)
    src = rng.standard_normal((n, nh4)) * 1e-2
    if not lh:
        src.reshape(n, -1, 4)[:, :, 2:] = 0.0
    sc = rng.random((n, 3))
    tc = sc + rng.choice([-1, 1], (n, 3)) * (1.5 + rng.random((n, 3)))
    tbox = 0.2 + 0.1 * rng.random((n, 3))
    trad = np.linalg.norm(tbox, axis=1)
    maxinf = 1 + rng.random(n)
    eps = 1e-6
    out = np.zeros((n, nh4))
    pu = gpu_m2l(ctx, out, tc, src, sc, p, lh, em, eps, tbox, trad, maxinf)
    for k in range(n):
        ref = O.expansion(p)
        pr, ok = C.c_int(), C.c_int()
        O.lib().oracle_m2l(O.dptr(ref), O.dptr(tc[k].copy()), O.dptr(tbox[k].copy()), trad[k], maxinf[k],
                           O.dptr(src[k].copy()), O.dptr(sc[k].copy()), p, lh, em, eps, 1, C.byref(pr),
                           C.byref(ok))
        exp_pu = pr.value if ok.value else -pr.value - 1
        assert pu[k] == exp_pu, (k, pu[k], exp_pu)
        scale = np.abs(ref).max()
        np.testing.assert_allclose(out[k], ref, rtol=0, atol=1e-12 * scale)


@pytest.mark.parametrize("p,lh", [(6, 0), (12, 1), (20, 0)])
def test_m2m_l2l_batch_match_oracle(ctx, p, lh):
    rng = np.random.default_rng(p + lh)
    n = 32
    nh4 = 4 * O.nh(p)
    src = rng.standard_normal((n, nh4))
    sc = rng.random((n, 3))
    tc = sc + 0.3 * rng.standard_normal((n, 3))
    for op, ofn in ((L.lib().fmm_op_m2m, O.lib().oracle_m2m), (L.lib().fmm_op_l2l, O.lib().oracle_l2l)):
        out = np.zeros((n, nh4))
        ctx.check(op(ctx.handle, n, d(out), d(tc), d(src), d(sc), p, lh))
        for k in range(n):
            ref = O.expansion(p)
            ofn(O.dptr(ref), O.dptr(tc[k].copy()), O.dptr(src[k].copy()), O.dptr(sc[k].copy()), p, lh)
            if not lh:
                ref.reshape(-1, 4)[:, 2:] = 0.0
            # unit-normal coefficients up to degree 20 (no decay with n) amplify summation-order differences
            np.testing.assert_allclose(out[k], ref, rtol=0, atol=1e-10 * np.abs(ref).max())


@pytest.mark.parametrize("kind,p", [(L.FMM_POINT_SOURCE, 10), (L.FMM_POINT_VORTEX, 12)])
def test_p2m_matches_oracle(ctx, kind, p):
    rng = np.random.default_rng(kind * 7 + p)
    n = 50
    dd = 5 if kind == L.FMM_POINT_SOURCE else 7
    buf = np.zeros((n, dd))
    buf[:, :3] = rng.random((n, 3))
    buf[:, 4:] = rng.standard_normal((n, dd - 4))
    ctr = np.array([0.45, 0.52, 0.49])
    M = O.expansion(p)
    ctx.check(L.lib().fmm_op_p2m(ctx.handle, kind, d(buf), dd, n, d(ctr), p, d(M)))
    ref = O.expansion(p)
    O.lib().oracle_p2m(kind, O.dptr(buf), dd, n, O.dptr(ctr), p, O.dptr(ref))
    np.testing.assert_allclose(M, ref, rtol=0, atol=1e-13 * np.abs(ref).max())


@pytest.mark.parametrize("p,lh", [(6, 0), (12, 1)])
def test_l2p_matches_oracle(ctx, p, lh):
    rng = np.random.default_rng(3 + p)
    Lx = rng.standard_normal(4 * O.nh(p))
    if not lh:
        Lx.reshape(-1, 4)[:, 2:] = 0
    n = 40
    dx = 0.3 * rng.standard_normal((n, 3))
    out = np.zeros((n, 13))
    ctx.check(L.lib().fmm_op_l2p(ctx.handle, n, d(dx), d(Lx), p, lh, 1, 1, 1, d(out)))
    for k in range(n):
        phi, g, H = np.zeros(1), np.zeros(3), np.zeros(9)
        O.lib().oracle_l2p(O.dptr(dx[k].copy()), O.dptr(Lx), p, lh, 1, 1, 1, O.dptr(phi), O.dptr(g), O.dptr(H))
        ref = np.concatenate([phi, g, H])
        np.testing.assert_allclose(out[k], ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_measured_fp32_peak_is_plausible():
    # the near field's roofline denominator: independent FMA chains on every SM of a B200
    # (nominal 148 SMs x 128 lanes x 2 flop x ~1.9 GHz = 74 TFLOP/s)
    for packed in (0, 1):
        v = C.c_double(0.0)
        assert L.lib().fmm_measure_fp32_peak(0, packed, C.byref(v)) == L.FMM_OK
        assert 20.0 < v.value < 90.0, (packed, v.value)
