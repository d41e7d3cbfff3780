"""Pin the FP64 oracle against the reference test suite's golden vectors.

Every case comes from FastMultipole.jl's own tests (extracted as text by
tests/golden/make_golden.py); tolerances are the reference tests' own.
"""
import json
import math
import os

import numpy as np
import pytest
from scipy.special import factorial, lpmv

import oracle_lib as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))["cases"]


def comp(e, p, set_=0):
    n = O.nh(p)
    return np.stack([e[2 * set_: 4 * n: 4], e[2 * set_ + 1: 4 * n: 4]], axis=1)


def test_m2l_coaxial():
    c = GOLD["m2l_z"]
    p = c["p"]
    src = O.full_to_expansion(c["src"], p)
    out = O.expansion(p)
    O.lib().oracle_translate_multipole_to_local_z(O.dptr(src), c["r"], p, 0, O.dptr(out))
    np.testing.assert_allclose(comp(out, p), O.full_compressed(c["expected"], p), rtol=0, atol=c["atol"])


def test_m2m_coaxial():
    c = GOLD["m2m_z"]
    p = c["p"]
    src = O.expansion(p)
    for i, (re, im) in enumerate(c["src_compressed"]):
        src[4 * i], src[4 * i + 1] = re, im
    out = O.expansion(p)
    O.lib().oracle_translate_multipole_z(O.dptr(src), c["r"], p, 0, O.dptr(out))
    np.testing.assert_allclose(comp(out, p), O.full_compressed(c["expected"], p), rtol=0, atol=c["atol"])


def test_l2l_coaxial():
    c = GOLD["l2l_z"]
    p = c["p"]
    src = O.full_to_expansion(c["src"], p)
    out = O.expansion(p)
    O.lib().oracle_translate_local_z(O.dptr(src), c["r"], p, 0, O.dptr(out))
    np.testing.assert_allclose(comp(out, p), O.full_compressed(c["expected"], p), rtol=0, atol=c["atol"])


def test_m2l_point_and_shoot():
    c = GOLD["m2l_point_and_shoot"]
    p = c["p"]
    src = O.full_to_expansion(c["src"], p)
    out = O.expansion(p)
    tc, sc, box = np.array(c["target_center"]), np.array(c["source_center"]), np.zeros(3)
    pu, ok = O.C.c_int(), O.C.c_int()
    O.lib().oracle_m2l(O.dptr(out), O.dptr(tc), O.dptr(box), 0.0, 0.0, O.dptr(src), O.dptr(sc), p, 0, 0, 0.0, 1,
                       O.C.byref(pu), O.C.byref(ok))
    assert pu.value == p and ok.value == 1
    np.testing.assert_allclose(comp(out, p), O.full_compressed(c["expected"], p), rtol=0, atol=c["atol"])


def test_p2m_and_m2m_point_and_shoot():
    c = GOLD["m2m_point_and_shoot"]
    p = c["p"]
    x = np.array(c["x"])
    xs = x + np.array(c["offset"])
    buf = np.array([[*xs, 0.0, c["mass"]]])
    M = O.expansion(p)
    O.lib().oracle_p2m(O.POINT_SOURCE, O.dptr(buf), 5, 1, O.dptr(x), p, O.dptr(M))
    M2 = O.expansion(p)
    x2 = x + np.array(c["shift"])
    O.lib().oracle_m2m(O.dptr(M2), O.dptr(x2), O.dptr(M), O.dptr(x), p, 0)
    exp = O.full_compressed(c["expected"], 10)[: O.nh(p)]
    np.testing.assert_allclose(comp(M2, p), exp, rtol=0, atol=c["atol"])


def test_l2l_point_and_shoot():
    c = GOLD["l2l_point_and_shoot"]
    p = c["p"]
    src = O.full_to_expansion(c["src"], p)
    out = O.expansion(p)
    tc, sc = np.array(c["target_center"]), np.array(c["source_center"])
    O.lib().oracle_l2l(O.dptr(out), O.dptr(tc), O.dptr(src), O.dptr(sc), p, 0)
    np.testing.assert_allclose(comp(out, p), O.full_compressed(c["expected"], p), rtol=0, atol=c["atol"])


def test_l2p_point_mass():
    c = GOLD["l2p_point_mass"]
    p = c["p"]
    L = O.full_to_expansion(c["local"], p)
    xt, ctr, xs, mass = map(np.array, (c["x_target"], c["center"], c["source"], c["mass"]))
    dx = xt - ctr
    phi, g, H = np.zeros(1), np.zeros(3), np.zeros(9)
    O.lib().oracle_l2p(O.dptr(dx), O.dptr(L), p, 0, 1, 1, 1, O.dptr(phi), O.dptr(g), O.dptr(H))
    d = xt - xs
    r = np.linalg.norm(d)
    np.testing.assert_allclose(phi[0], mass / r / 4 / np.pi, atol=c["atol_phi"], rtol=0)
    np.testing.assert_allclose(g, d / r**3 * mass / 4 / np.pi, atol=c["atol_grad"], rtol=0)
    h_test = -np.array([[2 * d[0]**2 - d[1]**2 - d[2]**2, 3 * d[0] * d[1], 3 * d[0] * d[2]],
                        [3 * d[0] * d[1], -d[0]**2 + 2 * d[1]**2 - d[2]**2, 3 * d[1] * d[2]],
                        [3 * d[0] * d[2], 3 * d[1] * d[2], -d[0]**2 - d[1]**2 + 2 * d[2]**2]]) / r**5 * mass / 4 / np.pi
    # SMatrix(h...) column-major 9-vector vs the symmetric analytic hessian
    np.testing.assert_allclose(H, h_test.flatten(order="F"), atol=c["atol_hess"], rtol=0)


@pytest.mark.parametrize("name", ["lh_multipole", "lh_local"])
def test_lamb_helmholtz_transforms(name):
    # the transforms are exercised through the coaxial ops at r=... via a zero-length translation? No: call the
    # M2M/L2L chain would rotate.  The oracle exposes the transforms inside the translation chain only, so this
    # case is checked through the C++ test hook below.
    c = GOLD[name]
    p = c["p"]
    e = O.full_to_expansion(c["phi"], p)
    O.full_to_expansion(c["chi"], p, 1, e)
    fn = O.lib().oracle_lh_transform
    fn.argtypes = [O.C.POINTER(O.C.c_double), O.C.c_double, O.C.c_int, O.C.c_int]
    fn(O.dptr(e), c["r"], p, 1 if name == "lh_local" else 0)
    np.testing.assert_allclose(comp(e, p, 0), O.full_compressed(c["expected_phi"], p), rtol=0, atol=c["atol"])
    np.testing.assert_allclose(comp(e, p, 1), O.full_compressed(c["expected_chi"], p), rtol=0, atol=c["atol"])


@pytest.mark.parametrize("name", ["lh_m2m", "lh_m2l", "lh_l2l"])
def test_lamb_helmholtz_translations(name):
    c = GOLD[name]
    p = c["p"]
    src = O.full_to_expansion(c["phi"], p)
    O.full_to_expansion(c["chi"], p, 1, src)
    out = O.expansion(p)
    tc, sc = np.array(c["target_center"]), np.array(c["source_center"])
    if name == "lh_m2m":
        O.lib().oracle_m2m(O.dptr(out), O.dptr(tc), O.dptr(src), O.dptr(sc), p, 1)
    elif name == "lh_l2l":
        O.lib().oracle_l2l(O.dptr(out), O.dptr(tc), O.dptr(src), O.dptr(sc), p, 1)
    else:
        box = np.zeros(3)
        pu, ok = O.C.c_int(), O.C.c_int()
        O.lib().oracle_m2l(O.dptr(out), O.dptr(tc), O.dptr(box), 0.0, 0.0, O.dptr(src), O.dptr(sc), p, 1, 0, 0.0,
                           1, O.C.byref(pu), O.C.byref(ok))
    k = O.nh(c["n_check"])
    rtol = c.get("rtol", 0.0)
    for s, key in ((0, "expected_phi"), (1, "expected_chi")):
        np.testing.assert_allclose(comp(out, p, s)[:k], O.full_compressed(c[key], p)[:k], rtol=rtol, atol=c["atol"])


def test_lamb_helmholtz_vorton():
    c = GOLD["lh_vorton"]
    p = c["p"]
    M = O.full_to_expansion(c["phi"], p)
    O.full_to_expansion(c["chi"], p, 1, M)
    # the golden multipole is P2M of the vorton about source_center
    xs, G, sc = map(np.array, (c["x_source"], c["gamma"], c["source_center"]))
    Mp = O.expansion(p)
    buf = np.array([[*xs, 0.0, *G]])
    O.lib().oracle_p2m(O.POINT_VORTEX, O.dptr(buf), 7, 1, O.dptr(sc), p, O.dptr(Mp))
    np.testing.assert_allclose(Mp, M, rtol=0, atol=1e-12)
    L = O.expansion(p)
    tc, box = np.array(c["target_center"]), np.zeros(3)
    pu, ok = O.C.c_int(), O.C.c_int()
    O.lib().oracle_m2l(O.dptr(L), O.dptr(tc), O.dptr(box), 0.0, 0.0, O.dptr(M), O.dptr(sc), p, 1, 0, 0.0, 1,
                       O.C.byref(pu), O.C.byref(ok))
    xt = np.array(c["x_target"])
    dx = xt - tc
    phi, g, H = np.zeros(1), np.zeros(3), np.zeros(9)
    O.lib().oracle_l2p(O.dptr(dx), O.dptr(L), p, 1, 1, 1, 1, O.dptr(phi), O.dptr(g), O.dptr(H))
    d = xt - xs
    r = np.linalg.norm(d)
    grad = -np.cross(d, G) / r**3 / (4 * np.pi)
    np.testing.assert_allclose(g, grad, atol=c["atol_grad"], rtol=0)
    r5 = r**5
    g11 = -3 * (-G[2] * d[1] + G[1] * d[2]) * d[0]**2 / r5
    g12 = -G[2] / r**3 - 3 * (-G[2] * d[1] + G[1] * d[2]) * d[1]**2 / r5
    g13 = G[1] / r**3 - 3 * (-G[2] * d[1] + G[1] * d[2]) * d[2]**2 / r5
    g21 = G[2] / r**3 - 3 * (G[2] * d[0] - G[0] * d[2]) * d[0]**2 / r5
    g22 = -3 * (G[2] * d[0] - G[0] * d[2]) * d[1]**2 / r5
    g23 = -G[0] / r**3 - 3 * (G[2] * d[0] - G[0] * d[2]) * d[2]**2 / r5
    g31 = -G[1] / r**3 - 3 * (-G[1] * d[0] + G[0] * d[1]) * d[0]**2 / r5
    g32 = G[0] / r**3 - 3 * (-G[1] * d[0] + G[0] * d[1]) * d[1]**2 / r5
    g33 = -3 * (-G[1] * d[0] + G[0] * d[1]) * d[2]**2 / r5
    hess = np.array([g11, g21, g31, g12, g22, g32, g13, g23, g33]) / (4 * np.pi)
    np.testing.assert_allclose(H, hess, atol=c["atol_hess"], rtol=0)


def _table_blocks(name):
    c = GOLD[name]
    return c, c["mats"]


def test_wigner_pi2_tables():
    c, mats = _table_blocks("H_pi2")
    p = 10
    Hs = np.zeros(O.lib().oracle_length_Hs(p))
    O.lib().oracle_tables(p, O.dptr(Hs), None, None, None, None)
    for n, M in zip((1, 2, 3, 4), mats):
        off = (n) * (n + 1) * (n + 2) // 6
        for m in range(n + 1):
            for mp in range(m + 1):
                got = Hs[off + m * (m + 1) // 2 + mp]
                assert abs(got - M[n + mp][n + m]) <= c["atol"], (n, m, mp)


def test_wigner_T_3pi7():
    c, mats = _table_blocks("T_3pi7")
    p = c["p"]
    Ts = np.zeros(O.lib().oracle_length_Ts(p))
    O.lib().oracle_update_Ts(p, 3 * np.pi / 7, O.dptr(Ts))
    for n, M in zip((1, 2, 3, 4), mats):
        off = n * (n + 1) * (2 * n + 1) // 6
        for m in range(n + 1):
            for mp in range(-m, m + 1):
                got = Ts[off + m * m + mp + m]
                assert abs(got - M[n + mp][n + m]) <= c["atol"], (n, m, mp)


def test_solid_harmonics_closed_form():
    # test/harmonics_test.jl:1-29 (Gumerov normalization vs associated Legendre closed form)
    p, rho, th, ph = 7, 1.7, 3 * np.pi / 8, 5 * np.pi / 3
    h = np.zeros(4 * O.nh(p + 2))
    O.lib().oracle_regular_harmonics(rho, th, ph, p, O.dptr(h))
    for n in range(p + 1):
        for m in range(n + 1):
            R = (-1)**n * (1j)**m * rho**n * lpmv(m, n, np.cos(th)) * np.exp(1j * m * ph) / factorial(n + m)
            i = n * (n + 1) // 2 + m
            assert abs(R.real - h[4 * i]) < 1e-12 and abs(R.imag - h[4 * i + 1]) < 1e-12
    O.lib().oracle_irregular_harmonics(rho, th, ph, p, O.dptr(h))
    for n in range(p + 1):
        for m in range(n + 1):
            S = (-1)**m * (1j)**m * rho**(-n - 1) * lpmv(m, n, np.cos(th)) * np.exp(1j * m * ph) * factorial(n - m)
            i = n * (n + 1) // 2 + m
            assert abs(S.real - h[4 * i]) < 1e-12 and abs(S.imag - h[4 * i + 1]) < 1e-12


def test_legendre_and_power_norms():
    # test/rotate_test.jl:1-15 and test/multipole_power_test.jl:1-31
    P = 10
    th = np.pi / 7
    out = np.zeros(O.nh(P))
    O.lib().oracle_compute_Pnms(P, np.sin(th), np.cos(th), O.dptr(out))
    for n in range(P + 1):
        for m in range(n + 1):
            np.testing.assert_allclose(out[n * (n + 1) // 2 + m], lpmv(m, n, np.cos(th)), rtol=1e-12)
    Mt, Lt = np.zeros(O.nh(21)), np.zeros(O.nh(21))
    O.lib().oracle_tables(21, None, None, None, O.dptr(Mt), O.dptr(Lt))
    i = 0
    for n in range(6):
        for m in range(n + 1):
            a, b = math.factorial(n + m), math.factorial(n - m)
            assert abs(Mt[i] - math.sqrt(a * b / (2 * n + 1))) < 1e-12
            assert abs(Lt[i] - math.sqrt(1 / (a * b * (2 * n + 1)))) < 1e-12
            i += 1


def test_fmm_five_masses_vs_direct():
    # test/fmm_test.jl:70-109: 5 masses, p=24, MAC 0.5 -> fmm! potential == direct! potential (atol 1e-12)
    xs = np.array([[1.2, 1.1, 0.8], [0.8, 0.9, 0.2], [0.1, 0.2, 0.9], [0.1, 0.3, 0.2], [0.2, 0.25, 0.4]])
    ms = np.array([0.8, 1.1, 2.2, 0.5, 1.9])
    buf = np.zeros((5, 5))
    buf[:, :3] = xs
    buf[:, 4] = ms
    opt = O.options(expansion_order=24, multipole_acceptance=0.5, leaf_size_source=20, scalar_potential=1)
    res = O.fmm(buf, O.POINT_SOURCE, opt)
    d = O.direct(buf, O.POINT_SOURCE)
    np.testing.assert_allclose(res["out"][:, 3], d[:, 3], atol=1e-12, rtol=0)


def test_fmm_converges_to_direct():
    # test/fmm_test.jl:459-495 asks fmm! == direct! at high order; the reference draws its bodies from Julia's
    # RNG, so this uses seeded bodies of its shape with the far field active and checks geometric convergence.
    rng = np.random.default_rng(7)
    n = 300
    buf = np.zeros((n, 5))
    buf[:, :3] = rng.random((n, 3))
    buf[:, 4] = rng.random(n) / n
    d = O.direct(buf, O.POINT_SOURCE)
    errs = []
    for p in (8, 16, 24):
        opt = O.options(expansion_order=p, leaf_size_source=4, multipole_acceptance=0.5, scalar_potential=1)
        r = O.fmm(buf, O.POINT_SOURCE, opt, want_tree=True)
        assert len(r["m2l"]) > 0
        errs.append(np.abs(r["out"][:, 3:7] - d[:, 3:7]).max())
    assert errs[0] > errs[1] > errs[2] and errs[2] < 1e-10


def test_tree_five_bodies():
    # test/tree_test.jl:1-60: 5 bodies, leaf_size 1 (SelfTuning split rule), no shrinking
    xs = np.array([[1.2, 1.1, 0.8], [0.8, 0.9, 0.2], [0.1, 0.2, 0.9], [0.1, 0.3, 0.2], [0.2, 0.25, 0.4]])
    buf = np.zeros((5, 5))
    buf[:, :3] = xs
    buf[:, 4] = 1.0
    opt = O.options(expansion_order=2, leaf_size_source=1, shrink_recenter=0, list_method=O.LIST_SELF_TUNING)
    t = O.fmm(buf, O.POINT_SOURCE, opt, want_tree=True)["source_tree"]
    r1 = t["target_box"][0].max()
    r2 = t["target_box"][1].max()
    c2 = t["target_center"][1]
    expected = [
        (5, [0.65, 0.65, 0.55], np.sqrt(3) * r1),
        (2, [0.65 - r1 / 2, 0.65 - r1 / 2, 0.55 - r1 / 2], np.sqrt(3) * r2),
        (1, [0.65 + r1 / 2, 0.65 + r1 / 2, 0.55 - r1 / 2], np.sqrt(3) * r2),
        (1, [0.65 - r1 / 2, 0.65 - r1 / 2, 0.55 + r1 / 2], np.sqrt(3) * r2),
        (1, [0.65 + r1 / 2, 0.65 + r1 / 2, 0.55 + r1 / 2], np.sqrt(3) * r2),
        (1, c2 - r2 / 2, np.sqrt(3) * r2 / 2),
        (1, [c2[0] - r2 / 2, c2[1] - r2 / 2, c2[2] + r2 / 2], np.sqrt(3) * r2 / 2),
    ]
    assert t["n_branches"] == len(expected)
    for i, (cnt, ctr, rad) in enumerate(expected):
        assert t["body_count"][i] == cnt
        np.testing.assert_allclose(t["target_center"][i], ctr, atol=1e-7)
        np.testing.assert_allclose(t["target_radius"][i], rad, atol=1e-7)
    # leaf numbering follows branch order (test/tree_test.jl:181-198)
    leaves = [i for i in range(t["n_branches"]) if t["n_children"][i] == 0]
    assert [t["i_leaf"][i] for i in leaves] == list(range(len(leaves)))


def test_tree_shrinking_geometry():
    # test/tree_test.jl:63-179: leaves with one body shrink onto it; source boxes include radii
    xs = np.array([[1.2, 1.1, 0.8], [0.8, 0.9, 0.2], [0.1, 0.2, 0.9], [0.1, 0.3, 0.2], [0.2, 0.25, 0.4]])
    radii = np.random.default_rng(123).random(5)
    buf = np.zeros((5, 5))
    buf[:, :3] = xs
    buf[:, 3] = radii
    buf[:, 4] = 1.0
    opt = O.options(expansion_order=2, leaf_size_source=1, shrink_recenter=1, list_method=O.LIST_SELF_TUNING)
    t = O.fmm(buf, O.POINT_SOURCE, opt, want_tree=True)["source_tree"]
    si = t["sort_index"]
    for i in range(2, 7):
        j = si[t["body_start"][i]]
        np.testing.assert_allclose(t["target_center"][i], xs[j], atol=1e-12)
        np.testing.assert_allclose(t["source_center"][i], xs[j], atol=1e-12)
        assert abs(t["target_radius"][i]) < 1e-12
        np.testing.assert_allclose(t["source_radius"][i], radii[j], atol=1e-12)
        np.testing.assert_allclose(t["source_box"][i], [radii[j]] * 3, atol=1e-12)
    # branch 2 (two bodies)
    bi = 1
    ids = si[t["body_start"][bi]: t["body_start"][bi] + t["body_count"][bi]]
    P, R = xs[ids], radii[ids]
    np.testing.assert_allclose(t["target_center"][bi], P.mean(axis=0), atol=1e-12)
    lo, hi = (P - R[:, None]).min(0), (P + R[:, None]).max(0)
    np.testing.assert_allclose(t["source_center"][bi], (lo + hi) / 2, atol=1e-12)
    np.testing.assert_allclose(t["source_box"][bi], (hi - lo) / 2, atol=1e-12)
    np.testing.assert_allclose(t["target_radius"][bi],
                               np.linalg.norm(P - t["target_center"][bi], axis=1).max(), atol=1e-12)
    np.testing.assert_allclose(t["source_radius"][bi],
                               (np.linalg.norm(P - t["source_center"][bi], axis=1) + R).max(), atol=1e-12)


def test_lists_sorted_by_target():
    # test/interaction_list_test.jl:1-26 (sortedness of the target-sorted lists), at a smaller N
    rng = np.random.default_rng(456)
    n = 20000
    buf = np.zeros((n, 5))
    buf[:, :3] = rng.random((n, 3))
    buf[:, 4] = rng.random(n)
    opt = O.options(expansion_order=2, leaf_size_source=100, multipole_acceptance=0.5)
    r = O.fmm(buf, O.POINT_SOURCE, opt, want_tree=True)
    assert np.all(np.diff(r["m2l"][:, 0]) >= 0) and np.all(np.diff(r["direct"][:, 0]) >= 0)
    # every (target leaf, source leaf) body pair is covered exactly once by near + far field
    tt, st = r["target_tree"], r["source_tree"]
    assert sorted(tt["sort_index"]) == list(range(n))
