"""GPU end-to-end parity through fmm_solve / fmm_direct against the FP64 oracle.

* octree (permutation, branch ranges, centres, radii, boxes, leaf numbering) and the
  interaction lists: bit-exact;
* FP64 fmm! results: within 1e-10 of the oracle's, relative to the field's magnitude;
* MIXED results: relative L2 error vs the FP64 all-pairs direct sum within the bound
  the configuration states.
"""
import numpy as np
import pytest

import fastmultipole_b200 as fm
from fastmultipole_b200 import _lib as L
import oracle_lib as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = fm.Context(0)
    yield c
    c.close()


def uniform(n, seed, kind=1, radius=0.0):
    rng = np.random.default_rng(seed)
    d = 5 if kind == 1 else 7
    b = np.zeros((n, d))
    b[:, :3] = rng.random((n, 3))
    b[:, 3] = radius * rng.random(n)
    if kind == 1:
        b[:, 4] = rng.random(n)
    else:
        b[:, 4:7] = (2 * rng.random((n, 3)) - 1) / n
    return b


def clustered(n, seed):
    rng = np.random.default_rng(seed)
    b = np.zeros((n, 5))
    nb = n // 10
    centres = rng.random((8, 3))
    k = rng.integers(0, 8, n - nb)
    b[: n - nb, :3] = centres[k] + 0.05 * rng.standard_normal((n - nb, 3))
    b[n - nb:, :3] = rng.random((nb, 3))
    b[:, 4] = 2 * rng.random(n) - 1
    return b


def ring(n, seed):
    rng = np.random.default_rng(seed)
    phi = 2 * np.pi * rng.random(n)
    off = 0.05 * rng.standard_normal((n, 2))
    R = 1.0 + off[:, 0]
    b = np.zeros((n, 7))
    b[:, 0] = R * np.cos(phi)
    b[:, 1] = R * np.sin(phi)
    b[:, 2] = off[:, 1]
    t = np.stack([-np.sin(phi), np.cos(phi), np.zeros(n)], axis=1)
    b[:, 4:7] = t / n + 1e-3 * rng.standard_normal((n, 3)) / n
    return b


def opt_pair(**kw):
    o_gpu = fm.make_options(**{k: v for k, v in kw.items() if k != "n_threads"})
    o_orc = O.options(expansion_order=o_gpu.expansion_order, leaf_size_source=o_gpu.leaf_size_source,
                      leaf_size_target=o_gpu.leaf_size_target, multipole_acceptance=o_gpu.multipole_acceptance,
                      error_method=o_gpu.error_method, error_tolerance=o_gpu.error_tolerance,
                      bonus_expansion=o_gpu.bonus_expansion, shrink_recenter=o_gpu.shrink_recenter,
                      list_method=o_gpu.list_method, farfield=o_gpu.farfield, nearfield=o_gpu.nearfield,
                      self_induced=o_gpu.self_induced, scalar_potential=o_gpu.scalar_potential,
                      gradient=o_gpu.gradient, hessian=o_gpu.hessian)
    return o_gpu, o_orc


def compare_trees(g, o):
    assert g["n_branches"] == o["n_branches"]
    for k in ("body_start", "body_count", "n_children", "parent", "i_leaf"):
        np.testing.assert_array_equal(g[k], o[k], err_msg=k)
    # child_start of leaves is the running counter in both implementations
    np.testing.assert_array_equal(g["child_start"], o["child_start"])
    np.testing.assert_array_equal(g["sort_index"], o["sort_index"])
    np.testing.assert_array_equal(g["leaf_index"], o["leaf_index"])
    np.testing.assert_array_equal(g["levels_start"], o["levels_start"])
    for k in ("target_center", "source_center", "target_radius", "source_radius", "target_box", "source_box"):
        np.testing.assert_array_equal(g[k], o[k], err_msg=k)


def compare_lists(gm, gd, om, od):
    # the reference's lists bit for bit: rows by target (sort_by_target, stable) and, inside a
    # row, the order of the depth-first recursion
    for a, b in ((gm, om), (gd, od)):
        assert len(a) == len(b)
        np.testing.assert_array_equal(a, b)


CASES = [
    dict(name="uniform10k_p6_ls50", gen=lambda: uniform(10000, 1), kw=dict(expansion_order=6, leaf_size_source=50,
                                                                            multipole_acceptance=0.5,
                                                                            scalar_potential=True)),
    dict(name="uniform_radius_barba", gen=lambda: uniform(6000, 2, radius=0.01),
         kw=dict(expansion_order=5, leaf_size_source=30, multipole_acceptance=0.6,
                 interaction_list_method=fm.Barba())),
    dict(name="uniform_selftuning_noshrink", gen=lambda: uniform(5000, 3),
         kw=dict(expansion_order=4, leaf_size_source=25, multipole_acceptance=0.4, shrink_recenter=False,
                 interaction_list_method=fm.SelfTuning())),
    dict(name="clustered20k_p10", gen=lambda: clustered(20000, 2),
         kw=dict(expansion_order=10, leaf_size_source=64, multipole_acceptance=0.5)),
    # ~4,000 target rows: the near field's 4-warp CTAs and the one-warp M2L rows (launches of fewer
    # rows than 4 per SM take wider CTAs, which the smaller cases here exercise)
    dict(name="uniform60k_p4_ls20", gen=lambda: uniform(60000, 31), kw=dict(expansion_order=4, leaf_size_source=20,
                                                                           multipole_acceptance=0.5,
                                                                           scalar_potential=True)),
    # the lane kernel's highest order
    dict(name="uniform6k_p12", gen=lambda: uniform(6000, 8), kw=dict(expansion_order=12, leaf_size_source=40,
                                                                     multipole_acceptance=0.5,
                                                                     scalar_potential=True)),
    # low orders run the thread-per-pair M2L; leaves of ~5 bodies split the P2P lanes over sources
    dict(name="uniform8k_p3_ls5", gen=lambda: uniform(8000, 4), kw=dict(expansion_order=3, leaf_size_source=5,
                                                                       multipole_acceptance=0.6,
                                                                       scalar_potential=True)),
    # leaves of up to 565 bodies: several target tiles and source leaves larger than one P2P batch
    dict(name="uniform20k_p2_ls200", gen=lambda: uniform(20000, 5), kw=dict(expansion_order=2, leaf_size_source=200,
                                                                           multipole_acceptance=0.5,
                                                                           scalar_potential=True)),
]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_tree_lists_and_fmm_match_oracle(ctx, case):
    buf = case["gen"]()
    og, oo = opt_pair(**case["kw"])
    out, res = fm.solve_buffers(buf, L.FMM_POINT_SOURCE, og, ctx=ctx)
    ref = O.fmm(buf, O.POINT_SOURCE, oo, want_tree=True)
    compare_trees(fm.get_tree(ctx, 1), ref["source_tree"])
    compare_trees(fm.get_tree(ctx, 0), ref["target_tree"])
    gm, gd = fm.get_lists(ctx)
    compare_lists(gm, gd, ref["m2l"], ref["direct"])
    rows = slice(3, 7) if og.scalar_potential else slice(4, 7)
    scale = np.abs(ref["out"][:, rows]).max()
    np.testing.assert_allclose(out[:, rows], ref["out"][:, rows], rtol=0, atol=1e-10 * scale)
    np.testing.assert_array_equal(out[:, :3], buf[:, :3])
    assert res.p_max == ref["pmax"] or len(ref["m2l"]) == 0


def test_vortex_ring_velocity_and_gradient(ctx):
    buf = ring(20000, 3)
    og, oo = opt_pair(expansion_order=12, leaf_size_source=80, multipole_acceptance=0.4, hessian=True)
    out, res = fm.solve_buffers(buf, L.FMM_POINT_VORTEX, og, ctx=ctx)
    ref = O.fmm(buf, O.POINT_VORTEX, oo, want_tree=True)
    compare_trees(fm.get_tree(ctx, 1), ref["source_tree"])
    gm, gd = fm.get_lists(ctx)
    compare_lists(gm, gd, ref["m2l"], ref["direct"])
    for rows in (slice(4, 7), slice(7, 16)):
        scale = np.abs(ref["out"][:, rows]).max()
        np.testing.assert_allclose(out[:, rows], ref["out"][:, rows], rtol=0, atol=1e-10 * scale)


@pytest.mark.parametrize("p,ls", [(3, 10), (2, 200)])
def test_vortex_low_order_and_large_leaves(ctx, p, ls):
    buf = ring(12000, 6)
    og, oo = opt_pair(expansion_order=p, leaf_size_source=ls, multipole_acceptance=0.5, hessian=True)
    out, res = fm.solve_buffers(buf, L.FMM_POINT_VORTEX, og, ctx=ctx)
    ref = O.fmm(buf, O.POINT_VORTEX, oo)
    for rows in (slice(4, 7), slice(7, 16)):
        scale = np.abs(ref["out"][:, rows]).max()
        np.testing.assert_allclose(out[:, rows], ref["out"][:, rows], rtol=0, atol=1e-10 * scale)


@pytest.mark.parametrize("p", [4, 6, 9, 10])
def test_vortex_lane_m2l_orders_match_oracle(ctx, p):
    # plain vortex M2L from order 4 runs the lane-per-pair Lamb-Helmholtz kernel, one template
    # instance per order; degrees >= 8 stage more rows than a warp has lanes
    buf = ring(8000, 10 + p)
    og, oo = opt_pair(expansion_order=p, leaf_size_source=30, multipole_acceptance=0.5, hessian=True)
    out, res = fm.solve_buffers(buf, L.FMM_POINT_VORTEX, og, ctx=ctx)
    assert res.n_m2l > 0
    ref = O.fmm(buf, O.POINT_VORTEX, oo)
    for rows in (slice(4, 7), slice(7, 16)):
        scale = np.abs(ref["out"][:, rows]).max()
        np.testing.assert_allclose(out[:, rows], ref["out"][:, rows], rtol=0, atol=1e-10 * scale)


def test_many_rows_vortex_and_mixed(ctx):
    # ~4,000 target rows (the narrow near-field and M2L launches): FP64 vortex particles against the
    # oracle, and the mixed point-source solve against the FP64 one
    buf = ring(50000, 32)
    og, oo = opt_pair(expansion_order=6, leaf_size_source=16, multipole_acceptance=0.5, hessian=True)
    out, res = fm.solve_buffers(buf, L.FMM_POINT_VORTEX, og, ctx=ctx)
    ref = O.fmm(buf, O.POINT_VORTEX, oo)
    for rows in (slice(4, 7), slice(7, 16)):
        scale = np.abs(ref["out"][:, rows]).max()
        np.testing.assert_allclose(out[:, rows], ref["out"][:, rows], rtol=0, atol=1e-10 * scale)
    pts = uniform(60000, 31)
    outs = {}
    for prec in ("f64", "mixed"):
        og = fm.make_options(expansion_order=6, leaf_size_source=20, multipole_acceptance=0.5,
                             error_tolerance=fm.PowerRelativeGradient(1e-6), scalar_potential=True, precision=prec)
        outs[prec], res = fm.solve_buffers(pts, L.FMM_POINT_SOURCE, og, ctx=ctx)
        assert res.n_m2l > 0
    assert rel_l2(outs["mixed"][:, 4:7], outs["f64"][:, 4:7]) < 1e-5


def test_chunked_near_field_probes_match_oracle(ctx):
    # 10,000 probes around 200,000 sources: 456 target rows, a few of them with most of the pairs,
    # so the near field cuts the rows into chunks of source leaves (summed in chunk order)
    rng = np.random.default_rng(4)
    buf = uniform(200000, 41)
    probes = np.ascontiguousarray(-0.5 + 2.0 * rng.random((10000, 3)))
    og, oo = opt_pair(expansion_order=8, leaf_size_source=50, multipole_acceptance=0.5, scalar_potential=True)
    out, res = fm.solve_buffers(buf, L.FMM_POINT_SOURCE, og, target_pos=probes, ctx=ctx)
    ref = O.fmm(buf, O.POINT_SOURCE, oo, target_pos=probes)
    rows = slice(3, 7)
    scale = np.abs(ref["out"][:, rows]).max()
    np.testing.assert_allclose(out[:, rows], ref["out"][:, rows], rtol=0, atol=1e-10 * scale)
    omx = fm.make_options(expansion_order=8, leaf_size_source=50, multipole_acceptance=0.5, scalar_potential=True,
                          precision="mixed")
    mx, _ = fm.solve_buffers(buf, L.FMM_POINT_SOURCE, omx, target_pos=probes, ctx=ctx)
    assert rel_l2(mx[:, 4:7], out[:, 4:7]) < 1e-5


def test_mixed_vortex_matches_f64(ctx):
    # FP32 near field (batch sums promoted to FP64): relative L2 deviation from the FP64 solve below 1e-5
    buf = ring(20000, 7)
    for ls in (80, 6):
        og64, _ = opt_pair(expansion_order=8, leaf_size_source=ls, multipole_acceptance=0.4, hessian=True)
        ogmx, _ = opt_pair(expansion_order=8, leaf_size_source=ls, multipole_acceptance=0.4, hessian=True,
                           precision="mixed")
        o64, _ = fm.solve_buffers(buf, L.FMM_POINT_VORTEX, og64, ctx=ctx)
        omx, _ = fm.solve_buffers(buf, L.FMM_POINT_VORTEX, ogmx, ctx=ctx)
        for rows in (slice(4, 7), slice(7, 16)):
            assert rel_l2(omx[:, rows], o64[:, rows]) < 1e-5


@pytest.mark.parametrize("p", [4, 12])
def test_mixed_vortex_far_field_matches_f64(ctx, p):
    # far field only: the mixed path's lane-per-pair Lamb-Helmholtz M2L (FP32 rotations of
    # scaled multipoles) against its FP64 instance (pinned to the oracle above), velocity and
    # velocity gradient
    buf = ring(30000, 9)
    outs = {}
    for prec in ("f64", "mixed"):
        og = fm.make_options(expansion_order=p, leaf_size_source=40, multipole_acceptance=0.4, nearfield=False,
                             hessian=True, precision=prec)
        outs[prec], res = fm.solve_buffers(buf, L.FMM_POINT_VORTEX, og, ctx=ctx)
        assert res.n_m2l > 0
    for rows in (slice(4, 7), slice(7, 16)):
        assert rel_l2(outs["mixed"][:, rows], outs["f64"][:, rows]) < 1e-5


@pytest.mark.parametrize("em", [fm.PowerRelativeGradient(1e-6), fm.PowerAbsoluteGradient(1e-4),
                                fm.RotatedCoefficientsRelativeGradient(1e-6), fm.PowerAbsolutePotential(1e-3),
                                fm.PowerRelativePotential(1e-6)], ids=["prg", "pag", "rcrg", "pap", "prp"])
def test_error_controlled_orders_match_oracle(ctx, em):
    buf = clustered(15000, 5)
    og, oo = opt_pair(expansion_order=10, leaf_size_source=64, multipole_acceptance=0.5, error_tolerance=em)
    out, res = fm.solve_buffers(buf, L.FMM_POINT_SOURCE, og, ctx=ctx)
    ref = O.fmm(buf, O.POINT_SOURCE, oo, want_tree=True)
    if em.code in (L.FMM_POWER_RELATIVE_GRADIENT, L.FMM_ROTATED_COEFFICIENTS_RELATIVE_GRADIENT,
                   L.FMM_POWER_RELATIVE_POTENTIAL):
        g = fm.get_tree(ctx, 0)
        np.testing.assert_allclose(g["max_influence"], ref["target_tree"]["max_influence"], rtol=1e-11, atol=0)
    assert res.p_max == ref["pmax"]
    assert bool(res.error_success) == ref["error_success"]
    gm, gd = fm.get_lists(ctx)
    compare_lists(gm, gd, ref["m2l"], ref["direct"])
    scale = np.abs(ref["out"][:, 4:7]).max()
    np.testing.assert_allclose(out[:, 4:7], ref["out"][:, 4:7], rtol=0, atol=1e-10 * scale)


def test_dual_tree_probes(ctx):
    src = uniform(20000, 4)
    rng = np.random.default_rng(44)
    probes = -0.5 + 2.0 * rng.random((3000, 3))
    og, oo = opt_pair(expansion_order=8, leaf_size_source=40, multipole_acceptance=0.5, scalar_potential=True)
    out, res = fm.solve_buffers(src, L.FMM_POINT_SOURCE, og, target_pos=probes, ctx=ctx)
    ref = O.fmm(src, O.POINT_SOURCE, oo, target_pos=probes, want_tree=True)
    compare_trees(fm.get_tree(ctx, 0), ref["target_tree"])
    gm, gd = fm.get_lists(ctx)
    compare_lists(gm, gd, ref["m2l"], ref["direct"])
    scale = np.abs(ref["out"][:, 3:7]).max()
    np.testing.assert_allclose(out[:, 3:7], ref["out"][:, 3:7], rtol=0, atol=1e-10 * scale)


@pytest.mark.parametrize("kind", [1, 3])
def test_direct_matches_oracle(ctx, kind):
    buf = uniform(3000, 9, kind=kind)
    tgt = np.zeros((3000, 16))
    src = L.SourceSystem(kind, 3000, buf.shape[1], buf.ctypes.data, 0)
    tsys = L.TargetSystem(3000, None, 0, tgt.ctypes.data, 0)
    import ctypes as C
    ctx.check(L.lib().fmm_direct(ctx.handle, C.byref(tsys), C.byref(src), 1, 1, 1, 0))
    ref = O.direct(buf, kind, ps=1, gs=1, hs=1)
    rows = slice(3, 7) if kind == 1 else slice(4, 16)
    np.testing.assert_allclose(tgt[:, rows], ref[:, rows], rtol=0, atol=1e-12 * np.abs(ref[:, rows]).max())


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_mixed_precision_error_bounds(ctx):
    # The error-controlled FP64 method itself leaves ~2e-6 at PowerRelativeGradient(1e-6) on this set and
    # ~1e-7 at 1e-7 (oracle).  The mixed path must stay within 1e-6 of FP64 direct at 1e-7 and must not add
    # more than 10% to the method's own error at 1e-6.
    buf = clustered(30000, 11)
    ids = np.random.default_rng(0).choice(len(buf), 2000, replace=False)
    ref = O.direct_subset(buf, O.POINT_SOURCE, ids)
    errs = {}
    for eps in (1e-6, 1e-7):
        for prec in ("f64", "mixed"):
            og, _ = opt_pair(expansion_order=10, leaf_size_source=64, multipole_acceptance=0.5,
                             error_tolerance=fm.PowerRelativeGradient(eps), precision=prec)
            out, _ = fm.solve_buffers(buf, L.FMM_POINT_SOURCE, og, ctx=ctx)
            errs[eps, prec] = rel_l2(out[ids, 4:7], ref[:, 4:7])
    assert errs[1e-7, "mixed"] < 1e-6, errs
    assert errs[1e-6, "mixed"] < 1.1 * errs[1e-6, "f64"] + 1e-7, errs


def test_mixed_low_order_m2l_and_influence_match_f64(ctx):
    # orders <= 3 (the influence estimate's order) run the single-precision M2L in the mixed
    # path: the far field must agree with the FP64 solve to FP32 accuracy (1e-5 relative L2,
    # far below the order-3 truncation error of ~1e-3), and the influence estimate of a
    # relative error method (max_influence per target branch) to 1e-4
    buf = clustered(40000, 13)
    outs = {}
    for prec in ("f64", "mixed"):
        og = fm.make_options(expansion_order=3, leaf_size_source=20, multipole_acceptance=0.5, nearfield=False,
                             scalar_potential=True, precision=prec)
        outs[prec], res = fm.solve_buffers(buf, L.FMM_POINT_SOURCE, og, ctx=ctx)
        assert res.n_m2l > 0
    for rows in (slice(3, 4), slice(4, 7)):
        assert rel_l2(outs["mixed"][:, rows], outs["f64"][:, rows]) < 1e-5
    inf = {}
    for prec in ("f64", "mixed"):
        og = fm.make_options(expansion_order=8, leaf_size_source=40, multipole_acceptance=0.5,
                             error_tolerance=fm.PowerRelativeGradient(1e-6), precision=prec)
        fm.solve_buffers(buf, L.FMM_POINT_SOURCE, og, ctx=ctx)
        inf[prec] = fm.get_tree(ctx, 0)["max_influence"]
    np.testing.assert_allclose(inf["mixed"], inf["f64"], rtol=1e-4, atol=0)


@pytest.mark.parametrize("ls,p", [(5, 3), (6, 8)])
def test_mixed_small_leaves_match_f64(ctx, ls, p):
    # leaves of ~5 bodies run the warp-per-row packed near field and the grouped L2P on the
    # mixed path: the result must agree with the FP64 solve to FP32 accuracy
    buf = clustered(30000, 17)
    outs = {}
    for prec in ("f64", "mixed"):
        og = fm.make_options(expansion_order=p, leaf_size_source=ls, multipole_acceptance=0.5,
                             scalar_potential=True, precision=prec)
        outs[prec], res = fm.solve_buffers(buf, L.FMM_POINT_SOURCE, og, ctx=ctx)
        assert res.n_direct > 0 and res.n_m2l > 0
    for rows in (slice(3, 4), slice(4, 7)):
        assert rel_l2(outs["mixed"][:, rows], outs["f64"][:, rows]) < 1e-5


def test_python_api_systems(ctx):
    rng = np.random.default_rng(5)
    n = 4000
    sys_ = fm.PointSources(rng.random((n, 3)), rng.random(n) / n)
    fm.fmm(sys_, expansion_order=12, leaf_size=30, multipole_acceptance=0.5, scalar_potential=True, context=ctx)
    fmm_phi = sys_.potential[:, 0].copy()
    fmm_grad = sys_.potential[:, 4:7].copy()
    sys_.potential[:] = 0
    fm.direct(sys_, scalar_potential=True, context=ctx)
    np.testing.assert_allclose(fmm_phi, sys_.potential[:, 0], rtol=0, atol=1e-7 * np.abs(fmm_phi).max())
    np.testing.assert_allclose(fmm_grad, sys_.potential[:, 4:7], rtol=0, atol=1e-6 * np.abs(fmm_grad).max())


def test_empty_and_tiny_systems(ctx):
    og, oo = opt_pair(expansion_order=4, leaf_size_source=10)
    for n in (1, 2, 7):
        buf = uniform(n, n)
        out, res = fm.solve_buffers(buf, L.FMM_POINT_SOURCE, og, ctx=ctx)
        ref = O.fmm(buf, O.POINT_SOURCE, oo)
        np.testing.assert_allclose(out[:, 4:7], ref["out"][:, 4:7], rtol=1e-12, atol=1e-300)
    out, res = fm.solve_buffers(np.zeros((0, 5)), L.FMM_POINT_SOURCE, og, target_pos=np.random.rand(5, 3), ctx=ctx)
    assert np.all(out[:, 3:] == 0)


def test_invalid_arguments_are_errors_not_faults(ctx):
    buf = uniform(100, 1)
    og, _ = opt_pair(expansion_order=40)
    with pytest.raises(fm.FMMError) as e:
        fm.solve_buffers(buf, L.FMM_POINT_SOURCE, og, ctx=ctx)
    assert e.value.status == L.FMM_ERR_ARGUMENT
    og, _ = opt_pair(expansion_order=4, leaf_size_source=1)
    dup = np.zeros((50, 5))
    dup[:, 4] = 1.0  # coincident bodies: the octree cannot separate them
    with pytest.raises(fm.FMMError) as e:
        fm.solve_buffers(dup, L.FMM_POINT_SOURCE, og, ctx=ctx)
    assert e.value.status == L.FMM_ERR_TREE_DEPTH
    # the context stays usable
    out, _ = fm.solve_buffers(buf, L.FMM_POINT_SOURCE, fm.make_options(expansion_order=4), ctx=ctx)
    assert np.isfinite(out).all()


def test_tuple_of_point_sources_and_vortices(ctx):
    # fmm_solve_multi: one octree over a tuple of systems (point sources and vortex
    # particles, Tree(systems::Tuple, ...)) against the oracle's tuple mode: trees and lists
    # bit for bit, the target buffer at 1e-10 (the potential too: with a vortex system the
    # reference runs the Lamb-Helmholtz form, whose scalar potential it warns is not
    # meaningful, and the restatement must reproduce it all the same)
    src = uniform(8000, 21)
    vort = ring(6000, 22)
    rng = np.random.default_rng(23)
    probes = np.ascontiguousarray(-0.5 + 2.0 * rng.random((4000, 3)))
    for p, em in ((12, None), (8, fm.PowerRelativeGradient(1e-7))):
        og, oo = opt_pair(expansion_order=p, leaf_size_source=40, multipole_acceptance=0.4, scalar_potential=True,
                          error_tolerance=em)
        out, res = fm.solve_multi_buffers([(src, L.FMM_POINT_SOURCE), (vort, L.FMM_POINT_VORTEX)], og, probes,
                                          ctx=ctx)
        ref = O.fmm_multi([(src, O.POINT_SOURCE), (vort, O.POINT_VORTEX)], oo, probes, want_tree=True)
        compare_trees(fm.get_tree(ctx, 1), ref["source_tree"])
        compare_trees(fm.get_tree(ctx, 0), ref["target_tree"])
        gm, gd = fm.get_lists(ctx)
        compare_lists(gm, gd, ref["m2l"], ref["direct"])
        assert res.p_max == ref["pmax"] and bool(res.error_success) == ref["error_success"]
        for rows in (slice(3, 4), slice(4, 7)):
            scale = np.abs(ref["out"][:, rows]).max()
            np.testing.assert_allclose(out[:, rows], ref["out"][:, rows], rtol=0, atol=1e-10 * scale)
        np.testing.assert_array_equal(out[:, :3], probes)
        # the far field of both kernels is exercised
        assert res.n_m2l > 0
    # the velocity is the sum of both systems' fields, to the FMM's accuracy
    d1 = O.direct(src, O.POINT_SOURCE, ps=1, gs=1, hs=0, target_pos=probes)
    d3 = O.direct(vort, O.POINT_VORTEX, ps=0, gs=1, hs=0, target_pos=probes)
    assert rel_l2(out[:, 4:7], d1[:, 4:7] + d3[:, 4:7]) < 1e-6
    # the Barba rule splits on per-system counts: rejected, not silently different
    ob, _ = opt_pair(expansion_order=6, leaf_size_source=40, interaction_list_method=fm.Barba())
    with pytest.raises(fm.FMMError):
        fm.solve_multi_buffers([(src, L.FMM_POINT_SOURCE), (vort, L.FMM_POINT_VORTEX)], ob, probes, ctx=ctx)
    # the Python fmm() on a tuple of systems of both kernels (self evaluation of the tuple)
    ps = fm.PointSources(src[:, :3], src[:, 4])
    vs = fm.VortexParticles(vort[:, :3], vort[:, 4:7])
    fm.fmm((ps, vs), expansion_order=8, leaf_size=40, multipole_acceptance=0.5, context=ctx)
    assert np.isfinite(ps.potential).all() and np.isfinite(vs.potential).all()


def test_tuple_edge_cases(ctx):
    # a tuple of two point-source systems is the concatenation of their bodies (one octree,
    # systems one after another inside each leaf): the single-system solve of the concatenated
    # buffer to rounding (per-system P2M and P2P batches sum in another order); an empty system
    # in a tuple changes nothing; three systems agree with the oracle's tuple mode
    a = uniform(5000, 31)
    b = uniform(4000, 32)
    v = ring(3000, 33)
    rng = np.random.default_rng(34)
    probes = np.ascontiguousarray(rng.random((2500, 3)))
    og, oo = opt_pair(expansion_order=7, leaf_size_source=30, multipole_acceptance=0.5, scalar_potential=True)
    out2, _ = fm.solve_multi_buffers([(a, L.FMM_POINT_SOURCE), (b, L.FMM_POINT_SOURCE)], og, probes, ctx=ctx)
    cat, _ = fm.solve_buffers(np.concatenate([a, b]), L.FMM_POINT_SOURCE, og, target_pos=probes, ctx=ctx)
    np.testing.assert_array_equal(out2[:, :3], cat[:, :3])
    np.testing.assert_allclose(out2[:, 3:7], cat[:, 3:7], rtol=0, atol=1e-12 * np.abs(cat[:, 3:7]).max())
    empty = np.zeros((0, 7))
    out3, _ = fm.solve_multi_buffers([(a, L.FMM_POINT_SOURCE), (empty, L.FMM_POINT_VORTEX), (v, L.FMM_POINT_VORTEX)],
                                     og, probes, ctx=ctx)
    out3b, _ = fm.solve_multi_buffers([(a, L.FMM_POINT_SOURCE), (v, L.FMM_POINT_VORTEX)], og, probes, ctx=ctx)
    np.testing.assert_array_equal(out3, out3b)
    out4, res = fm.solve_multi_buffers([(a, L.FMM_POINT_SOURCE), (v, L.FMM_POINT_VORTEX), (b, L.FMM_POINT_SOURCE)],
                                       og, probes, ctx=ctx)
    ref = O.fmm_multi([(a, O.POINT_SOURCE), (v, O.POINT_VORTEX), (b, O.POINT_SOURCE)], oo, probes, want_tree=True)
    compare_trees(fm.get_tree(ctx, 1), ref["source_tree"])
    gm, gd = fm.get_lists(ctx)
    compare_lists(gm, gd, ref["m2l"], ref["direct"])
    for rows in (slice(3, 4), slice(4, 7)):
        scale = np.abs(ref["out"][:, rows]).max()
        np.testing.assert_allclose(out4[:, rows], ref["out"][:, rows], rtol=0, atol=1e-10 * scale)
