"""Host side of the Python mirror of fmm!/direct! (no device calls).

* make_options maps the keyword arguments of fmm! (src/fmm.jl:862-923) onto the C options struct;
* the source buffers follow source_system_to_buffer! (x y z radius strength..., body-major);
* results go back through each system's buffer_to_target_system!, with the reference test
  systems' semantics (Gravitational assigns, VortexParticles and probes accumulate);
* a system that misses an overload fails with the reference's "not overloaded" message.
"""
import numpy as np
import pytest

import fastmultipole_b200 as fm
from fastmultipole_b200 import _lib as L
from fastmultipole_b200 import api


def test_make_options_maps_keywords():
    o = fm.make_options(expansion_order=9, leaf_size_source=33, leaf_size_target=12, multipole_acceptance=0.55,
                        shrink_recenter=False, interaction_list_method=fm.Barba(), farfield=False,
                        self_induced=False, scalar_potential=True, hessian=True, precision="mixed")
    assert (o.expansion_order, o.leaf_size_source, o.leaf_size_target) == (9, 33, 12)
    assert o.multipole_acceptance == 0.55
    assert (o.shrink_recenter, o.list_method) == (0, L.FMM_LIST_BARBA)
    assert (o.farfield, o.nearfield, o.self_induced) == (0, 1, 0)
    assert (o.scalar_potential, o.gradient, o.hessian) == (1, 1, 1)
    assert o.precision == L.FMM_PRECISION_MIXED
    # no leaf_size_target: the target tree takes the source leaf size (0 in the struct)
    assert fm.make_options(leaf_size_source=7).leaf_size_target == 0
    assert fm.make_options().precision == L.FMM_PRECISION_F64
    assert fm.make_options().list_method == L.FMM_LIST_SELF_TUNING_TREE_STOP
    with pytest.raises(KeyError):
        fm.make_options(precision="f16")


@pytest.mark.parametrize("ctor,code", [(fm.PowerAbsoluteGradient, L.FMM_POWER_ABSOLUTE_GRADIENT),
                                       (fm.PowerRelativeGradient, L.FMM_POWER_RELATIVE_GRADIENT),
                                       (fm.RotatedCoefficientsAbsoluteGradient,
                                        L.FMM_ROTATED_COEFFICIENTS_ABSOLUTE_GRADIENT),
                                       (fm.RotatedCoefficientsRelativeGradient,
                                        L.FMM_ROTATED_COEFFICIENTS_RELATIVE_GRADIENT)])
def test_error_methods(ctor, code):
    o = fm.make_options(error_tolerance=ctor(3e-7))
    assert (o.error_method, o.error_tolerance, o.bonus_expansion) == (code, 3e-7, 1)
    assert fm.make_options(error_tolerance=ctor(1e-4, False)).bonus_expansion == 0
    assert fm.make_options().error_method == L.FMM_ERROR_NONE


def test_source_buffers_follow_the_reference_layout():
    rng = np.random.default_rng(0)
    pos, q, rad = rng.random((4, 3)), rng.random(4), rng.random(4)
    ps = fm.PointSources(pos, q, radius=rad)
    g = rng.random((3, 3))
    vp = fm.VortexParticles(rng.random((3, 3)), g, sigma=np.full(3, 0.1))
    b = api._source_buffer([ps], L.FMM_POINT_SOURCE)
    np.testing.assert_array_equal(b, np.column_stack([pos, rad, q]))
    b = api._source_buffer([vp], L.FMM_POINT_VORTEX)
    np.testing.assert_array_equal(b, np.column_stack([vp.position, np.full(3, 0.1), g]))
    # several systems: concatenated in order
    ps2 = fm.PointSources(rng.random((2, 3)), rng.random(2))
    b = api._source_buffer([ps, ps2], L.FMM_POINT_SOURCE)
    assert b.shape == (6, 5)
    np.testing.assert_array_equal(b[4:, 4], ps2.strength)
    np.testing.assert_array_equal(api._positions([ps, ps2]), np.vstack([pos, ps2.position]))


def test_buffer_to_target_system_semantics():
    rng = np.random.default_rng(1)
    out = rng.random((5, 16))
    sw = fm.DerivativesSwitch(scalar_potential=True, gradient=True, hessian=False)
    # Gravitational (test/gravitational.jl:106-119): assignment; quantities not asked for are zeroed
    ps = fm.PointSources(rng.random((2, 3)), rng.random(2))
    ps.potential[:] = 7.0
    vp = fm.VortexParticles(rng.random((3, 3)), rng.random((3, 3)))
    vp.gradient_stretching[:] = 1.0
    vp.potential[:] = 2.0
    api._scatter([ps, vp], out, sw)
    np.testing.assert_array_equal(ps.potential[:, 0], out[:2, 3])
    np.testing.assert_array_equal(ps.potential[:, 4:7], out[:2, 4:7])
    assert not ps.potential[:, 7:16].any()
    # VortexParticles (test/vortex.jl:130-146): accumulation of the velocity (and its gradient)
    np.testing.assert_array_equal(vp.gradient_stretching[:, 0:3], 1.0 + out[2:, 4:7])
    np.testing.assert_array_equal(vp.potential[:, 4:13], 2.0)  # hessian not requested
    # probes accumulate every requested quantity
    pr = fm.ProbeSystem(rng.random((5, 3)))
    pr.buffer_to_target_system(out, fm.DerivativesSwitch(True, True, True))
    pr.buffer_to_target_system(out, fm.DerivativesSwitch(True, False, False))
    np.testing.assert_array_equal(pr.scalar_potential, 2 * out[:, 3])
    np.testing.assert_array_equal(pr.gradient, out[:, 4:7])
    np.testing.assert_array_equal(pr.hessian, out[:, 7:16])


def test_missing_overloads_and_kernels():
    class Bare(fm.System):
        pass

    with pytest.raises(NotImplementedError, match="not overloaded"):
        Bare().get_n_bodies()
    with pytest.raises(NotImplementedError, match="source_system_to_buffer! not overloaded"):
        Bare().source_system_to_buffer(None)

    class Odd(fm.PointSources):
        kernel = "dipole"

    with pytest.raises(ValueError):
        api._kind([Odd(np.zeros((1, 3)), np.ones(1))])
    ps = fm.PointSources(np.zeros((1, 3)), np.ones(1))
    vp = fm.VortexParticles(np.zeros((1, 3)), np.ones((1, 3)))
    assert api._kind([ps]) == L.FMM_POINT_SOURCE and api._kind([vp]) == L.FMM_POINT_VORTEX
    with pytest.raises(NotImplementedError):
        api._kind([ps, vp])
