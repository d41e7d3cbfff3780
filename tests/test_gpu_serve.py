"""fmm_serve_*: concurrent requests on one device.

* a request's result is bit-for-bit the same served alone (fmm_solve) and mixed
  with other requests on several workers;
* FMM_PENDING before completion, the solve's status after it, errors and the HBM
  budget reported per request.
"""
import numpy as np
import pytest

import fastmultipole_b200 as fm
from fastmultipole_b200 import _lib as L

pytestmark = pytest.mark.gpu


def bodies(n, kind, seed, clustered=False):
    rng = np.random.default_rng(seed)
    d = 5 if kind == L.FMM_POINT_SOURCE else 7
    b = np.zeros((n, d))
    if clustered:
        c = rng.random((4, 3))
        b[:, :3] = c[rng.integers(0, 4, n)] + 0.05 * rng.standard_normal((n, 3))
    else:
        b[:, :3] = rng.random((n, 3))
    if kind == L.FMM_POINT_SOURCE:
        b[:, 4] = 2 * rng.random(n) - 1
    else:
        b[:, 4:7] = (2 * rng.random((n, 3)) - 1) / n
    return b


REQUESTS = [
    dict(n=30000, kind=1, seed=1, p=8, ls=40, err=fm.PowerRelativeGradient(1e-7), clustered=True),
    dict(n=4000, kind=3, seed=2, p=6, ls=30, err=None, hs=True),
    dict(n=60000, kind=1, seed=3, p=10, ls=64, err=None, precision="mixed"),
    dict(n=2000, kind=1, seed=4, p=4, ls=20, err=None, probes=1500),
    dict(n=12000, kind=3, seed=5, p=12, ls=50, err=None),
    dict(n=9000, kind=1, seed=6, p=5, ls=25, err=fm.RotatedCoefficientsAbsoluteGradient(1e-6)),
]


def make(r):
    buf = bodies(r["n"], r["kind"], r["seed"], r.get("clustered", False))
    opt = fm.make_options(expansion_order=r["p"], leaf_size_source=r["ls"], multipole_acceptance=0.5,
                          error_tolerance=r["err"], scalar_potential=r["kind"] == 1, hessian=r.get("hs", False),
                          precision=r.get("precision", "f64"))
    tp = None
    if r.get("probes"):
        tp = np.random.default_rng(r["seed"] + 9).random((r["probes"], 3))
    return buf, opt, tp


def test_mixed_requests_match_alone_bitwise():
    ctx = fm.Context(0)
    try:
        alone = []
        for r in REQUESTS:
            buf, opt, tp = make(r)
            out, res = fm.solve_buffers(buf, r["kind"], opt, tp, ctx=ctx)
            alone.append(out)
        server = fm.Server(n_workers=3, ctx=ctx)
        for rounds in range(2):
            ids = []
            for r in REQUESTS:
                buf, opt, tp = make(r)
                ids.append(server.submit(buf, r["kind"], opt, tp))
            for k, rid in enumerate(reversed(ids)):
                rc, out, res = server.poll(rid, timeout_ms=-1)
                assert rc == L.FMM_OK
                np.testing.assert_array_equal(out, alone[len(ids) - 1 - k])
        server.stop()
    finally:
        ctx.close()


def test_pending_errors_and_budget():
    ctx = fm.Context(0)
    try:
        server = fm.Server(n_workers=2, hbm_budget=2 << 30, ctx=ctx)
        big = bodies(600000, 1, 11)
        opt = fm.make_options(expansion_order=10, leaf_size_source=64, multipole_acceptance=0.5)
        rid = server.submit(big, 1, opt)
        rc, out, _ = server.poll(rid, timeout_ms=0)
        assert rc in (L.FMM_PENDING, L.FMM_OK)
        if rc == L.FMM_PENDING:
            rc, out, _ = server.poll(rid, timeout_ms=-1)
        assert rc == L.FMM_OK and np.isfinite(out[:, 4:7]).all()
        # a request larger than the whole budget fails alone
        huge = bodies(8_000_000, 1, 12)
        rid = server.submit(huge, 1, opt)
        assert server.poll(rid)[0] == L.FMM_ERR_MEMORY
        # an invalid request fails with its own status; the next one still runs
        bad = fm.make_options(expansion_order=10, leaf_size_source=0)
        rid_bad = server.submit(bodies(100, 1, 13), 1, bad)
        rid_ok = server.submit(bodies(5000, 1, 14), 1, opt)
        assert server.poll(rid_bad)[0] == L.FMM_ERR_ARGUMENT
        assert server.poll(rid_ok)[0] == L.FMM_OK
        server.stop()
        with pytest.raises(fm.FMMError):
            server.submit(bodies(10, 1, 15), 1, opt)
    finally:
        ctx.close()


def test_requests_wait_for_memory_instead_of_failing():
    # a budget that holds one of these requests but not three: each one fits (it waits for
    # the memory the others hand back), none fails, and the results equal the solves alone
    ctx = fm.Context(0)
    try:
        opt = fm.make_options(expansion_order=8, leaf_size_source=64, multipole_acceptance=0.5)
        bufs = [bodies(900_000, 1, 20 + k) for k in range(3)]
        alone = [fm.solve_buffers(b, 1, opt, ctx=ctx)[0] for b in bufs]
        budget = int(1.5 * fm.request_footprint(bufs[0], 1, opt))
        server = fm.Server(n_workers=3, hbm_budget=budget, ctx=ctx)
        ids = [server.submit(b, 1, opt) for b in bufs]
        for k, rid in enumerate(ids):
            rc, out, _ = server.poll(rid, timeout_ms=-1)
            assert rc == L.FMM_OK
            np.testing.assert_array_equal(out, alone[k])
        server.stop()
    finally:
        ctx.close()
