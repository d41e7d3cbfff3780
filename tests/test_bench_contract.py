"""bench.py on CPU: the pieces of its output contract that need no GPU.

* the GPU arm and the reference arm describe the workload with the same config object;
* the serving mix is seeded (the same 4,096 requests every run), and a request's bodies are
  regenerated identically from its seed;
* the settings tried for the mixed-vs-FP64 pair at <= 1e-6 error are loosest first.
"""
import numpy as np

import bench


def test_reference_and_gpu_arms_share_the_config():
    w = bench.WORKLOADS["c2"]
    a = bench.config_of(w, w["n"], 1)
    b = bench.config_of(w, w["n"], 1)
    assert a == b and a["n_bodies"] == 1_000_000 and a["workload"] == w["workload"]


def test_serving_mix_is_seeded_and_regenerated_identically():
    w = bench.WORKLOADS["c5"]
    s1, s2 = bench.serve_specs(w), bench.serve_specs(w)
    assert len(s1) == 4096 and s1 == s2
    kinds = {sp[1] for sp in s1}
    assert kinds == {1, 3}
    ns = np.array([sp[0] for sp in s1])
    assert ns.min() >= 1000 and ns.max() <= 500_000
    small = min(s1, key=lambda sp: sp[0])
    np.testing.assert_array_equal(bench.serve_bodies(small), bench.serve_bodies(small))
    assert bench.serve_bodies(small).shape == (small[0], 5 if small[1] == 1 else 7)


def test_accuracy_candidates_loosest_first():
    eps = [c[0] for c in bench.MATCHED_CANDIDATES]
    assert eps == sorted(eps, reverse=True)
    assert all(p <= 20 and 0 < mac < 1 for _, p, mac in bench.MATCHED_CANDIDATES)


def test_every_near_field_workload_has_an_instruction_count():
    # the roofline's instruction view needs the packed loop's operation count for each
    # near-field-dominated workload the GPU arm times
    for key in ("c1", "c2", "c3"):
        w = bench.WORKLOADS[key]
        assert (w["kind"], w["ps"], w["hs"]) in bench.NEAR_F32X2_OPS, key
