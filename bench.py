#!/usr/bin/env python
"""Benchmark of the B200 FMM evaluation path (one JSON line on rank 0).

Default workload (the headline configuration): N = 1,000,000 Laplace point
sources in 8 isotropic Gaussian clusters (sigma 0.05, centres uniform in the
unit cube) plus 10% uniform background, strengths uniform in [-1, 1], seed 2;
expansion_order 10, leaf_size 64, multipole_acceptance 0.5,
PowerRelativeGradient(1e-6); potential and gradient at every body.  A step is
one fmm! (tree, lists, influence estimate, all passes, unsort).

* value   : bodies/s of the MIXED-precision solve with inputs resident in HBM
* e2e     : bodies/s through fmm_solve with pinned host buffers (H2D of the
            source buffer and D2H of the 16-row target buffer inside each step)
* f64_*   : the same for the plain FP64 drop-in
* rel_err : relative L2 error of the gradient vs FP64 all-pairs direct on a
            20,000-target subsample
Multi-GPU (torchrun): independent replicas, one per GPU ("scaling": "weak").
`--impl reference` times the CPU restatement of the reference algorithm (the
Julia package cannot run on this image) on all host cores.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


# ---------------------------------------------------------------------------
# synthetic workloads (seeded; shapes and distributions of the configurations)
def gen_uniform(n, seed):
    rng = np.random.default_rng(seed)
    b = np.zeros((n, 5))
    b[:, :3] = rng.random((n, 3))
    b[:, 4] = rng.random(n)
    return b


def gen_clustered(n, seed):
    rng = np.random.default_rng(seed)
    b = np.zeros((n, 5))
    nb = n // 10
    centres = rng.random((8, 3))
    k = rng.integers(0, 8, n - nb)
    b[: n - nb, :3] = centres[k] + 0.05 * rng.standard_normal((n - nb, 3))
    b[n - nb:, :3] = rng.random((nb, 3))
    b[:, 4] = 2 * rng.random(n) - 1
    return b


def gen_ring(n, seed):
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


def gen_c4(n, seed):
    rng = np.random.default_rng(seed)
    b = np.zeros((n, 5))
    b[:, :3] = rng.random((n, 3))
    b[:, 4] = rng.random(n)
    return b


METRIC = "FMM bodies/sec at <=1e-6 rel err vs FP64 direct, mixed vs FP64"

WORKLOADS = {
    "c2": dict(workload="clustered-8-gaussian point sources N=1e6 (10% uniform), p<=10, leaf 64, MAC 0.5, "
                        "PowerRelativeGradient(1e-6)",
               n=1_000_000, gen=gen_clustered, seed=2, kind=1, p=10, ls=64, mac=0.5, err=1e-6,
               ps=True, gs=True, hs=False, flops_per_pair=20, n_cpu=100_000),
    "c1": dict(workload="uniform point sources N=1e4, p=6, leaf 50, MAC 0.5", n=10_000, gen=gen_uniform, seed=1,
               kind=1, p=6, ls=50, mac=0.5, err=None, ps=True, gs=True, hs=False, flops_per_pair=20,
               n_cpu=10_000),
    "c4": dict(workload="adjoint: 200k sources U[0,1]^3, 10k probes U[-0.5,1.5]^3, p=8, loss sum(phi^2), "
                        "gradients wrt strengths and positions", n=200_000, n_probes=10_000, gen=gen_c4, seed=4,
               kind=1, p=8, ls=50, mac=0.5, err=None, ps=True, gs=True, hs=False, flops_per_pair=20,
               n_cpu=20_000),
    "c5": dict(workload="serving: requests with N log-uniform [1e3, 5e5], half point sources / half vortex, uniform "
                        "cube or 8 Gaussians, PowerRelativeGradient tolerance log-uniform [1e-8, 1e-4] (p <= 16), "
                        "Poisson arrivals at 70% of the sequential plain-FP64 capacity", n_requests=4096, seed=5, workers=4,
               kind=1, n=0, n_cpu=0),
    "c3": dict(workload="vortex ring N=2e6 (R=1, core sigma 0.05), p=12, leaf 80, MAC 0.4, velocity + gradient",
               n=2_000_000, gen=gen_ring, seed=3, kind=3, p=12, ls=80, mac=0.4, err=None, ps=False, gs=True,
               hs=True, flops_per_pair=72, n_cpu=40_000),
}


# settings tried, loosest first, for the mixed vs FP64 comparison at <= 1e-6 relative error
# (tolerance, expansion order, multipole acceptance); MAC 0.5 converges like 0.5^(p+1) in the worst case
MATCHED_CANDIDATES = [(1e-7, 12, 0.5), (3e-8, 12, 0.5), (1e-8, 12, 0.5), (1e-8, 16, 0.5)]

# f32x2 operations the packed near-field loop issues per source and pair of targets, by
# (kind, scalar potential, velocity gradient): point sources phi + grad 13 (grad alone 12),
# vortex particles u + grad u 32
NEAR_F32X2_OPS = {(1, True, False): 13, (1, False, False): 12, (3, False, True): 32}

# DRAM bytes (read + write) of the solve's near-field launch, one ncu capture of the full-size
# workload (dram__bytes_read.sum + dram__bytes_write.sum)
NEAR_TRAFFIC = {"c2": 311889408 + 46925568, "c3": 5638054144 + 197501696}


def options(fm, w, precision):
    err = fm.PowerRelativeGradient(w["err"]) if w["err"] else None
    return fm.make_options(expansion_order=w["p"], leaf_size_source=w["ls"], multipole_acceptance=w["mac"],
                           error_tolerance=err, scalar_potential=w["ps"], gradient=w["gs"], hessian=w["hs"],
                           precision=precision)


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU: the restatement of the reference algorithm on all host cores
def cpu_run(w, n, seed, buf=None):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    buf = w["gen"](n, seed) if buf is None else buf
    em = O.ERR_POWER_REL_GRAD if w["err"] else O.ERR_NONE
    o = O.options(expansion_order=w["p"], leaf_size_source=w["ls"], multipole_acceptance=w["mac"], error_method=em,
                  error_tolerance=w["err"] or 0.0, scalar_potential=int(w["ps"]), gradient=int(w["gs"]),
                  hessian=int(w["hs"]), n_threads=0)
    t0 = time.perf_counter()
    O.fmm(buf, w["kind"], o)
    return time.perf_counter() - t0


def cpu_baseline(w, n=None):
    n = n or w["n_cpu"]
    dt = cpu_run(w, n, w["seed"] + 1000)
    return {"value": n / dt, "unit": "bodies/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{n:,} bodies of the same distribution, one fmm! of the C++ FP64 restatement, {dt:.2f} s"}


def max_over_ranks(value, world, device="cpu"):
    """The largest of the ranks' values (every rank passes its own and gets the max): the
    slowest replica's time is the job's time."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(n_per_rank, world, ms_per_step):
    """Whole-job throughput of world replicas of n_per_rank bodies each, at the slowest rank's time."""
    return world * n_per_rank / (ms_per_step * 1e-3)


def reference_arm(args, w, rank):
    """The CPU restatement of the reference's fmm! on the GPU arm's workload: the same
    bodies (same generator and seed), the same options, one full solve per timed step on
    all host cores.  Warm-up steps run a 10,000-body sample (they only page the library
    and the thread pool in; a full-size warm-up would add minutes and no information)."""
    if rank != 0:
        return
    n = w["n"]
    buf = w["gen"](n, w["seed"])
    for _ in range(args.warmup):
        cpu_run(w, 10_000, w["seed"] + 1000)
    ts = [cpu_run(w, n, w["seed"], buf=buf) for _ in range(args.steps)]
    v = n / (sum(ts) / len(ts))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "bodies/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(ts) / len(ts),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(w, n, 1),
            "cpu_baseline": {"value": v, "unit": "bodies/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"the full workload ({n:,} bodies, the GPU arm's bodies and options) per "
                                       "step; warm-up steps on 10,000 bodies; the Julia reference itself is "
                                       "unavailable on this image"},
            "e2e": {"value": v, "unit": "bodies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_of(w, n, world):
    """The workload's config object, identical for the GPU arm and the reference arm."""
    return {"workload": w["workload"], "n_bodies": n, "parallelism": f"replicas x{world}",
            "l2": "inputs + 256 MB buffer written between timed steps (GPU arm)"}


# ---------------------------------------------------------------------------
def gpu_arm(args, w, rank, world, local_rank):
    import torch
    import fastmultipole_b200 as fm
    from fastmultipole_b200 import _lib as L

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)
    ctx = fm.Context(local_rank)
    ctx.set_stream(stream.cuda_stream)
    lib = L.lib()
    n, kind = w["n"], w["kind"]
    buf = w["gen"](n, w["seed"])
    d = buf.shape[1]
    src_dev = torch.from_numpy(buf).to(dev)
    out_dev = torch.empty((n, 16), dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    src_d = L.SourceSystem(kind, n, d, src_dev.data_ptr(), L.FMM_MEMORY_DEVICE)
    tgt_d = L.TargetSystem(n, None, 0, out_dev.data_ptr(), L.FMM_MEMORY_DEVICE)
    buf_pin = torch.from_numpy(buf).pin_memory()
    out_pin = torch.empty((n, 16), dtype=torch.float64).pin_memory()
    src_h = L.SourceSystem(kind, n, d, buf_pin.data_ptr(), L.FMM_MEMORY_HOST)
    tgt_h = L.TargetSystem(n, None, 0, out_pin.data_ptr(), L.FMM_MEMORY_HOST)
    res = L.Result()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    def timed(opt, src, tgt, steps, warmup):
        ctx.set_timing(False)
        for _ in range(warmup):
            ctx.check(lib.fmm_solve(ctx.handle, C.byref(tgt), C.byref(src), C.byref(opt), C.byref(res)))
        barrier()
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.check(lib.fmm_solve(ctx.handle, C.byref(tgt), C.byref(src), C.byref(opt), C.byref(res)))
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        barrier()
        return max_over_ranks(total, world, dev) / steps  # ms per step, max over ranks

    opt_mixed = options(fm, w, "mixed")
    opt_f64 = options(fm, w, "f64")
    with ClockSampler(local_rank) as clk:
        ms_mixed = timed(opt_mixed, src_d, tgt_d, args.steps, args.warmup)
    launches = res.n_kernel_launches
    ms_f64 = timed(opt_f64, src_d, tgt_d, args.steps, max(1, args.warmup // 2))
    ms_e2e = timed(opt_mixed, src_h, tgt_h, args.steps, 1)

    # stage times of one solve (roofline of the dominant kernel)
    def staged(opt):
        ctx.set_timing(True)
        flush.zero_()
        ctx.check(lib.fmm_solve(ctx.handle, C.byref(tgt_d), C.byref(src_d), C.byref(opt), C.byref(res)))
        ctx.set_timing(False)
        return {k: getattr(res, k) for k, _ in L.Result._fields_}

    st_mixed = staged(opt_mixed)
    st_f64 = staged(opt_f64)

    # accuracy vs FP64 all-pairs direct on a 20k-target subsample
    ids = np.random.default_rng(7).choice(n, min(n, 20_000), replace=False)
    tpos = np.ascontiguousarray(buf[ids, :3])
    ref = np.zeros((len(ids), 16))
    tsub = L.TargetSystem(len(ids), tpos.ctypes.data, 3, ref.ctypes.data, L.FMM_MEMORY_HOST)
    ctx.check(lib.fmm_direct(ctx.handle, C.byref(tsub), C.byref(src_d), 1, 1, 0, L.FMM_PRECISION_F64))
    rows = slice(4, 7)  # gradient (point sources) / velocity (vortex particles)

    def accuracy(opt):
        """(relative L2 error of the gradient rows vs FP64 direct on the subsample, error_success, p_max)"""
        ctx.check(lib.fmm_solve(ctx.handle, C.byref(tgt_d), C.byref(src_d), C.byref(opt), C.byref(res)))
        got = out_dev.cpu().numpy()[ids]
        e = float(np.linalg.norm(got[:, rows] - ref[:, rows]) / np.linalg.norm(ref[:, rows]))
        return e, bool(res.error_success), int(res.p_max)

    errs, succ = {}, {}
    for name, opt in (("mixed", opt_mixed), ("f64", opt_f64)):
        errs[name], succ[name], _ = accuracy(opt)

    # mixed vs FP64 at the metric's accuracy: the loosest candidate setting whose mixed and
    # FP64 solves both reach <= 1e-6 relative error on the subsample, both timed
    matched = None
    tried = []
    if w["err"] and not args.no_matched:
        for eps, pmax, mac in MATCHED_CANDIDATES:
            wm = dict(w, err=eps, p=pmax, mac=mac)
            om, of = options(fm, wm, "mixed"), options(fm, wm, "f64")
            em_, sm_, pm_ = accuracy(om)
            ef_, sf_, pf_ = accuracy(of)
            tried.append({"setting": f"PowerRelativeGradient({eps:g}), p<={pmax}, MAC {mac}", "mixed": em_,
                          "f64": ef_})
            if max(em_, ef_) <= 1e-6:
                tm = timed(om, src_d, tgt_d, args.steps, 1)
                tf = timed(of, src_d, tgt_d, args.steps, 1)
                matched = {"error_tolerance": f"PowerRelativeGradient({eps:g})", "expansion_order": pmax,
                           "multipole_acceptance": mac,
                           "value": job_rate(n, world, tm), "ms_per_step": tm, "rel_err_vs_direct": em_,
                           "error_success": sm_, "p_max": pm_,
                           "f64_value": job_rate(n, world, tf), "f64_ms_per_step": tf, "f64_rel_err_vs_direct": ef_,
                           "f64_error_success": sf_, "f64_p_max": pf_, "speedup_mixed_vs_f64": tf / tm}
                break
        if matched is None:
            matched = {"unavailable": "no candidate setting reached <= 1e-6 on the subsample"}
        matched["tried"] = tried

    if rank != 0:
        return
    pk = peaks()
    sm_max = pk.get("sm_max_mhz", 1965.0)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    nominal_fp32 = sms * 128 * 2 * sm_max * 1e6 / 1e12
    # measured CUDA-core FP32 throughput (independent FMA chains, packed and scalar): the
    # near field's denominator; the nominal figure is kept beside it
    meas = {}
    for name, packed in (("packed_f32x2", 1), ("scalar", 0)):
        v = C.c_double(0.0)
        ctx.check(lib.fmm_measure_fp32_peak(local_rank, packed, C.byref(v)))
        meas[name] = v.value
    fp32_peak = max(meas.values())
    fp64_peak = nominal_fp32 / 2
    near_flops = st_mixed["n_p2p_pairs"] * w["flops_per_pair"]
    stages = {"nearfield": st_mixed["t_nearfield_ms"], "horizontal": st_mixed["t_horizontal_ms"],
              "upward": st_mixed["t_upward_ms"], "downward": st_mixed["t_downward_ms"],
              "tree": st_mixed["t_tree_ms"], "lists": st_mixed["t_lists_ms"],
              "influence_estimate": st_mixed["t_influence_ms"]}
    dom = max(("nearfield", "horizontal"), key=lambda k: stages[k])
    if dom == "nearfield":
        ach = near_flops / (stages["nearfield"] * 1e-3) / 1e12
        traffic = NEAR_TRAFFIC.get(args.config) if not args.bodies else None
        roof = {"kernel": "k_p2p (FP32, mixed)", "bound": "fp32", "achieved": ach, "peak": fp32_peak,
                "unit": "TFLOP/s", "frac": ach / fp32_peak, "traffic": traffic,
                "work": f"{st_mixed['n_p2p_pairs']:.3e} pairs x {w['flops_per_pair']} flop",
                "peak_source": "measured on this GPU in this run (fmm_measure_fp32_peak: independent FMA chains; "
                               "MEASURED_PEAKS.json holds no CUDA-core figure)",
                "peak_measured": meas, "peak_nominal": nominal_fp32, "frac_of_nominal": ach / nominal_fp32}
        ops = NEAR_F32X2_OPS.get((w["kind"], w["ps"], w["hs"]))
        if ops:
            # the packed loop's own bound: its f32x2 operations per source and target pair at the
            # measured f32x2 rate (4 flop per f32x2 FMA), independent of the flop convention above
            bound_ms = st_mixed["n_p2p_pairs"] * ops / 2 / (meas["packed_f32x2"] * 1e12 / 4) * 1e3
            roof["instruction_view"] = {
                "f32x2_ops_per_source_and_two_targets": ops, "bound_ms": bound_ms,
                "frac": bound_ms / stages["nearfield"],
                "note": "operations counted in the packed loop (rsqrt runs on the XU pipe beside them); "
                        "frac divides by the near field's event window, which also holds the concurrent far field"}
        if traffic:
            gbs = traffic / (stages["nearfield"] * 1e-3) / 1e9
            roof["hbm_view"] = {"achieved_gbs": gbs, "peak_gbs": pk.get("hbm_gbs"),
                                "frac": gbs / pk["hbm_gbs"] if pk.get("hbm_gbs") else None,
                                "note": "DRAM bytes of one launch (ncu) over its event time: not HBM-bound"}
    else:
        ach = st_mixed["m2l_flops"] / (stages["horizontal"] * 1e-3) / 1e12
        roof = {"kernel": "k_m2l (FP64)", "bound": "fp64", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": ach / fp64_peak, "traffic": None, "work": f"{st_mixed['m2l_flops']:.3e} algorithmic flop",
                "peak_source": "nominal FP64 CUDA-core peak (half the FP32 rate)"}
    value = job_rate(n, world, ms_mixed)
    line = {
        "metric": METRIC,
        "value": value, "unit": "bodies/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded)",
        "config": config_of(w, n, world), "precision": "mixed",
        "rel_err_vs_direct": errs["mixed"], "f64_rel_err_vs_direct": errs["f64"],
        "error_success": succ["mixed"], "f64_error_success": succ["f64"],
        "at_1e-6": matched,
        "f64_value": job_rate(n, world, ms_f64), "f64_ms_per_step": ms_f64,
        "speedup_mixed_vs_f64": ms_f64 / ms_mixed,
        "e2e": {"value": job_rate(n, world, ms_e2e), "unit": "bodies/s", "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": int(buf.nbytes), "d2h_bytes_per_step": int(n * 16 * 8)},
        "gpu_launches": int(launches) * args.steps,
        "stages_ms": stages, "f64_stages_ms": {"nearfield": st_f64["t_nearfield_ms"],
                                               "horizontal": st_f64["t_horizontal_ms"],
                                               "upward": st_f64["t_upward_ms"], "downward": st_f64["t_downward_ms"],
                                               "tree": st_f64["t_tree_ms"], "lists": st_f64["t_lists_ms"],
                                               "influence_estimate": st_f64["t_influence_ms"]},
        "p_max": st_mixed["p_max"], "n_m2l": st_mixed["n_m2l"], "n_direct": st_mixed["n_direct"],
        "n_p2p_pairs": st_mixed["n_p2p_pairs"],
        "roofline": roof,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(w)
    print(json.dumps(line), flush=True)
    ctx.close()


def vjp_arm(args, w):
    """Adjoint workload: one step = forward solve at the probes (phi), then fmm_vjp with
    dL/dphi = 2 phi (L = sum phi^2); device-resident inputs; CUDA-event timing.  Both
    precisions are timed (value: the FP64 drop-in) and both gradients are checked by central
    finite differences of the exact loss (FP64 all-pairs) on the same 64 coordinates."""
    import torch
    import fastmultipole_b200 as fm
    from fastmultipole_b200 import _lib as L
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    ctx = fm.Context(0)
    ctx.set_stream(stream.cuda_stream)
    lib = L.lib()
    n, npr = w["n"], w["n_probes"]
    buf = w["gen"](n, w["seed"])
    probes = -0.5 + 2.0 * np.random.default_rng(w["seed"] + 1).random((npr, 3))
    src_dev = torch.from_numpy(buf).to(dev)
    pr_dev = torch.from_numpy(probes).to(dev)
    out_dev = torch.empty((npr, 16), dtype=torch.float64, device=dev)
    dout = torch.zeros((npr, 16), dtype=torch.float64, device=dev)
    dq = torch.empty(n, dtype=torch.float64, device=dev)
    dx = torch.empty((n, 3), dtype=torch.float64, device=dev)
    dy = torch.empty((npr, 3), dtype=torch.float64, device=dev)
    src = L.SourceSystem(1, n, 5, src_dev.data_ptr(), L.FMM_MEMORY_DEVICE)
    tgt = L.TargetSystem(npr, pr_dev.data_ptr(), 3, out_dev.data_ptr(), L.FMM_MEMORY_DEVICE)
    res = L.Result()
    dp = L._dp

    def run(precision):
        opt = fm.make_options(expansion_order=w["p"], leaf_size_source=w["ls"], multipole_acceptance=w["mac"],
                              scalar_potential=True, gradient=True, precision=precision)

        def step():
            ctx.check(lib.fmm_solve(ctx.handle, C.byref(tgt), C.byref(src), C.byref(opt), C.byref(res)))
            dout[:, 3] = 2.0 * out_dev[:, 3]
            ctx.check(lib.fmm_vjp(ctx.handle, C.byref(tgt), C.byref(src), C.byref(opt),
                                  C.cast(dout.data_ptr(), dp), C.cast(dq.data_ptr(), dp),
                                  C.cast(dx.data_ptr(), dp), C.cast(dy.data_ptr(), dp), C.byref(res)))

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / args.steps, dq.cpu().numpy(), dx.cpu().numpy(), dy.cpu().numpy()

    ms, gq, gx, gy = run("f64")
    ms_mx, gq_mx, gx_mx, gy_mx = run("mixed")
    # central finite differences of the exact loss (all-pairs direct) on 64 coordinates
    phi = np.zeros((npr, 16))

    def loss(b, pr):
        bb = np.ascontiguousarray(b)
        pp = np.ascontiguousarray(pr)
        s_ = L.SourceSystem(1, n, 5, bb.ctypes.data, L.FMM_MEMORY_HOST)
        t_ = L.TargetSystem(npr, pp.ctypes.data, 3, phi.ctypes.data, L.FMM_MEMORY_HOST)
        ctx.check(lib.fmm_direct(ctx.handle, C.byref(t_), C.byref(s_), 1, 0, 0, L.FMM_PRECISION_F64))
        return float(np.sum(phi[:, 3] ** 2))

    rng = np.random.default_rng(9)
    errs, errs_mx = [], []
    h = 1e-6
    for _ in range(64):
        which = rng.integers(0, 3)
        if which == 0:
            i = rng.integers(0, n)
            bp, bm = buf.copy(), buf.copy()
            hq = 1e-3 * buf[i, 4]
            bp[i, 4] += hq
            bm[i, 4] -= hq
            fd = (loss(bp, probes) - loss(bm, probes)) / (2 * hq)
            errs.append(abs(gq[i] - fd) / np.abs(gq).max())
            errs_mx.append(abs(gq_mx[i] - fd) / np.abs(gq).max())
        elif which == 1:
            i, k = rng.integers(0, n), rng.integers(0, 3)
            bp, bm = buf.copy(), buf.copy()
            bp[i, k] += h
            bm[i, k] -= h
            fd = (loss(bp, probes) - loss(bm, probes)) / (2 * h)
            errs.append(abs(gx[i, k] - fd) / np.abs(gx).max())
            errs_mx.append(abs(gx_mx[i, k] - fd) / np.abs(gx).max())
        else:
            i, k = rng.integers(0, npr), rng.integers(0, 3)
            pp, pm = probes.copy(), probes.copy()
            pp[i, k] += h
            pm[i, k] -= h
            fd = (loss(buf, pp) - loss(buf, pm)) / (2 * h)
            errs.append(abs(gy[i, k] - fd) / np.abs(gy).max())
            errs_mx.append(abs(gy_mx[i, k] - fd) / np.abs(gy).max())
    line = {"metric": "FMM loss gradient (forward + adjoint) sources/s", "value": n / (ms * 1e-3),
            "unit": "sources/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": w["workload"], "n_sources": n, "n_probes": npr, "solves_per_step": 3},
            "fd_max_rel_dev": float(max(errs)), "fd_coordinates": len(errs),
            "mixed": {"value": n / (ms_mx * 1e-3), "ms_per_step": ms_mx, "fd_max_rel_dev": float(max(errs_mx))}}
    print(json.dumps(line), flush=True)
    ctx.close()


def serve_specs(w):
    """The request mix of the serving workload (seeded): per request (n, kind, tolerance,
    clustered, seed of its bodies).  Bodies are generated from the seed when the request is
    submitted, so that 4,096 requests need not sit in host memory at once."""
    rng = np.random.default_rng(w["seed"])
    specs = []
    for k in range(w["n_requests"]):
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(5e5))))
        kind = 1 if k % 2 == 0 else 3
        tol = float(np.exp(rng.uniform(np.log(1e-8), np.log(1e-4))))
        clustered = bool(rng.random() < 0.5)
        specs.append((n, kind, tol, clustered, int(rng.integers(1 << 30))))
    return specs


def serve_bodies(spec):
    n, kind, _, clustered, seed = spec
    b = gen_clustered(n, seed) if clustered else gen_uniform(n, seed)
    if kind == 3:
        rng = np.random.default_rng(seed + 1)
        v = np.zeros((n, 7))
        v[:, :4] = b[:, :4]
        v[:, 4:7] = (2 * rng.random((n, 3)) - 1) / n
        b = v
    return b


def serve_arm(args, w):
    """Serving workload against sequential plain FP64 solves on the same GPU.

    Both run the seeded request mix back to back (capacity), then replay one Poisson
    arrival stream at 70% of the sequential capacity (a rate fixed by the baseline, so
    that latencies compare across builds); latency = completion - arrival.  The capacity
    pass keeps a window of requests queued (the server never idles) rather than all of
    them at once, and every request's bodies are generated just before it is submitted
    (outside the timed intervals of the sequential passes), so host memory stays bounded.
    Every worker's buffers are grown before timing (growing frees and reallocates device
    memory, which waits for the whole device)."""
    import collections
    import threading
    import fastmultipole_b200 as fm
    from fastmultipole_b200 import _lib as L
    specs = serve_specs(w)
    ns = np.array([sp[0] for sp in specs])
    window = 64

    def opt_of(kind, tol):
        return fm.make_options(expansion_order=16, leaf_size_source=64 if kind == 1 else 80,
                               multipole_acceptance=0.5, error_tolerance=fm.PowerRelativeGradient(tol),
                               scalar_potential=kind == 1, precision="f64")

    def largest(limit=None):
        out = {}
        for sp in specs:
            if limit is not None and sp[0] > limit:
                continue
            if sp[1] not in out or sp[0] > out[sp[1]][0]:
                out[sp[1]] = sp
        return list(out.values())

    arrive = None
    # sequential plain FP64 solves on one context (generation of the next request's bodies is
    # excluded from the capacity time)
    seq_ctx = fm.Context(0)
    for sp in largest():
        fm.solve_buffers(serve_bodies(sp), sp[1], opt_of(sp[1], sp[2]), ctx=seq_ctx)
    busy = 0.0
    for sp in specs:
        b = serve_bodies(sp)
        t0 = time.perf_counter()
        fm.solve_buffers(b, sp[1], opt_of(sp[1], sp[2]), ctx=seq_ctx)
        busy += time.perf_counter() - t0
    seq_cap = len(specs) / busy
    rate = 0.7 * seq_cap
    arrive = np.cumsum(np.random.default_rng(w["seed"] + 1).exponential(1.0 / rate, len(specs)))
    # the Poisson replay: a request whose arrival has passed is solved at once
    seq_lat = np.zeros(len(specs))
    t0 = time.perf_counter()
    for k, sp in enumerate(specs):
        b = serve_bodies(sp)
        delay = t0 + arrive[k] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        fm.solve_buffers(b, sp[1], opt_of(sp[1], sp[2]), ctx=seq_ctx)
        seq_lat[k] = 1e3 * (time.perf_counter() - (t0 + arrive[k]))
    seq_ctx.close()

    ctx = fm.Context(0)
    server = fm.Server(n_workers=w["workers"], hbm_budget=150 << 30, ctx=ctx)
    n_express = max(1, w["workers"] // 2)
    ids = [server.submit(serve_bodies(sp), sp[1], opt_of(sp[1], sp[2])) for sp in largest()
           for _ in range(w["workers"])]
    ids += [server.submit(serve_bodies(sp), sp[1], opt_of(sp[1], sp[2])) for sp in largest(65536)
            for _ in range(n_express)]
    for rid in ids:
        server.poll(rid)
    # capacity: a window of requests queued at all times; the bodies of request k + window are
    # generated while the server works on the window
    bodies = collections.deque(serve_bodies(sp) for sp in specs[:window])
    t0 = time.perf_counter()
    live = collections.deque()
    nxt = 0
    while nxt < len(specs) or live:
        while nxt < len(specs) and len(live) < window:
            sp = specs[nxt]
            live.append(server.submit(bodies.popleft(), sp[1], opt_of(sp[1], sp[2])))
            if nxt + window < len(specs):
                bodies.append(serve_bodies(specs[nxt + window]))
            nxt += 1
        rc, _, _ = server.poll(live.popleft())
        assert rc == L.FMM_OK
    cap = len(specs) / (time.perf_counter() - t0)
    done_at = {}
    outstanding = {}
    lock = threading.Lock()
    finished = threading.Event()

    def poller():
        while not (finished.is_set() and not outstanding):
            with lock:
                items = list(outstanding.items())
            for rid, k in items:
                rc, _, _ = server.poll(rid, 0)
                if rc != L.FMM_PENDING:
                    done_at[k] = time.perf_counter()
                    with lock:
                        outstanding.pop(rid, None)
            time.sleep(1e-4)

    th = threading.Thread(target=poller)
    th.start()
    t0 = time.perf_counter()
    for k, sp in enumerate(specs):
        b = serve_bodies(sp)
        delay = t0 + arrive[k] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        rid = server.submit(b, sp[1], opt_of(sp[1], sp[2]))
        with lock:
            outstanding[rid] = k
    finished.set()
    th.join()
    lat = np.array([1e3 * (done_at[k] - (t0 + arrive[k])) for k in range(len(specs))])
    server.stop()
    ctx.close()
    line = {"metric": "serve latency p50 ms", "value": float(np.percentile(lat, 50)), "unit": "ms",
            "p99_ms": float(np.percentile(lat, 99)), "p90_ms": float(np.percentile(lat, 90)),
            "sequential_p50_ms": float(np.percentile(seq_lat, 50)),
            "sequential_p99_ms": float(np.percentile(seq_lat, 99)),
            "offered_requests_per_s": rate, "capacity_requests_per_s": cap,
            "sequential_requests_per_s": seq_cap,
            "capacity_bodies_per_s": float(ns.sum() * cap / len(specs)),
            "sequential_bodies_per_s": float(ns.sum() * seq_cap / len(specs)), "capacity_vs_sequential": cap / seq_cap,
            "n_gpus": 1, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": w["workload"], "requests": len(specs), "workers": w["workers"],
                       "express_workers": n_express, "bodies_total": int(ns.sum()), "hbm_budget_gb": 150,
                       "arrivals": "Poisson at 70% of the sequential capacity", "capacity_window": window}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-matched", action="store_true", help="skip the mixed vs FP64 pair at <= 1e-6 error")
    ap.add_argument("--bodies", type=int, default=None, help="override N (small cases for profiling)")
    args = ap.parse_args()
    w = WORKLOADS[args.config]
    if args.bodies:
        w = dict(w, n=args.bodies, workload=w["workload"] + f" [N overridden: {args.bodies}]")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.config == "c5":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference runs one fmm! at a time "
                                  "(Julia, absent on this image); no serving loop to time"}))
            return
        if rank == 0:
            serve_arm(args, w)
        return
    if args.config == "c4":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference differentiates fmm! with "
                                  "ReverseDiff (Julia), absent on this image; the CPU port has no adjoint"}))
            return
        if rank == 0:
            vjp_arm(args, w)
        return
    if args.impl == "reference":
        reference_arm(args, w, rank)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        gpu_arm(args, w, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
