"""bench.py under torchrun (N > 1 replicas) on CPU: two gloo ranks.

* every rank gets the slowest rank's time (max over ranks), and the job rate counts all
  replicas' bodies at that time;
* the reference arm runs on rank 0 only: the other ranks exit 0 without work or output.
"""
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
dist.init_process_group("gloo", rank=int(os.environ["RANK"]), world_size=int(os.environ["WORLD_SIZE"]))
rank = dist.get_rank()
t = bench.max_over_ranks(10.0 * rank + 1.0, dist.get_world_size())
print("max", t, "rate", bench.job_rate(1000, dist.get_world_size(), t), flush=True)
dist.barrier()
dist.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_with_two_gloo_ranks():
    port = free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(out.split())
    for o in outs:
        # rank 0 contributed 1 ms, rank 1 11 ms: both see 11 ms; 2 replicas x 1000 bodies / 11 ms
        assert float(o[1]) == 11.0
        assert abs(float(o[3]) - 2 * 1000 / 11e-3) < 1e-6


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
