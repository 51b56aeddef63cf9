"""Multi-rank plumbing of bench.py (replicas: one box per rank, no data-path
collective): max-over-ranks time and summed work, run as two gloo ranks on
CPU."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank), LBM_BENCH_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench
    w, r, _ = bench.dist_setup(world)
    assert (w, r) == (world, rank)
    t = bench.dist_max(1.0 + rank, w)            # rank times 1, 2 -> max 2
    u = bench.dist_sum(10.0 * (rank + 1), w)     # work 10 + 20
    bench.barrier(w)
    out[rank] = (t, u)
    import torch.distributed as dist
    dist.destroy_process_group()


def test_max_time_and_summed_work_over_two_gloo_ranks():
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    assert out[0] == out[1] == (2.0, 30.0)


def test_reference_arm_on_nonzero_rank_is_silent():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line_small_box():
    """The reference arm times the reference CPU solver (oracle/_ref) and prints
    one JSON line with impl=reference, cpu_baseline and e2e."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--size", "32", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if "unavailable" in line:
        return
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] == 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["value"] > 0
