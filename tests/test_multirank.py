"""The multi-GPU paths of bench.py on the CPU, with two gloo ranks: the max-over-ranks timing
rule, the sum of the ranks' pair counts when the replica ensemble is dealt round-robin, and
a torchrun launch of the reference arm in which rank 0 alone runs and prints."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2,
                            timeout=datetime.timedelta(seconds=60))
    try:
        out.put((rank, bench.reduce_max([rank + 1.0, 10.0 - rank, 0.5], dist, "cpu")
                 + bench.reduce_sum([100.0 * (rank + 1), 7.0], dist, "cpu")))
    finally:
        dist.destroy_process_group()


def test_reduce_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0] == got[1] == [2.0, 10.0, 0.5, 300.0, 14.0]


def test_reduce_max_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max([1, 2.5], None, "cpu") == [1.0, 2.5]
    assert bench.reduce_sum([1, 2.5], None, "cpu") == [1.0, 2.5]


def test_round_robin_deals_every_replica_once():
    """rank r of N takes replicas r, r + N, ...: every replica on exactly one rank."""
    sys.path.insert(0, os.path.join(ROOT, "mdcore-history_b200"))
    import workloads as W
    ens = W.argon_replicas(nrep=10, seed=1)
    for world in (1, 2, 3, 4):
        dealt = [s.name for r in range(world) for s in ens[r::world]]
        assert sorted(dealt) == sorted(s.name for s in ens) and len(set(dealt)) == len(ens)


def test_reference_arm_under_torchrun_prints_one_line():
    """Two ranks of `bench.py --impl reference`: rank 0 times the reference's CPU step and
    prints the line, rank 1 exits 0 without work."""
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--workload", "argon", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" not in d:
        assert d["n_gpus"] == 2 and d["value"] > 0 and d["cpu_baseline"]["kind"] == "reference"
