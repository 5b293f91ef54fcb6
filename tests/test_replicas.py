"""Multi-rank host logic of the replicas-only multi-GPU mode, on CPU with gloo (world size 2).

Covers what bench.py and a multi-GPU job rely on: max / sum over ranks, per-rank workload seeds and shards,
a rank that fails before a collective (the other rank gets an error from the short process-group timeout
instead of waiting for good), and the reference arm of bench.py under torchrun (rank 0 alone prints one JSON
line, the other rank exits 0 without work).
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})


def _reductions(rank, world, port, q):
    sys.path.insert(0, ROOT)
    _env(rank, world, port)
    from distance_transform_benchmarks_b200.replicas import ReplicaGroup
    from distance_transform_benchmarks_b200 import workloads as wl
    g = ReplicaGroup().init("gloo", timeout_s=30)
    try:
        step_ms = [12.5, 20.25][rank]
        px = [1000, 234][rank]
        g.barrier()
        specs = wl.config3_specs(seed=g.seed(3), n=4)
        q.put((rank, g.max(step_ms), g.sum(px), g.shard(range(10)), [s[1:3] for s in specs]))
    finally:
        g.close()


def _one_rank_fails(rank, world, port, q):
    sys.path.insert(0, ROOT)
    _env(rank, world, port)
    from distance_transform_benchmarks_b200.replicas import ReplicaGroup
    g = ReplicaGroup().init("gloo", timeout_s=5)
    if rank == 1:
        q.put((rank, "left"))
        q.close()
        q.join_thread()  # the message is out before the process ends
        os._exit(0)  # leaves between steps: no collective of its own in flight
    try:
        g.max(1.0)
        q.put((rank, "no error"))
    except Exception as e:  # the peer is gone: gloo reports it (connection closed or timeout)
        q.put((rank, "error: %s" % type(e).__name__))


def _spawn(fn, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=fn, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda t: t[0]), [p.exitcode for p in procs]


def test_max_sum_seed_and_shard_over_two_ranks():
    out, codes = _spawn(_reductions)
    assert codes == [0, 0]
    (r0, mx0, sm0, sh0, sp0), (r1, mx1, sm1, sh1, sp1) = out
    assert mx0 == mx1 == 20.25
    assert sm0 == sm1 == 1234
    assert sh0 == [0, 2, 4, 6, 8] and sh1 == [1, 3, 5, 7, 9]
    assert sp0 != sp1  # each rank generates its own images (weak scaling)


def test_a_rank_that_leaves_makes_the_other_fail_not_hang():
    out, _ = _spawn(_one_rank_fails)
    assert out[1] == (1, "left")
    assert out[0][1].startswith("error"), out


def test_bench_reference_arm_under_torchrun_two_ranks(tmp_path):
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "0", "--images", "16", "--ref-mpx", "0.5"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
