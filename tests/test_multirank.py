"""Multi-rank paths of bench.py on CPU: gloo process group, world size 2."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

import helpers as H

ROOT = H.ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _max_worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5 * rank], world, "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_max_worker, args=(world, port, out), nprocs=world, join=True)
        got = dict(out)
    assert got[0] == got[1] == [2.0, 10.0, 0.5]


def test_reference_arm_under_torchrun_prints_once():
    """`--impl reference` with two ranks: rank 0 alone times the CPU path and prints one
    JSON line; the other rank exits 0 without work."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--config", "plain", "--gaussians", "1500", "--steps", "2", "--warmup", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0


def _partition_worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import importlib
    batch = importlib.import_module("3dgs-isaac-sim-xpbd_b200").batch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        objs = batch.make_objects(count=9, seed=4, n_min=300, n_max=3000)
        mine = batch.partition(objs, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        out[rank] = (got, [batch.object_cost(objs[k][0]) for k in range(len(objs))])
    finally:
        dist.destroy_process_group()


def test_batched_partition_gloo():
    """Each rank derives the same object partition: disjoint, covering, load-balanced."""
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_partition_worker, args=(world, port, out), nprocs=world, join=True)
        got = dict(out)
    parts, cost = got[0]
    assert got[1][0] == parts
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(cost)))
    loads = [sum(cost[k] for k in p) for p in parts]
    assert max(loads) - min(loads) <= max(cost)


def test_render_reference_arm_prints_one_line():
    """`--impl reference --config render`: the CPU restatement times one small frame of
    the splatting workload and prints the contract's JSON line."""
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "render",
           "--gaussians", "3000", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "frames/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["d2h_bytes_per_step"] == 0


def _served_partition_worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sessions = H.pkg.serve.make_sessions(200.0, 2.0, seed=0, n_min=5000, n_max=500000, max_frames=120)
        mine = H.pkg.serve.partition_sessions(sessions, world)[rank]
        parts = [None] * world
        dist.all_gather_object(parts, mine)
        out[rank] = (len(sessions), parts)
    finally:
        dist.destroy_process_group()


def test_served_sessions_partition_over_ranks_gloo():
    """Served sessions split over two ranks (one arena each, nothing exchanged while
    serving): every session on exactly one rank, each rank's share in arrival order, the
    ranks' work within the largest session's of each other."""
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_served_partition_worker, args=(world, port, out), nprocs=world, join=True)
        got = dict(out)
    total, parts = got[0]
    assert got[1][1] == parts
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(total))
    assert all(p == sorted(p) for p in parts)
    sessions = H.pkg.serve.make_sessions(200.0, 2.0, seed=0, n_min=5000, n_max=500000, max_frames=120)
    work = [sum(sessions[k][1] * sessions[k][2] for k in p) for p in parts]
    assert abs(work[0] - work[1]) <= max(s[1] * s[2] for s in sessions)
