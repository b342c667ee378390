"""Host logic of the multi-GPU bench path on CPU (gloo, two ranks).

``bench.py --gpus N`` runs N independent replicas (the step does not shard
at the workload size); each rank times its own replica on the device and the
job reports the slowest rank's time and the sum of the replicas' steps/s.
Here two gloo ranks check the max-over-ranks reduction and the replica
accounting; the reference arm exits without work on ranks other than 0.
"""
import importlib.util
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    b = _bench()
    ms = b.dist_max(2.0 + 3.0 * rank)  # rank 1 is the slower replica
    q.put((rank, ms, b.replica_value(world, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, ms, value in got:
        assert ms == 5.0                      # both ranks see the slowest time
        assert value == pytest.approx(400.0)  # 2 replicas x 1000 / 5 ms


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_ensemble_members_match_the_parity_tests():
    """bench.py's 48-run ensemble draws the same grids, Re, Ro and seeds as
    the ensemble parity tests (run m: default_rng(1000 + m))."""
    b = _bench()
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import numpy as np
    mem = b.ensemble_members()
    assert len(mem) == 48
    for m in (0, 12, 24, 36, 47):
        c = mem[m]
        mx, my, mz = b.ENSEMBLE_SIZES[m // 12]
        r = np.random.default_rng(1000 + m)
        assert (c["mx"], c["my"], c["mz"], c["seed"], c["dt"]) == (mx, my, mz, 1000 + m, 0.002)
        assert c["Re"] == r.uniform(500.0, 3000.0) and c["Ro"] == r.uniform(0.0, 0.3)


def test_other_workloads_report_failures(monkeypatch):
    """A failing extra workload leaves an error entry instead of losing the
    headline line."""
    b = _bench()

    def boom(args):
        raise RuntimeError("no device")
    monkeypatch.setattr(b, "run_solve", boom)
    monkeypatch.setattr(b, "run_ensemble", boom)
    import argparse
    res = b.other_workloads(argparse.Namespace(steps=5, warmup=3, solve_grid="576,576,768"))
    assert res == {"solve_384x193x384": {"error": "RuntimeError: no device"},
                   "ensemble_48_runs": {"error": "RuntimeError: no device"}}


def test_gpus_n_launches_n_ranks():
    """``bench.py --gpus 2`` started without torchrun starts two ranks itself
    (gloo here, no device work) and reports n_gpus = 2."""
    import json
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--check-launch"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["n_gpus"] == 2 and line["ranks_joined"] == 2


def test_gpus_n_must_match_world_size():
    env = dict(os.environ, RANK="0", WORLD_SIZE="2", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "3", "--check-launch"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "WORLD_SIZE=2" in r.stderr
