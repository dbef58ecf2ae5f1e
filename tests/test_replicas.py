"""The N > 1 path of bench.py on the CPU: two `gloo` ranks run the replica
logic (springback-precomp_b200/replicas.py) as torchrun would - each its own
seed, the barrier, the slowest rank's time taken by every rank, the
whole-job rate - and the reference arm leaves ranks above 0 without work."""
from __future__ import annotations

import importlib
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    rep = importlib.import_module("springback-precomp_b200.replicas")
    r, w, local = rep.rank_env()
    assert (r, w, local) == (rank, world, rank)
    assert rep.init(w, "gloo", timeout_s=60.0)
    rep.barrier(w)
    ms = 10.0 * (r + 1)  # rank 1 is the slow one
    slowest = rep.max_over_ranks(ms, w)
    rate = rep.job_rate(1000, w, slowest / 1e3)
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump({"seed": rep.replica_seed(7, r), "slowest": slowest, "rate": rate}, f)
    rep.finish(w)


def test_two_gloo_ranks_agree_on_the_slowest_time(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert [g["seed"] for g in got] == [7, 8]  # independent meshes
    assert all(g["slowest"] == 20.0 for g in got)
    assert all(g["rate"] == pytest.approx(2 * 1000 / 0.020) for g in got)


def test_reference_arm_leaves_other_ranks_idle():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
