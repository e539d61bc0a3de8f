"""The multi-GPU host logic on CPU: two gloo ranks, each solving its own rows with the oracle, agree on the MAX time
and the SUM of counts, and their rows together give the single-process result bit for bit (cells never couple)."""

import json
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

from maxichem_b200 import replicas

ROOT = Path(__file__).resolve().parent.parent


def test_rows_cover_the_batch_once():
    for total in (0, 1, 7, 64, 1000):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in replicas.rows(total, r, world)]
            assert got == list(range(total))
            sizes = [len(replicas.rows(total, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.rows(10, 2, 2)


def test_single_process_needs_no_group():
    import torch

    assert replicas.max_over_ranks(3.5, torch.device("cpu")) == 3.5
    t = torch.arange(12)
    assert replicas.sum_counts(t).tolist() == t.tolist()
    assert replicas.throughput(1000, 4, 2.0) == 2000.0
    assert replicas.seed(1000, 3) == 1003


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out: str) -> None:
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import oracle
    from maxichem_b200 import synthetic, tables

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), OMP_NUM_THREADS="1")  # fmt: skip
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        net = synthetic.network("cho41")
        w = synthetic.workload(net, "column", 16, seed=5)
        mine = replicas.rows(16, rank, world)
        o = oracle.Oracle(tables.build(net, True))
        r = o.call(w.x[mine.start : mine.stop], w.T[mine.start : mine.stop], w.P[mine.start : mine.stop],
                   w.dt[mine.start : mine.stop], w.h[mine.start : mine.stop], J=w.J[mine.start : mine.stop],
                   threads=1)  # fmt: skip
        fake_ms = 10.0 + rank  # each rank's own time; the job's time is the slowest rank's
        ms = replicas.max_over_ranks(fake_ms, torch.device("cpu"))
        counts = replicas.sum_counts(torch.as_tensor(r["count"].astype(np.int64)))
        gathered = [None] * world
        dist.all_gather_object(gathered, {"x": r["x"].tolist(), "count": r["count"].tolist()})
        if rank == 0:
            Path(out).write_text(json.dumps({"ms": ms, "counts": counts.tolist(), "parts": gathered}))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_time_counts_and_results(tmp_path, networks):
    import oracle
    from maxichem_b200 import synthetic, tables

    out = tmp_path / "rank0.json"
    mp.start_processes(_rank, args=(2, _free_port(), str(out)), nprocs=2, join=True, start_method="spawn")
    got = json.loads(out.read_text())
    assert got["ms"] == 11.0
    net = networks("cho41")
    w = synthetic.workload(net, "column", 16, seed=5)
    whole = oracle.Oracle(tables.build(net, True)).call(w.x, w.T, w.P, w.dt, w.h, J=w.J, threads=1)
    parts = np.concatenate([np.asarray(p["x"]) for p in got["parts"]])
    assert np.array_equal(parts, whole["x"])
    per_rank = np.sum([p["count"] for p in got["parts"]], axis=0)
    assert got["counts"] == per_rank.tolist()
    assert got["counts"][1:-1] == whole["count"][1:-1].tolist()


RANK_SCRIPT = """
import datetime, json, sys
import torch
import torch.distributed as dist
sys.path.insert(0, {root!r})
from maxichem_b200 import replicas
rank, local, world = replicas.rank_from_env()
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
ms = replicas.max_over_ranks(10.0 + rank, torch.device("cpu"))
counts = replicas.sum_counts(torch.full((12,), rank + 1, dtype=torch.int64))
if rank == 0:
    open(sys.argv[1], "w").write(json.dumps({{"world": world, "ms": ms, "counts": counts.tolist(),
                                              "value": replicas.throughput(1000, world, ms * 1e-3)}}))
dist.destroy_process_group()
"""


def test_the_launcher_starts_the_ranks_and_they_take_the_slowest_time(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT.format(root=str(ROOT)))
    out = tmp_path / "out.json"
    cmd = replicas.torchrun_command(2, str(script), [str(out)], port=1234)
    assert cmd[1:9] == ["-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2", "--master-addr",
                        "127.0.0.1"]  # fmt: skip
    assert replicas.relaunch(2, str(script), [str(out)], timeout=240) == 0
    got = json.loads(out.read_text())
    assert got["world"] == 2 and got["ms"] == 11.0 and got["counts"] == [3] * 12
    assert got["value"] == 2 * 1000 / 11e-3


def test_bench_refuses_more_gpus_than_are_visible():
    import subprocess

    import torch

    if torch.cuda.is_available():
        pytest.skip("checks the refusal on a machine without enough GPUs")
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2"], capture_output=True, text=True,
                       timeout=300, env=env)  # fmt: skip
    assert r.returncode != 0
    assert "bench.py --gpus 2: only 0 CUDA devices are visible" in r.stderr
