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
