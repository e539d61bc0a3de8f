"""Replicas of the per-call solve on several GPUs of one node: one process per GPU (launched by torchrun), each with
its own CudaSolver and its own cells.

Cells never couple (the reference's call kernel has no cross-cell data, maxichem/kernels/call.cuh:33-176), so the
data path has no exchange at all: a rank solves its own contiguous rows of the global batch, or, in the weak-scaling
bench, its own batch of the same size on every rank. Ranks only agree on the time of a region (MAX over ranks) and
may add up their counts (SUM). Both are one small collective on the process group (NCCL on GPUs, gloo on CPU).
"""

from __future__ import annotations

import os
import socket
import subprocess
import sys
from typing import NamedTuple

import torch
import torch.distributed as dist


class Rank(NamedTuple):
    rank: int
    local: int
    world: int


def rank_from_env() -> Rank:
    """The torchrun environment of this process (a single process without it)."""
    return Rank(int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
                int(os.environ.get("WORLD_SIZE", "1")))  # fmt: skip


def rows(total: int, rank: int, world: int) -> range:
    """The contiguous rows of a global batch of `total` cells that `rank` of `world` solves (sizes differ by at most
    one; every row belongs to exactly one rank)."""
    if world < 1 or not 0 <= rank < world or total < 0:
        raise ValueError(f"rank {rank} of {world} ranks over {total} cells")
    return range(rank * total // world, (rank + 1) * total // world)


def seed(base: int, rank: int) -> int:
    """The input seed of rank's own batch in the weak-scaling bench: every rank solves different cells."""
    return base + rank


def _active() -> bool:
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def max_over_ranks(value: float, device: torch.device) -> float:
    """The largest value over ranks (the time of a region every rank ran), on the process group's device."""
    if not _active():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_counts(total: torch.Tensor) -> torch.Tensor:
    """The counts of all ranks added up (a copy; the solver's own total is left alone)."""
    out = total.to(torch.int64).clone()
    if _active():
        dist.all_reduce(out, op=dist.ReduceOp.SUM)
    return out


def throughput(cells_per_rank: int, world: int, seconds: float) -> float:
    """Whole-job cells/s: the cells of all ranks over the slowest rank's time."""
    return world * cells_per_rank / seconds


def free_port() -> int:
    """A free TCP port on 127.0.0.1 for a rendezvous."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return int(s.getsockname()[1])


def under_launcher() -> bool:
    """True in a rank that torchrun (torch.distributed.run) started."""
    return "RANK" in os.environ and "WORLD_SIZE" in os.environ


def torchrun_command(n: int, script: str, argv: list[str], port: int | None = None) -> list[str]:
    """The command that runs ``script argv`` as n ranks of one node under torch.distributed.run, with the rendezvous on
    127.0.0.1 (the host name may not resolve)."""
    if n < 1:
        raise ValueError(f"ranks: at least 1 expected, got {n}")
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", str(n),
            "--master-addr", "127.0.0.1", "--master-port", str(port or free_port()), script, *argv]  # fmt: skip


def relaunch(n: int, script: str, argv: list[str], timeout: float | None = None) -> int:
    """Run ``script argv`` as n ranks under torch.distributed.run and wait for them; return the launcher's exit code
    (non-zero when a rank failed). Each rank reads its rank and world size from the environment (rank_from_env)."""
    proc = subprocess.run(torchrun_command(n, script, argv), timeout=timeout)
    return proc.returncode
