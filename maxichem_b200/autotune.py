"""The autotuner: picks the cell-to-warp mapping and the call kernel's grid for a network and a batch by timing them.

The reference sizes its launch by recompiling its kernels with growing cells per block and keeping the fastest that
does not spill (``maxichem/kincuda.py:184-218``), and takes 2 or 4 warps per cell by the network's size
(``maxichem/_constants.py:70-72``). Here the kernels are compiled once, for 2 and for 4 warps per cell; what is left
to choose is the mapping (2 warps: half the registers per cell, so twice the cells per SM when registers rather than
shared memory bound the occupancy, as for small networks; 4 warps: more threads per cell for its LU and sums) and
the grid: 1 .. k persistent CTAs per SM over the cell queue (k the occupancy limit), or one CTA per cell. A batch with
a wide spread of step counts favours the queue, a uniform batch is indifferent. The tuner times calls of each choice
on the caller's own inputs and keeps the fastest; results do not depend on the choice (the same sums in the same
orders), and the solver's counts are left as they were.
"""

from __future__ import annotations

from typing import Any

import torch

from .solver import CudaSolver, check_inputs, check_photolysis

_CACHE: dict[tuple[Any, ...], int] = {}


def _key(solver: CudaSolver, cells: int) -> tuple[Any, ...]:
    tab = solver.tab
    return (tab.ns, tab.nr, tab.nj, hash(tab.perm.tobytes()), hash(tab.rc.tobytes()), max(cells, 1).bit_length())


def cached(solver: CudaSolver, cells: int) -> int | None:
    """The grid an earlier tuning chose for this network and a batch of about this size (a power of two), if any."""
    return _CACHE.get(_key(solver, cells))


def tune_grid(solver: CudaSolver, x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor,
              h: torch.Tensor, *, J: torch.Tensor | None = None, rtol: float = 1e-3, atol: float = 1e-25,
              max_steps: int = 4000, choices: list[int] | None = None, repeats: int = 1) -> dict[str, Any]:
    """Time `repeats` calls per grid choice (after one untimed call) and set the fastest on the solver.

    choices: CTAs per SM, 0 for one CTA per cell; default 0 and every count up to the occupancy limit. Returns
    {"best": choice, "ms": {choice: milliseconds per call}}.
    """
    B = check_inputs(solver.dev, solver.ns, x, T, P, dt, h, rtol, atol, max_steps)
    jx = check_photolysis(J, B, solver.nj, solver.dev)
    if choices is None:
        choices = [0, *range(1, solver.info["call_ctas_per_sm"] + 1)]
    saved = solver.total.clone()
    stream = torch.cuda.current_stream(solver.dev)
    out = None
    ms: dict[int, float] = {}
    try:
        for choice in choices:
            solver.set_grid(choice)
            kw = dict(rtol=rtol, atol=atol, max_steps=max_steps, J=jx)
            out = solver.launch_raw(x, T, P, dt, h, out=out, **kw)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(repeats):
                out = solver.launch_raw(x, T, P, dt, h, out=out, **kw)
            e1.record(stream)
            e1.synchronize()
            ms[choice] = e0.elapsed_time(e1) / repeats
    finally:
        solver.total.copy_(saved)
    best = min(ms, key=ms.__getitem__)
    solver.set_grid(best)
    _CACHE[_key(solver, B)] = best
    return {"best": best, "ms": ms}


def tune(net: Any, device: torch.device | str, x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor,
         h: torch.Tensor, *, J: torch.Tensor | None = None, photo: bool = True, warps: tuple[int, ...] = (2, 4),
         repeats: int = 1, **solver_kw: Any) -> tuple[CudaSolver, dict[str, Any]]:
    """The mapping and the grid together: a solver per warps-per-cell choice, its grid tuned (tune_grid), and the
    fastest kept. Returns the chosen solver (its grid set; the others closed) and {"warps", "grid", "ms": {(warps,
    grid): milliseconds per call}}."""
    best: tuple[float, CudaSolver | None, int, int] = (float("inf"), None, 0, 0)
    table: dict[tuple[int, int], float] = {}
    for w in warps:
        solver = CudaSolver(net, device, photo=photo, warps=w, **solver_kw)
        got = tune_grid(solver, x, T, P, dt, h, J=J, repeats=repeats)
        for grid, ms in got["ms"].items():
            table[(w, grid)] = ms
        ms = got["ms"][got["best"]]
        if ms < best[0]:
            if best[1] is not None:
                best[1].close()
            best = (ms, solver, w, got["best"])
        else:
            solver.close()
    _, solver, w, grid = best
    return solver, {"warps": w, "grid": grid, "ms": table}
