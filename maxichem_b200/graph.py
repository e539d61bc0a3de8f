"""A GCM call loop captured in one CUDA graph.

A GCM advances the same cells call after call: call k + 1 starts from call k's x and h, with the column's T, P, dt
and J of that step. ``CallLoop`` captures `calls` such calls (the call, recovery and count kernels of each, with
their count resets) in one CUDA graph, so a replay launches the whole loop with one host call and no host
synchronisation in between; the refusal check the Python call makes after every call is made once per replay, on the
counts the loop added to ``solver.total`` (``run(check=True)``, one small read-back after the replay). Outputs
alternate between two sets of buffers.
"""

from __future__ import annotations

import torch

from .constants import COUNTS
from .solver import CudaSolver, check_inputs, check_photolysis


class CallLoop:
    """`calls` chained calls of `solver` on fixed forcing (T, P, dt, J), captured once, replayed by ``run``.

    x and h are copied into the loop's input buffers (``x_in``, ``h_in``); write new starting states there between
    runs, or call ``carry`` to start the next run from the last call's result.
    """

    def __init__(self, solver: CudaSolver, x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor,
                 h: torch.Tensor, *, J: torch.Tensor | None = None, calls: int = 100, rtol: float = 1e-3,
                 atol: float = 1e-25, max_steps: int = 4000) -> None:
        if calls < 1:
            raise ValueError(f"calls: at least 1 expected, got {calls}")
        B = check_inputs(solver.dev, solver.ns, x, T, P, dt, h, rtol, atol, max_steps)
        jx = check_photolysis(J, B, solver.nj, solver.dev)
        self.solver, self.calls, self.cells = solver, calls, B
        self.x_in, self.h_in = x.contiguous().clone(), h.contiguous().clone()
        self.T, self.P, self.dt = (a.contiguous().clone() for a in (T, P, dt))
        self.J = None if jx is None else jx.clone()
        self.kw = dict(rtol=rtol, atol=atol, max_steps=max_steps)
        self.outs = [self._outputs(), self._outputs()]
        # one eager call first: loads the kernels and sizes the solver's recompute list outside the capture
        saved = solver.total.clone()
        solver.launch_raw(self.x_in, self.T, self.P, self.dt, self.h_in, J=self.J, out=self.outs[0], **self.kw)
        torch.cuda.synchronize(solver.dev)
        solver.total.copy_(saved)
        self.graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(solver.dev)
        side.wait_stream(torch.cuda.current_stream(solver.dev))
        with torch.cuda.stream(side), torch.cuda.graph(self.graph, stream=side):
            x_k, h_k = self.x_in, self.h_in
            for k in range(calls):
                out = self.outs[k % 2]
                solver.launch_raw(x_k, self.T, self.P, self.dt, h_k, J=self.J, out=out, **self.kw)
                x_k, h_k = out["x"], out["h"]
        torch.cuda.current_stream(solver.dev).wait_stream(side)
        self.last = self.outs[(calls - 1) % 2]

    def _outputs(self) -> dict[str, torch.Tensor]:
        dev, B, ns = self.solver.dev, self.cells, self.solver.ns
        f = torch.empty(B, dtype=torch.float64, device=dev)
        return {"x": torch.empty(B, ns, dtype=torch.float64, device=dev), "h": f, "steps": torch.empty_like(f),
                **{k: torch.empty(B, dtype=torch.int32, device=dev) for k in ("done", "flag", "status")}}  # fmt: skip

    def run(self, check: bool = True) -> dict[str, torch.Tensor]:
        """Replay the loop on torch's current stream; return the last call's outputs (buffers of the loop).

        With ``check`` the counts the replay added to ``solver.total`` are read back once (the loop's one host
        synchronisation) and ValueError is raised if any call of the loop refused a cell (bad input, or T outside
        the solver's range), as the Python call does after each call. ``check=False`` leaves the replay
        asynchronous (for timing); ``refused`` then reads the counts later."""
        before = self.solver.total.clone() if check else None
        self.graph.replay()
        if check:
            refused = self.refused(before)
            if any(refused.values()):
                raise ValueError(
                    "the call loop refused cells: "
                    + ", ".join(f"{n} {kind}" for kind, n in refused.items() if n)
                    + f" over its {self.calls} calls (cell-calls); check the loop's inputs with a plain call"
                )
        return self.last

    def refused(self, before: torch.Tensor) -> dict[str, int]:
        """Refused cell-calls (bad_input, cold, hot) added to ``solver.total`` since it held ``before``."""
        added = (self.solver.total - before).tolist()
        return {kind: int(added[1 + COUNTS.index(kind)]) for kind in ("bad_input", "cold", "hot")}

    def carry(self) -> None:
        """Make the last call's x and h the next run's starting state."""
        self.x_in.copy_(self.last["x"])
        self.h_in.copy_(self.last["h"])

    def close(self) -> None:
        """Release the graph (before the solver is closed)."""
        self.graph.reset()
