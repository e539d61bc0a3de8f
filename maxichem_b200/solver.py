"""CudaSolver: the reference's per-call chemistry solver surface over the sm_100a C-ABI library.

Same constructor, call, results, counts, errors and lifetime as imalsky/maxichem ``CudaSolver``
(``maxichem/kincuda.py:72-373``, ``maxichem/_solver.py:42-234``), so a caller switches by changing the import. Inputs are
float64 CUDA tensors; a call runs on torch's current stream of the solver's device, launches the library's kernels
through ``mx_call`` and reads the counts back once (its one host synchronisation) to refuse bad cells.
"""

from __future__ import annotations

import ctypes
import math
import operator
from pathlib import Path
from typing import Any, NamedTuple

import numpy as np
import torch

from . import abi, tables
from .constants import ATOL, COUNTS, DEFAULT_MAX_STEPS, DEFAULT_RTOL, DRIFT, REC_STEPS, T_MAX, T_MIN, X_SUM_TOL
from .network import VulcanNetwork

__all__ = ["ATOL", "COUNTS", "DRIFT", "REC_STEPS", "T_MAX", "T_MIN", "X_SUM_TOL", "CallResult", "CudaSolver",
           "LaunchResult"]  # fmt: skip

_ERRLEN = 1024
INFO_FIELDS = ("warps", "rows_per_lane", "smem", "call_ctas_per_sm", "recover_ctas_per_sm", "sms", "ld",
               "grid_ctas_per_sm", "list_cells", "mixed_smem", "mixed_ctas_per_sm", "precision", "sweeps")
PRECISIONS = {"fp64": 0, "mixed": 1}
MIXED_TOL = 1.0  # MX_MIXED_TOL of include/maxichem_b200.h
MAX_SWEEPS = 4  # MX_MIXED_MAX_SWEEPS
# The default warps per cell is 2 when at least this many cells of the network fit one SM's shared memory: half again
# the 4-warp kernels' 4 cells per SM (41 species: 2 warps measured 11-19 % faster; 69 species, 4 cells a SM either
# way: 4 warps 16 % faster)
TWO_WARP_CELLS = 6


class CallResult(NamedTuple):
    """What a call returns per cell: x [B, S] mole fractions, h [B] the next starting step (s), done [B] bool (the call
    finished and its result passed the guard), steps [B] accepted steps (float64)."""

    x: torch.Tensor
    h: torch.Tensor
    done: torch.Tensor
    steps: torch.Tensor


class LaunchResult(NamedTuple):
    """CallResult's fields and the flag [B] int32: 0 passed the guard, 1 recomputed and passes, 2 still fails."""

    x: torch.Tensor
    h: torch.Tensor
    done: torch.Tensor
    steps: torch.Tensor
    flag: torch.Tensor


def _device_of(device: torch.device | str) -> torch.device:
    dev = torch.device(device)
    if dev.type != "cuda":
        raise ValueError(f"a CUDA device expected, got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


def check_tensor(name: str, a: torch.Tensor, shape: tuple[int, ...], device: torch.device) -> None:
    """Refuse a tensor that is not float64 of this shape on this device (_solver.py:34-39)."""
    if a.dtype != torch.float64 or a.device != device or tuple(a.shape) != shape:
        raise ValueError(
            f"{name}: float64 {list(shape)} on {device} expected, got {a.dtype} {list(a.shape)} on {a.device}"
        )


def check_inputs(dev: torch.device, ns: int, x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor,
                 h: torch.Tensor, rtol: float, atol: float, max_steps: int) -> int:
    """Refuse inputs of the wrong form or range before any launch; return B (_solver.py:42-70)."""
    if x.dim() != 2 or x.shape[1] != ns:
        raise ValueError(f"x: [B, {ns}] expected, got {list(x.shape)}")
    B = x.shape[0]
    check_tensor("x", x, (B, ns), dev)
    for name, a in (("T", T), ("P", P), ("dt", dt), ("h", h)):
        check_tensor(name, a, (B,), dev)
    if not (math.isfinite(rtol) and rtol > 0.0 and math.isfinite(atol) and atol > 0.0):
        raise ValueError(f"rtol and atol finite and positive expected, got {rtol}, {atol}")
    try:
        ms = operator.index(max_steps)
    except TypeError:
        raise ValueError(f"max_steps: an integer expected, got {max_steps!r}") from None
    most = int(np.iinfo(np.int32).max)
    if ms < 1 or REC_STEPS * ms > most:
        raise ValueError(f"max_steps from 1 to {most // REC_STEPS} expected, got {ms}")
    return int(B)


def check_photolysis(J: torch.Tensor | None, cells: int, branches: int, device: torch.device) -> torch.Tensor | None:
    """The call's J, None without photolysis (_solver.py:73-92)."""
    if not branches:
        if J is None:
            return None
        if J.dim() != 2 or J.shape[1] != 0:
            raise ValueError(
                f"J: none or an empty [{cells}, 0] one expected, since this solver has no photolysis; got "
                f"{list(J.shape)}"
            )
        check_tensor("J", J, (cells, 0), device)
        return None
    if J is None:
        raise ValueError(f"J [B, {branches}] is required with photolysis: pass zeros for dark cells")
    check_tensor("J", J, (cells, branches), device)
    return J.contiguous()


def _first(mask: torch.Tensor) -> int:
    return int(torch.nonzero(mask)[0, 0])


def _ptr(a: torch.Tensor | None) -> int | None:
    return None if a is None else a.data_ptr()


class CudaSolver:
    """Batched chemistry solver on one B200: ``solver(x, T, P, dt, h, J=J)`` advances each cell by dt.

    Parameters are the reference's: ``net`` (its species order is x's), ``device`` (a CUDA device), and keyword-only
    ``drift`` (the guard's element-drift allowance, DRIFT if None) and ``photo`` (the network's photolysis branches
    enter the call, which then takes J). Calls run one at a time on torch's current stream: the scratch, the queues
    and the counts are shared.

    Beyond the reference: ``precision`` "fp64" (the reference's arithmetic) or "mixed" (each try's linear algebra in
    row-scaled FP32, every stage solve refined ``sweeps`` times against an FP64 residual; a try whose last correction
    exceeds ``tol`` times the error-control scale has its cell redone in FP64 in the same call, counted in
    ``escalated``). Results, counts, flags and refusals have the same meaning in both. ``warps``: warps per cell of
    the call, 2 or 4, the same results bit for bit; by default 2 for a network of which at least TWO_WARP_CELLS cells
    fit one SM's shared memory (the 2-warp kernels then hold 6-8 cells per SM, registers allowing 8, against the
    4-warp kernels' 4), else 4, as the reference chooses its warps per cell by the network's size
    (maxichem/_constants.py:67-72) by its own rule. The derivatives need 4.
    """

    def __init__(self, net: VulcanNetwork, device: torch.device | str, *, drift: float | None = None,
                 photo: bool = False, precision: str = "fp64", sweeps: int = 1, tol: float = MIXED_TOL,
                 warps: int | None = None) -> None:
        self._handle: ctypes.c_void_p | None = None
        if precision not in PRECISIONS:
            raise ValueError(f"precision: one of {sorted(PRECISIONS)} expected, got {precision!r}")
        if not (isinstance(sweeps, int) and 1 <= sweeps <= MAX_SWEEPS):
            raise ValueError(f"sweeps: an integer from 1 to {MAX_SWEEPS} expected, got {sweeps!r}")
        if not (math.isfinite(tol) and tol > 0.0):
            raise ValueError(f"tol: a finite value above 0 expected, got {tol}")
        if photo and (not net.photo or net.photo_missing):
            raise ValueError(
                "photo=True needs a network with photolysis branches whose species are all in its species "
                f"list (branches {len(net.photo)}, missing species {net.photo_missing})"
            )
        value = float(DRIFT if drift is None else drift)
        if not (math.isfinite(value) and value >= 0.0):
            raise ValueError(f"drift: a finite allowance of at least 0 expected, got {drift}")
        self.drift = value
        self.net = net
        self.dev = _device_of(device)
        self._lib = abi.library()
        tab = None
        if warps is None:
            self.warps, tab = self._default_warps(net, photo)
        else:
            self.warps = int(warps)
        if not self._lib.mx_warps_supported(self.warps):
            raise ValueError(f"warps: 2 or 4 warps per cell expected, got {warps}")
        self.tab = tab if tab is not None else tables.build(net, photo, warps=self.warps)
        self.ns, self.nr, self.nj = self.tab.ns, self.tab.nr, self.tab.nj
        self.count = torch.zeros(abi.COUNT_SLOTS, dtype=torch.int32, device=self.dev)
        self.total = torch.zeros(abi.COUNT_SLOTS, dtype=torch.int64, device=self.dev)
        self.flag: torch.Tensor | None = None
        struct = abi.NetworkStruct(self.tab)
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(_ERRLEN)
        rc = self._lib.mx_create(struct.ref(), self.drift, self.dev.index, ctypes.byref(handle), err, _ERRLEN)
        if rc:
            raise (ValueError if rc in (1, 3) else RuntimeError)(err.value.decode())
        self._handle = handle
        self.precision, self.sweeps, self.tol = precision, int(sweeps), float(tol)
        if self._lib.mx_set_precision(self._handle, PRECISIONS[precision], self.sweeps, self.tol):
            raise ValueError(f"precision {precision!r}, sweeps {sweeps}, tol {tol}: refused by the library")
        self.escalated = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self._lib.mx_set_escalation_counter(self._handle, self.escalated.data_ptr())
        self.info: dict[str, Any] = self.layout()
        self.info.update(ns=self.ns, nr=self.nr, nj=self.nj, drift=self.drift, flops=dict(self.tab.flops))

    def _default_warps(self, net: VulcanNetwork, photo: bool) -> tuple[int, tables.Tables | None]:
        """2 when at least TWO_WARP_CELLS cells of the network fit one SM's shared memory, else the library's default
        (4); the tables already built for the choice, or None."""
        four = int(self._lib.mx_warps_per_cell())
        tab = tables.build(net, photo, warps=four)
        cells = int(self._lib.mx_cells_per_sm(abi.NetworkStruct(tab).ref(), self.dev.index))
        if cells >= TWO_WARP_CELLS and self._lib.mx_warps_supported(2):
            return 2, None
        return four, tab

    # lifetime (_solver.py:142-167)
    def close(self) -> None:
        """Release the device tables and scratch; the solver cannot be called afterwards, its counts stay readable."""
        if self._handle is not None:
            torch.cuda.synchronize(self.dev)
            self._lib.mx_destroy(self._handle)
            self._handle = None

    def __enter__(self) -> CudaSolver:
        return self

    def __exit__(self, *exception: object) -> None:
        self.close()

    def __del__(self) -> None:
        try:
            if getattr(self, "_handle", None) is not None:
                self._lib.mx_destroy(self._handle)
                self._handle = None
        except Exception:
            pass

    def _require_open(self) -> None:
        if self._handle is None:
            raise RuntimeError("this solver was closed; build a new one")

    def launch(self, x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor, h: torch.Tensor, *,
               rtol: float = DEFAULT_RTOL, atol: float = ATOL, max_steps: int = DEFAULT_MAX_STEPS,
               J: torch.Tensor | None = None) -> LaunchResult:
        """Run the call, the guard and the recovery; read the counts; refuse bad input and T out of range.

        Returns x, h, done, accepted steps and the per-cell flag (also ``self.flag``). The counts go to ``self.count``
        and are added to ``self.total``. Raises ValueError (after the kernels, counts kept) if a cell was refused.
        """
        self.flag = None
        self._require_open()
        B = check_inputs(self.dev, self.ns, x, T, P, dt, h, rtol, atol, max_steps)
        x, T, P, dt, h = (a.contiguous() for a in (x, T, P, dt, h))
        jx = check_photolysis(J, B, self.nj, self.dev)
        out = self.launch_raw(x, T, P, dt, h, rtol=rtol, atol=atol, max_steps=max_steps, J=jx)
        self._refuse(x, T, P, dt, jx, out["status"])
        self.flag = out["flag"]
        return LaunchResult(out["x"], out["h"], out["done"].bool(), out["steps"], out["flag"])

    def launch_raw(self, x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor, h: torch.Tensor, *,
                   rtol: float, atol: float, max_steps: int, J: torch.Tensor | None,
                   out: dict[str, torch.Tensor] | None = None) -> dict[str, torch.Tensor]:
        """The launches alone, on checked contiguous inputs, with no host synchronisation (CUDA-graph capturable
        when ``out`` supplies preallocated outputs)."""
        self._require_open()
        B = x.shape[0]
        if out is None:
            out = {
                "x": torch.empty_like(x), "h": torch.empty_like(h), "steps": torch.empty_like(h),
                **{k: torch.empty(B, dtype=torch.int32, device=self.dev) for k in ("done", "flag", "status")},
            }  # fmt: skip
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        err = ctypes.create_string_buffer(_ERRLEN)
        rc = self._lib.mx_call(
            self._handle, _ptr(x), _ptr(T), _ptr(P), _ptr(dt), _ptr(h), _ptr(J), B, float(rtol), float(atol),
            int(max_steps), _ptr(out["x"]), _ptr(out["h"]), _ptr(out["done"]), _ptr(out["steps"]), _ptr(out["flag"]),
            _ptr(out["status"]), _ptr(self.count), _ptr(self.total), stream, err, _ERRLEN,
        )  # fmt: skip
        if rc:
            raise (ValueError if rc == 1 else RuntimeError)(err.value.decode())
        return out

    def __call__(self, x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor, h: torch.Tensor, *,
                 rtol: float = DEFAULT_RTOL, atol: float = ATOL, max_steps: int = DEFAULT_MAX_STEPS,
                 J: torch.Tensor | None = None) -> CallResult:
        """Advance each cell by dt: ``launch`` without the flag in its result (``self.flag`` keeps it)."""
        r = self.launch(x, T, P, dt, h, rtol=rtol, atol=atol, max_steps=max_steps, J=J)
        return CallResult(r.x, r.h, r.done, r.steps)

    def export(self, folder: str | Path) -> Path:
        """Write what a caller without Python needs to build this solver (include/maxichem_b200.hpp and
        mx_create_from_export load it): meta.txt and tables/<name>.bin, the network's tables, names and the drift
        allowance (kincuda.py:363-373). The kernels are the library's own, so no kernel code is written."""
        self._require_open()
        from .export import write_export

        return write_export(self.tab, folder, drift=self.drift, species=list(self.net.species),
                            elements=list(self.net.elements))  # fmt: skip

    def set_grid(self, ctas_per_sm: int) -> None:
        """The call kernel's grid for later calls: 1 .. info["call_ctas_per_sm"] persistent CTAs per SM over the cell
        queue, 0 one CTA per cell, -1 the default (the occupancy limit). Results do not depend on it."""
        self._require_open()
        if self._lib.mx_set_grid(self._handle, int(ctas_per_sm)):
            most = max(self.info["call_ctas_per_sm"], self.info["mixed_ctas_per_sm"])
            raise ValueError(f"ctas_per_sm from -1 to {most} expected, got {ctas_per_sm}")
        values = (ctypes.c_int32 * len(INFO_FIELDS))()
        self._lib.mx_info(self._handle, values, len(INFO_FIELDS))
        self.info["grid_ctas_per_sm"] = int(values[INFO_FIELDS.index("grid_ctas_per_sm")])

    def layout(self) -> dict[str, int]:
        """The library's current launch layout (mx_info), read afresh: ``info``'s fields as they are now."""
        self._require_open()
        values = (ctypes.c_int32 * len(INFO_FIELDS))()
        self._lib.mx_info(self._handle, values, len(INFO_FIELDS))
        return dict(zip(INFO_FIELDS, list(values)))

    def call_host(self, x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor, h: torch.Tensor, *,
                  rtol: float = DEFAULT_RTOL, atol: float = ATOL, max_steps: int = DEFAULT_MAX_STEPS,
                  J: torch.Tensor | None = None, chunks: int = 4,
                  out: dict[str, torch.Tensor] | None = None) -> CallResult:
        """The call on host (CPU) tensors, with the copies overlapped: the batch goes in `chunks` pieces, each copied
        in, solved and copied out on three streams, so piece k + 1 is copied in and piece k - 1 copied out while
        piece k is solved (4 pieces measured best for 1M cells: more pieces add more kernel tails). Cells are independent, so the results, counts, flag and refusal are those of one call on
        the whole batch. Pinned inputs overlap; `out` may hold pinned host outputs x, h, steps (float64), done (bool),
        flag and status (int32) to write into (allocated, pinned, when None)."""
        self._require_open()
        self.flag = None
        cpu = torch.device("cpu")
        B = check_inputs(cpu, self.ns, x, T, P, dt, h, rtol, atol, max_steps)
        jx = check_photolysis(J, B, self.nj, cpu)
        if chunks < 1:
            raise ValueError(f"chunks: at least 1 expected, got {chunks}")
        if out is None:
            f = lambda *shape, dtype=torch.float64: torch.empty(*shape, dtype=dtype).pin_memory()
            out = {"x": f(B, self.ns), "h": f(B), "steps": f(B), "done": f(B, dtype=torch.bool),
                   "flag": f(B, dtype=torch.int32), "status": f(B, dtype=torch.int32)}  # fmt: skip
        ins = [a.contiguous() for a in (x, T, P, dt, h)] + ([jx] if jx is not None else [])
        dev_in = [torch.empty(a.shape, dtype=a.dtype, device=self.dev) for a in ins]
        dev_out = {
            "x": torch.empty(B, self.ns, dtype=torch.float64, device=self.dev),
            **{k: torch.empty(B, dtype=torch.float64, device=self.dev) for k in ("h", "steps")},
            **{k: torch.empty(B, dtype=torch.int32, device=self.dev) for k in ("done", "flag", "status")},
        }  # fmt: skip
        main = torch.cuda.current_stream(self.dev)
        s_in, s_run, s_out = (torch.cuda.Stream(self.dev) for _ in range(3))
        for s in (s_in, s_run, s_out):
            s.wait_stream(main)
        before = self.total.clone()
        step = -(-B // chunks) if B else 1
        for a in range(0, B, step):
            b = min(B, a + step)
            with torch.cuda.stream(s_in):
                for d, src in zip(dev_in, ins):
                    d[a:b].copy_(src[a:b], non_blocking=True)
            s_run.wait_stream(s_in)
            with torch.cuda.stream(s_run):
                sl = [d[a:b] for d in dev_in]
                self.launch_raw(*sl[:5], J=sl[5] if jx is not None else None, rtol=rtol, atol=atol,
                                max_steps=max_steps, out={k: v[a:b] for k, v in dev_out.items()})  # fmt: skip
            s_out.wait_stream(s_run)
            with torch.cuda.stream(s_out):
                for k, v in dev_out.items():
                    out[k][a:b].copy_(v[a:b], non_blocking=True)
        main.wait_stream(s_out)
        main.synchronize()
        self.count.copy_((self.total - before).to(torch.int32))  # the counts of the whole call
        self._refuse(*ins[:4], ins[5] if jx is not None else None, out["status"])
        self.flag = out["flag"]
        return CallResult(out["x"], out["h"], out["done"], out["steps"])

    @property
    def fallback(self) -> dict[str, int]:
        """The last call's counts (one small copy from the device)."""
        return dict(zip(COUNTS, self.count[1:-1].tolist(), strict=True))

    def _refuse(self, x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor, J: torch.Tensor | None,
                status: torch.Tensor) -> None:
        """Raise ValueError if the call refused a cell, naming the first of each kind (_solver.py:183-224)."""
        n = self.fallback
        if not (n["bad_input"] or n["cold"] or n["hot"]):
            return
        refused = status != 0
        cold, hot = refused & (T < T_MIN), refused & (T > T_MAX)
        problems = []
        for kind, cells, side in (("cold", cold, f"below {T_MIN:g} K"), ("hot", hot, f"above {T_MAX:g} K")):
            if n[kind]:
                i = _first(cells)
                problems.append(
                    f"{n[kind]} cells {side}, outside the solver's range {T_MIN:g}-{T_MAX:g} K (first: cell {i}, "
                    f"T = {float(T[i]):g} K); leave them out of the call"
                )
        if n["bad_input"]:
            i = _first(refused & torch.logical_not(cold | hot))
            where = (
                f"cell {i}: sum(x) - 1 = {float(x[i].sum() - 1.0):g} (added in another order than the kernel's, so "
                f"it can differ in the last bits), min(x) = {float(x[i].min()):g}, "
                f"T = {float(T[i]):g} K, P = {float(P[i]):g} dyn cm^-2, dt = {float(dt[i]):g} s"
                + ("" if J is None else f", min(J) = {float(J[i].min()):g} s^-1")
            )
            problems.append(
                f"{n['bad_input']} cells of bad input: x negative or non-finite, |sum(x) - 1| above {X_SUM_TOL:g} "
                "or no x above 0; T non-finite, P non-finite, not above 0 or so large that P / (k_B T) overflows, dt "
                f"negative or non-finite, or J negative or non-finite (first: {where}); pass x normalized to sum 1 in "
                "float64, clamped at 0"
            )
        raise ValueError("the call refused cells: " + "; ".join(problems))

    def check(self) -> dict[str, int]:
        """The counts since construction (one small copy); raise if any cell was outside [T_MIN, T_MAX]."""
        n = dict(zip(COUNTS, self.total[1:-1].tolist(), strict=True))
        if n["cold"] or n["hot"]:
            raise ValueError(
                f"{n['cold']} cells below {T_MIN:g} K and {n['hot']} above {T_MAX:g} K: outside the chemistry "
                "solver's range"
            )
        return n

    def guard(self, x0: torch.Tensor, xout: torch.Tensor, done: torch.Tensor, steps: torch.Tensor,
              status: torch.Tensor, atol: float = ATOL) -> torch.Tensor:
        """The guard alone on given states (the reference's guard kernel launched by hand): corrects xout in place,
        returns the per-cell flag (0/1) and leaves the counts in ``self.count``."""
        self._require_open()
        B = x0.shape[0]
        flag = torch.empty(B, dtype=torch.int32, device=self.dev)
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        err = ctypes.create_string_buffer(_ERRLEN)
        rc = self._lib.mx_guard(self._handle, _ptr(x0), _ptr(xout), _ptr(done), _ptr(steps), _ptr(status), B,
                                float(atol), _ptr(flag), _ptr(self.count), stream, err, _ERRLEN)
        if rc:
            raise RuntimeError(err.value.decode())
        return flag
