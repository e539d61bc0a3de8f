"""ADSolver: the tangent of one call, the reference's derivative surface over the sm_100a library.

Same constructor, ``jvp`` arguments, results, flags, counts and errors as imalsky/maxichem ``ADSolver``
(``maxichem/kincuda_ad.py:118-453``): each call returns the result of ``CudaSolver.launch`` bit for bit (with lm and
rc at their defaults) and its derivative along up to ``DMAX`` directions. The two contracts, frozen and adaptive, are
the reference's (its ``docs/method.md``, "Derivatives"). Calls run one at a time on torch's current stream.
"""

from __future__ import annotations

import ctypes
import operator
from typing import NamedTuple

import torch

from .constants import ARRHENIUS_COLUMNS, ATOL, CAP, DEFAULT_MAX_STEPS, DEFAULT_RTOL, DMAX, REC_STEPS
from .network import VulcanNetwork
from .solver import _ERRLEN, CudaSolver, _ptr, check_inputs, check_photolysis, check_tensor

__all__ = ["ADSolver", "Cotangents", "JvpResult", "VjpResult"]


class JvpResult(NamedTuple):
    """What ``ADSolver.jvp`` returns, per cell (``self.flag`` holds the per-cell flag): x [B, S], h [B], done [B]
    (bool), steps [B] as ``CudaSolver.launch``; dx [B, S] or [D, B, S] and dh [B] or [D, B], the tangents of x and h
    (float64), with the leading axis of D directions if the input tangents have it."""

    x: torch.Tensor
    h: torch.Tensor
    done: torch.Tensor
    steps: torch.Tensor
    dx: torch.Tensor
    dh: torch.Tensor


class Cotangents(NamedTuple):
    """The cotangents of ``ADSolver.vjp``'s inputs, float64, each per unit of its input (kincuda_ad.py:63-91): x [B, S];
    T, P, dt, h [B] (per K, per dyn cm^-2, per s, per s); lm [B, R]; rc [R, 9], the rate table's Arrhenius columns,
    a sum over the cells; J [B, branches], None without photolysis."""

    x: torch.Tensor
    T: torch.Tensor
    P: torch.Tensor
    dt: torch.Tensor
    h: torch.Tensor
    lm: torch.Tensor
    rc: torch.Tensor
    J: torch.Tensor | None


class VjpResult(NamedTuple):
    """What ``ADSolver.vjp`` returns (``self.flag`` holds the per-cell flag): x, h, done, steps as
    ``CudaSolver.launch``, and the ``Cotangents`` of the inputs (kincuda_ad.py:94-108)."""

    x: torch.Tensor
    h: torch.Tensor
    done: torch.Tensor
    steps: torch.Tensor
    cotangents: Cotangents


class ADSolver(CudaSolver):
    """One solver call with its tangent on one B200 (kincuda_ad.py:118-148).

    Parameters are the reference's: ``net``, ``device``, and keyword-only ``cap`` (attempts stored per cell before the
    adjoint checkpoints; it bounds max_steps as the reference's does), ``drift`` and ``photo``. The result of each call
    is ``CudaSolver.launch``'s; the guard lists the cells the solver would recompute, and those are differentiated
    along the recovery's path. A cell that still fails has flag 2 and NaN tangents.
    """

    def __init__(self, net: VulcanNetwork, device: torch.device | str, *, cap: int = CAP,
                 drift: float | None = None, photo: bool = False) -> None:
        try:
            cap = operator.index(cap)
        except TypeError:
            raise ValueError(f"cap: an integer expected, got {cap!r}") from None
        if cap < 1:
            raise ValueError(f"cap: at least 1 stored attempt expected, got {cap}")
        super().__init__(net, device, drift=drift, photo=photo, warps=4)  # the derivative kernels take 4
        self.cap = cap
        self._rc0 = torch.as_tensor(self.tab.rc, dtype=torch.float64).to(self.dev)

    @property
    def rc0(self) -> torch.Tensor:
        """The network's rate table [R, 14], which a call uses unless given another (kincuda_ad.py:217-221)."""
        self._require_open()
        return self._rc0

    def _check_tangents(self, tangents: dict[str, torch.Tensor | None], cells: int) -> int:
        """Refuse a tangent of the wrong form, naming it; return the directions (kincuda_ad.py:304-339)."""
        dx = tangents["dx"]
        if dx.dim() not in (2, 3):
            raise ValueError(f"dx: [B, S] or [D, B, S] expected, got {list(dx.shape)}")
        one = dx.dim() == 2
        directions = 1 if one else dx.shape[0]
        if not 1 <= directions <= DMAX:
            raise ValueError(f"dx: from 1 to {DMAX} directions on the leading axis expected, got {list(dx.shape)}")
        lead = () if one else (directions,)
        dJ = tangents["dJ"]
        if dJ is not None and not self.nj and (dJ.dim() != len(lead) + 2 or dJ.shape[-1] != 0):
            raise ValueError(
                f"dJ: none or an empty {[*lead, cells, 0]} one expected, since this solver has no photolysis; "
                f"got {list(dJ.shape)}"
            )
        shapes = {"dx": (*lead, cells, self.ns), "dT": (*lead, cells), "dP": (*lead, cells), "ddt": (*lead, cells),
                  "dh": (*lead, cells), "dlm": (*lead, cells, self.nr), "drc": (*lead, self.nr, ARRHENIUS_COLUMNS),
                  "dJ": (*lead, cells, self.nj)}  # fmt: skip
        for name, a in tangents.items():
            if a is not None:
                check_tensor(name, a, shapes[name], self.dev)
        return directions

    def jvp(self, x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor, h: torch.Tensor,
            dx: torch.Tensor, dT: torch.Tensor, dP: torch.Tensor, ddt: torch.Tensor, dh: torch.Tensor, *,
            lm: torch.Tensor | None = None, dlm: torch.Tensor | None = None, rc: torch.Tensor | None = None,
            drc: torch.Tensor | None = None, adapt: bool = True, rtol: float = DEFAULT_RTOL, atol: float = ATOL,
            max_steps: int = DEFAULT_MAX_STEPS, J: torch.Tensor | None = None,
            dJ: torch.Tensor | None = None) -> JvpResult:
        """Run the call and its tangent (kincuda_ad.py:341-453). Everything after dh is keyword only.

        x, T, P, dt, h and J as ``CudaSolver.launch``; dx, dT, dP, ddt, dh their tangents in the same shapes, or with a
        leading axis of D <= DMAX directions on every tangent, which then share one call. lm [B, R]: per-cell log rate
        multipliers (None: none); dlm their tangent. rc [R, 14]: the rate table (``rc0`` if None); drc [R, 9] the
        tangent of its nine Arrhenius columns. dJ: the tangent of J (without photolysis None or an empty one). adapt:
        differentiate the step control too; False holds the accepted steps fixed (dh is then 0). Raises ValueError as
        ``CudaSolver.launch`` if a cell was refused (``self.flag`` is then None).
        """
        self.flag = None
        self._require_open()
        B = check_inputs(self.dev, self.ns, x, T, P, dt, h, rtol, atol, max_steps)
        limit = (2 * self.cap) ** 2 // REC_STEPS  # what the recovery's checkpoints reach
        if max_steps > limit:
            raise ValueError(f"max_steps: at most {limit} at cap {self.cap} expected, got {max_steps}")
        if lm is not None:
            check_tensor("lm", lm, (B, self.nr), self.dev)
            lm = lm.contiguous()
        if rc is not None:
            check_tensor("rc", rc, tuple(self._rc0.shape), self.dev)
            rc = rc.contiguous()
        jx = check_photolysis(J, B, self.nj, self.dev)
        tangents = {"dx": dx, "dT": dT, "dP": dP, "ddt": ddt, "dh": dh, "dlm": dlm, "drc": drc, "dJ": dJ}
        D = self._check_tangents(tangents, B)
        one = dx.dim() == 2
        lead = (lambda a: a.unsqueeze(0)) if one else (lambda a: a)
        tan = [lead(a).contiguous() for a in (dx, dT, dP, ddt, dh)]
        dJ = dJ if self.nj else None  # an empty dJ without photolysis is none, as an empty J
        dlm, drc, dJ = (None if a is None else lead(a).contiguous() for a in (dlm, drc, dJ))
        x, T, P, dt, h = (a.contiguous() for a in (x, T, P, dt, h))
        xo, ho, steps = torch.empty_like(x), torch.empty_like(h), torch.empty_like(h)
        done, flag, status = (torch.empty(B, dtype=torch.int32, device=self.dev) for _ in range(3))
        dxo = torch.empty((D, B, self.ns), dtype=torch.float64, device=self.dev)
        dho = torch.empty((D, B), dtype=torch.float64, device=self.dev)
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        err = ctypes.create_string_buffer(_ERRLEN)
        code = self._lib.mx_jvp(
            self._handle, _ptr(x), _ptr(T), _ptr(P), _ptr(dt), _ptr(h), _ptr(jx), _ptr(lm), _ptr(rc), B, float(rtol),
            float(atol), int(max_steps), int(bool(adapt)), D, *(_ptr(a) for a in tan), _ptr(dlm), _ptr(drc), _ptr(dJ),
            _ptr(xo), _ptr(ho), _ptr(done), _ptr(steps), _ptr(flag), _ptr(status), _ptr(dxo), _ptr(dho),
            _ptr(self.count), _ptr(self.total), stream, err, _ERRLEN,
        )  # fmt: skip
        if code:
            raise (ValueError if code == 1 else RuntimeError)(err.value.decode())
        self._refuse(x, T, P, dt, jx, status)
        self.flag = flag
        return JvpResult(xo, ho, done.bool(), steps, dxo[0] if one else dxo, dho[0] if one else dho)

    def vjp(self, x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor, h: torch.Tensor,
            gx: torch.Tensor, *, gh: torch.Tensor | None = None, lm: torch.Tensor | None = None,
            rc: torch.Tensor | None = None, adapt: bool = True, rtol: float = DEFAULT_RTOL, atol: float = ATOL,
            max_steps: int = DEFAULT_MAX_STEPS, J: torch.Tensor | None = None) -> VjpResult:
        """Run the call and the cotangents of its inputs (kincuda_ad.py:455-556). Everything after gx is keyword only.

        x, T, P, dt, h, lm, rc, adapt, rtol, atol, max_steps and J as ``jvp``; gx [B, S] the cotangent of the output
        x, gh [B] that of the output h (adaptive only). A cell with flag 2 (``self.flag``) has NaN in its own
        cotangents and is left out of rc's sum; ``fallback["still_failed"]`` counts the cells left out. Raises
        ValueError as ``CudaSolver.launch`` if a cell was refused (``self.flag`` is then None).
        """
        self.flag = None
        self._require_open()
        B = check_inputs(self.dev, self.ns, x, T, P, dt, h, rtol, atol, max_steps)
        limit = (2 * self.cap) ** 2 // REC_STEPS  # what the recovery's checkpoints reach
        if max_steps > limit:
            raise ValueError(f"max_steps: at most {limit} at cap {self.cap} expected, got {max_steps}")
        if lm is not None:
            check_tensor("lm", lm, (B, self.nr), self.dev)
            lm = lm.contiguous()
        if rc is not None:
            check_tensor("rc", rc, tuple(self._rc0.shape), self.dev)
            rc = rc.contiguous()
        jx = check_photolysis(J, B, self.nj, self.dev)
        check_tensor("gx", gx, (B, self.ns), self.dev)
        gx = gx.contiguous()
        if gh is not None:
            check_tensor("gh", gh, (B,), self.dev)
            gh = gh.contiguous()
        x, T, P, dt, h = (a.contiguous() for a in (x, T, P, dt, h))
        xo, ho, steps = torch.empty_like(x), torch.empty_like(h), torch.empty_like(h)
        done, flag, status = (torch.empty(B, dtype=torch.int32, device=self.dev) for _ in range(3))
        f64 = lambda *shape: torch.empty(*shape, dtype=torch.float64, device=self.dev)  # noqa: E731
        g = Cotangents(x=torch.empty_like(x), T=f64(B), P=f64(B), dt=f64(B), h=f64(B), lm=f64(B, self.nr),
                       rc=f64(self.nr, ARRHENIUS_COLUMNS), J=f64(B, self.nj) if self.nj else None)  # fmt: skip
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        err = ctypes.create_string_buffer(_ERRLEN)
        code = self._lib.mx_vjp(
            self._handle, _ptr(x), _ptr(T), _ptr(P), _ptr(dt), _ptr(h), _ptr(jx), _ptr(lm), _ptr(rc), B, float(rtol),
            float(atol), int(max_steps), int(bool(adapt)), self.cap, _ptr(gx), _ptr(gh), _ptr(xo), _ptr(ho),
            _ptr(done), _ptr(steps), _ptr(flag), _ptr(status), _ptr(g.x), _ptr(g.T), _ptr(g.P), _ptr(g.dt),
            _ptr(g.h), _ptr(g.lm), _ptr(g.rc), _ptr(g.J), _ptr(self.count), _ptr(self.total), stream, err, _ERRLEN,
        )  # fmt: skip
        if code:
            raise (ValueError if code == 1 else RuntimeError)(err.value.decode())
        self._refuse(x, T, P, dt, jx, status)
        self.flag = flag
        return VjpResult(xo, ho, done.bool(), steps, g)
