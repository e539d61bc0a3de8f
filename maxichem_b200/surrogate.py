"""The learned part of the call: a BF16 MLP surrogate trained on the GPU by the library's own kernels, and the gated
call that solves with Rodas3 only the cells it cannot vouch for (no counterpart in the reference).

``Surrogate`` wraps the library's mx_sur_* entry points: the network (features -> 4 hidden layers of 512 with SiLU ->
4 heads of (delta log10 x per species, log10 h)), its standardisation, its training (``fit``: Adam on minibatches,
every GEMM a tcgen05 kernel) and its forward pass. ``pairs`` generates training pairs with the plain FP64 solver over
the column-grid distributions (settled calls, night cells, cold starts). ``GatedSolver`` is the call: the network
proposes each cell's end-of-call state; a proposal is accepted only inside the training range, under the heads'
spread threshold and when its element-share projection is small, and every rejected cell plus a seeded 1/64 audit
of the accepted ones is solved by Rodas3 in the same call, the audit reporting the surrogate's error.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from pathlib import Path
from typing import Any

import numpy as np
import torch

from . import abi, synthetic
from .constants import ATOL, DEFAULT_MAX_STEPS, DEFAULT_RTOL, DRIFT
from .solver import CallResult, CudaSolver, check_inputs, check_photolysis

_ERRLEN = 1024
X_FLOOR = 1e-30
AUDIT_FLOOR = 1e-20
STD_FLOOR = 1e-4  # the smallest target deviation (dex) the standardisation divides by
STATS = ("accepted", "audited", "out_of_range", "spread", "projection", "unusable")
INFO = ("nf", "kin", "nt", "kout", "params", "layers", "hidden", "heads", "steps")


def quantile(v: torch.Tensor, q: float) -> float:
    """The q-quantile of a 1-d tensor (linear interpolation; any size, unlike torch.quantile)."""
    n = v.numel()
    if n == 0:
        return 0.0
    s = torch.sort(v.reshape(-1).double()).values
    pos = q * (n - 1)
    lo = int(math.floor(pos))
    hi = min(lo + 1, n - 1)
    return float(s[lo] + (s[hi] - s[lo]) * (pos - lo))


def raw_features(x: torch.Tensor, T: torch.Tensor, P: torch.Tensor, dt: torch.Tensor, h: torch.Tensor,
                 J: torch.Tensor | None) -> torch.Tensor:
    """The features before standardisation, as the library's features kernel forms them (FP32 [B][nf])."""
    cols = [torch.log10(x.clamp_min(X_FLOOR)), torch.log10(T)[:, None], torch.log10(P)[:, None],
            torch.log10(dt.clamp_min(X_FLOOR))[:, None], torch.log10(h.clamp_min(X_FLOOR))[:, None]]  # fmt: skip
    if J is not None and J.shape[1]:
        cols.append(torch.log10(J + X_FLOOR))
    return torch.cat(cols, 1).float()


def targets(x_in: torch.Tensor, x_out: torch.Tensor, h_out: torch.Tensor) -> torch.Tensor:
    """The unstandardised targets: log10 x_out - log10 x_in per species (floored), then log10 h_out (FP32 [B][nt])."""
    d = torch.log10(x_out.clamp_min(X_FLOOR)) - torch.log10(x_in.clamp_min(X_FLOOR))
    return torch.cat([d, torch.log10(h_out)[:, None]], 1).float()


@dataclass
class Pairs:
    """Training pairs on the device: inputs of a call and its plain-solver outcome."""

    x: torch.Tensor
    T: torch.Tensor
    P: torch.Tensor
    dt: torch.Tensor
    h: torch.Tensor
    J: torch.Tensor
    x_out: torch.Tensor
    h_out: torch.Tensor

    def __len__(self) -> int:
        return int(self.x.shape[0])

    def select(self, idx: torch.Tensor) -> "Pairs":
        return Pairs(*(getattr(self, f)[idx] for f in ("x", "T", "P", "dt", "h", "J", "x_out", "h_out")))

    @staticmethod
    def cat(parts: list["Pairs"]) -> "Pairs":
        return Pairs(*(torch.cat([getattr(p, f) for p in parts]) for f in ("x", "T", "P", "dt", "h", "J", "x_out", "h_out")))


def pairs(solver: CudaSolver, cells: int, calls: int, seed: int, cold_share: float = 0.25, dt: float = 300.0) -> Pairs:
    """Pairs from the plain solver on the column grid (config-1/2 distributions): `calls` chained calls of dt from a
    solar start, half of the columns at night, and after the first call a `cold_share` of cells re-started cold
    (x perturbed log-normally, h 1e-10 s) in every call. Cells the call does not finish are left out."""
    dev = solver.dev
    w = synthetic.workload(solver.net, "uneven", cells, seed=seed)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)  # noqa: E731
    x, T, P, DT, h, J = t(w.x), t(w.T), t(w.P), t(w.dt), t(w.h), t(w.J)
    DT.fill_(dt)
    out = []
    rng = np.random.default_rng(seed + 1)
    for k in range(calls):
        if k > 0 and cold_share > 0:
            xc, hc, _ = synthetic.cold_start(x.cpu().numpy(), h.cpu().numpy(), seed=int(rng.integers(1 << 30)),
                                             share=cold_share)  # fmt: skip
            x, h = t(xc), t(hc)
        r = solver.launch(x, T, P, DT, h, J=J)
        ok = r.done & (r.flag == 0)
        out.append(Pairs(x[ok], T[ok], P[ok], DT[ok], h[ok], J[ok], r.x[ok], r.h[ok]))
        x, h = r.x, r.h
    return Pairs.cat(out)


class Surrogate:
    """The network and its training, over the library's mx_sur_* entry points (device `dev`)."""

    def __init__(self, ns: int, nj: int, atoms: np.ndarray, device: torch.device | str, *, hidden: int = 512,
                 layers: int = 4, heads: int = 4, seed: int = 0) -> None:
        self._handle: ctypes.c_void_p | None = None
        self.dev = torch.device(device)
        self._lib = abi.library()
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(_ERRLEN)
        rc = self._lib.mx_sur_create(ns, nj, atoms.shape[1], atoms.ctypes.data, hidden, layers, heads,
                                     self.dev.index or 0, ctypes.byref(handle), err, _ERRLEN)  # fmt: skip
        if rc:
            raise (ValueError if rc == 1 else RuntimeError)(err.value.decode())
        self._handle = handle
        self.ns, self.nj, self.hidden, self.layers, self.heads = ns, nj, hidden, layers, heads
        self.info = self._info()
        self.nf, self.kin, self.nt, self.kout = (self.info[k] for k in ("nf", "kin", "nt", "kout"))
        self.shapes = [(hidden if l < layers else self.kout, self.kin if l == 0 else hidden) for l in range(layers + 1)]
        self.set_params(self.initial(seed))
        self.scaling: dict[str, np.ndarray] | None = None

    def _info(self) -> dict[str, int]:
        v = (ctypes.c_int64 * len(INFO))()
        self._lib.mx_sur_info(self._handle, v, len(INFO))
        return dict(zip(INFO, [int(q) for q in v]))

    def close(self) -> None:
        if self._handle is not None:
            torch.cuda.synchronize(self.dev)
            self._lib.mx_sur_destroy(self._handle)
            self._handle = None

    def __del__(self) -> None:
        try:
            if getattr(self, "_handle", None) is not None:
                self._lib.mx_sur_destroy(self._handle)
        except Exception:
            pass

    # parameters: W_l [out][in] then b_l [out], layer by layer
    def initial(self, seed: int) -> np.ndarray:
        """He-uniform weights for SiLU layers and a small output layer; zero biases; padding rows of the heads 0."""
        rng = np.random.default_rng(seed)
        parts = []
        for l, (rows, cols) in enumerate(self.shapes):
            bound = math.sqrt(6.0 / cols) * (0.1 if l == self.layers else 1.0)
            w = rng.uniform(-bound, bound, (rows, cols)).astype(np.float32)
            if l == 0:
                w[:, self.nf:] = 0.0
            if l == self.layers:
                w[self.heads * self.nt:] = 0.0
            parts += [w.ravel(), np.zeros(rows, np.float32)]
        return np.concatenate(parts)

    def params(self, which: int = 0) -> np.ndarray:
        out = np.empty(self.info["params"], np.float32)
        if self._lib.mx_sur_params(self._handle, which, out.ctypes.data, out.size):
            raise RuntimeError("mx_sur_params failed")
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if self._lib.mx_sur_set_params(self._handle, p.ctypes.data, p.size):
            raise ValueError(f"{p.size} parameters given, {self.info['params']} expected")

    def unpack(self, p: np.ndarray) -> list[tuple[np.ndarray, np.ndarray]]:
        out, off = [], 0
        for rows, cols in self.shapes:
            w = p[off : off + rows * cols].reshape(rows, cols)
            off += rows * cols
            out.append((w, p[off : off + rows]))
            off += rows
        return out

    def set_scaling(self, raw: torch.Tensor, tgt: torch.Tensor, target_scale: float | None = None) -> None:
        """Standardisation and training range from raw features [N][nf] and unstandardised targets [N][nt]; the
        targets' scale is their deviation, or one fixed `target_scale` (dex) for all of them with no shift."""
        f = raw.double()
        t = tgt.double()
        if target_scale is None:
            tmean, tstd = t.mean(0), t.std(0).clamp_min(STD_FLOOR)
        else:
            tmean, tstd = torch.zeros_like(t[0]), torch.full_like(t[0], float(target_scale))
        sc = {"fmean": f.mean(0), "fstd": f.std(0), "flo": f.min(0).values, "fhi": f.max(0).values,
              "tmean": tmean, "tstd": tstd}  # fmt: skip
        self.scaling = {k: v.float().cpu().numpy() for k, v in sc.items()}
        self._push_scaling()

    def _push_scaling(self) -> None:
        a = {k: np.ascontiguousarray(v, dtype=np.float32) for k, v in self.scaling.items()}
        rc = self._lib.mx_sur_set_scaling(self._handle, *(a[k].ctypes.data for k in
                                                          ("fmean", "fstd", "flo", "fhi", "tmean", "tstd")))  # fmt: skip
        if rc:
            raise ValueError("mx_sur_set_scaling refused the scaling")

    def features(self, x, T, P, dt, h, J) -> tuple[torch.Tensor, torch.Tensor]:
        B = x.shape[0]
        feat = torch.empty(B, self.kin, dtype=torch.bfloat16, device=self.dev)
        inr = torch.empty(B, dtype=torch.int32, device=self.dev)
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        rc = self._lib.mx_sur_features(self._handle, x.data_ptr(), T.data_ptr(), P.data_ptr(), dt.data_ptr(),
                                       h.data_ptr(), None if J is None else J.data_ptr(), B, feat.data_ptr(),
                                       inr.data_ptr(), stream)  # fmt: skip
        if rc:
            raise RuntimeError(f"mx_sur_features failed ({rc})")
        return feat, inr

    def propose(self, x, T, P, dt, h, J, *, drift: float = DRIFT, atol: float = ATOL) -> tuple[torch.Tensor, torch.Tensor]:
        """The gate's projected proposal of every cell [B][ns] and its measures [B][4]: spread (dex), projection size
        (inf on drift), 1 when usable and in range, proposed h (mx_sur_propose)."""
        B = x.shape[0]
        xp = torch.empty(B, self.ns, dtype=torch.float64, device=self.dev)
        diag = torch.empty(B, 4, dtype=torch.float64, device=self.dev)
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        rc = self._lib.mx_sur_propose(self._handle, x.data_ptr(), T.data_ptr(), P.data_ptr(), dt.data_ptr(),
                                      h.data_ptr(), None if J is None else J.data_ptr(), B, float(drift), float(atol),
                                      xp.data_ptr(), diag.data_ptr(), stream)  # fmt: skip
        if rc:
            raise RuntimeError(f"mx_sur_propose failed ({rc})")
        return xp, diag

    def forward(self, feat: torch.Tensor) -> torch.Tensor:
        pred = torch.empty(feat.shape[0], self.kout, dtype=torch.float32, device=self.dev)
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        if self._lib.mx_sur_forward(self._handle, feat.data_ptr(), feat.shape[0], pred.data_ptr(), stream):
            raise RuntimeError("mx_sur_forward failed")
        return pred

    def train_step(self, feat: torch.Tensor, tgt: torch.Tensor, wts: torch.Tensor, lr: float,
                   loss: torch.Tensor | None = None, delta: float = 0.0) -> None:
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        rc = self._lib.mx_sur_train_step(self._handle, feat.data_ptr(), tgt.data_ptr(), wts.data_ptr(), feat.shape[0],
                                         float(lr), float(delta), None if loss is None else loss.data_ptr(), stream)  # fmt: skip
        if rc:
            raise ValueError(f"mx_sur_train_step refused the batch ({rc}): rows a multiple of 64 expected")

    def check(self) -> None:
        flag = ctypes.c_int32()
        self._lib.mx_sur_error(self._handle, ctypes.byref(flag))
        if flag.value:
            raise RuntimeError("a tensor-core GEMM gave up waiting on its pipeline")

    def standardised_targets(self, tgt: torch.Tensor) -> torch.Tensor:
        m = torch.as_tensor(self.scaling["tmean"], device=self.dev)
        s = torch.as_tensor(self.scaling["tstd"], device=self.dev)
        return ((tgt - m) / s).float().contiguous()

    def fit(self, data: Pairs, *, epochs: int = 8, batch: int = 8192, lr: float = 2e-3, seed: int = 0,
            target_scale: float | None = None, delta: float = 0.0, log: list | None = None) -> dict[str, Any]:
        """Train on `data`: standardisation from the data (the targets' own deviations, or one fixed `target_scale` in
        dex), each head on its own Poisson(1) bootstrap weights, the square error (delta 0) or the Huber loss of
        width delta, Adam with a cosine decay from lr. Returns the loss per epoch."""
        raw = raw_features(data.x, data.T, data.P, data.dt, data.h, data.J)
        tgt = targets(data.x, data.x_out, data.h_out)
        self.set_scaling(raw, tgt, target_scale)
        feat, _ = self.features(data.x, data.T, data.P, data.dt, data.h, data.J)
        y = self.standardised_targets(tgt)
        gen = torch.Generator(device=self.dev)
        gen.manual_seed(seed)
        wts = torch.poisson(torch.ones(len(data), self.heads, device=self.dev), generator=gen).float()
        n = len(data) // batch * batch
        if n == 0:
            raise ValueError(f"{len(data)} pairs: at least one batch of {batch} expected")
        steps = epochs * (n // batch)
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        history, k = [], 0
        for _ in range(epochs):
            order = torch.randperm(len(data), device=self.dev, generator=gen)[:n]
            loss.zero_()
            for b in range(0, n, batch):
                idx = order[b : b + batch]
                rate = lr * 0.5 * (1.0 + math.cos(math.pi * k / steps))
                self.train_step(feat[idx].contiguous(), y[idx].contiguous(), wts[idx].contiguous(), rate, loss, delta)
                k += 1
            history.append(float(loss.item()) / (n // batch))
            if log is not None:
                log.append(history[-1])
        self.check()
        return {"loss": history, "steps": k, "pairs": len(data)}

    def heads_of(self, pred: torch.Tensor) -> torch.Tensor:
        """The heads' unstandardised outputs [B][heads][nt] from a forward pass."""
        m = torch.as_tensor(self.scaling["tmean"], device=self.dev)
        s = torch.as_tensor(self.scaling["tstd"], device=self.dev)
        return pred[:, : self.heads * self.nt].reshape(-1, self.heads, self.nt) * s + m

    def save(self, path: str | Path) -> None:
        np.savez(path, params=self.params(), shape=np.array([self.ns, self.nj, self.hidden, self.layers, self.heads]),
                 **self.scaling)  # fmt: skip

    def load(self, path: str | Path) -> None:
        d = np.load(path)
        if list(d["shape"]) != [self.ns, self.nj, self.hidden, self.layers, self.heads]:
            raise ValueError(f"{path}: a network of another shape ({list(d['shape'])})")
        self.set_params(d["params"])
        self.scaling = {k: d[k] for k in ("fmean", "fstd", "flo", "fhi", "tmean", "tstd")}
        self._push_scaling()


def calibrate(sur: "Surrogate", data: Pairs, *, target: float = 1e-3, quantile_: float = 0.999,
              proj_max: float = 1e-2, margin: float = 0.5, drift: float = DRIFT, atol: float = ATOL) -> dict[str, float]:
    """The gate's spread threshold from held-out pairs (not trained on): accepting eligible cells (inputs usable and in
    range, projection at most proj_max, drift test passed) in order of increasing spread, the largest threshold under
    which the call's per-species relative error against the plain solver (over every cell and species above 1e-20;
    a rejected cell carries Rodas3's result, error 0) stays within `target` at `quantile_`, with only `margin` of the
    allowed share of values beyond it spent. Returns {"spread_max", "proj_max", "accept"} (accept: the share of
    `data`'s cells the threshold accepts; spread_max 0 when none can be)."""
    xp, diag = sur.propose(data.x, data.T, data.P, data.dt, data.h, data.J, drift=drift, atol=atol)
    truth = data.x_out
    big = truth > AUDIT_FLOOR
    err = torch.where(big, (xp - truth).abs() / truth.clamp_min(1e-300), torch.zeros_like(truth))
    bad = (err > target).sum(1).double()
    budget = (1.0 - quantile_) * float(big.sum()) * margin
    eligible = (diag[:, 2] == 1) & (diag[:, 1] <= proj_max)
    spread = torch.where(eligible, diag[:, 0], torch.full_like(diag[:, 0], math.inf))
    order = torch.argsort(spread)
    fine = (torch.cumsum(bad[order], 0) <= budget) & torch.isfinite(spread[order])
    k = int(fine.long().cumprod(0).sum())  # the longest admissible prefix
    if k == 0:
        return {"spread_max": 0.0, "proj_max": proj_max, "accept": 0.0}
    return {"spread_max": float(spread[order[k - 1]]), "proj_max": proj_max, "accept": k / len(data)}


class GatedSolver:
    """The gated call over a CudaSolver (its precision is the fallback's) and a trained Surrogate:
    ``solver(x, T, P, dt, h, J=J) -> CallResult``, the reference call's surface, with ``stats`` and ``audit``."""

    def __init__(self, solver: CudaSolver, sur: Surrogate, *, spread_max: float, proj_max: float = 1e-3,
                 audit_every: int = 64, seed: int = 0, audit_cap: int = 1 << 16) -> None:
        if sur.ns != solver.ns or sur.nj != solver.nj:
            raise ValueError("the surrogate and the solver are for different networks")
        self.solver, self.sur = solver, sur
        self.spread_max, self.proj_max, self.audit_every, self.seed = spread_max, proj_max, audit_every, seed
        dev = solver.dev
        self.stats = torch.zeros(len(STATS), dtype=torch.int64, device=dev)
        self.audit_cap = audit_cap
        self.audit_cells = torch.zeros(audit_cap, dtype=torch.int32, device=dev)
        self.audit_x = torch.zeros(audit_cap, solver.ns, dtype=torch.float64, device=dev)
        self.audit_err = torch.zeros(audit_cap, solver.ns, dtype=torch.float32, device=dev)
        self.audit_count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.calls = 0

    def launch_raw(self, x, T, P, dt, h, *, rtol=DEFAULT_RTOL, atol=ATOL, max_steps=DEFAULT_MAX_STEPS, J=None,
                   out=None) -> dict[str, torch.Tensor]:
        s = self.solver
        B = x.shape[0]
        if out is None:
            out = {"x": torch.empty_like(x), "h": torch.empty_like(h), "steps": torch.empty_like(h),
                   **{k: torch.empty(B, dtype=torch.int32, device=s.dev) for k in ("done", "flag", "status")}}  # fmt: skip
        p = lambda a: None if a is None else a.data_ptr()  # noqa: E731
        err = ctypes.create_string_buffer(_ERRLEN)
        stream = torch.cuda.current_stream(s.dev).cuda_stream
        rc = s._lib.mx_sur_call(
            self.sur._handle, s._handle, p(x), p(T), p(P), p(dt), p(h), p(J), B, float(rtol), float(atol),
            int(max_steps), float(self.spread_max), float(self.proj_max), int(self.audit_every),
            (self.seed * 1000003 + self.calls) & 0xFFFFFFFF, p(out["x"]), p(out["h"]), p(out["done"]), p(out["steps"]),
            p(out["flag"]), p(out["status"]), p(s.count), p(s.total), p(self.stats), p(self.audit_cells),
            p(self.audit_x), p(self.audit_err), p(self.audit_count), self.audit_cap, stream, err, _ERRLEN,
        )  # fmt: skip
        if rc:
            raise (ValueError if rc == 1 else RuntimeError)(err.value.decode())
        self.calls += 1
        return out

    def __call__(self, x, T, P, dt, h, *, rtol=DEFAULT_RTOL, atol=ATOL, max_steps=DEFAULT_MAX_STEPS, J=None) -> CallResult:
        s = self.solver
        s._require_open()
        B = check_inputs(s.dev, s.ns, x, T, P, dt, h, rtol, atol, max_steps)
        x, T, P, dt, h = (a.contiguous() for a in (x, T, P, dt, h))
        jx = check_photolysis(J, B, s.nj, s.dev)
        out = self.launch_raw(x, T, P, dt, h, rtol=rtol, atol=atol, max_steps=max_steps, J=jx)
        s._refuse(x, T, P, dt, jx, out["status"])
        s.flag = out["flag"]
        return CallResult(out["x"], out["h"], out["done"].bool(), out["steps"])

    def call_host(self, x, T, P, dt, h, *, rtol=DEFAULT_RTOL, atol=ATOL, max_steps=DEFAULT_MAX_STEPS, J=None,
                  out: dict[str, torch.Tensor] | None = None) -> CallResult:
        """The gated call on host (CPU) tensors: the inputs copied to the device, the call, the outputs copied back
        (into `out`'s pinned host tensors x, h, steps, done, flag, status when given), one stream, one synchronisation
        for the refusal check."""
        s = self.solver
        dev = s.dev
        ins = [torch.as_tensor(a).to(dev, non_blocking=True) for a in (x, T, P, dt, h)]
        jd = None if J is None else torch.as_tensor(J).to(dev, non_blocking=True)
        r = self.launch_raw(*ins, rtol=rtol, atol=atol, max_steps=max_steps, J=jd)
        if out is None:
            out = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in r.items()}
        for k, v in r.items():
            out[k].copy_(v, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        s._refuse(*ins[:4], jd, r["status"])
        return CallResult(out["x"], out["h"], out["done"].bool(), out["steps"])

    def counts(self) -> dict[str, int]:
        return dict(zip(STATS, [int(v) for v in self.stats.tolist()]))

    def audit(self) -> dict[str, Any]:
        """The last call's audit: per-species relative errors of the audited proposals against Rodas3 (species above
        1e-20), their quantiles, and the audited cells."""
        n = min(int(self.audit_count.item()), self.audit_cap)
        e = self.audit_err[:n].double()
        vals = e[e > 0] if n else e.new_zeros(0)
        q = lambda p: quantile(vals, p)  # noqa: E731
        return {"cells": n, "p50": q(0.5), "p99": q(0.99), "p999": q(0.999),
                "max": float(vals.max()) if vals.numel() else 0.0}  # fmt: skip
