"""TEST INFRASTRUCTURE ONLY: the CPU oracle of the per-call chemistry solve (oracle/mx_oracle.c) and of its tangent
(oracle/mx_oracle_ad.c) through ctypes.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this package: as the oracle the CUDA path
is compared with, or as the timed CPU baseline. The product (maxichem_b200) never imports it.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path
from typing import Any

import numpy as np

from maxichem_b200.abi import COUNT_SLOTS, NetworkStruct
from maxichem_b200.tables import Tables

HERE = Path(__file__).resolve().parent
SOURCES = [HERE / "mx_oracle.c", HERE / "mx_oracle_ad.c"]
LIBRARY = HERE / "_build" / "libmx_oracle.so"
# -O3 with the x86-64-v3 level (AVX2, BMI2) rather than -march=native: the built library travels to machines whose
# CPUs may differ from the build machine's; -ffp-contract=off keeps every multiply-add unfused unless written as fma.
FLAGS = ["-O3", "-march=x86-64-v3", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
         "-std=c11", "-Wall"]  # fmt: skip

_lib: ctypes.CDLL | None = None


def build(force: bool = False) -> Path:
    """Compile the oracle with gcc (no contraction of multiply-adds: every fma is explicit)."""
    LIBRARY.parent.mkdir(exist_ok=True)
    header = HERE.parent / "include" / "maxichem_b200.h"
    newest = max(p.stat().st_mtime for p in [*SOURCES, header])
    stale = not LIBRARY.exists() or newest > LIBRARY.stat().st_mtime
    if force or stale:
        tmp = LIBRARY.with_suffix(".tmp.so")
        subprocess.run(["gcc", *FLAGS, *map(str, SOURCES), "-o", str(tmp), "-lm"], check=True)
        tmp.replace(LIBRARY)
    return LIBRARY


def library() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIBRARY))
        P, I64, D, I32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int32
        lib.mxo_call.restype = ctypes.c_int
        lib.mxo_call.argtypes = [P, D, P, P, P, P, P, P, I64, D, D, I32, P, P, P, P, P, P, P, ctypes.c_int]
        lib.mxo_rates.restype = None
        lib.mxo_rates.argtypes = [P, D, D, P, P, P, P]
        lib.mxo_rhs_jacobian.restype = D
        lib.mxo_rhs_jacobian.argtypes = [P, P, P, D, P, P, P]
        lib.mxo_check_cell.restype = ctypes.c_int
        lib.mxo_check_cell.argtypes = [P, P, P, ctypes.c_int, D, D, D]
        lib.mxo_dense_lu.restype = None
        lib.mxo_dense_lu.argtypes = [ctypes.c_int, P, P, P]
        lib.mxo_dense_solve.restype = None
        lib.mxo_dense_solve.argtypes = [ctypes.c_int, P, P, P, P, P]
        lib.mxo_screen.restype = ctypes.c_int
        lib.mxo_screen.argtypes = [P, P, D, D, D, P, P]
        lib.mxo_threads.restype = ctypes.c_int
        lib.mxo_jvp.restype = ctypes.c_int
        lib.mxo_jvp.argtypes = [P, D, P, P, P, P, P, P, P, P, I64, D, D, I32, I32, I32] + [P] * 8 + [P] * 9 + [
            ctypes.c_int]
        lib.mxo_debug_try.restype = None
        lib.mxo_debug_try.argtypes = [P, P, D, D, D, P, D, D, P]
        _lib = lib
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _f64(a: Any) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    """The oracle for one network's tables: ``call`` mirrors CudaSolver.launch on host arrays."""

    def __init__(self, tab: Tables, drift: float = 1e-6) -> None:
        self.tab = tab
        self.net = NetworkStruct(tab)
        self.drift = float(drift)
        self.lib = library()

    def call(self, x: Any, T: Any, P: Any, dt: Any, h: Any, *, rtol: float = 1e-3, atol: float = 1e-25,
             max_steps: int = 4000, J: Any = None, threads: int = 0) -> dict[str, np.ndarray]:
        """One call on the CPU: x, h, done (bool), steps, flag, status and the counts (int32 [12])."""
        x, T, P, dt, h = (_f64(a) for a in (x, T, P, dt, h))
        B, ns = x.shape
        Jc = _f64(J if J is not None and self.tab.nj else np.zeros((B, self.tab.nj)))
        xo, ho, steps = np.empty_like(x), np.empty(B), np.empty(B)
        done, flag, status = (np.empty(B, np.int32) for _ in range(3))
        count = np.zeros(COUNT_SLOTS, np.int32)
        self.lib.mxo_call(self.net.ref(), self.drift, _p(x), _p(T), _p(P), _p(dt), _p(h), _p(Jc), B, rtol, atol,
                          max_steps, _p(xo), _p(ho), _p(done), _p(steps), _p(flag), _p(status), _p(count), threads)
        return {"x": xo, "h": ho, "done": done.astype(bool), "steps": steps, "flag": flag, "status": status,
                "count": count}  # fmt: skip

    def jvp(self, x: Any, T: Any, P: Any, dt: Any, h: Any, dx: Any = None, dT: Any = None, dP: Any = None,
            ddt: Any = None, dh: Any = None, *, lm: Any = None, dlm: Any = None, rc: Any = None, drc: Any = None,
            J: Any = None, dJ: Any = None, adapt: bool = True, rtol: float = 1e-3, atol: float = 1e-25,
            max_steps: int = 4000, threads: int = 0) -> dict[str, np.ndarray]:
        """One call and its tangent on the CPU (dual numbers through the oracle's call): the outputs of ``call`` and
        dx [D, B, S], dh [D, B]. Every tangent has a leading axis of D directions (None: zeros; all None: D = 0, the
        primal alone, which takes lm and rc as the tangent call does)."""
        tab = self.tab
        x, T, P, dt, h = (_f64(a) for a in (x, T, P, dt, h))
        B, ns = x.shape
        nr, nj = tab.nr, tab.nj
        given = [a for a in (dx, dT, dP, ddt, dh, dlm, drc, dJ) if a is not None]
        D = int(np.shape(given[0])[0]) if given else 0
        z = lambda *s: np.zeros(s)
        dx, dT, dP, ddt, dh = (_f64(a) if a is not None else z(D, *shape)
                               for a, shape in ((dx, (B, ns)), (dT, (B,)), (dP, (B,)), (ddt, (B,)), (dh, (B,))))
        opt = lambda a: None if a is None else _f64(a)
        lm, dlm, rc, drc, dJ = (opt(a) for a in (lm, dlm, rc, drc, dJ))
        Jc = _f64(J if J is not None and nj else np.zeros((B, nj)))
        if dJ is not None and not nj:
            dJ = None
        xo, ho, steps = np.empty_like(x), np.empty(B), np.empty(B)
        done, flag, status = (np.empty(B, np.int32) for _ in range(3))
        count = np.zeros(COUNT_SLOTS, np.int32)
        dxo, dho = np.empty((D, B, ns)), np.empty((D, B))
        q = lambda a: None if a is None else _p(a)
        self.lib.mxo_jvp(self.net.ref(), self.drift, _p(x), _p(T), _p(P), _p(dt), _p(h), _p(Jc), q(lm), q(rc), B, rtol,
                         atol, max_steps, int(adapt), D, _p(dx), _p(dT), _p(dP), _p(ddt), _p(dh), q(dlm), q(drc), q(dJ),
                         _p(xo), _p(ho), _p(done), _p(steps), _p(flag), _p(status), _p(count), _p(dxo), _p(dho),
                         threads)  # fmt: skip
        return {"x": xo, "h": ho, "done": done.astype(bool), "steps": steps, "flag": flag, "status": status,
                "count": count, "dx": dxo, "dh": dho}  # fmt: skip

    def debug_try(self, x: Any, T: float, P: float, h: float, J: Any = None, rtol: float = 1e-3,
                  atol: float = 1e-25) -> dict[str, np.ndarray]:
        """One fresh try of one cell with every stage (the layout of the library's mx_debug_try)."""
        tab = self.tab
        out = np.empty(debug_size(tab))
        Jc = _f64(J if J is not None and tab.nj else np.zeros(tab.nj))
        self.lib.mxo_debug_try(self.net.ref(), _p(_f64(x)), T, P, h, _p(Jc), rtol, atol, _p(out))
        return split_debug(tab, out)

    def rates(self, T: float, P: float, J: Any = None) -> tuple[np.ndarray, np.ndarray]:
        tab = self.tab
        kf, kr = np.empty(tab.nr), np.empty(tab.nr)
        g = np.empty(tab.ns + 1)
        Jc = _f64(J if J is not None else np.zeros(tab.nj))
        nd = P / (1.380649e-16 * T)
        self.lib.mxo_rates(self.net.ref(), T, nd, _p(Jc), _p(kf), _p(kr), _p(g))
        return kf, kr

    def rhs_jacobian(self, kf: np.ndarray, kr: np.ndarray, Y: np.ndarray, nd: float) -> tuple[Any, ...]:
        """F, u0, -Jn (dense, elimination order) and n_tot at the state Y (elimination order)."""
        ns = self.tab.ns
        k = _f64(np.concatenate([kf, kr]))
        Y = _f64(Y)
        F, u0, A = np.empty(ns), np.empty(ns), np.empty((ns, ns))
        ntot = self.lib.mxo_rhs_jacobian(self.net.ref(), _p(k), _p(Y), nd, _p(F), _p(u0), _p(A))
        return F, u0, A, ntot


def dense_lu(a: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """The recovery's threshold-pivoted dense LU: factors, 1 / pivots, row order."""
    a = _f64(a).copy()
    n = a.shape[0]
    dinv, pr = np.empty(n), np.empty(n, np.int32)
    library().mxo_dense_lu(n, _p(a), _p(dinv), _p(pr))
    return a, dinv, pr


def dense_solve(a: np.ndarray, dinv: np.ndarray, pr: np.ndarray, y: np.ndarray) -> np.ndarray:
    y = _f64(y).copy()
    work = np.empty_like(y)
    library().mxo_dense_solve(len(y), _p(_f64(a)), _p(_f64(dinv)), _p(np.ascontiguousarray(pr, np.int32)), _p(y),
                              _p(work))
    return y


def threads() -> int:
    return int(library().mxo_threads())


def debug_size(tab: Tables) -> int:
    return 2 * tab.nr + 10 * tab.ns + 2 * tab.ns * tab.ns + 2


def split_debug(tab: Tables, out: np.ndarray) -> dict[str, np.ndarray]:
    """Name the stages of a one-try dump."""
    ns, nr = tab.ns, tab.nr
    parts = [("kf", nr), ("kr", nr), ("F", ns), ("u0", ns), ("Jn", ns * ns), ("w", ns), ("LU", ns * ns), ("dinv", ns),
             ("K1", ns), ("K2", ns), ("K3", ns), ("K4", ns), ("Y", ns), ("err", 1), ("ok", 1)]  # fmt: skip
    d, o = {}, 0
    for name, n in parts:
        d[name] = out[o : o + n]
        o += n
    return d
