"""mx_call_static, the call that allocates nothing, against mx_call through the C-ABI.

Some callers cannot allocate device memory during their time loop: a GCM whose framework reserved the GPU's memory for
its own pool at start-up (a cudaMalloc then fails or fragments that pool), or a loop that cannot afford the
device-wide synchronisation cudaMalloc and cudaFree may imply. mx_call_static serves them: its one piece of scratch,
the recompute list, is a static device array instead of solver-owned memory. This file checks that it gives mx_call's
results bit for bit on two calls in a row whose guard lists cells, so the recovery really reads the static list, and
that a solver called only through it never sizes a list of its own. It is collected last and also passes alone in a
fresh process (the static array's address is looked up at each call).
"""

import ctypes

import numpy as np
import pytest
import torch

from maxichem_b200 import abi, synthetic
from maxichem_b200.constants import COUNTS
from maxichem_b200.solver import CudaSolver

pytestmark = pytest.mark.gpu
ERRLEN = 512
MAX_CELLS = 1048576  # MX_STATIC_MAX_CELLS of include/maxichem_b200.h
RECOMPUTED = 1 + COUNTS.index("recomputed")  # count slot (slot 0 is the cell queue)
MAX_STEPS = 30  # a cold start needs ~140 steps: every cell is left unfinished, listed, and recovered (300 tries)


def outputs(B, ns, dev):
    f = lambda *shape: torch.empty(*shape, dtype=torch.float64, device=dev)
    i = lambda: torch.empty(B, dtype=torch.int32, device=dev)
    return {"x": f(B, ns), "h": f(B), "done": i(), "steps": f(B), "flag": i(), "status": i(),
            "count": torch.zeros(12, dtype=torch.int32, device=dev), "total": torch.zeros(12, dtype=torch.int64, device=dev)}  # fmt: skip


def c_call(entry, solver, inp, out, B=None, max_steps=4000):
    """One call of mx_call or mx_call_static through ctypes on device tensors; returns (status, message)."""
    p = lambda t: t.data_ptr()
    err = ctypes.create_string_buffer(ERRLEN)
    x, T, P, dt, h, J = inp
    rc = entry(solver._handle, p(x), p(T), p(P), p(dt), p(h), p(J), x.shape[0] if B is None else B, 1e-3, 1e-25,
               max_steps, p(out["x"]), p(out["h"]), p(out["done"]), p(out["steps"]), p(out["flag"]), p(out["status"]),
               p(out["count"]), p(out["total"]), torch.cuda.current_stream(solver.dev).cuda_stream, err, ERRLEN)  # fmt: skip
    return rc, err.value.decode()


def host(out):
    return {k: v.cpu().numpy() for k, v in out.items()}


def test_the_static_call_matches_the_call_twice_in_a_row(gpu, networks):
    net = networks("cho41")
    B = 512
    w = synthetic.workload(net, "column", B, seed=21)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=gpu)
    lib = abi.library()
    # two fresh solvers: one called only through mx_call, the other only through mx_call_static
    with CudaSolver(net, gpu, photo=True) as plain, CudaSolver(net, gpu, photo=True) as static:
        ns = plain.ns
        inp_a = inp_b = (t(w.x), t(w.T), t(w.P), t(w.dt), t(w.h), t(w.J))
        ref, got = outputs(B, ns, gpu), outputs(B, ns, gpu)
        for k in range(2):  # a cold start cut short at MAX_STEPS tries, then a 1e10 s dark call from its results
            for o in (ref, got):
                o["x"].fill_(float("nan"))
            rc, msg = c_call(lib.mx_call, plain, inp_a, ref, max_steps=MAX_STEPS)
            assert rc == 0, msg
            rc, msg = c_call(lib.mx_call_static, static, inp_b, got, max_steps=MAX_STEPS)
            assert rc == 0, msg
            torch.cuda.synchronize(gpu)
            r, g = host(ref), host(got)
            assert r["count"][RECOMPUTED] > 0, (k, r["count"])  # the guard listed cells: the list was written and read
            for name in ("x", "h", "done", "steps", "flag", "status", "count"):
                assert np.array_equal(g[name], r[name], equal_nan=True), (k, name)
            assert np.array_equal(g["total"], r["total"]), k
            assert (r["flag"] > 0).sum() == r["count"][RECOMPUTED]
            long = torch.full_like(inp_a[3], 1e10)  # hundreds of steps: again beyond MAX_STEPS, so listed again
            inp_a = (ref["x"].clone(), inp_a[1], inp_a[2], long, ref["h"].clone(), torch.zeros_like(inp_a[5]))
            inp_b = (got["x"].clone(), inp_b[1], inp_b[2], long, got["h"].clone(), torch.zeros_like(inp_b[5]))
        assert static.layout()["list_cells"] == 0  # the static solver never sized a recompute list of its own
        assert plain.layout()["list_cells"] >= B


def test_the_static_call_refuses_more_cells_than_its_scratch(gpu, networks):
    net = networks("cho41")
    w = synthetic.workload(net, "column", 4, seed=2)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=gpu)
    with CudaSolver(net, gpu, photo=True) as solver:
        out = outputs(4, solver.ns, gpu)
        rc, msg = c_call(abi.library().mx_call_static, solver, (t(w.x), t(w.T), t(w.P), t(w.dt), t(w.h), t(w.J)), out,
                         B=MAX_CELLS + 1)  # fmt: skip
    assert rc == 1
    assert "MX_STATIC_MAX_CELLS = 1048576" in msg and "1048577" in msg
