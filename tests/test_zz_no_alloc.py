"""mx_call_static, the call that allocates nothing (for a GCM whose framework keeps the GPU's memory in its own pool,
or whose time loop must not pay cudaMalloc's synchronisation), against mx_call through the C-ABI: two calls in a row,
the second from the first's results, give the same outputs and counts (collected last, and correct in a fresh
process too: its first call on the device looks up the static scratch)."""

import ctypes

import numpy as np
import pytest
import torch

import parity
from maxichem_b200 import abi, synthetic
from maxichem_b200.solver import CudaSolver

pytestmark = pytest.mark.gpu
ERRLEN = 512
MAX_CELLS = 1048576  # MX_STATIC_MAX_CELLS of include/maxichem_b200.h


def outputs(B, ns, dev):
    f = lambda *shape: torch.empty(*shape, dtype=torch.float64, device=dev)
    i = lambda: torch.empty(B, dtype=torch.int32, device=dev)
    return {"x": f(B, ns), "h": f(B), "done": i(), "steps": f(B), "flag": i(), "status": i(),
            "count": torch.zeros(12, dtype=torch.int32, device=dev), "total": torch.zeros(12, dtype=torch.int64, device=dev)}  # fmt: skip


def c_call(entry, solver, inp, out, B=None):
    """One call of mx_call or mx_call_static through ctypes on device tensors; returns (status, message)."""
    p = lambda t: t.data_ptr()
    err = ctypes.create_string_buffer(ERRLEN)
    x, T, P, dt, h, J = inp
    rc = entry(solver._handle, p(x), p(T), p(P), p(dt), p(h), p(J), x.shape[0] if B is None else B, 1e-3, 1e-25,
               4000, p(out["x"]), p(out["h"]), p(out["done"]), p(out["steps"]), p(out["flag"]), p(out["status"]),
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
    with CudaSolver(net, gpu, photo=True) as solver:
        ns = solver.ns
        inp_a = inp_b = (t(w.x), t(w.T), t(w.P), t(w.dt), t(w.h), t(w.J))
        for k in range(2):  # two calls in a row: a cold start, then a settling call from its results
            ref, got = outputs(B, ns, gpu), outputs(B, ns, gpu)
            rc, msg = c_call(lib.mx_call, solver, inp_a, ref)
            assert rc == 0, msg
            rc, msg = c_call(lib.mx_call_static, solver, inp_b, got)
            assert rc == 0, msg
            torch.cuda.synchronize(gpu)
            r, g = host(ref), host(got)
            assert np.array_equal(g["status"], r["status"]) and np.array_equal(g["done"], r["done"])
            assert np.array_equal(g["flag"], r["flag"]) and np.array_equal(g["steps"], r["steps"])
            assert np.array_equal(g["count"], r["count"]) and np.array_equal(g["total"], r["total"])
            big = (np.abs(r["x"]) > parity.FLOOR) & (np.abs(g["x"]) > parity.FLOOR)
            rel = np.abs(g["x"] - r["x"])[big] / np.abs(r["x"])[big]
            assert rel.max(initial=0.0) <= parity.RTOL, (k, rel.max())
            assert np.allclose(g["h"], r["h"], rtol=parity.H_RTOL, atol=0)
            inp_a = (ref["x"], inp_a[1], inp_a[2], inp_a[3], ref["h"], inp_a[5])
            inp_b = (got["x"], inp_b[1], inp_b[2], inp_b[3], got["h"], inp_b[5])


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
