"""The CUDA path against the CPU oracle on the synthetic networks: same inputs, same method, parity within RTOL."""

import numpy as np
import pytest
import torch

import oracle
import parity
from maxichem_b200 import synthetic
from maxichem_b200.solver import CudaSolver

pytestmark = pytest.mark.gpu


def run_both(net, w, device, calls=1, photo=True, rtol=1e-3, atol=1e-25, max_steps=4000, drift=None):
    """Chain `calls` calls on the GPU and on the oracle from the same inputs; each call starts both sides from the
    oracle's previous result. Returns one parity report per call."""
    solver = CudaSolver(net, device, photo=photo, drift=drift)
    ref = oracle.Oracle(solver.tab, drift=solver.drift)
    x, h = w.x.copy(), w.h.copy()
    reports = []
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=device)
    for _ in range(calls):
        J = t(w.J) if photo else None
        out = solver.launch_raw(t(x), t(w.T), t(w.P), t(w.dt), t(h), J=J, rtol=rtol, atol=atol, max_steps=max_steps)
        g = {k: v.cpu().numpy() for k, v in out.items()}
        g["done"] = g["done"].astype(bool)
        g["count"] = solver.count.cpu().numpy()
        r = ref.call(x, w.T, w.P, w.dt, h, J=w.J if photo else None, rtol=rtol, atol=atol, max_steps=max_steps)
        reports.append(parity.compare(g, r, x, net.atoms))
        x, h = r["x"], r["h"]
    solver.close()
    return reports


@pytest.mark.parametrize("name,cells", [("cho41", 512), ("chno69", 256), ("sncho91", 128)])
def test_gcm_calls_match_the_oracle(gpu, networks, name, cells):
    # 300 s calls on the column grid with upper-layer J: a cold start from solar gas, then a settling call
    net = networks(name)
    w = synthetic.workload(net, "column", cells, seed=1)
    for rep in run_both(net, w, gpu, calls=2):
        print(name, rep)
        assert parity.passed(rep), rep


def test_long_dark_call_matches_the_oracle(gpu, networks):
    # the 41-species network's first call: 512 cells, T 500-2500 K, P 1e-2..1e8, dark, dt 1e10 s from solar gas
    net = networks("cho41")
    w = synthetic.workload(net, "cfg0", 512, seed=1)
    (rep,) = run_both(net, w, gpu, calls=1)
    print("cho41 cfg0", rep)
    assert parity.passed_long(rep), rep
