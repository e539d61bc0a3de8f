"""The CUDA path against the CPU oracle on the synthetic networks: same inputs, same method.

A settled GCM call (a few steps) must agree to RTOL = 1e-9 per species above 1e-20 on at least 99% of the cells
whose steps match (none beyond 1e-8), with identical statuses, flags and counts. A cold start or a 1e10 s dark call amplifies last-bit differences through hundreds of stiff steps; there the
bar is the oracle's own response to a one-ulp change of T (parity.passed_calibrated).
"""

import numpy as np
import pytest
import torch

import oracle
import parity
from maxichem_b200 import synthetic
from maxichem_b200.solver import CudaSolver

pytestmark = pytest.mark.gpu


def run_both(net, w, device, calls=1, photo=True, rtol=1e-3, atol=1e-25, max_steps=4000, drift=None, forcing=None):
    """Chain calls on the GPU and on the oracle from the same inputs; each call starts both sides from the oracle's
    previous result. forcing: (dt, J) per call (default `calls` calls of w.dt and w.J). Returns, per call, the
    GPU-oracle report and the oracle's one-ulp self-report."""
    solver = CudaSolver(net, device, photo=photo, drift=drift)
    ref = oracle.Oracle(solver.tab, drift=solver.drift)
    x, h = w.x.copy(), w.h.copy()
    out_reports = []
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=device)
    kw = dict(rtol=rtol, atol=atol, max_steps=max_steps)
    for dt, Jc in forcing or [(w.dt, w.J)] * calls:
        J = t(Jc) if photo else None
        out = solver.launch_raw(t(x), t(w.T), t(w.P), t(dt), t(h), J=J, **kw)
        g = {k: v.cpu().numpy() for k, v in out.items()}
        g["done"] = g["done"].astype(bool)
        g["count"] = solver.count.cpu().numpy()
        Jh = Jc if photo else None
        r = ref.call(x, w.T, w.P, dt, h, J=Jh, **kw)
        nudged = ref.call(x, np.nextafter(w.T, np.inf), w.P, dt, h, J=Jh, **kw)
        out_reports.append((parity.compare(g, r, x, net.atoms), parity.compare(nudged, r, x, net.atoms)))
        x, h = r["x"], r["h"]
    solver.close()
    return out_reports


@pytest.mark.parametrize("name,cells", [("cho41", 512), ("chno69", 256), ("sncho91", 128)])
def test_gcm_calls_match_the_oracle(gpu, networks, name, cells):
    # 300 s calls on the column grid with upper-layer J: a cold start from solar gas, then two settling calls
    net = networks(name)
    w = synthetic.workload(net, "column", cells, seed=1)
    reports = run_both(net, w, gpu, calls=3)
    for k, (rep, floor) in enumerate(reports):
        print(name, k, rep, "one-ulp floor:", {q: floor[q] for q in ("worst_rel", "share_within_rtol", "flips")})
        assert parity.passed_calibrated(rep, floor), rep
    for rep, _ in reports[1:]:  # settled calls: the strict bar
        assert parity.passed(rep), rep


def test_long_dark_call_matches_the_oracle(gpu, networks):
    # the 41-species network's first call: 512 cells, T 500-2500 K, P 1e-2..1e8, dark, dt 1e10 s from solar gas
    net = networks("cho41")
    w = synthetic.workload(net, "cfg0", 512, seed=1)
    ((rep, floor),) = run_both(net, w, gpu, calls=1)
    print("cho41 cfg0", rep, "one-ulp floor:", floor)
    assert parity.passed_calibrated(rep, floor), rep


def test_the_cpu_configuration_matches_the_oracle(gpu, networks):
    # the 41-species network's CPU-runnable case: 512 cells, T 500-2500 K, P 1e-2..1e8, one dark 1e10 s call from
    # solar gas, then five 300 s calls with J log-uniform in 1e-10..1e-3 s^-1 where P < 1e3 dyn cm^-2
    net = networks("cho41")
    w = synthetic.workload(net, "cfg0", 512, seed=1)
    J = synthetic.photolysis_rates(w.P, len(net.photo), np.random.default_rng(2))
    forcing = [(w.dt, np.zeros_like(J))] + [(np.full(512, 300.0), J)] * 5
    reports = run_both(net, w, gpu, forcing=forcing)
    for k, (rep, floor) in enumerate(reports):
        print("cho41 cpu case call", k, rep, "one-ulp floor:", {q: floor[q] for q in ("worst_rel", "share_within_rtol")})
        assert parity.passed_calibrated(rep, floor), (k, rep)
        if k > 0:  # the lit 300 s calls after the dark one: the strict bar
            assert parity.passed(rep), (k, rep)


def test_the_sulfur_network_over_600_s_calls(gpu, networks):
    # the 91-species network on 256 cells of the column grid, two 600 s calls: a cold start, then a settling call
    net = networks("sncho91")
    w = synthetic.workload(net, "column", 256, seed=4)
    dt = np.full(256, 600.0)
    reports = run_both(net, w, gpu, forcing=[(dt, w.J)] * 2)
    for k, (rep, floor) in enumerate(reports):
        print("sncho91 600 s call", k, rep, "one-ulp floor:", {q: floor[q] for q in ("worst_rel", "share_within_rtol")})
        assert parity.passed_calibrated(rep, floor), (k, rep)
    assert parity.passed(reports[1][0]), reports[1][0]


@pytest.mark.parametrize("name,dt", [("chno69", 300.0), ("sncho91", 600.0)])
def test_a_4096_cell_sample_of_the_configuration_grid(gpu, networks, name, dt):
    # every 16th cell of a 65,536-cell column grid (64 levels x 1,024 columns: the 69-species configuration's grid;
    # the sulfur configuration's calls are 600 s): a cold start from solar gas, then two settling calls
    net = networks(name)
    full = synthetic.workload(net, "column", 65536, seed=7)
    pick = np.arange(0, 65536, 16)
    w = synthetic.Workload(full.x[pick], full.T[pick], full.P[pick], np.full(len(pick), dt), full.h[pick],
                           full.J[pick])  # fmt: skip
    reports = run_both(net, w, gpu, calls=3)
    for k, (rep, floor) in enumerate(reports):
        print(name, "4096-cell sample, call", k, {q: rep[q] for q in ("share_within_rtol", "worst_rel", "flips",
                                                                        "flip_dex", "share_rel")},
              "one-ulp floor:", {q: floor[q] for q in ("worst_rel", "share_within_rtol", "flips")})  # fmt: skip
        assert parity.passed_calibrated(rep, floor), (k, rep)
    for rep, _ in reports[1:]:
        assert parity.passed(rep), rep
        assert parity.passed_strict(rep), rep
