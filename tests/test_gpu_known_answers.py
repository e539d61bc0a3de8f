"""The CUDA path through the public CudaSolver against answers known without the solver (the reference's
tests/test_known_answers.py and tests/test_order.py on the GPU): photolysis decay, NASA-9 equilibria, recombination,
photolysis branches, the exact first Rodas3 trial, third order, and a rejected first try."""

import json
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest
import torch

import invented
import test_oracle
from maxichem_b200.solver import CudaSolver

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).parent / "golden"
P_TEST, T_TEST = 1e6, 1500.0


def call(solver, dev, x, T, P, dt, h, J=None, **kw):
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    Jt = None if J is None else t(J)
    r = solver.launch(t(x), t(T), t(P), t(dt), t(h), J=Jt, **kw)
    out = {k: getattr(r, k).cpu().numpy() for k in r._fields}
    out["count"] = solver.count.cpu().numpy()
    return out


def test_photolysis_decay_at_constant_pressure(gpu, tmp_path):
    net = invented.decay(tmp_path)
    times = np.array([0.1, 0.5, 1.0, 2.0])
    with CudaSolver(net, gpu, photo=True) as s:
        r = call(s, gpu, invented.state(net, 4, N2_1=1.0), np.full(4, T_TEST), np.full(4, P_TEST), times,
                 1e-6 * np.ones(4), J=np.full((4, 1), 2.0), rtol=1e-6)  # fmt: skip
    a, b = invented.decay_answer(2.0 * times)
    assert r["done"].all()
    assert np.allclose(r["x"][:, net.species.index("N2_1")], a, rtol=2e-5, atol=0)
    assert np.allclose(r["x"][:, net.species.index("N_1")], b, rtol=2e-5, atol=0)


@pytest.mark.parametrize("T", [800.0, 1500.0, 2500.0])
def test_long_call_reaches_the_nasa9_equilibrium(gpu, tmp_path, T):
    net, thermo = invented.hydrogen(tmp_path)
    x0 = invented.state(net, 2, H=0.1, H2=0.6, OH=0.05, H2O=0.1, O=0.05, He=0.1)
    P = 1e7
    with CudaSolver(net, gpu) as s:
        r = call(s, gpu, x0, np.full(2, T), np.full(2, P), np.full(2, 1e10), np.full(2, 1e-10))
    assert r["done"].all()
    x = {q: r["x"][0, net.species.index(q)] for q in ("H", "H2", "OH", "O", "H2O")}
    g = {q: invented.gibbs_rt(thermo[q], T) for q in x}
    assert x["H2"] * x["O"] / (x["H"] * x["OH"]) == pytest.approx(np.exp(-(g["H2"] + g["O"] - g["H"] - g["OH"])), rel=1e-12)
    assert x["OH"] * x["H2"] / (x["H"] * x["H2O"]) == pytest.approx(np.exp(-(g["OH"] + g["H2"] - g["H"] - g["H2O"])), rel=1e-12)
    k3 = np.exp(-(g["H2"] - 2.0 * g["H"])) * P / invented.STANDARD_PRESSURE
    assert x["H2"] / x["H"] ** 2 == pytest.approx(k3, rel=1e-12)


def test_recombination_at_constant_pressure(gpu, tmp_path):
    net, _ = invented.recombination(tmp_path)
    left = np.array([0.8, 0.5, 0.3])
    t = invented.recombination_time(left, P_TEST)
    with CudaSolver(net, gpu) as s:
        r = call(s, gpu, invented.state(net, 3, H=1.0), np.full(3, invented.RECOMBINATION_T), np.full(3, P_TEST), t,
                 1e-3 * t, rtol=1e-8)  # fmt: skip
    assert r["done"].all()
    assert np.allclose(r["x"][:, net.species.index("H")], 2.0 * left / (1.0 + left), rtol=1e-6, atol=0)


def test_each_photolysis_branch_takes_its_own_rate(gpu, tmp_path):
    net = test_oracle.photolysis_network(tmp_path)
    times = np.array([0.3, 1.0, 3.0])
    J = np.array([[test_oracle.BRANCHES[(r["absorber"], r["branch"])][0] for r in net.photo]] * 3)
    with CudaSolver(net, gpu, photo=True) as s:
        r = call(s, gpu, invented.state(net, 3, **test_oracle.ABSORBED), np.full(3, T_TEST), np.full(3, P_TEST),
                 times, 1e-6 * times, J=J, rtol=1e-8)  # fmt: skip
    assert r["done"].all()
    for c, t in enumerate(times):
        for q, want in test_oracle.photolysis_answer(t).items():
            assert r["x"][c, net.species.index(q)] == pytest.approx(want, rel=1e-6)


def test_one_rodas3_step_is_the_exact_rational_one(gpu, tmp_path):
    g = json.loads((GOLDEN / "first_trial.json").read_text())
    new = [Fraction(*q) for q in g["new"]]
    z = Fraction(*g["z"])
    net = invented.decay(tmp_path)
    J = 2.0
    dt = float(z) / J
    with CudaSolver(net, gpu, photo=True) as s:
        r = call(s, gpu, invented.state(net, 1, N2_1=1.0), np.full(1, T_TEST), np.full(1, P_TEST), np.full(1, dt),
                 np.full(1, dt), J=np.full((1, 1), J), rtol=1e6, max_steps=1)  # fmt: skip
    assert r["done"].all() and r["steps"][0] == 1.0
    total = new[0] + new[1]
    assert r["x"][0, net.species.index("N2_1")] == pytest.approx(float(new[0] / total), rel=1e-14)
    assert r["x"][0, net.species.index("N_1")] == pytest.approx(float(new[1] / total), rel=1e-14)


def test_rodas3_is_third_order(gpu, tmp_path):
    net = invented.decay(tmp_path)
    a = net.species.index("N2_1")
    errors = []
    with CudaSolver(net, gpu, photo=True) as s:
        for steps in (4, 8, 16, 32):
            dt = 1.0 / steps
            x = invented.state(net, 1, N2_1=1.0)
            for _ in range(steps):
                r = call(s, gpu, x, np.full(1, T_TEST), np.full(1, P_TEST), np.full(1, dt), np.full(1, dt),
                         J=np.full((1, 1), 1.0), rtol=1e6)  # fmt: skip
                assert r["done"].all() and r["steps"][0] == 1.0
                x = r["x"]
            errors.append(abs(x[0, a] - invented.decay_answer(1.0)[0]))
    slope = np.polyfit(np.log(1.0 / np.array([4, 8, 16, 32])), np.log(errors), 1)[0]
    assert 2.7 <= slope <= 3.3, (errors, slope)


def test_a_rejected_first_try_is_retried(gpu, tmp_path):
    net = invented.decay(tmp_path)
    J = np.full((1, 1), 2.0)
    dt = np.full(1, 5.0 / 2.0)  # J dt = 5: a first try of h = dt is rejected
    args = (invented.state(net, 1, N2_1=1.0), np.full(1, T_TEST), np.full(1, P_TEST), dt, dt.copy())
    with CudaSolver(net, gpu, photo=True) as s:
        r = call(s, gpu, *args, J=J, rtol=1e-6)
        steps = int(r["steps"][0])
        short = call(s, gpu, *args, J=J, rtol=1e-6, max_steps=steps)
    assert r["done"].all()
    assert r["x"][0, net.species.index("N2_1")] == pytest.approx(invented.decay_answer(5.0)[0], rel=2e-5)
    assert short["count"][5] == 1  # unfinished at max_steps = the accepted steps: some try was rejected
