"""The CPU oracle pinned: rate coefficients against the reference tests' written-out laws, the recovery's dense LU
against the reference test's threshold-pivoting rule, and whole calls against answers known without the solver."""

import json
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

import invented
import oracle
from maxichem_b200 import synthetic, tables

GOLDEN = Path(__file__).parent / "golden"
P_TEST = 1e6  # dyn cm^-2
T_TEST = 1500.0  # K


@pytest.mark.parametrize("name", list(synthetic.NETWORKS))
def test_rates_match_the_written_out_laws(networks, name):
    g = np.load(GOLDEN / "rates.npz")
    tab = tables.build(networks(name), False)
    ref = oracle.Oracle(tab)
    for c, (T, P) in enumerate(g["conditions"]):
        kf, kr = ref.rates(float(T), float(P))
        for mine, want in ((kf, g[f"{name}/kf"][c]), (kr, g[f"{name}/kr"][c])):
            big = np.abs(want) > 1e-300
            rel = np.abs(mine - want)[big] / np.abs(want[big])
            assert rel.max() < 1e-11, (T, P, rel.max())
            assert np.array_equal(mine[~big] == 0, want[~big] == 0)


def test_dense_lu_pivots_by_the_threshold_rule():
    g = np.load(GOLDEN / "dense_lu.npz")
    for a, factors, order in zip(g["a"], g["factors"], g["orders"]):
        f, dinv, pr = oracle.dense_lu(a)
        assert pr.tolist() == order.tolist()
        assert np.allclose(f, factors, rtol=1e-10, atol=1e-10 * np.abs(factors).max())
        assert np.array_equal(dinv, 1.0 / np.diag(f))
        y = np.random.default_rng(0).standard_normal(len(a))
        x = oracle.dense_solve(f, dinv, pr, y)
        assert np.abs(a @ x - y).max() < 1e-9 * np.abs(y).max() * np.abs(a).max() * len(a)
    assert oracle.dense_lu(g["a"][-1])[2][0] == 3  # a tie for the largest |entry| goes to the lower row


def _one(net, photo=True):
    return oracle.Oracle(tables.build(net, photo))


def test_photolysis_decay_at_constant_pressure(tmp_path):
    net = invented.decay(tmp_path)
    times = np.array([0.1, 0.5, 1.0, 2.0])
    J = np.full((4, 1), 2.0)
    x0 = invented.state(net, 4, N2_1=1.0)
    r = _one(net).call(x0, np.full(4, T_TEST), np.full(4, P_TEST), times, 1e-6 * np.ones(4), rtol=1e-6, J=J)
    a, b = invented.decay_answer(2.0 * times)
    assert r["done"].all()
    assert np.allclose(r["x"][:, net.species.index("N2_1")], a, rtol=2e-5, atol=0)
    assert np.allclose(r["x"][:, net.species.index("N_1")], b, rtol=2e-5, atol=0)


@pytest.mark.parametrize("T", [800.0, 1500.0, 2500.0])
def test_long_call_reaches_the_nasa9_equilibrium(tmp_path, T):
    net, thermo = invented.hydrogen(tmp_path)
    x0 = invented.state(net, 2, H=0.1, H2=0.6, OH=0.05, H2O=0.1, O=0.05, He=0.1)
    P = 1e7
    r = _one(net, photo=False).call(x0, np.full(2, T), np.full(2, P), np.full(2, 1e10), np.full(2, 1e-10))
    assert r["done"].all()
    x = {q: r["x"][0, net.species.index(q)] for q in ("H", "H2", "OH", "O", "H2O")}
    g = {q: invented.gibbs_rt(thermo[q], T) for q in x}
    assert x["H2"] * x["O"] / (x["H"] * x["OH"]) == pytest.approx(np.exp(-(g["H2"] + g["O"] - g["H"] - g["OH"])), rel=1e-12)
    assert x["OH"] * x["H2"] / (x["H"] * x["H2O"]) == pytest.approx(np.exp(-(g["OH"] + g["H2"] - g["H"] - g["H2O"])), rel=1e-12)
    k3 = np.exp(-(g["H2"] - 2.0 * g["H"])) * P / invented.STANDARD_PRESSURE
    assert x["H2"] / x["H"] ** 2 == pytest.approx(k3, rel=1e-12)


def test_recombination_at_constant_pressure(tmp_path):
    net, _ = invented.recombination(tmp_path)
    left = np.array([0.8, 0.5, 0.3])
    t = invented.recombination_time(left, P_TEST)
    r = _one(net, photo=False).call(invented.state(net, 3, H=1.0), np.full(3, invented.RECOMBINATION_T),
                                    np.full(3, P_TEST), t, 1e-3 * t, rtol=1e-8)  # fmt: skip
    assert r["done"].all()
    assert np.allclose(r["x"][:, net.species.index("H")], 2.0 * left / (1.0 + left), rtol=1e-6, atol=0)


PHOTOLYSIS = """# Invented: three absorbers, one with two branches; thermal rows of zero rate
# Two-body Reactions
1 [ N2_1 + N_1 -> N_1 + N2_1 ] 0.0 0.0 0.0
3 [ N2_2 + N_2 -> N_2 + N2_2 ] 0.0 0.0 0.0
5 [ N2_3 + N_3 -> N_3 + N2_3 ] 0.0 0.0 0.0
7 [ N2_3 + N_4 -> N_4 + N2_3 ] 0.0 0.0 0.0

# reverse stops
# photo disscoiation (no reversals)
9 [ N2_1 -> N_1 + N_1 ] N2_1 1
11 [ N2_2 -> N_2 + N_2 ] N2_2 1
13 [ N2_3 -> N_3 + N_3 ] N2_3 1
15 [ N2_3 -> N_4 + N_4 ] N2_3 2
"""
BRANCHES = {("N2_1", 1): (0.7, "N_1"), ("N2_2", 1): (2.3, "N_2"), ("N2_3", 1): (0.4, "N_3"), ("N2_3", 2): (1.1, "N_4")}
ABSORBED = {"N2_1": 0.3, "N2_2": 0.3, "N2_3": 0.4}


def photolysis_answer(t):
    n = {}
    for absorber, n0 in ABSORBED.items():
        total = sum(j for (a, _), (j, _) in BRANCHES.items() if a == absorber)
        n[absorber] = n0 * np.exp(-total * t)
        for (a, _), (j, product) in BRANCHES.items():
            if a == absorber:
                n[product] = 2.0 * n0 * j / total * (1.0 - np.exp(-total * t))
    s = sum(n.values())
    return {q: v / s for q, v in n.items()}


def photolysis_network(folder):
    thermo = {q: invented.constant_cp(0.0) for q in ("N2_1", "N_1", "N2_2", "N_2", "N2_3", "N_3", "N_4", "He")}
    return invented.write(folder, PHOTOLYSIS, thermo)


def test_each_photolysis_branch_takes_its_own_rate(tmp_path):
    net = photolysis_network(tmp_path)
    times = np.array([0.3, 1.0, 3.0])
    J = np.array([[BRANCHES[(r["absorber"], r["branch"])][0] for r in net.photo]] * 3)
    x0 = invented.state(net, 3, **ABSORBED)
    r = _one(net).call(x0, np.full(3, T_TEST), np.full(3, P_TEST), times, 1e-6 * times, rtol=1e-8, J=J)
    assert r["done"].all()
    for c, t in enumerate(times):
        for q, want in photolysis_answer(t).items():
            assert r["x"][c, net.species.index(q)] == pytest.approx(want, rel=1e-6)


def test_one_rodas3_step_is_the_exact_rational_one(tmp_path):
    # one step of A -> 2 B from (1, 0) at J h = 1/10, exactly in rationals (golden), against the oracle's single try
    g = json.loads((GOLDEN / "first_trial.json").read_text())
    new = [Fraction(*q) for q in g["new"]]
    z = Fraction(*g["z"])
    net = invented.decay(tmp_path)
    J = 2.0
    dt = float(z) / J
    x0 = invented.state(net, 1, N2_1=1.0)
    r = _one(net).call(x0, np.full(1, T_TEST), np.full(1, P_TEST), np.full(1, dt), np.full(1, dt), rtol=1e6,
                       max_steps=1, J=np.full((1, 1), J))  # fmt: skip
    assert r["done"].all() and r["steps"][0] == 1.0
    total = new[0] + new[1]
    assert r["x"][0, net.species.index("N2_1")] == pytest.approx(float(new[0] / total), rel=1e-14)
    assert r["x"][0, net.species.index("N_1")] == pytest.approx(float(new[1] / total), rel=1e-14)


def test_rodas3_is_third_order(tmp_path):
    net = invented.decay(tmp_path)
    o = _one(net)
    a = net.species.index("N2_1")
    errors = []
    for steps in (4, 8, 16, 32):
        dt = 1.0 / steps
        x = invented.state(net, 1, N2_1=1.0)
        for _ in range(steps):
            r = o.call(x, np.full(1, T_TEST), np.full(1, P_TEST), np.full(1, dt), np.full(1, dt), rtol=1e6,
                       J=np.full((1, 1), 1.0))  # fmt: skip
            assert r["done"].all() and r["steps"][0] == 1.0
            x = r["x"]
        errors.append(abs(x[0, a] - invented.decay_answer(1.0)[0]))
    slope = np.polyfit(np.log(1.0 / np.array([4, 8, 16, 32])), np.log(errors), 1)[0]
    assert 2.7 <= slope <= 3.3, (errors, slope)


def test_a_rejected_first_try_is_retried(tmp_path):
    net = invented.decay(tmp_path)
    o = _one(net)
    J = np.full((1, 1), 2.0)
    dt = np.full(1, 5.0 / 2.0)  # J dt = 5: a first try of h = dt is rejected
    x0 = invented.state(net, 1, N2_1=1.0)
    args = (x0, np.full(1, T_TEST), np.full(1, P_TEST), dt, dt.copy())
    r = o.call(*args, rtol=1e-6, J=J)
    steps = int(r["steps"][0])
    assert r["done"].all()
    assert r["x"][0, net.species.index("N2_1")] == pytest.approx(invented.decay_answer(5.0)[0], rel=2e-5)
    short = o.call(*args, rtol=1e-6, J=J, max_steps=steps)
    assert short["count"][5] == 1  # unfinished at max_steps = the accepted steps: some try was rejected


def test_screening_refuses_bad_cells_and_counts_them(networks):
    net = networks("cho41")
    o = _one(net)
    w = synthetic.workload(net, "column", 8, seed=5)
    x, T, P, dt, h = w.x.copy(), w.T.copy(), w.P.copy(), w.dt.copy(), w.h.copy()
    x[0, 0] = np.nan
    x[1] *= 0.9
    T[2], T[3] = 250.0, 3000.5
    P[4] = 0.0
    dt[5] = -1.0
    h[6] = np.inf
    r = o.call(x, T, P, dt, h, J=w.J)
    assert r["status"].tolist() == [2, 2, 1, 3, 2, 2, 0, 0]
    c = r["count"]
    assert (c[1], c[2], c[3], c[10]) == (4, 1, 1, 1)
    assert not r["done"][:6].any() and r["done"][6:].all()
