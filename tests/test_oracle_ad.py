"""The tangent oracle (oracle/mx_oracle_ad.c) pinned before it checks the CUDA tangent.

Its primal must be the primal oracle's bit for bit (dual numbers carry the same value operations), and its tangent the
derivative of that primal: central differences of the oracle's own call judge it the way the reference judges its
tangent kernels (tests/test_ad.py of imalsky/maxichem: per cell the best error over a plateau of step sizes, the
log-x tangent of species above 1e-20, p90 within 1e-4 and the worst within 1e-2).
"""

import numpy as np
import pytest

from maxichem_b200 import synthetic, tables
from maxichem_b200.constants import COUNTS
from oracle import Oracle

FD_STEPS = (1e-4, 1e-5, 1e-6, 1e-7)
FD_P90 = 1e-4
FD_P90_H = 1e-3  # the starting step: its tangent reaches x only through the step control, so differences are noisy
FD_MAX = 1e-2
FD_COVERAGE = 0.75  # share of judged cells with a plateau (the start-step class sits near step-count branches)
SCALING_TANGENT = 1e-12  # relative to max x: the frozen tangent along x itself is 0 but rounding


@pytest.fixture(scope="module")
def case():
    net = synthetic.network("cho41")
    tab = tables.build(net, True, warps=4)
    w = synthetic.workload(net, "column", 256, seed=1)
    sel = np.arange(0, 256, 16)
    B = len(sel)
    rng = np.random.default_rng(5)
    return {
        "o": Oracle(tab), "tab": tab, "x": w.x[sel], "T": w.T[sel], "P": w.P[sel], "dt": np.full(B, 100.0),
        "h": np.full(B, 1e-10), "J": w.J[sel], "lm": 0.1 * rng.standard_normal((B, tab.nr)),
    }  # fmt: skip


def test_primal_is_the_oracle_call(case):
    o = case["o"]
    ref = o.call(case["x"], case["T"], case["P"], case["dt"], case["h"], J=case["J"])
    for adapt in (True, False):
        B, ns = case["x"].shape
        r = o.jvp(case["x"], case["T"], case["P"], case["dt"], case["h"], np.ones((1, B, ns)), J=case["J"],
                  adapt=adapt)  # fmt: skip
        for k in ("x", "h", "done", "steps", "flag", "status", "count"):
            assert np.array_equal(ref[k], r[k]), k


def _tangent_case(case, cls, seed):
    o, tab = case["o"], case["tab"]
    x, T, P, dt, h, J, lm = (case[k] for k in ("x", "T", "P", "dt", "h", "J", "lm"))
    B, ns = x.shape
    rng = np.random.default_rng(seed)
    t = {"dx": np.zeros((B, ns)), "dT": np.zeros(B), "dP": np.zeros(B), "ddt": np.zeros(B), "dh": np.zeros(B),
         "dlm": np.zeros((B, tab.nr)), "dJ": np.zeros(J.shape), "drc": np.zeros((tab.nr, 9))}  # fmt: skip
    if cls == "x":  # along sum(x) = 1: the call refuses a state off it
        d = x * rng.standard_normal(x.shape)
        t["dx"] = d - x * d.sum(1, keepdims=True)
    elif cls == "T":
        room = np.minimum(T - 300.0, 3000.0 - T) / FD_STEPS[0]
        t["dT"] = np.clip(T * rng.standard_normal(B), -room, room)
    elif cls == "P":
        t["dP"] = P * rng.standard_normal(B)
    elif cls == "dt":
        t["ddt"] = dt * rng.standard_normal(B)
    elif cls == "h":
        t["dh"] = h * rng.standard_normal(B)
    elif cls == "lm":
        t["dlm"] = rng.standard_normal((B, tab.nr))
    elif cls == "J":
        t["dJ"] = J * rng.standard_normal(J.shape)
    elif cls == "rc":
        t["drc"] = rng.standard_normal((tab.nr, 9)) * np.array([1.0, 0.1, 30.0] * 3)
    r = o.jvp(x, T, P, dt, h, *(t[k][None] for k in ("dx", "dT", "dP", "ddt", "dh")), lm=lm, dlm=t["dlm"][None],
              drc=t["drc"][None], J=J, dJ=t["dJ"][None])  # fmt: skip
    x1, k1 = r["x"], r["steps"]
    adl = r["dx"][0] / x1
    big = x1 > 1e-20
    fds, ks = [], []
    for e in FD_STEPS:
        side = []
        for sg in (1.0, -1.0):
            rc = tab.rc.copy()
            rc[:, :9] += sg * e * t["drc"]
            q = o.jvp(x + sg * e * t["dx"], T + sg * e * t["dT"], P + sg * e * t["dP"], dt + sg * e * t["ddt"],
                      h + sg * e * t["dh"], J=J + sg * e * t["dJ"], lm=lm + sg * e * t["dlm"], rc=rc)  # fmt: skip
            side.append((q["x"], q["steps"]))
        (xp, kp), (xm, km) = side
        fds.append((np.log(xp.clip(1e-300)) - np.log(xm.clip(1e-300))) / (2 * e))
        ks.append(np.where(kp == km, kp, -1))

    def mx(a):
        return np.where(big, np.abs(a), 0.0).max(1)

    S = np.maximum(mx(adl), np.max([mx(f) for f in fds], 0))
    best = np.full(B, np.inf)
    for q in range(len(fds) - 1):
        same = (ks[q] == k1) & (ks[q + 1] == k1)
        agree = mx(fds[q] - fds[q + 1]) <= 1e-2 * S
        for f in (fds[q], fds[q + 1]):
            best = np.where(same & agree, np.minimum(best, mx(f - adl) / S.clip(1e-300)), best)
    judged = S > 1e-6
    if cls == "J":
        judged &= (J > 0).any(1)
    return best[judged], int(judged.sum()), r


@pytest.mark.parametrize("cls", ["x", "T", "P", "dt", "h", "lm", "J", "rc"])
def test_tangent_against_differences(case, cls):
    errors, judged, r = _tangent_case(case, cls, 11)
    fin = errors[np.isfinite(errors)]
    assert judged >= 8 and np.isfinite(r["dx"]).all() and (r["flag"] != 2).all()
    assert len(fin) >= FD_COVERAGE * judged, (cls, len(fin), judged)
    p90 = FD_P90_H if cls == "h" else FD_P90
    assert np.quantile(fin, 0.9) <= p90 and fin.max() <= FD_MAX, (cls, np.quantile(fin, 0.9), fin.max())


def test_frozen_tangent_along_x_itself_is_zero(case):
    # the right-hand side is homogeneous of degree 1 in N: with the try sizes held, N -> c N scales every stage
    o = case["o"]
    r = o.jvp(case["x"], case["T"], case["P"], case["dt"], case["h"], case["x"][None], J=case["J"], adapt=False)
    worst = (np.abs(r["dx"][0]).max(1) / np.abs(r["x"]).max(1)).max()
    assert worst <= SCALING_TANGENT
    assert (r["dh"] == 0.0).all()  # the frozen contract gives h_out no tangent


def test_directions_share_one_call(case):
    o, tab = case["o"], case["tab"]
    x, T, P, dt, h, J, lm = (case[k] for k in ("x", "T", "P", "dt", "h", "J", "lm"))
    B, ns = x.shape
    rng = np.random.default_rng(2)
    tan = [rng.standard_normal((3, B, ns)) * x, rng.standard_normal((3, B)), rng.standard_normal((3, B)) * P,
           rng.standard_normal((3, B)), rng.standard_normal((3, B)) * h]  # fmt: skip
    dlm = rng.standard_normal((3, B, tab.nr))
    together = o.jvp(x, T, P, dt, h, *tan, lm=lm, dlm=dlm, J=J)
    for k in range(3):
        one = o.jvp(x, T, P, dt, h, *(a[k : k + 1] for a in tan), lm=lm, dlm=dlm[k : k + 1], J=J)
        assert np.array_equal(one["dx"][0], together["dx"][k]) and np.array_equal(one["dh"][0], together["dh"][k])


def test_non_finite_step_acts_as_twice_dt(case):
    # a non-finite starting step acts as dt with no tangent of its own: min(h, dt) = dt at h = 2 dt too
    o = case["o"]
    x, T, P, dt, J = (case[k] for k in ("x", "T", "P", "dt", "J"))
    B, ns = x.shape
    rng = np.random.default_rng(3)
    tan = [x * rng.standard_normal((1, B, ns)), rng.standard_normal((1, B)), np.zeros((1, B)),
           dt * rng.standard_normal((1, B)), rng.standard_normal((1, B))]  # fmt: skip
    two = o.jvp(x, T, P, dt, 2.0 * dt, *tan, J=J)
    nan = o.jvp(x, T, P, dt, np.full(B, np.nan), *tan, J=J)
    for k in ("x", "h", "steps", "dx", "dh"):
        assert np.array_equal(two[k], nan[k]), k
    assert nan["count"][1 + COUNTS.index("nonfinite_h")] == B


def test_non_finite_log_multiplier_fails_the_cell(case):
    o, tab = case["o"], case["tab"]
    x, T, P, dt, h, J, lm = (case[k] for k in ("x", "T", "P", "dt", "h", "J", "lm"))
    B, ns = x.shape
    bad = lm.copy()
    bad[0, 0] = np.nan
    r = o.jvp(x, T, P, dt, h, x[None], lm=bad, J=J)
    good = o.jvp(x, T, P, dt, h, x[None], lm=lm, J=J)
    assert r["flag"][0] == 2 and r["steps"][0] == 0 and not r["done"][0] and np.isnan(r["dx"][0, 0]).all()
    for k in ("x", "h", "steps", "flag", "dx"):
        a, b = (r[k][:, 1:] if k == "dx" else r[k][1:]), (good[k][:, 1:] if k == "dx" else good[k][1:])
        assert np.array_equal(a, b), k


def test_no_multipliers_are_zero_multipliers(case):
    # lm None is lm = 0: the tangent along dlm still scales both directions of each reaction
    o, tab = case["o"], case["tab"]
    x, T, P, dt, h, J = (case[k] for k in ("x", "T", "P", "dt", "h", "J"))
    B = x.shape[0]
    dlm = np.random.default_rng(4).standard_normal((1, B, tab.nr))
    none = o.jvp(x, T, P, dt, h, dlm=dlm, J=J)
    zero = o.jvp(x, T, P, dt, h, dlm=dlm, lm=np.zeros((B, tab.nr)), J=J)
    for k in ("x", "h", "steps", "dx", "dh"):
        assert np.array_equal(none[k], zero[k]), k
    assert np.abs(none["dx"]).max() > 0.0


@pytest.fixture(scope="module")
def recovered():
    # cold starts with max_steps 20: the call leaves them unfinished, the guard lists them, and the recovery (dense
    # pivoted W, ten times the tries) redoes them, so the tangent runs along the recovery's path
    net = synthetic.network("cho41")
    tab = tables.build(net, True, warps=4)
    w = synthetic.workload(net, "column", 64, seed=3)
    x, h, _ = synthetic.cold_start(w.x, w.h, seed=4, share=0.3)
    sel = np.arange(0, 64, 4)
    rng = np.random.default_rng(5)
    return {
        "o": Oracle(tab), "tab": tab, "x": x[sel], "T": w.T[sel], "P": w.P[sel], "dt": np.full(len(sel), 100.0),
        "h": h[sel], "J": w.J[sel], "lm": 0.1 * rng.standard_normal((len(sel), tab.nr)),
    }  # fmt: skip


@pytest.mark.parametrize("cls", ["x", "T", "lm", "rc"])
def test_recovered_tangent_against_differences(recovered, cls, monkeypatch):
    o = recovered["o"]
    jvp = o.jvp
    monkeypatch.setattr(o, "jvp", lambda *a, **k: jvp(*a, max_steps=20, **k))
    errors, judged, r = _tangent_case(recovered, cls, 13)
    assert (r["flag"] == 1).sum() >= 12, r["flag"]
    fin = errors[np.isfinite(errors)]
    assert len(fin) >= FD_COVERAGE * judged and judged >= 8, (cls, len(fin), judged)
    assert np.quantile(fin, 0.9) <= FD_P90 and fin.max() <= FD_MAX, (cls, np.quantile(fin, 0.9), fin.max())


def test_frozen_contract_has_no_dt_or_h_tangent(case):
    # the frozen contract holds every accepted try's size: neither dt nor the starting step reaches x or h_out
    o = case["o"]
    x, T, P, dt, h, J = (case[k] for k in ("x", "T", "P", "dt", "h", "J"))
    B, ns = x.shape
    rng = np.random.default_rng(6)
    r = o.jvp(x, T, P, dt, h, np.zeros((2, B, ns)), np.zeros((2, B)), np.zeros((2, B)),
              np.stack([dt * rng.standard_normal(B), np.zeros(B)]), np.stack([np.zeros(B), h * rng.standard_normal(B)]),
              J=J, adapt=False)  # fmt: skip
    assert (r["dx"] == 0.0).all() and (r["dh"] == 0.0).all()
    a = o.jvp(x, T, P, dt, h, np.zeros((1, B, ns)), np.zeros((1, B)), np.zeros((1, B)),
              (dt * rng.standard_normal(B))[None], np.zeros((1, B)), J=J)  # fmt: skip
    assert np.abs(a["dx"]).max() > 0.0  # the adaptive contract has one
