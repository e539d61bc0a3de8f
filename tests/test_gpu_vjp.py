"""The adjoint (ADSolver.vjp) on the GPU: dot products against the tangent, and the reference's adjoint cases.

<c, J v> (the tangent, itself pinned against the tangent oracle by tests/test_gpu_jvp.py) against <J^T c, v> (the
adjoint) per cell and input class, with the bars of the reference's tests/test_ad.py (p99 within 1e-6, the log
multipliers' within 1e-4, the worst within 1e-3, the rate table's batch sum within 1e-7); then the primal, the
checkpoints, determinism, failed cells and refusals.
"""

import numpy as np
import pytest
import torch

from maxichem_b200 import synthetic
from maxichem_b200.ad import ADSolver
from maxichem_b200.solver import CudaSolver

pytestmark = pytest.mark.gpu

DOT_P99 = 1e-6
DOT_P99_LM = 1e-4  # a fast balanced reaction's multiplier changes nothing in exact arithmetic; this is its rounding
DOT_MAX = 1e-3
RC_BATCH = 1e-7  # relative: a sum over cells, reactions and columns
ULP_T = 2.220446049250313e-16
FLOOR_FACTOR = 100.0  # a long call's cell is judged against its tangent's own change under a one-ulp change of T
LONG_MEDIAN = 1e-8
CLASSES = ("x", "T", "P", "dt", "h", "lm", "J")


class Case:
    def __init__(self, net, dev, cells=64, seed=3, cap=100):
        self.dev = dev
        self.cs = CudaSolver(net, dev, photo=True)
        self.ad = ADSolver(net, dev, photo=True, cap=cap)
        w = synthetic.workload(net, "column", cells, seed=seed)
        self.x, self.h, _ = synthetic.cold_start(w.x, w.h, seed=seed + 1, share=0.3)
        self.T, self.P, self.J = w.T, w.P, w.J
        self.dt = np.full(cells, 100.0)
        self.B, self.ns, self.nr, self.nj = cells, self.cs.ns, self.cs.nr, self.cs.nj
        self.lm = 0.1 * np.random.default_rng(seed).standard_normal((cells, self.nr))

    def t(self, a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=self.dev)

    def inputs(self):
        return [self.t(a) for a in (self.x, self.T, self.P, self.dt, self.h)]

    def close(self):
        self.cs.close()
        self.ad.close()


@pytest.fixture(scope="module", params=["cho41", "chno69", "sncho91"])
def case(request, gpu, networks):
    c = Case(networks(request.param), gpu)
    yield c
    c.close()


def tangent(c, cls, rng):
    B, ns, nr, nj = c.B, c.ns, c.nr, c.nj
    z = {"dx": np.zeros((B, ns)), "dT": np.zeros(B), "dP": np.zeros(B), "ddt": np.zeros(B), "dh": np.zeros(B),
         "dlm": np.zeros((B, nr)), "dJ": np.zeros((B, nj)), "drc": np.zeros((nr, 9))}  # fmt: skip
    if cls == "x":
        z["dx"] = c.x * rng.standard_normal((B, ns))
    elif cls == "T":
        z["dT"] = c.T * rng.standard_normal(B)
    elif cls == "P":
        z["dP"] = c.P * rng.standard_normal(B)
    elif cls == "dt":
        z["ddt"] = c.dt * rng.standard_normal(B)
    elif cls == "h":
        z["dh"] = c.h * rng.standard_normal(B)
    elif cls == "lm":
        z["dlm"] = rng.standard_normal((B, nr))
    elif cls == "J":
        z["dJ"] = np.maximum(c.J, 1e-8) * rng.standard_normal((B, nj))
    elif cls == "rc":
        z["drc"] = rng.standard_normal((nr, 9)) * np.array([1.0, 0.1, 30.0] * 3)
    return z


def dot_errors(c, adapt, seed, floors=None, **kw):
    """Per class: the cells' relative errors of <c, J v> against <J^T c, v>, and the rate table's batch error. With a
    dict `floors`, also per class and judged cell the change of <c, J v> under a one-ulp change of T (relative, inf
    where the accepted steps moved): the tangent's own conditioning."""
    rng = np.random.default_rng(seed)
    B, ns = c.B, c.ns
    base = c.ad.jvp(*c.inputs(), c.t(np.zeros((B, ns))), *(c.t(np.zeros(B)) for _ in range(4)), lm=c.t(c.lm),
                    J=c.t(c.J), adapt=adapt, **kw)  # fmt: skip
    x1, h1 = base.x.cpu().numpy(), base.h.cpu().numpy()
    cx = np.where(x1 > 1e-20, rng.standard_normal((B, ns)) / np.maximum(x1, 1e-300), 0.0)
    ch = rng.standard_normal(B) / h1 if adapt else None
    v = c.ad.vjp(*c.inputs(), c.t(cx), gh=None if ch is None else c.t(ch), lm=c.t(c.lm), J=c.t(c.J), adapt=adapt,
                 **kw)  # fmt: skip
    flag = c.ad.flag.cpu().numpy()
    g = {k: (a.cpu().numpy() if a is not None else None) for k, a in v.cotangents._asdict().items()}
    out = {}
    for cls in (*CLASSES, "rc"):
        if cls in ("dt", "h") and not adapt:
            continue
        z = tangent(c, cls, rng)
        j = c.ad.jvp(*c.inputs(), *(c.t(z[k]) for k in ("dx", "dT", "dP", "ddt", "dh")), lm=c.t(c.lm),
                     dlm=c.t(z["dlm"]), drc=c.t(z["drc"]), J=c.t(c.J), dJ=c.t(z["dJ"]), adapt=adapt, **kw)  # fmt: skip
        assert np.array_equal(c.ad.flag.cpu().numpy(), flag)
        lt = cx * j.dx.cpu().numpy()
        if adapt:
            lt = np.concatenate([lt, (ch * j.dh.cpu().numpy())[:, None]], 1)
        if cls == "rc":
            keep = flag != 2
            left, right = lt[keep].sum(), (g["rc"] * z["drc"]).sum()
            out[cls] = abs(left - right) / max(abs(left), abs(right), 1e-300)
            continue
        rt = {"x": g["x"] * z["dx"], "T": (g["T"] * z["dT"])[:, None], "P": (g["P"] * z["dP"])[:, None],
              "dt": (g["dt"] * z["ddt"])[:, None], "h": (g["h"] * z["dh"])[:, None], "lm": g["lm"] * z["dlm"],
              "J": g["J"] * z["dJ"]}[cls]  # fmt: skip
        sc = np.maximum(np.abs(lt).sum(1), np.abs(rt).sum(1))
        e = np.abs(lt.sum(1) - rt.sum(1)) / np.maximum(sc, 1e-300)
        judged = (sc > 1e-10 * np.abs(cx * x1).sum(1)) & (flag != 2)
        assert np.isfinite(e[flag != 2]).all(), cls
        out[cls] = e[judged]
        if floors is not None:
            x, T, P, dt, h = c.inputs()
            q = c.ad.jvp(x, T * (1.0 + ULP_T), P, dt, h, *(c.t(z[k]) for k in ("dx", "dT", "dP", "ddt", "dh")),
                         lm=c.t(c.lm), dlm=c.t(z["dlm"]), drc=c.t(z["drc"]), J=c.t(c.J), dJ=c.t(z["dJ"]),
                         adapt=adapt, **kw)  # fmt: skip
            lq = cx * q.dx.cpu().numpy()
            if adapt:
                lq = np.concatenate([lq, (ch * q.dh.cpu().numpy())[:, None]], 1)
            moved = q.steps.cpu().numpy() != j.steps.cpu().numpy()
            fl = np.abs(lq.sum(1) - lt.sum(1)) / np.maximum(sc, 1e-300)
            floors[cls] = np.where(moved, np.inf, fl)[judged]
    return out, flag, g


def check_dots(out):
    for cls, e in out.items():
        if cls == "rc":
            assert e <= RC_BATCH, (cls, e)
            continue
        assert len(e) >= 16, (cls, len(e))
        p99 = DOT_P99_LM if cls == "lm" else DOT_P99
        assert np.quantile(e, 0.99) <= p99 and e.max() <= DOT_MAX, (cls, np.quantile(e, 0.99), e.max())


@pytest.mark.parametrize("adapt", [True, False])
def test_primal_is_the_call(case, adapt):
    ref = case.cs.launch(*case.inputs(), J=case.t(case.J))
    v = case.ad.vjp(*case.inputs(), torch.zeros(case.B, case.ns, dtype=torch.float64, device=case.dev),
                    J=case.t(case.J), adapt=adapt)  # fmt: skip
    for a, b in zip(ref[:4], v[:4]):
        assert torch.equal(a, b)
    assert torch.equal(ref.flag, case.ad.flag) and torch.equal(case.cs.count, case.ad.count)


@pytest.mark.parametrize("adapt", [True, False])
def test_dot_products(case, adapt):
    out, flag, _ = dot_errors(case, adapt, 21)
    check_dots(out)


@pytest.mark.parametrize("adapt", [True, False])
def test_recovered_dot_products(gpu, networks, adapt):
    # max_steps 20 leaves the cold starts unfinished: the recovery redoes them (flag 1), a few still fail (flag 2)
    c = Case(networks("cho41"), gpu)
    try:
        out, flag, g = dot_errors(c, adapt, 23, max_steps=20)
        assert (flag == 1).sum() >= 32 and (flag == 2).sum() >= 1
        check_dots(out)
        failed = flag == 2
        for k, a in g.items():
            if k != "rc" and a is not None:
                assert np.isnan(a[failed]).all() and np.isfinite(a[~failed]).all(), k
        assert np.isfinite(g["rc"]).all()
    finally:
        c.close()


def test_checkpoints_give_the_same_bits(gpu, networks):
    # cap 8 stores 16 try states: the 20 tries of each cell's call and the recovery's up to 200 go through
    # checkpoints and recomputed segments, whose tries repeat the stored ones bit for bit
    net = networks("cho41")
    small, full = Case(net, gpu, cap=8), Case(net, gpu, cap=100)
    try:
        rng = np.random.default_rng(5)
        cx = rng.standard_normal((small.B, small.ns))
        ch = rng.standard_normal(small.B)
        a = small.ad.vjp(*small.inputs(), small.t(cx), gh=small.t(ch), lm=small.t(small.lm), J=small.t(small.J),
                         max_steps=20)  # fmt: skip
        b = full.ad.vjp(*full.inputs(), full.t(cx), gh=full.t(ch), lm=full.t(full.lm), J=full.t(full.J), max_steps=20)
        assert all(torch.equal(p, q) for p, q in zip(a[:4], b[:4]))
        for p, q in zip(a.cotangents, b.cotangents):
            if p is not None:
                assert torch.equal(p.nan_to_num(7.0), q.nan_to_num(7.0))
    finally:
        small.close()
        full.close()


def test_determinism(case):
    rng = np.random.default_rng(9)
    cx = case.t(rng.standard_normal((case.B, case.ns)))
    args = dict(lm=case.t(case.lm), J=case.t(case.J))
    a1 = case.ad.vjp(*case.inputs(), cx, **args).cotangents._asdict()
    a2 = case.ad.vjp(*case.inputs(), cx, **args).cotangents._asdict()
    assert all(torch.equal(a1[k], a2[k]) for k in a1 if a1[k] is not None)
    perm = torch.randperm(case.B, generator=torch.Generator().manual_seed(1)).to(case.dev)
    ins = [a[perm] for a in case.inputs()]
    a3 = case.ad.vjp(*ins, cx[perm], lm=case.t(case.lm)[perm], J=case.t(case.J)[perm]).cotangents._asdict()
    assert all(torch.equal(a1[k][perm], a3[k]) for k in a1 if k != "rc" and a1[k] is not None)


def test_failed_cell_is_left_out_of_the_rate_table(case):
    # the failed cell comes last: the others keep their places, and the rate table's sum its order
    rng = np.random.default_rng(11)
    cx = case.t(rng.standard_normal((case.B, case.ns)))
    lm = case.t(case.lm)
    bad = lm.clone()
    bad[-1, 0] = float("nan")
    x, T, P, dt, h = case.inputs()
    h = 2.0 * dt
    failed = case.ad.vjp(x, T, P, dt, h, cx, lm=bad, J=case.t(case.J))
    flag, counts = case.ad.flag.clone(), case.ad.fallback
    alone = case.ad.vjp(x[:-1], T[:-1], P[:-1], dt[:-1], h[:-1], cx[:-1], lm=bad[:-1], J=case.t(case.J)[:-1])
    assert int(flag[-1]) == 2 and counts["still_failed"] == 1
    assert all(torch.equal(a[:-1], b) for a, b in zip(failed[:4], alone[:4]))
    f, o = failed.cotangents._asdict(), alone.cotangents._asdict()
    for k in f:
        if f[k] is None:
            continue
        if k == "rc":
            assert torch.equal(f[k], o[k]) and bool(f[k].isfinite().all())
        else:
            assert torch.equal(f[k][:-1], o[k]) and bool(f[k][-1].isnan().all()), k


def test_a_nan_from_a_passing_cell_reaches_the_rate_table(case):
    rng = np.random.default_rng(13)
    cx = case.t(rng.standard_normal((case.B, case.ns)))
    cx[0, 0] = float("nan")
    x, T, P, dt, _ = case.inputs()
    g = case.ad.vjp(x, T, P, dt, 2.0 * dt, cx, lm=case.t(case.lm), J=case.t(case.J)).cotangents
    assert case.ad.fallback["still_failed"] == 0 and bool(g.rc.isnan().any())


def test_non_finite_step_acts_as_twice_dt(case):
    rng = np.random.default_rng(15)
    cx = case.t(rng.standard_normal((case.B, case.ns)))
    ch = case.t(rng.standard_normal(case.B))
    x, T, P, dt, _ = case.inputs()
    two = case.ad.vjp(x, T, P, dt, 2.0 * dt, cx, gh=ch, lm=case.t(case.lm), J=case.t(case.J))
    for q in (float("nan"), float("-inf")):
        bad = case.ad.vjp(x, T, P, dt, torch.full_like(dt, q), cx, gh=ch, lm=case.t(case.lm), J=case.t(case.J))
        assert all(torch.equal(a, b) for a, b in zip(two[:4], bad[:4]))
        for k, (a, b) in enumerate(zip(two.cotangents, bad.cotangents)):
            if a is not None and k != 4:  # h's own cotangent: zero for a non-finite h
                assert torch.equal(a, b)
        assert bool((bad.cotangents.h == 0).all()) and case.ad.fallback["nonfinite_h"] == case.B


def test_wrong_cotangents_are_refused_by_name(case):
    x, T, P, dt, h = case.inputs()
    with pytest.raises(ValueError, match="gx"):
        case.ad.vjp(x, T, P, dt, h, x[:, :-1], J=case.t(case.J))
    with pytest.raises(ValueError, match="gh"):
        case.ad.vjp(x, T, P, dt, h, x, gh=h[:-1], J=case.t(case.J))
    with pytest.raises(ValueError, match="max_steps"):
        case.ad.vjp(x, T, P, dt, h, x, J=case.t(case.J), max_steps=4001)


@pytest.mark.parametrize("adapt", [True, False])
def test_long_dark_calls(gpu, networks, adapt):
    # the 1e10 s dark call from a solar start (T log-uniform 500-2500 K, P 1e-2 to 1e8 dyn cm^-2): hundreds of tries
    # per cell, beyond the 2 cap = 200 stored states, so the reverse pass runs on checkpoints and recomputed segments
    net = networks("cho41")
    c = Case(net, gpu, cells=32)
    try:
        w = synthetic.workload(net, "cfg0", 32, seed=5)
        c.x, c.T, c.P, c.J, c.h, c.dt = w.x, w.T, w.P, w.J, w.h, w.dt
        # Over hundreds of step-size feedbacks the tangent is ill-conditioned in a few cells (a one-ulp change of T
        # moves it by up to 1e-4 relative), and tangent and adjoint each carry rounding of that size: such a cell is
        # judged against its own conditioning, the others against the reference's bar
        floors = {}
        out, flag, _ = dot_errors(c, adapt, 25, floors=floors)
        steps = c.cs.launch(*c.inputs(), J=c.t(c.J)).steps.cpu().numpy()
        assert steps.max() > 2 * c.ad.cap, steps.max()
        assert out["rc"] <= RC_BATCH, out["rc"]
        for cls, e in out.items():
            if cls == "rc":
                continue
            bound = np.maximum(DOT_P99_LM if cls == "lm" else DOT_P99, FLOOR_FACTOR * floors[cls])
            assert len(e) >= 16 and np.median(e) <= LONG_MEDIAN, (cls, len(e), np.median(e))
            assert (e <= bound).all(), (cls, e[e > bound], floors[cls][e > bound])
    finally:
        c.close()


def test_without_photolysis(gpu, networks):
    # photo=False: no photolysis branches, J None, no J cotangent; the primal is still the call's bit for bit and the
    # adjoint still the tangent's transpose
    net = networks("cho41")
    cs, ad = CudaSolver(net, gpu), ADSolver(net, gpu)
    try:
        B = 32
        w = synthetic.workload(net, "column", B, seed=7)
        x, h, _ = synthetic.cold_start(w.x, w.h, seed=8, share=0.3)
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=gpu)  # noqa: E731
        args = [t(x), t(w.T), t(w.P), t(np.full(B, 100.0)), t(h)]
        ref = cs.launch(*args)
        rng = np.random.default_rng(3)
        dx, dT = x * rng.standard_normal(x.shape), w.T * rng.standard_normal(B)
        zero = t(np.zeros(B))
        j = ad.jvp(*args, t(dx), t(dT), zero, zero, zero)
        assert all(torch.equal(a, b) for a, b in zip(ref[:4], j[:4]))
        x1 = j.x.cpu().numpy()
        c = np.where(x1 > 1e-20, rng.standard_normal(x1.shape) / np.maximum(x1, 1e-300), 0.0)
        v = ad.vjp(*args, t(c))
        assert v.cotangents.J is None and all(torch.equal(a, b) for a, b in zip(ref[:4], v[:4]))
        g = v.cotangents
        left = (c * j.dx.cpu().numpy()).sum(1)
        right = (g.x.cpu().numpy() * dx).sum(1) + g.T.cpu().numpy() * dT
        e = np.abs(left - right) / np.maximum(np.abs(left), np.abs(right)).clip(1e-300)
        assert np.quantile(e, 0.99) <= DOT_P99 and e.max() <= DOT_MAX, e.max()
    finally:
        cs.close()
        ad.close()
