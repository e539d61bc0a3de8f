"""The call surface on the GPU: refusals and their messages, the guard and the recovery, counts, flags, lifetime, and
results that do not depend on the batch (the behaviours the reference's tests/test_guard.py checks)."""

import numpy as np
import pytest
import torch

import invented
import oracle
import parity
from maxichem_b200 import synthetic
from maxichem_b200.constants import REC_STEPS, T_MAX, T_MIN, X_SUM_TOL
from maxichem_b200.solver import CallResult, CudaSolver, LaunchResult

pytestmark = pytest.mark.gpu


class Case:
    """The 41-species network on 64 cells of the column grid, settled by one 100 s call from a solar start."""

    def __init__(self, net, dev, cells=64, seed=3):
        self.net, self.dev = net, dev
        self.solver = CudaSolver(net, dev, photo=True)
        w = synthetic.workload(net, "column", cells, seed=seed)
        self.w = w
        t = self.t
        self.x0, self.T, self.P, self.J = t(w.x), t(w.T), t(w.P), t(w.J)
        r = self.solver(self.x0, self.T, self.P, self.full(100.0), t(w.h), J=self.J)
        self.xs, self.hs = r.x, r.h

    def t(self, a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=self.dev)

    def full(self, v, cells=None):
        return torch.full((cells or self.T.shape[0],), float(v), dtype=torch.float64, device=self.dev)


@pytest.fixture(scope="module")
def case(gpu, networks):
    c = Case(networks("cho41"), gpu)
    yield c
    c.solver.close()


def unrefused(solver, monkeypatch):
    monkeypatch.setattr(solver, "_refuse", lambda *_: None)


def test_nan_input_is_refused(case, monkeypatch):
    s, cells = case.solver, case.T.shape[0]
    x = case.xs.clone()
    x[3, 5] = float("nan")
    dt = case.full(1.0)
    with pytest.raises(ValueError, match=r"1 cells of bad input: .*\(first: cell 3: sum\(x\) - 1 = nan"):
        s(x, case.T, case.P, dt, case.hs, J=case.J)
    with monkeypatch.context() as m:
        unrefused(s, m)
        y, _, d, _ = s(x, case.T, case.P, dt, case.hs, J=case.J)
    counts = s.fallback
    keep = torch.arange(cells, device=case.dev) != 3
    y2, _, d2, _ = s(x[keep], case.T[keep], case.P[keep], dt[keep], case.hs[keep], J=case.J[keep])
    assert counts["bad_input"] == 1 and counts["recomputed"] == 0
    assert not bool(d[3]) and bool(torch.equal(y[3], x[3]) or not torch.isfinite(y[3]).all())
    assert torch.equal(y[keep], y2) and torch.equal(d[keep], d2) and bool(d2.all())


def test_forced_failure_is_recomputed(case):
    s, cells = case.solver, case.T.shape[0]
    x, h, dt = case.xs.clone(), case.hs.clone(), case.full(1.0)
    x[7], h[7], dt[7] = case.x0[7], 1e-10, 500.0  # cell 7: a cold start over 500 s
    y, _, d, n, flag = s.launch(x, case.T, case.P, dt, h, J=case.J, max_steps=10)
    counts = s.fallback
    assert counts["unfinished"] == 1 and counts["recomputed"] == 1
    assert counts["recovered"] + counts["still_failed"] == 1
    assert int(flag[7]) == (1 if bool(d[7]) else 2)
    others = torch.arange(cells, device=case.dev) != 7
    assert bool(d[others].all()) and int(flag[others].abs().sum()) == 0
    # the oracle's recovery of the same cell, judged as the other long calls are: against the oracle's own change
    # when T moves by one ulp (a recovery is a cold start of up to REC_STEPS x max_steps tries)
    ref = oracle.Oracle(s.tab, drift=s.drift)
    i = [7]
    args = (x[i].cpu().numpy(), case.w.T[i], case.w.P[i], dt[i].cpu().numpy(), h[i].cpu().numpy())
    r = ref.call(*args, J=case.w.J[i], max_steps=10)
    nudged = ref.call(args[0], np.nextafter(args[1], np.inf), *args[2:], J=case.w.J[i], max_steps=10)
    assert r["flag"][0] == int(flag[7]) and r["done"][0] == bool(d[7]) and r["steps"][0] == float(n[7])
    got = y[7].cpu().numpy()

    def worst(a, b):
        big = (np.abs(a) > 1e-20) & (np.abs(b) > 1e-20)
        return float((np.abs(a - b)[big] / np.abs(b[big])).max())

    assert worst(got, r["x"][0]) <= max(parity.RTOL, 10.0 * worst(nudged["x"][0], r["x"][0]))


def test_element_drift_is_recomputed(gpu, networks):
    # with allowance 0 every rounding change of an element share is flagged; atol 1e-18 (the default's clamping
    # allowance would cover rounding drift)
    net = networks("cho41")
    w = synthetic.workload(net, "column", 512, seed=11)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=gpu)
    args = (t(w.x), t(w.T), t(w.P), torch.full((512,), 500.0, dtype=torch.float64, device=gpu),
            torch.full((512,), 1e-10, dtype=torch.float64, device=gpu))  # fmt: skip
    with CudaSolver(net, gpu, photo=True, drift=0.0) as strict:
        y, _, dz, _, flag = strict.launch(*args, J=t(w.J), atol=1e-18)
        counts = strict.fallback
    with CudaSolver(net, gpu, photo=True) as plain:
        yk, _, _, _, flag0 = plain.launch(*args, J=t(w.J), atol=1e-18)
    passed = flag == 0
    assert counts["drift"] > 0
    assert counts["recomputed"] == counts["drift"] + counts["nonfinite"] + counts["unfinished"]
    assert counts["recovered"] + counts["still_failed"] == counts["recomputed"]
    assert int(flag0.sum()) == 0
    assert torch.equal(y[passed], yk[passed])
    assert not bool(dz[flag == 2].any())


def test_temperature_out_of_range_is_refused(case, monkeypatch):
    s = case.solver
    T = case.T.clone()
    T[0], T[1] = 250.0, T_MAX + 0.5
    T[2], T[3] = T_MIN, T_MAX
    args = (case.xs, T, case.P, case.full(500.0), case.full(1e-10))
    refused = r"1 cells below 300 K, .*\(first: cell 0, T = 250 K\).*; 1 cells above 3000 K, .*cell 1, T = 3000.5 K\)"
    with CudaSolver(case.net, case.dev, photo=True) as fresh:
        with pytest.raises(ValueError, match=refused):
            fresh(*args, J=case.J)
        with pytest.raises(ValueError, match="1 cells below 300 K and 1 above 3000 K"):
            fresh.check()
        with monkeypatch.context() as m:
            unrefused(fresh, m)
            _, _, d, _ = fresh(*args, J=case.J)
        counts = fresh.fallback
    assert counts["cold"] == 1 and counts["hot"] == 1
    assert not bool(d[:2].any()) and bool(d[2:4].all())


def test_bad_inputs_are_refused(case, monkeypatch):
    s, cells = case.solver, case.T.shape[0]
    xb, pb, dtb, hb = case.x0.clone(), case.P.clone(), case.full(50.0), case.full(1e-10)
    xb[3] = 0.0
    xb[7, 0] = -1e-3
    pb[5] = 0.0
    dtb[9] = -1.0
    xb[11] *= 0.9
    xb[13] *= 1.0 + 0.9 * X_SUM_TOL  # just inside the tolerance on either side: accepted
    xb[15] *= 1.0 - 0.9 * X_SUM_TOL
    Jb = case.J.clone()
    Jb[17, 0] = -1.0  # a negative photolysis rate
    bad = [3, 5, 7, 9, 11, 17]
    with pytest.raises(ValueError, match=r"6 cells of bad input: .*\(first: cell 3: sum\(x\) - 1 = -1 "):
        s(xb, case.T, pb, dtb, hb, J=Jb)
    with pytest.raises(ValueError, match=r"1 cells of bad input: .*\(first: cell 0: sum\(x\) - 1 = -0.1 "):
        s(xb[11:12], case.T[11:12], pb[11:12], dtb[11:12], hb[11:12], J=Jb[11:12])
    with monkeypatch.context() as m:
        unrefused(s, m)
        y, _, d, _ = s(xb, case.T, pb, dtb, hb, J=Jb)
    counts = s.fallback
    good = torch.ones(cells, dtype=torch.bool, device=case.dev)
    good[bad] = False
    yr, _, dr, _ = s(xb[good], case.T[good], pb[good], dtb[good], hb[good], J=Jb[good])
    assert counts["bad_input"] == len(bad) and counts["nonfinite"] == 0 and counts["recomputed"] == 0
    assert not bool(d[bad].any()) and bool(d[[13, 15]].all())
    assert torch.equal(y[good], yr) and torch.equal(d[good], dr)


def test_non_finite_and_overflowing_pressures_are_refused_and_named(case):
    s = case.solver
    P = case.P[:4].clone()
    P[1:] = case.t([float("inf"), float("nan"), 1e300])
    named = r"^the call refused cells: 3 cells of bad input: .*P non-finite, not above 0 or so large that P / \(k_B T\)"
    with pytest.raises(ValueError, match=rf"{named} overflows.*first: cell 1:"):
        s(case.x0[:4], case.T[:4], P, case.full(50.0, 4), case.full(1e-10, 4), J=case.J[:4])
    assert s.fallback["bad_input"] == 3


def test_just_outside_the_range_is_refused_and_named(case, monkeypatch):
    s = case.solver
    cold, hot = np.nextafter(T_MIN, 0.0), np.nextafter(T_MAX, np.inf)
    T = case.t([cold, hot, cold, hot])
    dt, h = case.t([0.0, 0.0, 500.0, 500.0]), case.full(1e-10, 4)
    refused = r"2 cells below 300 K, .*\(first: cell 0, T = 300 K\).*; 2 cells above 3000 K, .*\(first: cell 1, "
    with pytest.raises(ValueError, match=refused):
        s(case.x0[:4], T, case.P[:4], dt, h, J=case.J[:4])
    with monkeypatch.context() as m:
        unrefused(s, m)
        _, _, done, _ = s(case.x0[:4], T, case.P[:4], dt, h, J=case.J[:4])
    assert s.fallback["cold"] == 2 and s.fallback["hot"] == 2 and not bool(done.any())


def warp_order_sum(values):
    """x summed as the call kernel's screening warp adds it: lane l adds the values l, l + 32, ... (elimination
    order), then a butterfly over the 32 partial sums."""
    p = [0.0] * 32
    for i, v in enumerate(values):
        p[i % 32] += v
    for o in (16, 8, 4, 2, 1):
        p = [p[q] + p[q ^ o] for q in range(32)]
    return p[0]


def straddle(perm, warp_above, seed=0):
    """A row of comparable entries, one of them moved, whose sums in the warp's order and in the network's order fall
    on either side of 1 + X_SUM_TOL (the warp's above if warp_above). A row's two orders differ by a few ulps of one
    sign, so rows are drawn until one straddles the tolerance the asked way."""
    rng = np.random.default_rng(seed)
    for _ in range(200):
        row = rng.uniform(0.5, 1.5, len(perm))
        row = list(row / row.sum())
        big = int(np.argmax(row))
        base = row[big]
        for k in range(64):
            for sign in (1, -1):
                r = list(row)
                r[big] = base + (1.0 + X_SUM_TOL - sum(row)) + sign * k * np.spacing(base)
                warp = warp_order_sum([r[q] for q in perm]) - 1.0
                plain = sum(r) - 1.0
                if warp_above and warp > X_SUM_TOL >= plain or not warp_above and plain > X_SUM_TOL >= warp:
                    return r
    raise AssertionError("no straddling row found")


def test_sum_on_the_tolerance_is_judged_once(case):
    # only the warp's sum is judged: a row above the tolerance in the warp's order (below it in the network's) is
    # refused; the opposite row is accepted and stepped
    s = case.solver
    perm = [int(q) for q in s.tab.perm]
    above, below = straddle(perm, True), straddle(perm, False)
    dt, h = case.full(50.0, 1), case.full(1e-10, 1)
    with pytest.raises(ValueError, match=r"1 cells of bad input: .*\(first: cell 0: sum\(x\) - 1 = "):
        s(case.t([above]), case.T[:1], case.P[:1], dt, h, J=case.J[:1])
    _, _, done, _ = s(case.t([below]), case.T[:1], case.P[:1], dt, h, J=case.J[:1])
    assert bool(done.all()) and s.fallback["bad_input"] == 0


def test_non_finite_step_acts_as_dt(case):
    s = case.solver
    dt = case.full(50.0)
    ref = s(case.xs, case.T, case.P, dt, dt.clone(), J=case.J)
    assert s.fallback["nonfinite_h"] == 0
    for q in (np.nan, -np.inf, np.inf):
        out = s(case.xs, case.T, case.P, dt, case.full(q), J=case.J)
        assert all(torch.equal(a, b) for a, b in zip(out, ref, strict=True))
        assert s.fallback["nonfinite_h"] == case.T.shape[0]


def test_launch_adds_to_the_total(case):
    s = case.solver
    before = s.total.clone()
    s.launch(case.xs[:8], case.T[:8], case.P[:8], case.full(1.0, 8), case.full(1.0, 8), J=case.J[:8])
    assert torch.equal(s.total - before, s.count.to(torch.int64))


def test_call_and_launch_name_their_results(case):
    s = case.solver
    args = (case.x0[:8], case.T[:8], case.P[:8], case.full(50.0, 8), case.full(1e-10, 8))
    launched = s.launch(*args, J=case.J[:8], max_steps=2)  # few tries: the guard lists cells, so flags are not all 0
    assert isinstance(launched, LaunchResult)
    assert s.flag is launched.flag
    assert bool((launched.flag != 0).any())
    called = s(*args, J=case.J[:8], max_steps=2)
    assert isinstance(called, CallResult)
    assert all(torch.equal(getattr(called, name), getattr(launched, name)) for name in called._fields)
    assert torch.equal(s.flag, launched.flag)


def test_flag_is_none_after_a_call_that_raised(case):
    s = case.solver
    x, T, P, J = case.xs[:8], case.T[:8], case.P[:8], case.J[:8]
    dt = h = case.full(1.0, 8)
    bad = x.clone()
    bad[3, 0] = float("nan")
    s(x, T, P, dt, h, J=J)
    with pytest.raises(ValueError, match="refused cells"):
        s.launch(bad, T, P, dt, h, J=J)
    assert s.flag is None
    s(x, T, P, dt, h, J=J)
    with pytest.raises(ValueError, match=r"^T: "):
        s(x[:5], T[:5].cpu(), P[:5], dt[:5], h[:5], J=J[:5])
    assert s.flag is None


def test_wrong_inputs_raise_before_any_launch(case):
    s = case.solver
    x, T, P, J = case.xs, case.T, case.P, case.J
    dt = h = case.full(50.0)
    before = s.total.clone()
    with pytest.raises(ValueError, match=r"^T: .* on cpu$"):
        s(x, T.cpu(), P, dt, h, J=J)
    with pytest.raises(ValueError, match="required"):
        s(x, T, P, dt, h)
    with pytest.raises(ValueError, match=r"^max_steps from 1"):
        s(x, T, P, dt, h, J=J, max_steps=0)
    with pytest.raises(ValueError, match=r"^J: "):
        s(x, T, P, dt, h, J=J[:, :3])
    assert torch.equal(s.total, before)


def test_closed_solver_refuses_a_call(case):
    with CudaSolver(case.net, case.dev, photo=True) as solver:
        assert solver.fallback["cold"] == 0
    solver.close()  # closing twice does nothing
    with pytest.raises(RuntimeError, match="closed"):
        solver(case.xs[:8], case.T[:8], case.P[:8], case.full(1.0, 8), case.full(1.0, 8), J=case.J[:8])
    assert solver.check()["cold"] == 0  # the counts stay readable


def test_empty_j_is_none_without_photolysis(gpu, tmp_path):
    net, _ = invented.hydrogen(tmp_path)
    x = torch.as_tensor(invented.state(net, 4, H=0.1, H2=0.6, OH=0.05, H2O=0.1, O=0.05, He=0.1), device=gpu)
    T, P, dt, h = (torch.full((4,), q, dtype=torch.float64, device=gpu) for q in (1500.0, 1e6, 1e-3, 1e-3))
    empty = torch.zeros(4, 0, dtype=torch.float64, device=gpu)
    with CudaSolver(net, gpu) as solver:
        assert all(map(torch.equal, solver(x, T, P, dt, h), solver(x, T, P, dt, h, J=empty)))
        with pytest.raises(ValueError, match=r"^J: none or an empty \[4, 0\] one expected"):
            solver(x, T, P, dt, h, J=torch.zeros(4, 1, dtype=torch.float64, device=gpu))


def test_an_empty_batch_is_a_call(case):
    s = case.solver
    e = lambda *shape: torch.zeros(*shape, dtype=torch.float64, device=case.dev)
    r = s.launch(e(0, s.ns), e(0), e(0), e(0), e(0), J=e(0, s.nj))
    assert r.x.shape == (0, s.ns) and r.flag.shape == (0,)
    assert int(s.count.abs().sum()) == 0


def test_results_do_not_depend_on_the_batch(gpu, networks):
    net = networks("cho41")
    cells = 2048
    w = synthetic.workload(net, "column", cells, seed=7)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=gpu)
    args = (t(w.x), t(w.T), t(w.P), torch.full((cells,), 50.0, dtype=torch.float64, device=gpu),
            torch.full((cells,), 1e-10, dtype=torch.float64, device=gpu), t(w.J))  # fmt: skip
    with CudaSolver(net, gpu, photo=True) as s:
        run = lambda a: s.launch(*a[:5], J=a[5])
        big = run(args)
        sel = torch.arange(0, cells, 64, device=gpu)
        perm = torch.randperm(cells, generator=torch.Generator().manual_seed(3)).to(gpu)
        shuffled = run([q[perm] for q in args])
        inverse = torch.empty_like(perm)
        inverse[perm] = torch.arange(cells, device=gpu)
        alone = run([q[sel] for q in args])
        one = run([q[sel[:1]] for q in args])
    assert all(torch.equal(p[sel], q) for p, q in zip(big, alone, strict=True))
    assert all(torch.equal(p[sel[:1]], q) for p, q in zip(big, one, strict=True))
    assert all(torch.equal(p, q[inverse]) for p, q in zip(big, shuffled, strict=True))


ALLOWANCE = 1e-6
DRIFTS = (0.5, 0.99, 1.01, 2.0)  # the largest relative change of an element's share, in units of the allowance


def test_drift_beyond_the_allowance_is_flagged(gpu, tmp_path):
    # the guard alone on hand-made pairs of a state and a result whose He share moved by r times the allowance
    net, _ = invented.hydrogen(tmp_path)
    x0 = invented.state(net, 1, H=0.1, H2=0.6, OH=0.05, H2O=0.1, O=0.05, He=0.1)[0]
    atoms = np.asarray(net.atoms, dtype=float)
    share = (x0 @ atoms) / (x0 @ atoms).sum()
    he = net.species.index("He")
    col = int(np.argmax(atoms[he]))
    f = share[col]
    results = []
    for r in DRIFTS:
        d = r * ALLOWANCE / (1.0 - f - f * r * ALLOWANCE)
        x = x0.copy()
        x[he] *= 1.0 + d
        moved = (x @ atoms) / (x @ atoms).sum() / share - 1.0
        assert np.abs(moved).max() == pytest.approx(r * ALLOWANCE, rel=1e-6)
        results.append(x)
    cells = len(DRIFTS)
    t = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=gpu)
    with CudaSolver(net, gpu, drift=ALLOWANCE) as solver:
        flag = solver.guard(t([x0] * cells), t(results), torch.ones(cells, dtype=torch.int32, device=gpu),
                            t(np.ones(cells)), torch.zeros(cells, dtype=torch.int32, device=gpu))  # fmt: skip
        counts = solver.fallback
    assert flag.tolist() == [int(r > 1.0) for r in DRIFTS]
    assert counts["drift"] == counts["recomputed"] == sum(r > 1.0 for r in DRIFTS)


def test_recovery_tries_ten_times_the_steps(case):
    # a cell that cannot finish in 3 tries is recomputed with REC_STEPS times as many
    s = case.solver
    x, h, dt = case.x0[:4].clone(), case.full(1e-10, 4), case.full(500.0, 4)
    y, _, d, n, flag = s.launch(x, case.T[:4], case.P[:4], dt, h, J=case.J[:4], max_steps=3)
    counts = s.fallback
    assert counts["unfinished"] == int((flag > 0).sum()) > 0
    ref = oracle.Oracle(s.tab, drift=s.drift)
    r = ref.call(x.cpu().numpy(), case.w.T[:4], case.w.P[:4], dt.cpu().numpy(), h.cpu().numpy(), J=case.w.J[:4],
                 max_steps=3)  # fmt: skip
    assert r["flag"].tolist() == flag.tolist() and r["done"].tolist() == d.tolist()
    assert (n.cpu().numpy() <= 3 * REC_STEPS).all()


@pytest.mark.parametrize("chunks", [1, 5])
def test_the_host_call_is_the_device_call(case, chunks):
    # the call on host tensors, copies overlapped over pieces of the batch, gives the device call's bits and counts
    s = case.solver
    args = (case.xs, case.T, case.P, case.full(300.0), case.hs)
    ref = s.launch(*args, J=case.J)
    ref_count, ref_flag = s.count.clone(), ref.flag.clone()
    before = s.total.clone()
    pin = lambda a: a.cpu().pin_memory()
    got = s.call_host(*(pin(a) for a in args), J=pin(case.J), chunks=chunks)
    assert all(torch.equal(a.cpu(), b) for a, b in zip(ref[:4], got, strict=True))
    assert torch.equal(s.count, ref_count) and torch.equal(s.flag, ref_flag.cpu())
    assert torch.equal(s.total - before, ref_count.to(torch.int64))


def test_the_host_call_refuses_like_the_device_call(case):
    s = case.solver
    x = case.xs.cpu().clone()
    x[6, 2] = float("nan")
    T = case.T.cpu().clone()
    T[9] = 250.0
    with pytest.raises(ValueError, match=r"1 cells below 300 K, .*\(first: cell 9, T = 250 K\).*1 cells of bad input: .*"
                                         r"\(first: cell 6: sum\(x\) - 1 = nan"):
        s.call_host(x, T, case.P.cpu(), case.full(1.0).cpu(), case.hs.cpu(), J=case.J.cpu(), chunks=3)
    assert s.flag is None
    with pytest.raises(ValueError, match=r"^T: float64"):
        s.call_host(x, case.T, case.P.cpu(), case.full(1.0).cpu(), case.hs.cpu(), J=case.J.cpu())

