"""The tangent (ADSolver.jvp) on the GPU against the tangent oracle and the call.

The cases of the reference's tests/test_ad.py that judge a tangent alone: the primal is the call's bit for bit, the
frozen tangent along x itself is zero, directions share one call, a non-finite starting step acts as dt, a
non-finite log multiplier fails its cell, recovered cells are differentiated on the recovery's path. Where the
reference judges its tangent by central differences, the tangent here is judged against the tangent oracle
(oracle/mx_oracle_ad.c: dual numbers through the oracle's call, itself pinned against central differences by
tests/test_oracle_ad.py), a derivation independent of the kernel's.
"""

import numpy as np
import pytest
import torch

from maxichem_b200 import synthetic
from maxichem_b200.ad import ADSolver
from maxichem_b200.solver import CudaSolver
from oracle import Oracle

pytestmark = pytest.mark.gpu

# Per cell whose accepted steps and flag match the oracle's: max |dx_gpu - dx_oracle| over species, relative to the
# cell's largest |dx_oracle|. Both sides differentiate the same arithmetic; the primal differs in the last bits of the
# transcendentals. Most cells agree to DX_TIGHT (measured worst 3.1e-9 over the three networks); a cell whose tangent
# is ill-conditioned (deep in the high-pressure limit a falloff rate's sensitivity to its k0 columns is 1 / (1 + pr),
# and the step-size tangents follow err's, a difference of near-equal stages) is judged against the oracle's own
# change under a one-ulp change of T, times FLOOR_FACTOR.
DX_TIGHT = 1e-7
DX_TIGHT_SHARE = 0.95
DX_MEDIAN = 1e-12
FLOOR_FACTOR = 100.0
# dh against the oracle's: the next step size's tangent follows err's. Measured: median 1.5e-11.
DH_MEDIAN = 1e-9
ULP_T = 2.220446049250313e-16
SCALING_TANGENT = 1e-12  # relative to max x: the frozen tangent along x itself is 0 but rounding
CELLS = 128


class Case:
    def __init__(self, net, dev, drift=None, cells=CELLS, seed=3):
        self.dev = dev
        self.cs = CudaSolver(net, dev, photo=True, drift=drift)
        self.ad = ADSolver(net, dev, photo=True, drift=drift)
        self.o = Oracle(self.cs.tab, drift=self.cs.drift)
        w = synthetic.workload(net, "column", cells, seed=seed)
        x, h, _ = synthetic.cold_start(w.x, w.h, seed=seed + 1, share=0.3)
        self.x, self.T, self.P, self.J, self.h = x, w.T, w.P, w.J, h
        self.dt = np.full(cells, 100.0)
        self.B, self.ns, self.nr, self.nj = cells, self.cs.ns, self.cs.nr, self.cs.nj

    def t(self, a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=self.dev)

    def inputs(self):
        return [self.t(a) for a in (self.x, self.T, self.P, self.dt, self.h)]

    def directions(self, D, seed=7):
        """D tangents of every input class at once, and log multipliers."""
        rng = np.random.default_rng(seed)
        B, ns, nr = self.B, self.ns, self.nr
        dx = self.x * rng.standard_normal((D, B, ns))
        dx -= self.x * dx.sum(2, keepdims=True)
        return {
            "dx": dx, "dT": self.T * 0.01 * rng.standard_normal((D, B)), "dP": self.P * rng.standard_normal((D, B)),
            "ddt": self.dt * rng.standard_normal((D, B)), "dh": self.h * rng.standard_normal((D, B)),
            "dlm": rng.standard_normal((D, B, nr)), "dJ": self.J * rng.standard_normal((D, B, self.nj)),
            "drc": rng.standard_normal((D, nr, 9)) * np.array([1.0, 0.1, 30.0] * 3),
            "lm": 0.1 * rng.standard_normal((B, nr)),
        }  # fmt: skip

    def gpu_jvp(self, tan, adapt=True, lm=True, **kw):
        return self.ad.jvp(*self.inputs(), *(self.t(tan[k]) for k in ("dx", "dT", "dP", "ddt", "dh")),
                           lm=self.t(tan["lm"]) if lm else None, dlm=self.t(tan["dlm"]), drc=self.t(tan["drc"]),
                           J=self.t(self.J), dJ=self.t(tan["dJ"]), adapt=adapt, **kw)  # fmt: skip

    def close(self):
        self.cs.close()
        self.ad.close()


@pytest.fixture(scope="module", params=["cho41", "chno69", "sncho91"])
def case(request, gpu, networks):
    c = Case(networks(request.param), gpu)
    yield c
    c.close()


def zeros(c):
    return [torch.zeros(c.B, c.ns, dtype=torch.float64, device=c.dev)] + [
        torch.zeros(c.B, dtype=torch.float64, device=c.dev) for _ in range(4)
    ]


@pytest.mark.parametrize("adapt", [True, False])
def test_primal_is_the_call(case, adapt):
    ref = case.cs.launch(*case.inputs(), J=case.t(case.J))
    j = case.ad.jvp(*case.inputs(), *zeros(case), J=case.t(case.J), adapt=adapt)
    for a, b in zip(ref[:4], j[:4]):
        assert torch.equal(a, b)
    assert torch.equal(ref.flag, case.ad.flag)
    assert torch.equal(case.cs.count, case.ad.count)


def oracle_tangents(c, tan, adapt, lm=True, **kw):
    """The oracle's call and tangent, and per direction and cell its own relative change under T (1 +- one ulp)."""
    args = [tan[k] for k in ("dx", "dT", "dP", "ddt", "dh")]
    opt = dict(lm=tan["lm"] if lm else None, dlm=tan["dlm"], drc=tan["drc"], J=c.J, dJ=tan["dJ"], adapt=adapt, **kw)
    r = c.o.jvp(c.x, c.T, c.P, c.dt, c.h, *args, **opt)
    fx, fh = np.zeros(r["dx"].shape[:2]), np.zeros(r["dh"].shape)
    for sg in (1.0, -1.0):
        q = c.o.jvp(c.x, c.T * (1.0 + sg * ULP_T), c.P, c.dt, c.h, *args, **opt)
        moved = q["steps"] != r["steps"]
        scale = np.maximum(np.abs(r["dx"]).max(2), 1e-300)
        fx = np.maximum(fx, np.where(moved, np.inf, np.abs(q["dx"] - r["dx"]).max(2) / scale))
        fh = np.maximum(fh, np.where(moved, np.inf, np.abs(q["dh"] - r["dh"]) / np.maximum(np.abs(r["dh"]), 1e-300)))
    return r, fx, fh


def compare(g, flag, r, fx, fh, adapt):
    gs, gf = g.steps.cpu().numpy(), flag.cpu().numpy()
    same = (gs == r["steps"]) & (gf == r["flag"])
    assert same.mean() >= 0.95, f"accepted steps or flags differ from the oracle's in {(~same).sum()} cells"
    gdx, gdh = g.dx.cpu().numpy(), g.dh.cpu().numpy()
    keep = same & (gf != 2)
    for d in range(gdx.shape[0]):
        a, b = gdx[d][keep], r["dx"][d][keep]
        e = np.abs(a - b).max(1) / np.maximum(np.abs(b).max(1), 1e-300)
        assert np.median(e) <= DX_MEDIAN and (e <= DX_TIGHT).mean() >= DX_TIGHT_SHARE, (d, np.median(e), e.max())
        bound = np.maximum(DX_TIGHT, FLOOR_FACTOR * fx[d][keep])
        assert (e <= bound).all(), (d, e[e > bound], fx[d][keep][e > bound])
        if adapt:
            hs = np.abs(gdh[d][keep] - r["dh"][d][keep]) / np.maximum(np.abs(r["dh"][d][keep]), 1e-300)
            assert np.median(hs) <= DH_MEDIAN, (d, np.median(hs))
            hb = np.maximum(DX_TIGHT, FLOOR_FACTOR * fh[d][keep])
            assert (hs <= hb).all(), (d, hs[hs > hb], fh[d][keep][hs > hb])
        else:
            assert (gdh[d][gf != 2] == 0.0).all()
    failed = gf == 2
    assert np.isnan(gdx[:, failed]).all() and np.isnan(gdh[:, failed]).all()
    assert np.isfinite(gdx[:, ~failed]).all()


@pytest.mark.parametrize("adapt", [True, False])
def test_tangent_is_the_oracles(case, adapt):
    tan = case.directions(3)
    g = case.gpu_jvp(tan, adapt=adapt)
    flag = case.ad.flag.clone()
    r, fx, fh = oracle_tangents(case, tan, adapt)
    compare(g, flag, r, fx, fh, adapt)


@pytest.mark.parametrize("adapt", [True, False])
def test_recovered_cells_follow_the_recovery(gpu, networks, adapt):
    # max_steps 20 leaves the cold starts unfinished, so the guard lists them and the recovery (ten times the tries,
    # dense pivoted W) redoes them: most pass (flag 1) and are differentiated along its path, a few still fail (flag 2,
    # NaN tangents)
    c = Case(networks("cho41"), gpu, cells=64)
    try:
        tan = c.directions(2, seed=9)
        ref = c.cs.launch(*c.inputs(), J=c.t(c.J), max_steps=20)
        g = c.gpu_jvp(tan, adapt=adapt, lm=False, max_steps=20)
        flag = c.ad.flag.clone()
        j0 = c.ad.jvp(*c.inputs(), *zeros(c), J=c.t(c.J), adapt=adapt, max_steps=20)
        for a, b in zip(ref[:4], j0[:4]):
            assert torch.equal(a, b)
        assert torch.equal(ref.flag, c.ad.flag) and torch.equal(ref.flag, flag)
        assert int((flag == 1).sum()) >= 32 and int((flag == 2).sum()) >= 1
        r, fx, fh = oracle_tangents(c, tan, adapt, lm=False, max_steps=20)
        compare(g, flag, r, fx, fh, adapt)
    finally:
        c.close()


def test_directions_share_one_call(case):
    tan = case.directions(3, seed=11)
    together = case.gpu_jvp(tan)
    for k in range(3):
        one = {n: (v[k] if n not in ("lm",) else v) for n, v in tan.items()}
        g = case.ad.jvp(*case.inputs(), *(case.t(one[n]) for n in ("dx", "dT", "dP", "ddt", "dh")),
                        lm=case.t(tan["lm"]), dlm=case.t(one["dlm"]), drc=case.t(one["drc"]), J=case.t(case.J),
                        dJ=case.t(one["dJ"]))  # fmt: skip
        assert torch.equal(g.dx, together.dx[k]) and torch.equal(g.dh, together.dh[k])
        assert torch.equal(g.x, together.x)


def test_frozen_tangent_along_x_itself_is_zero(case):
    # the right-hand side is homogeneous of degree 1 in N: with the try sizes held, N -> c N scales every stage
    z = zeros(case)
    out = case.ad.jvp(*case.inputs(), case.t(case.x), *z[1:], J=case.t(case.J), adapt=False)
    passed = case.ad.flag != 2
    worst = float((out.dx.abs().amax(1) / out.x.abs().amax(1))[passed].max())
    assert worst <= SCALING_TANGENT


def test_non_finite_step_acts_as_twice_dt(case):
    tan = case.directions(1, seed=13)
    x, T, P, dt, _ = case.inputs()
    args = [case.t(tan[k][0]) for k in ("dx", "dT", "dP", "ddt", "dh")]
    two = case.ad.jvp(x, T, P, dt, 2.0 * dt, *args, J=case.t(case.J))
    for q in (float("nan"), float("-inf")):
        bad = case.ad.jvp(x, T, P, dt, torch.full_like(dt, q), *args, J=case.t(case.J))
        assert all(torch.equal(a, b) for a, b in zip(two, bad))
        assert case.ad.fallback["nonfinite_h"] == case.B


def test_nan_log_multiplier_fails_the_cell(case):
    tan = case.directions(1, seed=15)
    lm = case.t(tan["lm"])
    bad = lm.clone()
    bad[0, 0] = float("nan")
    args = [case.t(tan[k][0]) for k in ("dx", "dT", "dP", "ddt", "dh")]
    x, T, P, dt, _ = case.inputs()
    h = 2.0 * dt
    jb = case.ad.jvp(x, T, P, dt, h, *args, lm=bad, J=case.t(case.J))
    counts, flag = case.ad.fallback, case.ad.flag.clone()
    j2 = case.ad.jvp(x, T, P, dt, h, *args, lm=lm, J=case.t(case.J))
    assert int(jb.steps[0]) == 0 and not bool(jb.done[0]) and int(flag[0]) == 2 and counts["still_failed"] == 1
    assert bool(jb.dx[0].isnan().all()) and bool(jb.dh[0].isnan())
    assert all(torch.equal(a[1:], b[1:]) for a, b in zip(jb, j2))


def test_no_multipliers_are_zero_multipliers(case):
    tan = case.directions(1, seed=17)
    args = [case.t(tan[k][0]) for k in ("dx", "dT", "dP", "ddt", "dh")]
    dlm = case.t(tan["dlm"][0])
    none = case.ad.jvp(*case.inputs(), *args, dlm=dlm, J=case.t(case.J))
    zero = case.ad.jvp(*case.inputs(), *args, lm=torch.zeros_like(dlm), dlm=dlm, J=case.t(case.J))
    assert all(torch.equal(a, b) for a, b in zip(none, zero))


def test_wrong_tangents_are_refused_by_name(case):
    x, T, P, dt, h = case.inputs()
    z = zeros(case)
    with pytest.raises(ValueError, match="dT"):
        case.ad.jvp(x, T, P, dt, h, z[0], z[1][:-1], *z[2:], J=case.t(case.J))
    with pytest.raises(ValueError, match="dlm"):
        case.ad.jvp(x, T, P, dt, h, *z, dlm=torch.zeros(case.B, case.nr + 1, dtype=torch.float64, device=case.dev),
                    J=case.t(case.J))  # fmt: skip
    with pytest.raises(ValueError, match="directions"):
        case.ad.jvp(x, T, P, dt, h, torch.zeros(17, case.B, case.ns, dtype=torch.float64, device=case.dev),
                    *(a.expand(17, -1) for a in z[1:]), J=case.t(case.J))  # fmt: skip
    with pytest.raises(ValueError, match="max_steps"):
        case.ad.jvp(x, T, P, dt, h, *z, J=case.t(case.J), max_steps=4001)


def test_a_callers_rate_table(gpu, networks):
    # rc replaces the network's table for the call: ln A of every thermal row moved by 0.1, against the oracle's call
    # on the same table, and the tangent's and the adjoint's primal alike bit for bit
    c = Case(networks("cho41"), gpu, cells=64)
    try:
        rc = c.cs.tab.rc.copy()
        rc[: c.cs.tab.nrt, 0] += 0.1
        z = zeros(c)
        j = c.ad.jvp(*c.inputs(), *z, rc=c.t(rc), J=c.t(c.J))
        flag = c.ad.flag.cpu().numpy()
        v = c.ad.vjp(*c.inputs(), torch.zeros_like(z[0]), rc=c.t(rc), J=c.t(c.J))
        assert all(torch.equal(a, b) for a, b in zip(j[:4], v[:4]))
        r = c.o.jvp(c.x, c.T, c.P, c.dt, c.h, rc=rc, J=c.J)
        same = (j.steps.cpu().numpy() == r["steps"]) & (flag == r["flag"])
        assert same.mean() >= 0.95
        a, b = j.x.cpu().numpy()[same], r["x"][same]
        big = (a > 1e-20) & (b > 1e-20)
        rel = np.abs(a - b) / np.maximum(a, b).clip(1e-300)
        assert (np.where(big, rel, 0).max(1) <= 1e-9).mean() >= 0.95 and rel[big].max() <= 1e-6
        ref = c.cs.launch(*c.inputs(), J=c.t(c.J))
        assert not torch.equal(ref.x, j.x)  # the table reached the call
    finally:
        c.close()
