"""The learned part on the GPU: features, the network's forward pass and gradients against the CPU reference
(oracle/surrogate_ref.py, rounding to BF16 where the kernels do), training, and the gated call (no acceptance gives
the plain call bit for bit; accepted cells conserve their element shares; audited cells carry Rodas3's result and the
audit measures the proposals' error)."""

import numpy as np
import pytest
import torch

import parity
from maxichem_b200 import surrogate as sg
from maxichem_b200 import synthetic
from maxichem_b200.solver import CudaSolver
from oracle import surrogate_ref as ref

pytestmark = pytest.mark.gpu
GRAD_RTOL = 5e-3  # per layer, norm-relative: the sums' FP32 order and the odd BF16 rounding flip of dZ


def t(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)


@pytest.fixture(scope="module")
def small(gpu, networks):
    """The 41-species network, its plain solver, and pairs of two chained 300 s calls on 4,096 column cells."""
    net = networks("cho41")
    solver = CudaSolver(net, gpu, photo=True)
    data = sg.pairs(solver, 4096, 2, seed=31)
    yield net, solver, data
    solver.close()


def test_features_are_the_standardised_logs(small, gpu):
    net, solver, data = small
    sur = sg.Surrogate(solver.ns, solver.nj, solver.tab.atoms, gpu, hidden=128, layers=2, heads=2)
    raw = sg.raw_features(data.x, data.T, data.P, data.dt, data.h, data.J)
    sur.set_scaling(raw, sg.targets(data.x, data.x_out, data.h_out))
    feat, inr = sur.features(data.x, data.T, data.P, data.dt, data.h, data.J)
    sc = sur.scaling
    want = (raw.cpu().numpy() - sc["fmean"]) / np.where(sc["fstd"] > 0, sc["fstd"], 1.0)
    got = feat.float().cpu().numpy()
    assert np.abs(got[:, : sur.nf] - ref.bf16(want)).max() <= 2**-7 * np.abs(want).max()
    assert (got[:, sur.nf :] == 0).all() and bool(inr.bool().all())
    shifted = data.T.clone()
    shifted[:5] = float(10.0 ** (float(sc["fhi"][solver.ns]) + 0.01))  # T above the training range
    _, inr2 = sur.features(data.x, shifted, data.P, data.dt, data.h, data.J)
    assert not bool(inr2[:5].bool().any()) and bool(inr2[5:].bool().all())
    sur.close()


@pytest.mark.parametrize("delta", [0.0, 0.5])
def test_gradients_match_the_cpu_reference_layer_by_layer(small, gpu, delta):
    net, solver, data = small
    sur = sg.Surrogate(solver.ns, solver.nj, solver.tab.atoms, gpu, seed=3)  # 4 x 512, 4 heads
    raw = sg.raw_features(data.x, data.T, data.P, data.dt, data.h, data.J)
    tg = sg.targets(data.x, data.x_out, data.h_out)
    sur.set_scaling(raw, tg)
    M = 256
    feat, _ = sur.features(data.x[:M], data.T[:M], data.P[:M], data.dt[:M], data.h[:M], data.J[:M])
    y = sur.standardised_targets(tg[:M])
    wts = torch.poisson(torch.ones(M, sur.heads, device=gpu)).float()
    p0 = sur.params()
    loss = torch.zeros(1, dtype=torch.float32, device=gpu)
    sur.train_step(feat, y, wts, 0.0, loss, delta)  # lr 0: the gradients alone (square error, or Huber)
    sur.check()
    gpu_grads = sur.unpack(sur.params(1))
    assert np.array_equal(sur.params(), p0)
    layers = ref.unpack(p0, sur.shapes)
    pred, a, z = ref.forward(feat.float().cpu().numpy(), layers)
    dpred, lossr = ref.loss_grad(pred, y.cpu().numpy(), wts.cpu().numpy(), sur.heads, sur.nt, delta)
    grads = ref.backward(dpred, layers, a, z)
    assert abs(float(loss.item()) - lossr) <= 1e-3 * lossr
    for l, ((gw, gb), (rw, rb)) in enumerate(zip(gpu_grads, grads)):
        ew = np.linalg.norm(gw - rw) / np.linalg.norm(rw)
        eb = np.linalg.norm(gb - rb) / max(np.linalg.norm(rb), 1e-30)
        assert ew <= GRAD_RTOL and eb <= GRAD_RTOL, (l, ew, eb)
    # the forward pass of the library equals the reference's: the same BF16 operands, FP32 sums in another order, so
    # an activation now and then rounds to the neighbouring BF16 value (2^-8 relative) and the five layers carry it on
    got = sur.forward(feat).cpu().numpy()
    assert np.abs(got - pred).max() <= 5e-3 * np.abs(pred).max()
    assert np.linalg.norm(got - pred) <= 1e-3 * np.linalg.norm(pred)
    sur.close()


def test_training_lowers_the_loss(small, gpu):
    net, solver, data = small
    sur = sg.Surrogate(solver.ns, solver.nj, solver.tab.atoms, gpu, seed=5)
    hist = sur.fit(data, epochs=6, batch=1024, lr=2e-3)["loss"]
    assert hist[-1] < 0.5 * hist[0], hist
    sur.close()


def test_a_gate_that_accepts_nothing_gives_the_plain_call(small, gpu):
    net, solver, data = small
    sur = sg.Surrogate(solver.ns, solver.nj, solver.tab.atoms, gpu, seed=7)
    sur.fit(data, epochs=1, batch=1024)
    w = synthetic.workload(net, "column", 2048, seed=41)
    args = [t(a, gpu) for a in (w.x, w.T, w.P, w.dt, w.h)]
    J = t(w.J, gpu)
    plain = solver.launch(*args, J=J)
    counts = solver.fallback
    gated = sg.GatedSolver(solver, sur, spread_max=0.0, proj_max=0.0, audit_every=0)
    r = gated(*args, J=J)
    assert torch.equal(r.x, plain.x) and torch.equal(r.h, plain.h) and torch.equal(r.steps, plain.steps)
    assert torch.equal(r.done, plain.done) and torch.equal(solver.flag, plain.flag)
    assert solver.fallback == counts
    assert gated.counts()["accepted"] == 0
    sur.close()


def test_accepted_cells_conserve_and_audited_cells_are_solved(small, gpu):
    net, solver, data = small
    sur = sg.Surrogate(solver.ns, solver.nj, solver.tab.atoms, gpu, seed=9)
    sur.fit(data, epochs=4, batch=1024)
    x, T, P, dt, h, J = data.x_out[:2048], data.T[:2048], data.P[:2048], data.dt[:2048], data.h_out[:2048], data.J[:2048]
    x = x / x.sum(1, keepdim=True)
    plain = solver.launch(x, T, P, dt, h, J=J)
    gated = sg.GatedSolver(solver, sur, spread_max=10.0, proj_max=1.0, audit_every=4, seed=3)  # a loose gate
    r = gated(x, T, P, dt, h, J=J)
    c = gated.counts()
    assert c["accepted"] > 0 and c["audited"] > 0
    acc = (r.steps == 0) & r.done
    # accepted: element shares of the input kept (the projection), sum 1
    sh = lambda q: parity.shares(q.cpu().numpy(), solver.tab.atoms)  # noqa: E731
    assert np.abs(sh(r.x[acc]) - sh(x[acc])).max() <= 1e-9
    assert torch.allclose(r.x[acc].sum(1), torch.ones_like(r.x[acc].sum(1)), rtol=0, atol=1e-12)
    # audited and rejected cells: Rodas3's result bit for bit
    solved = ~acc
    assert torch.equal(r.x[solved], plain.x[solved]) and torch.equal(r.steps[solved], plain.steps[solved])
    n = int(gated.audit_count.item())
    cells = gated.audit_cells[:n].long()
    assert bool((r.steps[cells] == plain.steps[cells]).all())
    prop, truth = gated.audit_x[:n], plain.x[cells]
    want = torch.where(truth > sg.AUDIT_FLOOR, (prop - truth).abs() / truth, torch.zeros_like(truth)).float()
    assert torch.allclose(gated.audit_err[:n], want, rtol=1e-6, atol=0)
    sur.close()


def test_the_gate_decides_on_the_proposals_measures(small, gpu):
    net, solver, data = small
    sur = sg.Surrogate(solver.ns, solver.nj, solver.tab.atoms, gpu, seed=11)
    sur.fit(data, epochs=3, batch=1024)
    n = 2048
    args = (data.x_out[:n] / data.x_out[:n].sum(1, keepdim=True), data.T[:n], data.P[:n], data.dt[:n], data.h_out[:n])
    J = data.J[:n]
    xp, diag = sur.propose(*args, J, drift=solver.drift)
    spread_max = float(torch.quantile(diag[:, 0][diag[:, 2] == 1], 0.5))
    gated = sg.GatedSolver(solver, sur, spread_max=spread_max, proj_max=0.05, audit_every=0)
    r = gated(*args, J=J)
    want = (diag[:, 2] == 1) & (diag[:, 0] <= spread_max) & (diag[:, 1] <= 0.05)
    acc = (r.steps == 0) & r.done
    assert torch.equal(acc, want) and int(want.sum()) > 0
    assert torch.equal(r.x[acc], xp[acc])
    assert gated.counts()["accepted"] == int(want.sum())
    sur.close()


def test_what_the_network_gains_over_the_method_without_it(small, gpu):
    """Train on pairs from the plain solver, calibrate the gate on held-out pairs, then run the gated call on cells of
    a third seed beside the plain call: the whole call's per-species error stays within rtol 1e-3 at the 99.9th
    percentile with every cell done (the bar), cells the gate rejects carry Rodas3's result bit for bit, and the gain
    is the share of cells the network answers (each one a Rodas3 solve saved). On these small synthetic sets the
    gain is measured, not required: the network's errors of a few percent leave the gate little to accept."""
    net, solver, data = small
    sur = sg.Surrogate(solver.ns, solver.nj, solver.tab.atoms, gpu, seed=13)
    sur.fit(data, epochs=6, batch=1024)
    held = sg.pairs(solver, 2048, 2, seed=41)
    cal = sg.calibrate(sur, held, target=1e-3)
    assert 0.0 <= cal["accept"] <= 1.0 and cal["spread_max"] >= 0.0
    test = sg.pairs(solver, 2048, 2, seed=43)
    args = (test.x, test.T, test.P, test.dt, test.h)
    plain = solver.launch(*args, J=test.J)
    gated = sg.GatedSolver(solver, sur, spread_max=cal["spread_max"], proj_max=cal["proj_max"], audit_every=64, seed=5)
    r = gated(*args, J=test.J)
    big = plain.x > 1e-20
    rel = ((r.x - plain.x).abs() / plain.x)[big]
    assert float(torch.quantile(rel.float(), 0.999)) <= 1e-3 and bool(r.done.all())
    acc = (r.steps == 0) & r.done
    assert torch.equal(r.x[~acc], plain.x[~acc])
    gain = float(acc.double().mean())
    print(f"the network answers {gain:.2%} of the test cells (calibrated on held-out: {cal['accept']:.2%}, "
          f"spread_max {cal['spread_max']:.2e} dex)")
    assert gated.counts()["accepted"] == int(acc.sum())
    sur.close()
