"""The conversions' kernels on the GPU: bit for bit the formulas with row sums in the warp's order, within rounding of
the reference's torch formulas, their problem bits, and a GCM step that keeps each cell's tracer mass and element
moles through a call."""

import numpy as np
import pytest
import torch

from maxichem_b200 import coupling, synthetic
from maxichem_b200.solver import CudaSolver

pytestmark = pytest.mark.gpu


def warp_rows(v):
    """Row sums of v [cells, n] as a warp forms them: lane l adds columns l, l + 32, ..., then a butterfly."""
    cells, n = v.shape
    R = -(-n // 32)
    pad = np.zeros((cells, 32 * R))
    pad[:, :n] = v
    p = np.zeros((cells, 32))
    for r in range(R):
        p = p + pad[:, 32 * r : 32 * (r + 1)]
    lanes = np.arange(32)
    for o in (16, 8, 4, 2, 1):
        p = p + p[:, lanes ^ o]
    return p[:, 0]


def inputs(networks, cells=4096, seed=0):
    net = networks("chno69")
    mw = coupling.molar_masses(net.atoms, net.elements)
    rng = np.random.default_rng(seed)
    q = rng.random((cells, len(mw))) * 10.0 ** rng.uniform(-12, -2, (cells, len(mw)))
    return net, mw.numpy(), q


def test_mass_to_mole_is_the_warp_order_formula(gpu, networks):
    _, mw, q = inputs(networks)
    x = coupling.mass_to_mole(torch.as_tensor(q, device=gpu), torch.as_tensor(mw, device=gpu)).cpu().numpy()
    n = q / mw
    want = n / warp_rows(n)[:, None]
    assert np.array_equal(x, want)
    ref = coupling.mass_to_mole(torch.as_tensor(q), torch.as_tensor(mw)).numpy()  # torch's own sum order
    assert (np.abs(x - ref) <= 1e-14 * np.abs(ref)).all()  # the sum's order moves the last bits only


def test_mole_to_mass_is_the_warp_order_formula(gpu, networks):
    _, mw, q = inputs(networks, seed=1)
    x = q / q.sum(1, keepdims=True)
    mass = q.sum(1)
    got = coupling.mole_to_mass(torch.as_tensor(x, device=gpu), torch.as_tensor(mw, device=gpu),
                                torch.as_tensor(mass, device=gpu)).cpu().numpy()  # fmt: skip
    xm = x * mw
    want = xm * (mass / warp_rows(xm))[:, None]
    assert np.array_equal(got, want)


def test_the_kernels_report_bad_rows(gpu, networks):
    _, mw, q = inputs(networks, cells=64, seed=2)
    t = lambda a: torch.as_tensor(a, device=gpu)
    bad = q.copy()
    bad[7, 3] = np.inf
    with pytest.raises(ValueError, match="q holds 1 non-finite entries"):
        coupling.mass_to_mole(t(bad), t(mw))
    bad = q.copy()
    bad[9, 1] = -1e-12
    with pytest.raises(ValueError, match="q holds negatives"):
        coupling.mass_to_mole(t(bad), t(mw))
    assert torch.isfinite(coupling.signed_mole_fractions(t(bad), t(mw))).all()
    bad = q.copy()
    bad[11] = 0.0
    with pytest.raises(ValueError, match="cell 11 holds no tracer mass"):
        coupling.mass_to_mole(t(bad), t(mw))
    x = q / q.sum(1, keepdims=True)
    mass = q.sum(1)
    mass[4] = -1.0
    with pytest.raises(ValueError, match="mass must be finite and not negative"):
        coupling.mole_to_mass(t(x), t(mw), t(mass))


def test_a_gcm_step_keeps_tracer_mass_and_element_moles(gpu, networks):
    net = networks("chno69")
    B = 512
    w = synthetic.workload(net, "column", B, seed=6)
    mw = coupling.molar_masses(net.atoms, net.elements).to(gpu)
    atoms = torch.as_tensor(np.asarray(net.atoms, dtype=np.float64), device=gpu)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=gpu)
    x0 = t(w.x)
    mass = torch.full((B,), 0.02, dtype=torch.float64, device=gpu)
    q = coupling.mole_to_mass(x0, mw, mass)  # the GCM's tracers
    with CudaSolver(net, gpu, photo=True) as solver:
        x = coupling.mass_to_mole(q, mw)
        x1, h1, done, steps = solver(x, t(w.T), t(w.P), t(w.dt), t(w.h), J=t(w.J))
        coupling.require_finished(done, t(w.T), t(w.P) / coupling.PA_TO_DYN_CM2, solver.fallback, "in the test")
        q1 = coupling.mole_to_mass(x1, mw, q.sum(1))
    assert torch.allclose(q1.sum(1), q.sum(1), rtol=1e-14, atol=0)
    e0, e1 = coupling.element_moles(q, mw, atoms), coupling.element_moles(q1, mw, atoms)
    assert ((e1 - e0).abs() <= 1e-9 * e0.abs() + 1e-30).all()
