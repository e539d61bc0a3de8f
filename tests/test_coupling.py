"""The GCM step's glue on CPU: molar masses, the conversions' formulas and checks, element totals, and the stop on
unfinished cells (the behaviour of the reference's coupling/composition.py and coupling/chemistry.py)."""

import numpy as np
import pytest
import torch

from maxichem_b200 import coupling


def net_mw(networks):
    net = networks("chno69")
    return net, coupling.molar_masses(net.atoms, net.elements)


def test_molar_masses_follow_the_atoms(networks):
    net, mw = net_mw(networks)
    i = net.species.index("H2O")
    assert float(mw[i]) == pytest.approx(2 * 1.008e-3 + 15.999e-3, rel=1e-15)
    with pytest.raises(ValueError, match=r"no atomic mass for \['Xe'\]"):
        coupling.molar_masses(np.ones((2, 1)), ["Xe"])
    with pytest.raises(ValueError, match="species rows \\[1\\] have no atoms"):
        coupling.molar_masses(np.array([[1.0], [0.0]]), ["H"])


def test_mass_and_mole_round_trip(networks):
    net, mw = net_mw(networks)
    rng = np.random.default_rng(0)
    q = torch.as_tensor(rng.random((16, len(mw))) * 1e-3)
    x = coupling.mass_to_mole(q, mw)
    assert torch.allclose(x.sum(1), torch.ones(16, dtype=torch.float64), rtol=1e-15, atol=0)
    mass = q.sum(1)
    back = coupling.mole_to_mass(x, mw, mass)
    assert torch.allclose(back, q, rtol=1e-13, atol=0)
    assert torch.allclose(back.sum(1), mass, rtol=1e-14, atol=0)


def test_the_checks_name_what_failed(networks):
    _, mw = net_mw(networks)
    q = torch.full((4, len(mw)), 1e-3, dtype=torch.float64)
    bad = q.clone()
    bad[1, 2] = float("nan")
    with pytest.raises(ValueError, match="q holds 1 non-finite entries"):
        coupling.mass_to_mole(bad, mw)
    bad = q.clone()
    bad[2, 5] = -1e-9
    with pytest.raises(ValueError, match="q holds negatives, the least -1e-09"):
        coupling.mass_to_mole(bad, mw)
    assert torch.isfinite(coupling.signed_mole_fractions(bad, mw)).all()
    bad = q.clone()
    bad[3] = 0.0
    with pytest.raises(ValueError, match="cell 3 holds no tracer mass"):
        coupling.mass_to_mole(bad, mw)
    with pytest.raises(ValueError, match=r"q must be \[cells, 69\]"):
        coupling.mass_to_mole(q[:, :5], mw)
    with pytest.raises(ValueError, match="mass must be finite and not negative"):
        coupling.mole_to_mass(coupling.mass_to_mole(q, mw), mw, torch.tensor([1.0, -1.0, 1.0, 1.0], dtype=torch.float64))


def test_element_totals(networks):
    net, mw = net_mw(networks)
    atoms = torch.as_tensor(np.asarray(net.atoms, dtype=np.float64))
    q = torch.full((3, len(mw)), 1e-3, dtype=torch.float64)
    e = coupling.element_moles(q, mw, atoms)
    assert e.shape == (3, len(net.elements))
    cell_mass = torch.tensor([1.0, 2.0, 3.0], dtype=torch.float64)
    t = coupling.tracer_totals(q, cell_mass, mw, atoms)
    assert float(t[0]) == pytest.approx(float(q.sum(1)[0]) * 6.0, rel=1e-14)
    assert torch.allclose(t[1:], (e * cell_mass[:, None]).sum(0), rtol=1e-14)


def test_require_finished_names_the_cause():
    done = torch.tensor([True, False, True, False])
    T, P = torch.tensor([1000.0, 1200.0, 900.0, 800.0]), torch.tensor([1e5, 2e5, 3e5, 4e5])
    coupling.require_finished(torch.ones(4, dtype=torch.bool), T, P, {}, "at cycle 1")
    with pytest.raises(coupling.UnfinishedCellsError, match=r"2 chemistry cell\(s\) not done at cycle 7; the first, "
                       r"cell 1: T 1200.0 K, P 2e\+05 Pa.*1 cell\(s\) still failing the guard after the recovery's 10"):
        coupling.require_finished(done, T, P, {"still_failed": 1, "unfinished": 1, "cold": 0}, "at cycle 7")
    with pytest.raises(coupling.UnfinishedCellsError, match="below the solver's 300-3000 K domain"):
        coupling.require_finished(done, T, P, {"cold": 2}, "here")
    with pytest.raises(coupling.UnfinishedCellsError, match="no count of the solver explains it"):
        coupling.require_finished(done, T, P, {}, "here")
    with pytest.raises(ValueError, match="done, T and P must all be"):
        coupling.require_finished(done[:2], T, P, {}, "here")
