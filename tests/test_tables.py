"""The kernel tables against the reference table builder's (golden): order, fill, rate rows, flags, species slots."""

from pathlib import Path

import numpy as np
import pytest

from maxichem_b200 import synthetic, tables

GOLDEN = Path(__file__).parent / "golden"


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN / "tables.npz")


@pytest.mark.parametrize("photo", [False, True])
@pytest.mark.parametrize("name", list(synthetic.NETWORKS))
def test_tables_match_the_reference_builder(golden, networks, name, photo):
    tab = tables.build(networks(name), photo)
    p = f"{name}/{int(photo)}"
    assert np.array_equal(tab.perm, golden[f"{p}/perm"])  # the pivots, so the factorisation's rounding
    k0 = int(golden[f"{p}/k0"])
    lead = {(int(i), int(j)) for i, j in golden[f"{p}/lead"]}
    mine = {(i, j) for i, j in zip(*np.nonzero(tab.fill)) if not (i >= k0 and j >= k0)}
    assert mine == lead
    rc = golden[f"{p}/rc"]
    assert np.array_equal(tab.rc[:, : rc.shape[1]], rc)
    assert np.array_equal(tab.rf, golden[f"{p}/rf"])
    assert np.array_equal(tab.rx, golden[f"{p}/rx"])


def test_term_lists_restate_the_stoichiometry(networks):
    net = networks("cho41")
    tab = tables.build(net, True)
    S = np.hstack([net.S, net.Sp])
    code = np.array([1.0, -1.0, 2.0, -2.0])
    dense = np.zeros((tab.ns, tab.nr))
    for i in range(tab.ns):
        for t in range(tab.sv_ptr[i], tab.sv_ptr[i + 1]):
            w = int(tab.sv_term[t])
            dense[i, w & 0xFFFF] = code[(w >> 16) & 3]
    assert np.array_equal(dense, S[tab.perm])
    # every Jacobian entry lies inside the fill pattern, and the fill contains the diagonal
    p, q = tab.jac_entry >> 16, tab.jac_entry & 0xFFFF
    assert tab.fill[p, q].all() and tab.fill.diagonal().all()


def test_work_counts(networks):
    f = tables.build(networks("chno69"), True).flops
    assert f["lu"] < f["dense_lu"]  # the fill pattern is sparser than dense
    assert f["fresh_try"] > f["retry"] > 0
