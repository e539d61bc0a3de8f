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


@pytest.mark.parametrize("threads", [128, 96])
@pytest.mark.parametrize("name", list(synthetic.NETWORKS))
def test_thread_streams_reproduce_the_plain_sums(networks, name, threads):
    # emulate the kernel's walk of each thread's word stream: every row and entry is written once, with the sums of
    # the plain term lists in the same order (so bit for bit)
    tab = tables.build(networks(name), True)
    st = tab.streams[threads]
    rng = np.random.default_rng(3)
    v = np.append(rng.standard_normal(tab.nr), 0.0)
    code = np.array([1.0, -1.0, 2.0, -2.0])
    P, row_ptr = tables.sv_row_pieces(tab)
    part = np.full(int(row_ptr[-1]), np.nan)
    for t in range(threads):
        s, piece = 0.0, 0
        for q in range(st["sv"].shape[0]):
            w = int(st["sv"][q, t])
            s = s + code[(w >> 11) & 3] * v[w & 0x7FF]
            if w & tables.SV_END:
                d = int(st["sv_rows"][piece, t])
                assert np.isnan(part[d])
                part[d], s, piece = s, 0.0, piece + 1
    assert not np.isnan(part).any()
    got = np.array([sum(part[row_ptr[i] + 1 : row_ptr[i + 1]], part[row_ptr[i]]) for i in range(tab.ns)])
    want = np.zeros(tab.ns)
    for i in range(tab.ns):  # the oracle's order: pieces of P terms summed from 0, added in order
        terms = list(tab.sv_term[tab.sv_ptr[i] : tab.sv_ptr[i + 1]])
        acc = 0.0
        for c in range(0, max(1, len(terms)), P):
            p = 0.0
            for term in terms[c : c + P]:
                p = p + code[(int(term) >> 16) & 3] * v[int(term) & 0xFFFF]
            acc = p if c == 0 else acc + p
        want[i] = acc
    assert np.array_equal(got, want)
    k = np.append(rng.standard_normal(2 * tab.nr), 0.0)
    n = np.append(rng.standard_normal(tab.ns), 1.0)
    ld = tab.ns | 1
    A = np.full(tab.ns * ld, np.nan)
    for t in range(threads):
        acc, e = 0.0, 0
        for q in range(st["jt"].shape[0]):
            w = int(st["jt"][q, t])
            acc = acc + code[(w >> 12) & 3] * (k[w & 0xFFF] * n[(w >> 16) & 255] * n[w >> 24])
            if w & tables.J_END:
                d = int(st["jac_dst"][e, t])
                assert np.isnan(A[d])
                A[d], acc, e = -acc, 0.0, e + 1
    for e in range(len(tab.jac_entry)):
        p, qq = int(tab.jac_entry[e]) >> 16, int(tab.jac_entry[e]) & 0xFFFF
        acc = 0.0
        for term in tab.jac_term[tab.jac_ptr[e] : tab.jac_ptr[e + 1]]:
            w = int(term)
            acc = acc + code[(w >> 12) & 3] * (k[w & 0xFFF] * n[(w >> 16) & 255] * n[w >> 24])
        assert A[p * ld + qq] == -acc
    assert np.isnan(A).sum() == tab.ns * ld - len(tab.jac_entry)
