"""The seeded workloads: the uneven batch's night half is dark, and cold starts stay normalised."""

import numpy as np

from maxichem_b200 import synthetic


def test_the_uneven_batch_has_a_dark_half(networks):
    net = networks("chno69")
    w = synthetic.workload(net, "uneven", 1024, seed=1)
    columns = np.arange(1024) // 64
    assert not w.J[columns >= 8].any()
    assert w.J[columns < 8].any()
    assert np.array_equal(w.T, synthetic.workload(net, "uneven", 1024, seed=1).T)


def test_cold_starts_are_a_quarter_and_normalised(networks):
    net = networks("chno69")
    w = synthetic.workload(net, "column", 4096, seed=2)
    x, h, cold = synthetic.cold_start(w.x, w.h, seed=3)
    assert 0.2 < cold.mean() < 0.3
    assert np.abs(x.sum(1) - 1.0).max() < 1e-14
    assert (h[cold] == 1e-10).all() and (h[~cold] == w.h[~cold]).all()
    assert np.array_equal(x[~cold], w.x[~cold]) and not np.array_equal(x[cold], w.x[cold])
