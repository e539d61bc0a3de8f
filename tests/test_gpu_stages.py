"""Each stage of one try on the GPU against the oracle's, on one cell (mx_debug_try against mxo_debug_try)."""

import numpy as np
import pytest
import torch

import oracle
from maxichem_b200 import abi, synthetic
from maxichem_b200.solver import CudaSolver

pytestmark = pytest.mark.gpu


def _rel(a, b):
    """Largest difference relative to the vector's largest entry (a component far below it carries the rounding of
    its larger neighbours, so it is not judged against itself)."""
    scale = max(np.abs(a).max(), np.abs(b).max())
    return float(np.abs(a - b).max() / scale) if scale > 0 else 0.0


@pytest.mark.parametrize("name", ["cho41", "chno69"])
def test_each_stage_of_one_try_matches_the_oracle(gpu, networks, name):
    net = networks(name)
    w = synthetic.workload(net, "column", 64, seed=2)
    with CudaSolver(net, gpu, photo=True) as solver:
        ref = oracle.Oracle(solver.tab)
        worst = {}
        for cell in (0, 10, 40, 63):
            out = torch.empty(oracle.debug_size(solver.tab), dtype=torch.float64, device=gpu)
            x = torch.tensor(w.x[cell], dtype=torch.float64, device=gpu)
            J = torch.tensor(w.J[cell], dtype=torch.float64, device=gpu)
            h = 1e-3
            rc = abi.library().mx_debug_try(solver._handle, x.data_ptr(), float(w.T[cell]), float(w.P[cell]), h,
                                            J.data_ptr(), 1e-3, 1e-25, out.data_ptr(), None)  # fmt: skip
            assert rc == 0
            torch.cuda.synchronize()
            g = oracle.split_debug(solver.tab, out.cpu().numpy())
            r = ref.debug_try(w.x[cell], float(w.T[cell]), float(w.P[cell]), h, J=w.J[cell])
            for k in g:
                worst[k] = max(worst.get(k, 0.0), _rel(g[k], r[k]))
        print(name, {k: f"{v:.1e}" for k, v in worst.items()})
        for k in ("kf", "kr", "F", "u0", "Jn", "dinv", "Y"):
            assert worst[k] < 1e-13, (k, worst[k])
        for k in ("w", "LU", "K1", "K2", "K3", "K4", "err"):
            assert worst[k] < 1e-10, (k, worst[k])
