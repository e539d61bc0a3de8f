"""Batching forms on the GPU: every grid choice (persistent CTAs per SM, or one CTA per cell) gives the same bits, the
autotuner picks one of them and leaves the counts alone, and a call loop captured in a CUDA graph gives the same
results and counts as the same calls made one by one."""

import numpy as np
import pytest
import torch

from maxichem_b200 import autotune, graph, synthetic
from maxichem_b200.solver import CudaSolver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def uneven(gpu, networks):
    net = networks("cho41")
    w = synthetic.workload(net, "uneven", 1024, seed=4)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=gpu)
    solver = CudaSolver(net, gpu, photo=True)
    x, h, _, _ = solver(t(w.x), t(w.T), t(w.P), t(w.dt), t(w.h), J=t(w.J))
    xc, hc, cold = synthetic.cold_start(x.cpu().numpy(), h.cpu().numpy(), seed=5)
    yield solver, (t(xc), t(w.T), t(w.P), t(w.dt), t(hc), t(w.J)), cold
    solver.close()


def call(solver, args):
    x, T, P, dt, h, J = args
    return solver.launch(x, T, P, dt, h, J=J)


def test_every_grid_gives_the_same_bits(uneven):
    solver, args, cold = uneven
    solver.set_grid(-1)
    ref = call(solver, args)
    assert solver.info["grid_ctas_per_sm"] == solver.info["call_ctas_per_sm"]
    for grid in (0, 1, solver.info["call_ctas_per_sm"]):
        solver.set_grid(grid)
        assert solver.info["grid_ctas_per_sm"] == grid
        got = call(solver, args)
        assert all(torch.equal(a, b) for a, b in zip(got, ref, strict=True)), grid
    solver.set_grid(-1)
    steps = ref.steps.cpu().numpy()
    assert steps[cold].mean() > 3 * steps[~cold].mean()  # the batch is uneven


def test_a_grid_beyond_the_occupancy_limit_is_refused(uneven):
    solver, _, _ = uneven
    most = max(solver.info["call_ctas_per_sm"], solver.info["mixed_ctas_per_sm"])  # each kernel takes at most its own
    with pytest.raises(ValueError, match="ctas_per_sm from -1 to"):
        solver.set_grid(most + 1)
    with pytest.raises(ValueError, match="ctas_per_sm from -1 to"):
        solver.set_grid(-2)


def test_the_tuner_picks_a_grid_and_keeps_the_counts(uneven):
    solver, (x, T, P, dt, h, J), _ = uneven
    before = solver.total.clone()
    got = autotune.tune_grid(solver, x, T, P, dt, h, J=J, choices=[0, 1, solver.info["call_ctas_per_sm"]])
    assert got["best"] in (0, 1, solver.info["call_ctas_per_sm"])
    assert set(got["ms"]) == {0, 1, solver.info["call_ctas_per_sm"]} and all(v > 0 for v in got["ms"].values())
    assert solver.info["grid_ctas_per_sm"] == got["best"]
    assert autotune.cached(solver, x.shape[0]) == got["best"]
    assert torch.equal(solver.total, before)
    solver.set_grid(-1)


def test_a_captured_loop_equals_the_calls_one_by_one(uneven):
    solver, (x, T, P, dt, h, J), _ = uneven
    calls = 3
    before = solver.total.clone()
    xs, hs, outs = x, h, []
    for _ in range(calls):
        r = solver.launch_raw(xs, T, P, dt, hs, rtol=1e-3, atol=1e-25, max_steps=4000, J=J)
        outs.append({k: v.clone() for k, v in r.items()})
        xs, hs = r["x"], r["h"]
    eager_total = solver.total - before
    loop = graph.CallLoop(solver, x, T, P, dt, h, J=J, calls=calls)
    mid = solver.total.clone()
    last = loop.run()
    torch.cuda.synchronize()
    for k in ("x", "h", "steps", "done", "flag", "status"):
        assert torch.equal(last[k], outs[-1][k]), k
    assert torch.equal(solver.total - mid, eager_total)
    loop.carry()
    assert torch.equal(loop.x_in, outs[-1]["x"]) and torch.equal(loop.h_in, outs[-1]["h"])
    loop.close()


def test_a_captured_loop_refuses_a_cold_cell(uneven):
    solver, (x, T, P, dt, h, J), _ = uneven
    n = 256
    T2 = T[:n].clone()
    T2[5] = 250.0  # below the solver's range: every call of the loop refuses it
    loop = graph.CallLoop(solver, x[:n], T2, P[:n], dt[:n], h[:n], J=J[:n], calls=2)
    with pytest.raises(ValueError, match=r"the call loop refused cells: 2 cold over its 2 calls"):
        loop.run()
    before = solver.total.clone()
    loop.run(check=False)
    assert loop.refused(before) == {"bad_input": 0, "cold": 2, "hot": 0}
    loop.close()


@pytest.mark.parametrize("name", ["cho41", "chno69", "sncho91"])
def test_two_warps_per_cell_give_the_same_bits(gpu, networks, name):
    net = networks(name)
    w = synthetic.workload(net, "uneven", 1024, seed=13)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=gpu)
    args = [t(a) for a in (w.x, w.T, w.P, w.dt, w.h)]
    with CudaSolver(net, gpu, photo=True, warps=4) as four, CudaSolver(net, gpu, photo=True, warps=2) as two:
        assert two.info["warps"] == 2 and four.info["warps"] == 4
        a = four.launch(*args, J=t(w.J))
        b = two.launch(*args, J=t(w.J))
        assert four.fallback == two.fallback
    for k in ("x", "h", "done", "steps", "flag"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k


def test_the_tuner_picks_a_mapping_and_a_grid(gpu, networks):
    net = networks("cho41")
    w = synthetic.workload(net, "uneven", 4096, seed=14)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=gpu)
    args = [t(a) for a in (w.x, w.T, w.P, w.dt, w.h)]
    solver, got = autotune.tune(net, gpu, *args, J=t(w.J))
    assert got["warps"] in (2, 4) and solver.info["warps"] == got["warps"]
    assert solver.info["grid_ctas_per_sm"] == got["grid"]
    assert {k[0] for k in got["ms"]} == {2, 4}
    r = solver.launch(*args, J=t(w.J))
    with CudaSolver(net, gpu, photo=True) as plain:
        assert torch.equal(plain.launch(*args, J=t(w.J)).x, r.x)
    solver.close()


def test_the_derivatives_refuse_two_warps(gpu, networks):
    import ctypes

    from maxichem_b200 import abi

    lib = abi.library()
    err = ctypes.create_string_buffer(256)
    with CudaSolver(networks("cho41"), gpu, photo=True, warps=2) as two:
        n = len(abi.SIGNATURES["mx_jvp"][1])
        args = [two._handle] + [None] * 8 + [0, 1e-3, 1e-25, 4000, 1, 1] + [None] * 18 + [None, err, 256]
        assert len(args) == n
        assert lib.mx_jvp(*args) == 3  # MX_ERR_NETWORK
    assert b"4 warps per cell" in err.value


def test_the_default_mapping_follows_the_network_size(gpu, networks):
    # 41 species: a cell's shared memory lets at least 6 cells share an SM, so 2 warps by default; 69 and 91 species
    # fit 4 or fewer, so 4 warps; the derivative solver takes 4 whatever the size
    from maxichem_b200 import abi, tables
    from maxichem_b200.ad import ADSolver
    from maxichem_b200.solver import TWO_WARP_CELLS

    lib = abi.library()
    for name, want in (("cho41", 2), ("chno69", 4), ("sncho91", 4)):
        net = networks(name)
        with CudaSolver(net, gpu, photo=True) as s:
            assert s.info["warps"] == want, name
        cells = lib.mx_cells_per_sm(abi.NetworkStruct(tables.build(net, True, warps=4)).ref(), gpu.index or 0)
        assert (cells >= TWO_WARP_CELLS) == (want == 2), (name, cells)
    with ADSolver(networks("cho41"), gpu, photo=True) as ad:
        assert ad.info["warps"] == 4
