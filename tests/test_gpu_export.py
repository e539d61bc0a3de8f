"""A caller without Python on the GPU: a C++ program (tests/cpp/call_export.cpp) builds a solver from a folder that
CudaSolver.export wrote and makes a call; its results equal the Python call's bit for bit (the reference's
tests/test_export_cpp.py checks the same of its C++ caller), and its refusal names the refused cells."""

import subprocess

import numpy as np
import pytest
import torch

import test_export
from maxichem_b200 import synthetic
from maxichem_b200.solver import CudaSolver

pytestmark = pytest.mark.gpu


def run(exe, folder, io, inputs, B):
    io.mkdir(exist_ok=True)
    for name, a in inputs.items():
        np.ascontiguousarray(a, dtype="<f8").tofile(io / f"{name}.bin")
    r = subprocess.run([str(exe), str(folder), str(io), str(B)], capture_output=True, text=True, timeout=300)
    out = {k: np.fromfile(io / f"{k}.bin", dtype="<f8") for k in ("x_out", "h_out", "steps")}
    out.update({k: np.fromfile(io / f"{k}.bin", dtype="<i4") for k in ("done", "flag", "status", "count")})
    return r, out


@pytest.mark.parametrize("name", ["cho41", "chno69"])
def test_the_cpp_call_equals_the_python_call(gpu, networks, tmp_path, name):
    net = networks(name)
    B = 256
    w = synthetic.workload(net, "column", B, seed=8)
    with CudaSolver(net, gpu, photo=True) as solver:
        solver.export(tmp_path / "export")
        t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=gpu)
        ref = solver.launch(t(w.x), t(w.T), t(w.P), t(w.dt), t(w.h), J=t(w.J))
        count = solver.count.cpu().numpy()
    exe = test_export.compile_caller(tmp_path / "call_export")
    r, out = run(exe, tmp_path / "export", tmp_path / "io", {"x": w.x, "T": w.T, "P": w.P, "dt": w.dt, "h": w.h,
                                                               "J": w.J}, B)  # fmt: skip
    assert r.returncode == 0, r.stdout + r.stderr
    assert np.array_equal(out["x_out"].reshape(B, -1), ref.x.cpu().numpy())
    assert np.array_equal(out["h_out"], ref.h.cpu().numpy()) and np.array_equal(out["steps"], ref.steps.cpu().numpy())
    assert np.array_equal(out["done"], ref.done.cpu().numpy().astype(np.int32))
    assert np.array_equal(out["flag"], ref.flag.cpu().numpy()) and np.array_equal(out["count"], count)


def test_the_cpp_call_refuses_and_names_bad_cells(gpu, networks, tmp_path):
    net = networks("cho41")
    B = 16
    w = synthetic.workload(net, "column", B, seed=9)
    x, T = w.x.copy(), w.T.copy()
    x[5, 3] = np.nan
    T[2] = 250.0
    with CudaSolver(net, gpu, photo=True) as solver:
        solver.export(tmp_path / "export")
    exe = test_export.compile_caller(tmp_path / "call_export")
    r, out = run(exe, tmp_path / "export", tmp_path / "io", {"x": x, "T": T, "P": w.P, "dt": w.dt, "h": w.h,
                                                               "J": w.J}, B)  # fmt: skip
    assert r.returncode == 3, r.stdout + r.stderr
    assert "1 cells below 300 K (first: cell 2)" in r.stdout
    assert "1 cells of bad input" in r.stdout and "(first: cell 5)" in r.stdout
    assert out["count"][1] == 1 and out["count"][2] == 1 and out["status"][5] == 2 and out["status"][2] == 1
