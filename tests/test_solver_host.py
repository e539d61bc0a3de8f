"""The Python surface's host logic without a GPU: keyword-only settings, named results, and the form checks that
refuse inputs before any launch (the reference's tests/test_call_interface.py and _solver.py:34-130)."""

import inspect

import numpy as np
import pytest
import torch

import invented
from maxichem_b200.constants import COUNTS
from maxichem_b200.solver import CallResult, CudaSolver, LaunchResult, check_inputs, check_photolysis

CPU = torch.device("cpu")
CALLS = {"call": (CudaSolver.__call__, 5), "launch": (CudaSolver.launch, 5)}


@pytest.mark.parametrize("name", [*CALLS, "constructor"])
def test_every_optional_argument_is_keyword_only(name):
    function = CALLS[name][0] if name in CALLS else CudaSolver.__init__
    parameters = list(inspect.signature(function).parameters.values())[1:]
    positional = [p for p in parameters if p.kind is not inspect.Parameter.KEYWORD_ONLY]
    assert [p.name for p in positional if p.default is not p.empty] == []
    assert len(positional) == (CALLS[name][1] if name in CALLS else 2)


@pytest.mark.parametrize("name", CALLS)
def test_settings_by_position_are_refused(name):
    function, inputs = CALLS[name]
    solver = object.__new__(CudaSolver)
    with pytest.raises(TypeError, match=r"positional arguments? but \d+ were given"):
        function(solver, *([None] * inputs), 1e-25)


def test_results_are_named_tuples_in_the_reference_order():
    assert CallResult._fields == ("x", "h", "done", "steps")
    assert LaunchResult._fields == ("x", "h", "done", "steps", "flag")


def test_counts_have_the_reference_order():
    assert COUNTS == ("bad_input", "cold", "hot", "nonfinite", "unfinished", "drift", "recomputed", "recovered",
                      "still_failed", "nonfinite_h")  # fmt: skip


def inputs(B=4, ns=6):
    x = torch.full((B, ns), 1.0 / ns, dtype=torch.float64)
    T, P, dt, h = (torch.full((B,), v, dtype=torch.float64) for v in (1000.0, 1e6, 1.0, 1e-3))
    return x, T, P, dt, h


def test_form_checks_pass_good_inputs():
    assert check_inputs(CPU, 6, *inputs(), 1e-3, 1e-25, 4000) == 4


@pytest.mark.parametrize(
    "change,message",
    [
        (lambda a: a.__setitem__(0, a[0][:, :5]), r"^x: \[B, 6\] expected, got \[4, 5\]"),
        (lambda a: a.__setitem__(0, a[0].float()), r"^x: float64 \[4, 6\] on cpu expected, got torch.float32"),
        (lambda a: a.__setitem__(1, a[1][:3]), r"^T: float64 \[4\] on cpu expected, got torch.float64 \[3\]"),
        (lambda a: a.__setitem__(2, a[2].reshape(4, 1)), r"^P: float64 \[4\]"),
        (lambda a: a.__setitem__(3, a[3].to(torch.int64)), r"^dt: float64"),
        (lambda a: a.__setitem__(4, a[4][None]), r"^h: float64"),
    ],
)  # fmt: skip
def test_wrong_forms_are_refused(change, message):
    a = list(inputs())
    change(a)
    with pytest.raises(ValueError, match=message):
        check_inputs(CPU, 6, *a, 1e-3, 1e-25, 4000)


@pytest.mark.parametrize("rtol,atol", [(0.0, 1e-25), (1e-3, -1.0), (float("nan"), 1e-25), (1e-3, float("inf"))])
def test_tolerances_must_be_finite_and_positive(rtol, atol):
    with pytest.raises(ValueError, match="rtol and atol finite and positive expected"):
        check_inputs(CPU, 6, *inputs(), rtol, atol, 4000)


@pytest.mark.parametrize("max_steps", [0, -1, 2**31 // 10 + 1, 2.5, "10"])
def test_max_steps_must_be_a_positive_integer_within_the_recovery_range(max_steps):
    with pytest.raises(ValueError, match="max_steps"):
        check_inputs(CPU, 6, *inputs(), 1e-3, 1e-25, max_steps)


def test_max_steps_accepts_numpy_integers():
    assert check_inputs(CPU, 6, *inputs(), 1e-3, 1e-25, np.int64(7)) == 4


def test_photolysis_rates_are_checked():
    J = torch.zeros(4, 3, dtype=torch.float64)
    assert check_photolysis(J, 4, 3, CPU) is not None
    with pytest.raises(ValueError, match=r"^J \[B, 3\] is required with photolysis"):
        check_photolysis(None, 4, 3, CPU)
    with pytest.raises(ValueError, match=r"^J: float64 \[4, 3\]"):
        check_photolysis(J[:, :2], 4, 3, CPU)
    assert check_photolysis(None, 4, 0, CPU) is None
    assert check_photolysis(torch.zeros(4, 0, dtype=torch.float64), 4, 0, CPU) is None
    with pytest.raises(ValueError, match=r"^J: none or an empty \[4, 0\] one expected"):
        check_photolysis(J, 4, 0, CPU)


def test_photo_needs_branches(tmp_path):
    net, _ = invented.hydrogen(tmp_path)
    with pytest.raises(ValueError, match="photo=True needs a network with photolysis branches"):
        CudaSolver(net, "cuda:0", photo=True)


@pytest.mark.parametrize("drift", [-1e-6, float("nan"), float("inf")])
def test_drift_must_be_finite_and_not_negative(tmp_path, drift):
    net, _ = invented.hydrogen(tmp_path)
    with pytest.raises(ValueError, match="drift: a finite allowance of at least 0 expected"):
        CudaSolver(net, "cuda:0", drift=drift)


def test_a_cpu_device_is_refused(tmp_path):
    net, _ = invented.hydrogen(tmp_path)
    with pytest.raises(ValueError, match="a CUDA device expected"):
        CudaSolver(net, "cpu")
