"""ADSolver's host logic without a GPU: the constructor's cap, and the tangents' forms and their refusals by name
(the reference's kincuda_ad.py:135-148 and 304-339; its tests/test_ad.py:721-757)."""

import pytest
import torch

from maxichem_b200 import synthetic
from maxichem_b200.ad import ADSolver
from maxichem_b200.constants import DMAX


@pytest.mark.parametrize("cap", [0, -3, 2.5, "8"])
def test_cap_is_checked_before_any_device_work(cap):
    net = synthetic.network("cho41")
    with pytest.raises(ValueError, match="cap"):
        ADSolver(net, "cuda:0", cap=cap, photo=True)


def solver_shape(ns=5, nr=7, nj=2):
    """An ADSolver's shape without a device: only the host checks run."""
    s = object.__new__(ADSolver)
    s.ns, s.nr, s.nj, s.dev = ns, nr, nj, torch.device("cpu")
    return s


def tangents(B, lead=(), ns=5, nr=7, nj=2):
    z = lambda *shape: torch.zeros(*lead, *shape, dtype=torch.float64)  # noqa: E731
    return {"dx": z(B, ns), "dT": z(B), "dP": z(B), "ddt": z(B), "dh": z(B), "dlm": z(B, nr),
            "drc": z(nr, 9), "dJ": z(B, nj)}  # fmt: skip


def test_one_direction_and_a_leading_axis():
    s = solver_shape()
    assert s._check_tangents(tangents(4), 4) == 1
    assert s._check_tangents(tangents(4, (3,)), 4) == 3
    assert s._check_tangents(tangents(4, (DMAX,)), 4) == DMAX


def test_too_many_directions_are_refused():
    s = solver_shape()
    with pytest.raises(ValueError, match=f"from 1 to {DMAX} directions"):
        s._check_tangents(tangents(4, (DMAX + 1,)), 4)


@pytest.mark.parametrize("name", ["dT", "dP", "ddt", "dh", "dlm", "drc", "dJ"])
def test_a_wrong_tangent_is_refused_by_name(name):
    s = solver_shape()
    t = tangents(4)
    t[name] = t[name][..., :-1] if t[name].dim() > 1 else t[name][:-1]
    with pytest.raises(ValueError, match=name):
        s._check_tangents(t, 4)


def test_a_wrong_dtype_is_refused_by_name():
    s = solver_shape()
    t = tangents(4)
    t["dP"] = t["dP"].float()
    with pytest.raises(ValueError, match="dP"):
        s._check_tangents(t, 4)


def test_dx_must_be_two_or_three_dimensional():
    s = solver_shape()
    t = tangents(4)
    t["dx"] = torch.zeros(20, dtype=torch.float64)
    with pytest.raises(ValueError, match="dx"):
        s._check_tangents(t, 4)


def test_without_photolysis_an_empty_dJ_counts_as_none():
    s = solver_shape(nj=0)
    t = tangents(4, nj=0)
    assert s._check_tangents(t, 4) == 1
    t["dJ"] = torch.zeros(4, 3, dtype=torch.float64)
    with pytest.raises(ValueError, match="dJ: none or an empty"):
        s._check_tangents(t, 4)
