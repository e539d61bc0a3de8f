"""The GCM step either side of a chemistry call: mass mixing ratios and mole fractions, element totals, and the stop
when a call leaves cells unfinished (the reference's maxichem/coupling/composition.py:48-235 and
maxichem/coupling/chemistry.py:15-96, with the same names, arguments, checks and messages).

The GCM carries each species as a mass mixing ratio q (kg per kg of gas); the call takes mole fractions. On CUDA
tensors the two conversions are the library's one-pass kernels (mx_mass_to_mole, mx_mole_to_mass: one warp per
cell, row sums in the warp's order); the checks read back one word of problem bits, and only a failed check looks
at the data again to say what failed. On CPU tensors they are the same formulas in torch.
"""

from __future__ import annotations

from collections.abc import Mapping, Sequence

import numpy as np
import torch

from . import abi
from .constants import REC_STEPS, T_MAX, T_MIN, X_SUM_TOL

__all__ = ["ATOMIC_MASS", "PA_TO_DYN_CM2", "UnfinishedCellsError", "element_moles", "mass_to_mole", "molar_masses",
           "mole_to_mass", "require_finished", "signed_mole_fractions", "tracer_totals"]  # fmt: skip

PA_TO_DYN_CM2 = 10.0  # the call takes pressure in dyn cm^-2: 1 Pa = 10 dyn cm^-2

# kg/mol, the atomic weights the reference's coupling uses (composition.py:28)
ATOMIC_MASS = {"H": 1.008e-3, "He": 4.002602e-3, "C": 12.011e-3, "N": 14.007e-3, "O": 15.999e-3, "S": 32.06e-3}


def _check_molar_masses(mw: torch.Tensor) -> None:
    if mw.dim() != 1:
        raise ValueError(f"mw must be [S], got shape {tuple(mw.shape)}")
    if not bool((torch.isfinite(mw) & (mw > 0)).all()):
        raise ValueError(f"mw must be finite and positive, its least value is {float(mw.min())!r} kg/mol")


def _check_shape(name: str, a: torch.Tensor, mw: torch.Tensor) -> None:
    _check_molar_masses(mw)
    if a.dim() != 2 or a.shape[1] != mw.shape[0]:
        raise ValueError(f"{name} must be [cells, {mw.shape[0]}], got shape {tuple(a.shape)}")


def _nonfinite(name: str, a: torch.Tensor) -> ValueError:
    return ValueError(f"{name} holds {int((~torch.isfinite(a)).sum())} non-finite entries")


def _check_per_cell(name: str, a: torch.Tensor, cells: int) -> None:
    if a.shape != (cells,):
        raise ValueError(f"{name} must be [{cells}], got shape {tuple(a.shape)}")
    if not bool((torch.isfinite(a) & (a >= 0)).all()):
        raise ValueError(f"{name} must be finite and not negative, its least value is {float(a.min())!r}")


def molar_masses(atoms: np.ndarray | torch.Tensor, elements: Sequence[str]) -> torch.Tensor:
    """Each species' molar mass from its atoms [S, E] and the columns' elements: kg/mol, float64 on the CPU."""
    missing = [e for e in elements if e not in ATOMIC_MASS]
    if missing:
        raise ValueError(f"no atomic mass for {missing}: add them to maxichem_b200.coupling.ATOMIC_MASS")
    a = torch.as_tensor(atoms, dtype=torch.float64).cpu()
    if a.dim() != 2 or a.shape[1] != len(elements):
        raise ValueError(f"atoms must be [species, {len(elements)}], got shape {tuple(a.shape)}")
    if not bool((torch.isfinite(a) & (a >= 0)).all()):
        raise ValueError("atoms must be finite and not negative: check the network's atoms table")
    mw = a @ torch.tensor([ATOMIC_MASS[e] for e in elements], dtype=torch.float64)
    empty = torch.nonzero(mw <= 0).flatten().tolist()
    if empty:
        raise ValueError(f"species rows {empty} have no atoms, so no molar mass: check the network's atoms table")
    return mw


def _device_pass(entry: str, args: list, dev: torch.device) -> int:
    bad = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = getattr(abi.library(), entry)(*args, bad.data_ptr(), stream)
    if rc:
        raise RuntimeError(f"{entry} failed with status {rc}")
    return int(bad.item())


def _to_mole(q: torch.Tensor, mw: torch.Tensor, signed: bool) -> torch.Tensor:
    _check_shape("q", q, mw)
    if q.dtype != mw.dtype:
        raise ValueError(f"q and mw must share one precision, got {q.dtype}, {mw.dtype}")
    if q.is_cuda and q.dtype == torch.float64:
        q, mw = q.contiguous(), mw.to(q.device).contiguous()
        x = torch.empty_like(q)
        bad = _device_pass("mx_mass_to_mole", [q.data_ptr(), mw.data_ptr(), q.shape[0], q.shape[1], int(signed),
                                               x.data_ptr()], q.device)  # fmt: skip
        if bad & 1:
            raise _nonfinite("q", q)
        if bad & 2:
            raise ValueError(f"q holds negatives, the least {float(q.min()):.3g}: clamp them before the conversion")
        if bad & 4:
            cell = int(torch.nonzero((q / mw).sum(1) <= 0)[0])
            raise ValueError(f"cell {cell} holds no tracer mass, so it has no mole fractions: check its tracers")
        return x
    if not bool(torch.isfinite(q).all()):
        raise _nonfinite("q", q)
    if not signed and bool((q < 0).any()):
        raise ValueError(f"q holds negatives, the least {float(q.min()):.3g}: clamp them before the conversion")
    n = q / mw
    total = n.sum(1, keepdim=True)
    if not signed and bool((total <= 0).any()):
        cell = int(torch.nonzero(total.flatten() <= 0)[0])
        raise ValueError(f"cell {cell} holds no tracer mass, so it has no mole fractions: check its tracers")
    return n / total


def mass_to_mole(q: torch.Tensor, mw: torch.Tensor) -> torch.Tensor:
    """Mole fractions [cells, S] of mass mixing ratios q [cells, S] (finite, not negative) with molar masses mw [S]:
    n / sum(n), n = q / mw (composition.py:102-127)."""
    return _to_mole(q, mw, signed=False)


def signed_mole_fractions(q: torch.Tensor, mw: torch.Tensor) -> torch.Tensor:
    """The same conversion for output, keeping the transport's negatives; never feed these to the chemistry
    (composition.py:130-151)."""
    return _to_mole(q, mw, signed=True)


def mole_to_mass(x: torch.Tensor, mw: torch.Tensor, mass: torch.Tensor) -> torch.Tensor:
    """Mass mixing ratios [cells, S] that hold each cell's tracer mass `mass` [cells]: x mw (mass / sum(x mw))
    (composition.py:154-182)."""
    _check_shape("x", x, mw)
    if not (x.dtype == mw.dtype == mass.dtype):
        raise ValueError(f"x, mw and mass must share one precision, got {x.dtype}, {mw.dtype}, {mass.dtype}")
    if mass.shape != (x.shape[0],):
        raise ValueError(f"mass must be [{x.shape[0]}], got shape {tuple(mass.shape)}")
    if x.is_cuda and x.dtype == torch.float64:
        x, mw, mass = x.contiguous(), mw.to(x.device).contiguous(), mass.contiguous()
        q = torch.empty_like(x)
        bad = _device_pass("mx_mole_to_mass", [x.data_ptr(), mw.data_ptr(), mass.data_ptr(), x.shape[0],
                                               x.shape[1], q.data_ptr()], x.device)  # fmt: skip
        if bad & 1:
            raise _nonfinite("x", x)
        if bad & 8:
            _check_per_cell("mass", mass, x.shape[0])
        if bad & 2:
            raise ValueError(f"x holds negatives, the least {float(x.min()):.3g}: the call's result is not usable")
        if bad & 4:
            cell = int(torch.nonzero((x * mw).sum(1) <= 0)[0])
            raise ValueError(f"cell {cell} has mole fractions of no mass (sum of x * mw <= 0): check the call's result")
        return q
    if not bool(torch.isfinite(x).all()):
        raise _nonfinite("x", x)
    _check_per_cell("mass", mass, x.shape[0])
    if bool((x < 0).any()):
        raise ValueError(f"x holds negatives, the least {float(x.min()):.3g}: the call's result is not usable")
    xm = x * mw
    weight = xm.sum(1)
    if bool((weight <= 0).any()):
        cell = int(torch.nonzero(weight <= 0)[0])
        raise ValueError(f"cell {cell} has mole fractions of no mass (sum of x * mw <= 0): check the call's result")
    return xm * (mass / weight)[:, None]


def element_moles(q: torch.Tensor, mw: torch.Tensor, atoms: torch.Tensor) -> torch.Tensor:
    """Each cell's moles of each element per kg of gas [cells, E]: (q / mw) atoms (composition.py:185-209)."""
    _check_shape("q", q, mw)
    if not bool(torch.isfinite(q).all()):
        raise _nonfinite("q", q)
    if atoms.dim() != 2 or atoms.shape[0] != mw.shape[0]:
        raise ValueError(f"atoms must be [{mw.shape[0]}, elements], got shape {tuple(atoms.shape)}")
    if not bool(torch.isfinite(atoms).all()):
        raise ValueError("atoms holds non-finite entries: check the network's atoms table")
    if not (q.dtype == mw.dtype == atoms.dtype):
        raise ValueError(f"q, mw and atoms must share one precision, got {q.dtype}, {mw.dtype}, {atoms.dtype}")
    return (q / mw) @ atoms


def tracer_totals(q: torch.Tensor, cell_mass: torch.Tensor, mw: torch.Tensor, atoms: torch.Tensor) -> torch.Tensor:
    """The tracers' mass (kg) and each element's moles summed over the cells [1 + E] (composition.py:212-234)."""
    moles = element_moles(q, mw, atoms)
    _check_per_cell("cell_mass", cell_mass, q.shape[0])
    mass = (q * cell_mass[:, None]).sum()
    return torch.cat([mass.view(1), (moles * cell_mass[:, None]).sum(0)])


class UnfinishedCellsError(RuntimeError):
    """A chemistry call returned cells that are not done."""


def _causes(counts: Mapping[str, int]) -> list[str]:
    out = []
    for name, side, edge in (("cold", "below", T_MIN), ("hot", "above", T_MAX)):
        if counts.get(name):
            out.append(
                f"{counts[name]} cell(s) {side} the solver's {T_MIN:g}-{T_MAX:g} K domain (refused at {edge:g} K). "
                f"No solver setting helps: the flow made them this {name}; look at the deck (its lid, its radiation) "
                "where they are"
            )
    if counts.get("bad_input"):
        out.append(
            f"{counts['bad_input']} cell(s) with bad input (non-finite or negative mole fractions, |sum(x) - 1| above "
            f"{X_SUM_TOL:g}, none above 0, P non-finite, P <= 0 or P / (k_B T) overflowing, a non-finite T, dt < 0 "
            "or a bad J). The driver's inputs to the call are wrong there: check the cells' tracers, their "
            "normalization, T and P"
        )
    if counts.get("still_failed"):
        out.append(
            f"{counts['still_failed']} cell(s) still failing the guard after the recovery's {REC_STEPS} times longer "
            f"try (in the call: {counts.get('unfinished', 0)} out of steps, {counts.get('nonfinite', 0)} non-finite, "
            f"{counts.get('drift', 0)} element drift). Run with a shorter --dt"
        )
    return out or ["no count of the solver explains it; report this with the counts above"]


def require_finished(done: torch.Tensor, T: torch.Tensor, P: torch.Tensor, counts: Mapping[str, int],
                     where: str) -> None:
    """Raise UnfinishedCellsError when the call left any cell not done, naming the cause from the call's counts
    (``CudaSolver.fallback``) and its fix (chemistry.py:54-96). P is in Pa, for the message."""
    if not (done.dim() == 1 and done.shape == T.shape == P.shape):
        shapes = [tuple(a.shape) for a in (done, T, P)]
        raise ValueError(f"done, T and P must all be [cells], got shapes {shapes}")
    bad = ~done.bool()
    if not bool(bad.any()):
        return
    i = int(torch.nonzero(bad)[0])
    risen = {k: int(v) for k, v in counts.items() if v}
    raise UnfinishedCellsError(
        f"{int(bad.sum())} chemistry cell(s) not done {where}; the first, cell {i}: T {float(T[i]):.1f} K, "
        f"P {float(P[i]):.4g} Pa. The call's counts: {risen}. " + ". ".join(_causes(risen)) + "."
    )
