"""The parity rule between the CUDA path and the CPU oracle, shared by the GPU tests.

Both sides run the same method on the same inputs; they differ only in the last bits of exp/log/pow (libm against
CUDA's), so a cell either takes the same accepted steps on both sides, and then agrees to a relative RTOL per species
above FLOOR, or (rarely) a rounding difference flips one accept/reject decision, and then the two results are two
valid Rodas3 answers within the integrator's tolerance. The flips are counted and bounded.
"""

import numpy as np

RTOL = 1e-9  # relative, per species above FLOOR, on cells whose accepted steps match
WITHIN_SHARE = 0.99  # share of step-matched cells that must be within RTOL on every species above FLOOR
WORST_RTOL = 1e-8  # the rest: a stiff species whose last-bit difference the few steps of the call amplified
FLOOR = 1e-20  # mole fraction
FLIP_SHARE = 2e-3  # share of cells whose accepted steps may differ (a rounding-flipped accept/reject)
FLIP_DEX = 0.1  # their worst difference above FLOOR, dex (the call's rtol 1e-3 on quantities far above atol)
SHARE_TOL = 1e-11  # element shares of a passing cell, relative to the input's
H_RTOL = 1e-4  # the next step size: err is a difference of near-equal stages, so its last bits move h this much


def shares(x: np.ndarray, atoms: np.ndarray) -> np.ndarray:
    e = x @ atoms
    return e / e.sum(1, keepdims=True)


def compare(gpu: dict, ref: dict, x0: np.ndarray, atoms: np.ndarray) -> dict:
    """Return the parity report of one call: GPU arrays (host numpy) against the oracle's."""
    rep = {}
    rep["status_equal"] = bool(np.array_equal(gpu["status"], ref["status"]))
    rep["done_equal"] = bool(np.array_equal(gpu["done"], ref["done"]))
    rep["flag_equal"] = bool(np.array_equal(gpu["flag"], ref["flag"]))
    rep["counts_gpu"] = [int(v) for v in gpu["count"][1:-1]]
    rep["counts_ref"] = [int(v) for v in ref["count"][1:-1]]
    stepped = gpu["status"] == 0
    same = (gpu["steps"] == ref["steps"]) & stepped
    flips = stepped & ~same
    rep["cells"] = int(len(gpu["steps"]))
    rep["flips"] = int(flips.sum())
    a, b = gpu["x"][same], ref["x"][same]
    big = (np.abs(a) > FLOOR) & (np.abs(b) > FLOOR)
    rel = np.abs(a - b) / np.maximum(np.abs(a), np.abs(b)).clip(1e-300)
    rep["worst_rel"] = float(rel[big].max()) if big.any() else 0.0
    cell_rel = np.where(big, rel, 0.0).max(1) if big.size else np.zeros(0)
    rep["share_within_rtol"] = float((cell_rel <= RTOL).mean()) if cell_rel.size else 1.0
    per_cell = np.where(big, rel, 0.0).max(1)
    idx = np.flatnonzero(same)[np.argsort(per_cell)[::-1][:4]]
    rep["worst_cells"] = [
        (int(c), float(np.where(big, rel, 0.0).max(1)[list(np.flatnonzero(same)).index(c)]), float(gpu["steps"][c]),
         int(gpu["flag"][c]), int(ref["flag"][c]), float(gpu["h"][c]), float(ref["h"][c]))
        for c in idx
    ]
    hr = np.abs(gpu["h"][same] - ref["h"][same]) / np.abs(ref["h"][same]).clip(1e-300)
    rep["worst_h_rel"] = float(hr.max()) if hr.size else 0.0
    if flips.any():
        la = np.log10(np.maximum(gpu["x"][flips], FLOOR))
        lb = np.log10(np.maximum(ref["x"][flips], FLOOR))
        rep["flip_dex"] = float(np.abs(la - lb).max())
    else:
        rep["flip_dex"] = 0.0
    ok = (gpu["flag"] == 0) & stepped & np.isfinite(gpu["x"]).all(1)
    if ok.any():
        s0, s1 = shares(x0[ok], atoms), shares(gpu["x"][ok], atoms)
        m = s0 > 1e-14
        rep["share_rel"] = float((np.abs(s1 - s0)[m] / s0[m]).max())
    else:
        rep["share_rel"] = 0.0
    return rep


def passed(rep: dict) -> bool:
    """The bar of a settled GCM-like call: at least WITHIN_SHARE of the step-matched cells within RTOL on every
    species above FLOOR and none beyond WORST_RTOL, identical statuses, and identical flags and counts unless a
    rounding flip of an accept/reject decision explains them."""
    return (
        rep["status_equal"]
        and (rep["done_equal"] or rep["flips"] > 0)
        and (rep["flag_equal"] or rep["flips"] > 0)
        and (rep["counts_gpu"] == rep["counts_ref"] or rep["flips"] > 0)
        and rep["share_within_rtol"] >= WITHIN_SHARE
        and rep["worst_rel"] <= WORST_RTOL
        and rep["worst_h_rel"] <= H_RTOL
        and rep["flips"] <= max(1, FLIP_SHARE * rep["cells"])
        and rep["flip_dex"] <= FLIP_DEX
        and rep["share_rel"] <= SHARE_TOL
    )


STRICT_SHARE = 0.999  # the configuration-grid samples: share of cells within RTOL
STRICT_FLIPS = 1e-3  # and of cells whose accepted steps differ


def passed_strict(rep: dict) -> bool:
    """The bar of a settled call on a sample of a configuration's grid, closer to a bitwise one: statuses, done
    flags, guard flags and counts identical with no rounding flip excused, at least STRICT_SHARE of the cells within
    RTOL on every species above FLOOR, none beyond WORST_RTOL, element shares to SHARE_TOL."""
    return (
        rep["status_equal"]
        and rep["done_equal"]
        and rep["flag_equal"]
        and rep["counts_gpu"] == rep["counts_ref"]
        and rep["share_within_rtol"] >= STRICT_SHARE
        and rep["worst_rel"] <= WORST_RTOL
        and rep["flips"] <= STRICT_FLIPS * rep["cells"]
        and rep["share_rel"] <= SHARE_TOL
    )


def passed_calibrated(rep: dict, floor: dict) -> bool:
    """The bar of a call whose own rounding sensitivity exceeds RTOL (a cold start, or a long dark call): the GPU
    may differ from the oracle by no more than the oracle differs from itself when T moves by one ulp (floor), up to
    a factor of ten, with the same statuses, and guard flags that differ only on drift-borderline cells."""
    mismatch = [a - b for a, b in zip(rep["counts_gpu"], rep["counts_ref"])]
    drift_only = all(d == 0 for k, d in enumerate(mismatch) if k not in (5, 6, 7, 8))  # drift .. still_failed
    allowed_flags = max(2, 3 * abs(floor["counts_gpu"][6] - floor["counts_ref"][6]), 0.01 * rep["cells"])
    return (
        rep["status_equal"]
        and drift_only
        and abs(mismatch[6]) <= allowed_flags
        and rep["worst_rel"] <= max(RTOL, 10.0 * floor["worst_rel"])
        and rep["share_within_rtol"] >= floor["share_within_rtol"] - 0.05
        and rep["flips"] <= max(1, FLIP_SHARE * rep["cells"], 2 * floor["flips"])
        and rep["share_rel"] <= SHARE_TOL
    )
