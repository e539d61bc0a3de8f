"""Write a solver's network tables for a caller without Python (include/maxichem_b200.hpp, mx_create_from_export).

The reference exports its specialised kernels and tables (``maxichem/_export.py:26-72``, read by
``cpp/maxichem.cpp``). Here the kernels live in the library, compiled once for sm_100a, so an export is the network's
tables alone: ``meta.txt`` (sizes, settings, names, and one ``table <name> <dtype> <count>`` line per table) and
``tables/<name>.bin`` (raw little-endian arrays), every field of ``mx_network`` in include/maxichem_b200.h. A call
through the export gives the same bits as the Python call.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np

from . import tables
from .constants import ATOL, COUNTS, T_MAX, T_MIN, X_SUM_TOL

EXPORT_FORMAT = 1

# every array of mx_network: (field, numpy dtype), then the per-group streams
_ARRAYS = [("perm", np.int32), ("rx", np.uint8), ("rc", np.float64), ("rf", np.int32), ("nasa", np.float64),
           ("atoms", np.float64), ("sv_ptr", np.int32), ("sv_term", np.uint32), ("jac_ptr", np.int32),
           ("jac_entry", np.uint32), ("jac_term", np.uint32), ("fill", np.uint8)]  # fmt: skip
_STREAMS = [("sv", "sv_stream", np.uint16), ("sv_rows", "sv_rows", np.uint16), ("jt", "jac_stream", np.uint32),
            ("jac_dst", "jac_dst", np.uint16)]  # fmt: skip


def write_export(tab: tables.Tables, folder: str | Path, *, drift: float, species: list[str],
                 elements: list[str]) -> Path:
    """Write `tab` (built with the solver's photolysis choice) and the drift allowance into `folder`."""
    folder = Path(folder)
    (folder / "tables").mkdir(parents=True, exist_ok=True)
    piece, row_ptr = tables.sv_row_pieces(tab)
    lines = [
        f"export_format {EXPORT_FORMAT}", f"ns {tab.ns}", f"nr {tab.nr}", f"nrt {tab.nrt}", f"nj {tab.nj}",
        f"nel {tab.nel}", f"n_entries {len(tab.jac_entry)}", f"has_troe {int(tab.has_troe)}",
        f"has_eff {int(tab.has_eff)}", f"sv_piece {piece}", f"n_pieces {int(row_ptr[-1])}", f"drift {drift!r}",
        f"atol {ATOL!r}", f"t_min {T_MIN!r}", f"t_max {T_MAX!r}", f"x_sum_tol {X_SUM_TOL!r}",
        f"counts {' '.join(COUNTS)}", f"species {' '.join(species)}", f"elements {' '.join(elements)}",
    ]  # fmt: skip

    def table(name: str, a: np.ndarray, dtype) -> None:
        c = np.ascontiguousarray(a, dtype=dtype)
        c.astype(c.dtype.newbyteorder("<"), copy=False).tofile(folder / "tables" / f"{name}.bin")
        lines.append(f"table {name} {np.dtype(dtype).name} {c.size}")

    for name, dtype in _ARRAYS:
        table(name, getattr(tab, name), dtype)
    table("sv_row_ptr", row_ptr, np.int32)
    for g, threads in enumerate(tab.stream_groups):
        st = tab.streams[threads]
        lines.append(f"group {g} {threads} {st['sv'].shape[0]} {st['sv_rows'].shape[0]} {st['jt'].shape[0]} "
                     f"{st['jac_dst'].shape[0]}")  # fmt: skip
        for key, name, dtype in _STREAMS:
            table(f"{name}{g}", st[key], dtype)
    (folder / "meta.txt").write_text("\n".join(lines) + "\n")
    return folder


def struct_fields() -> list[str]:
    """The pointer fields of mx_network an export holds (tests check every one is written)."""
    names = [name for name, _ in _ARRAYS] + ["sv_row_ptr"]
    return names + [f"{name}{g}" for g in (0, 1) for _, name, _ in _STREAMS]

