"""ctypes mirror of ``include/maxichem_b200.h``: the mx_network struct and the library's entry points."""

from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import Any

import numpy as np

from . import tables
from .tables import Tables

PACKAGE = Path(__file__).resolve().parent
LIBRARY = PACKAGE / "_build" / "libmaxichem_b200.so"
COUNT_SLOTS = 12


class MxNetwork(ctypes.Structure):
    """struct mx_network."""

    _fields_ = [
        ("ns", ctypes.c_int32),
        ("nr", ctypes.c_int32),
        ("nrt", ctypes.c_int32),
        ("nj", ctypes.c_int32),
        ("nel", ctypes.c_int32),
        ("n_entries", ctypes.c_int32),
        ("has_troe", ctypes.c_int32),
        ("has_eff", ctypes.c_int32),
        ("perm", ctypes.c_void_p),
        ("rx", ctypes.c_void_p),
        ("rc", ctypes.c_void_p),
        ("rf", ctypes.c_void_p),
        ("nasa", ctypes.c_void_p),
        ("atoms", ctypes.c_void_p),
        ("sv_ptr", ctypes.c_void_p),
        ("sv_term", ctypes.c_void_p),
        ("jac_ptr", ctypes.c_void_p),
        ("jac_entry", ctypes.c_void_p),
        ("jac_term", ctypes.c_void_p),
        ("fill", ctypes.c_void_p),
        ("sv_piece", ctypes.c_int32),
        ("n_pieces", ctypes.c_int32),
        ("sv_row_ptr", ctypes.c_void_p),
        ("stream_threads", ctypes.c_int32 * 2),
        ("sv_rounds", ctypes.c_int32 * 2),
        ("sv_nrows", ctypes.c_int32 * 2),
        ("jac_rounds", ctypes.c_int32 * 2),
        ("jac_nents", ctypes.c_int32 * 2),
        ("sv_stream", ctypes.c_void_p * 2),
        ("sv_rows", ctypes.c_void_p * 2),
        ("jac_stream", ctypes.c_void_p * 2),
        ("jac_dst", ctypes.c_void_p * 2),
    ]


class NetworkStruct:
    """An mx_network over a Tables' arrays; keeps the arrays alive while the struct is in use."""

    def __init__(self, tab: Tables) -> None:
        self._keep: list[np.ndarray] = []

        def ptr(a: np.ndarray, dtype: Any) -> int:
            c = np.ascontiguousarray(a, dtype=dtype)
            self._keep.append(c)
            return c.ctypes.data

        self.struct = MxNetwork(
            ns=tab.ns, nr=tab.nr, nrt=tab.nrt, nj=tab.nj, nel=tab.nel, n_entries=len(tab.jac_entry),
            has_troe=int(tab.has_troe), has_eff=int(tab.has_eff),
            perm=ptr(tab.perm, np.int32), rx=ptr(tab.rx, np.uint8), rc=ptr(tab.rc, np.float64),
            rf=ptr(tab.rf, np.int32), nasa=ptr(tab.nasa, np.float64), atoms=ptr(tab.atoms, np.float64),
            sv_ptr=ptr(tab.sv_ptr, np.int32), sv_term=ptr(tab.sv_term, np.uint32),
            jac_ptr=ptr(tab.jac_ptr, np.int32), jac_entry=ptr(tab.jac_entry, np.uint32),
            jac_term=ptr(tab.jac_term, np.uint32), fill=ptr(tab.fill, np.uint8),
        )  # fmt: skip
        piece, row_ptr = tables.sv_row_pieces(tab)
        self.struct.sv_piece, self.struct.n_pieces = piece, int(row_ptr[-1])
        self.struct.sv_row_ptr = ptr(row_ptr, np.int32)
        for g, threads in enumerate(tab.stream_groups):
            st = tab.streams.get(threads)
            if st is None:
                continue
            self.struct.stream_threads[g] = threads
            self.struct.sv_rounds[g], self.struct.sv_nrows[g] = st["sv"].shape[0], st["sv_rows"].shape[0]
            self.struct.jac_rounds[g], self.struct.jac_nents[g] = st["jt"].shape[0], st["jac_dst"].shape[0]
            self.struct.sv_stream[g] = ptr(st["sv"], np.uint16)
            self.struct.sv_rows[g] = ptr(st["sv_rows"], np.uint16)
            self.struct.jac_stream[g] = ptr(st["jt"], np.uint32)
            self.struct.jac_dst[g] = ptr(st["jac_dst"], np.uint16)

    def ref(self) -> Any:
        return ctypes.byref(self.struct)


_P = ctypes.c_void_p
_ERR = ctypes.c_char_p

# Every entry point that include/maxichem_b200.h declares, with its ctypes signature.
SIGNATURES: dict[str, tuple[Any, list[Any]]] = {
    "mx_create": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_int, ctypes.POINTER(_P), _ERR, ctypes.c_size_t]),
    "mx_create_from_export": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(_P), _ERR, ctypes.c_size_t]),
    "mx_call": (
        ctypes.c_int,
        [_P, _P, _P, _P, _P, _P, _P, ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
         _P, _P, _P, _P, _P, _P, _P, _P, _P, _ERR, ctypes.c_size_t],
    ),  # fmt: skip
    "mx_call_static": (
        ctypes.c_int,
        [_P, _P, _P, _P, _P, _P, _P, ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
         _P, _P, _P, _P, _P, _P, _P, _P, _P, _ERR, ctypes.c_size_t],
    ),  # fmt: skip
    "mx_jvp": (
        ctypes.c_int,
        [_P, _P, _P, _P, _P, _P, _P, _P, _P, ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
         ctypes.c_int32, ctypes.c_int32] + [_P] * 8 + [_P] * 10 + [_P, _ERR, ctypes.c_size_t],
    ),  # fmt: skip
    "mx_vjp": (
        ctypes.c_int,
        [_P, _P, _P, _P, _P, _P, _P, _P, _P, ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
         ctypes.c_int32, ctypes.c_int32] + [_P] * 18 + [_P, _ERR, ctypes.c_size_t],
    ),  # fmt: skip
    "mx_guard": (
        ctypes.c_int,
        [_P, _P, _P, _P, _P, _P, ctypes.c_int64, ctypes.c_double, _P, _P, _P, _ERR, ctypes.c_size_t],
    ),
    "mx_info": (ctypes.c_int, [_P, _P, ctypes.c_int32]),
    "mx_set_grid": (ctypes.c_int, [_P, ctypes.c_int32]),
    "mx_mass_to_mole": (ctypes.c_int, [_P, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, _P, _P, _P]),
    "mx_mole_to_mass": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, ctypes.c_int32, _P, _P, _P]),
    "mx_destroy": (ctypes.c_int, [_P]),
    "mx_set_try_counter": (ctypes.c_int, [_P, _P]),
    "mx_set_phase_counter": (ctypes.c_int, [_P, _P]),
    "mx_time_phases": (
        ctypes.c_int,
        [_P, _P, ctypes.c_double, ctypes.c_double, ctypes.c_double, _P, ctypes.c_int32, ctypes.c_int32, _P, _P],
    ),
    "mx_debug_try": (
        ctypes.c_int,
        [_P, _P, ctypes.c_double, ctypes.c_double, ctypes.c_double, _P, ctypes.c_double, ctypes.c_double, _P, _P],
    ),
    "mx_probe_fp64": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]),
    "mx_set_precision": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_double]),
    "mx_sur_create": (
        ctypes.c_int,
        [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
         ctypes.c_int32, ctypes.POINTER(_P), _ERR, ctypes.c_size_t],
    ),  # fmt: skip
    "mx_sur_info": (ctypes.c_int, [_P, _P, ctypes.c_int32]),
    "mx_sur_set_scaling": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "mx_sur_features": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, ctypes.c_int64, _P, _P, _P]),
    "mx_sur_forward": (ctypes.c_int, [_P, _P, ctypes.c_int64, _P, _P]),
    "mx_sur_train_step": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int64, ctypes.c_float, ctypes.c_float, _P, _P]),
    "mx_sur_params": (ctypes.c_int, [_P, ctypes.c_int32, _P, ctypes.c_int64]),
    "mx_sur_set_params": (ctypes.c_int, [_P, _P, ctypes.c_int64]),
    "mx_sur_error": (ctypes.c_int, [_P, _P]),
    "mx_sur_call": (
        ctypes.c_int,
        [_P, _P, _P, _P, _P, _P, _P, _P, ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
         ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_uint32] + [_P] * 13
        + [ctypes.c_int32, _P, _ERR, ctypes.c_size_t],
    ),  # fmt: skip
    "mx_sur_destroy": (ctypes.c_int, [_P]),
    "mx_sur_propose": (
        ctypes.c_int,
        [_P, _P, _P, _P, _P, _P, _P, ctypes.c_int64, ctypes.c_double, ctypes.c_double, _P, _P, _P],
    ),  # fmt: skip
    "mx_gemm_bf16": (
        ctypes.c_int,
        [_P, ctypes.c_int32, _P, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
         _P, _P, ctypes.c_int32, _P, ctypes.c_int32, _P, _P],
    ),  # fmt: skip
    "mx_gemm_bf16_split": (
        ctypes.c_int,
        [_P, ctypes.c_int32, _P, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, _P, _P,
         ctypes.c_int32, _P, _P],
    ),  # fmt: skip
    "mx_gemm_split_workspace": (ctypes.c_int64, [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32]),
    "mx_set_escalation_counter": (ctypes.c_int, [_P, _P]),
    "mx_debug_try_mixed": (
        ctypes.c_int,
        [_P, _P, ctypes.c_double, ctypes.c_double, ctypes.c_double, _P, ctypes.c_double, ctypes.c_double,
         ctypes.c_int32, _P, _P],
    ),  # fmt: skip
    "mx_version": (ctypes.c_char_p, []),
    "mx_warps_per_cell": (ctypes.c_int, []),
    "mx_warps_supported": (ctypes.c_int, [ctypes.c_int32]),
    "mx_cells_per_sm": (ctypes.c_int, [_P, ctypes.c_int32]),
}

_lib: ctypes.CDLL | None = None


def library() -> ctypes.CDLL:
    """Load the CUDA library (built by ``maxichem_b200.build``); raise if it is missing."""
    global _lib
    if _lib is None:
        path = Path(os.environ.get("MAXICHEM_B200_LIBRARY", LIBRARY))
        if not path.exists():
            raise RuntimeError(
                f"the maxichem_b200 CUDA library {path} is missing: build it with "
                "`python -c 'import maxichem_b200.build as b; b.build()'` (there is no CPU fallback)"
            )
        lib = ctypes.CDLL(str(path))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib
