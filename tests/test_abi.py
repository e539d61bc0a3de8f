"""The C-ABI library without a GPU: it loads, exports every entry point the header declares, and the ctypes mirror of
mx_network has the header's layout (checked against gcc's own offsets)."""

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from maxichem_b200 import abi

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "maxichem_b200.h"


def declared() -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s*(mx_\w+)\s*\(", text, flags=re.M)))


def test_the_header_declares_the_entry_points():
    names = declared()
    for want in ("mx_create", "mx_call", "mx_destroy", "mx_guard", "mx_info", "mx_version"):
        assert want in names


def test_the_library_exports_every_declared_entry_point():
    lib = abi.library()
    missing = [name for name in declared() if not hasattr(lib, name)]
    assert missing == []
    for name in declared():
        assert name in abi.SIGNATURES, f"{name} has no ctypes signature"


def test_the_version_names_the_architecture():
    assert b"sm_100a" in abi.library().mx_version()


def test_create_refuses_a_null_network_without_touching_a_device():
    lib = abi.library()
    handle = ctypes.c_void_p()
    err = ctypes.create_string_buffer(256)
    rc = lib.mx_create(None, 1e-6, 0, ctypes.byref(handle), err, 256)
    assert rc == 1 and handle.value is None
    assert b"null" in err.value


def test_destroy_and_info_accept_null():
    lib = abi.library()
    assert lib.mx_destroy(None) == 0
    values = (ctypes.c_int32 * 4)()
    assert lib.mx_info(None, values, 4) == 1


def test_the_network_struct_has_the_header_layout(tmp_path):
    fields = [name for name, _ in abi.MxNetwork._fields_]
    lines = "\n".join(f'  printf("{f} %zu\\n", offsetof(mx_network, {f}));' for f in fields)
    src = tmp_path / "layout.c"
    src.write_text(f"""#include <stddef.h>
#include <stdio.h>
#include "maxichem_b200.h"
int main(void) {{
{lines}
  printf("sizeof %zu\\n", sizeof(mx_network));
  return 0;
}}
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())  # fmt: skip
    for name in fields:
        assert int(got[name]) == getattr(abi.MxNetwork, name).offset, name
    assert int(got["sizeof"]) == ctypes.sizeof(abi.MxNetwork)


@pytest.mark.parametrize("name", ["cho41", "chno69", "sncho91"])
def test_a_network_struct_points_at_its_tables(networks, name):
    from maxichem_b200 import tables

    tab = tables.build(networks(name), True)
    s = abi.NetworkStruct(tab)
    st = s.struct
    assert (st.ns, st.nr, st.nj, st.nel) == (tab.ns, tab.nr, tab.nj, tab.atoms.shape[1])
    assert list(st.stream_threads) == list(tab.stream_groups) == [128, 96]
    assert abi.library().mx_warps_per_cell() == 4
    assert all(p for p in (st.perm, st.rx, st.rc, st.rf, st.nasa, st.atoms, st.sv_row_ptr))
