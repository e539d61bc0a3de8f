"""The export for callers without Python, on CPU: the folder holds every table of mx_network, the loader refuses a
broken folder before any CUDA work, and the C++ caller compiles against include/maxichem_b200.hpp."""

import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from maxichem_b200 import abi, export, tables

ROOT = Path(__file__).resolve().parent.parent
CUDA = Path("/usr/local/cuda")


def write(networks, tmp_path, name="cho41"):
    net = networks(name)
    tab = tables.build(net, True)
    return net, tab, export.write_export(tab, tmp_path / name, drift=1e-6, species=list(net.species),
                                         elements=list(net.elements))  # fmt: skip


def meta(folder):
    return {line.split()[0]: line.split()[1:] for line in (folder / "meta.txt").read_text().splitlines()}


def test_the_export_holds_every_table(networks, tmp_path):
    net, tab, folder = write(networks, tmp_path)
    m = meta(folder)
    assert m["export_format"] == ["1"] and int(m["ns"][0]) == tab.ns and int(m["nj"][0]) == tab.nj
    assert m["species"] == list(net.species) and m["elements"] == list(net.elements)
    names = [line.split()[1] for line in (folder / "meta.txt").read_text().splitlines() if line.startswith("table")]
    assert sorted(names) == sorted(export.struct_fields())
    assert np.array_equal(np.fromfile(folder / "tables" / "perm.bin", dtype="<i4"), tab.perm)
    assert np.array_equal(np.fromfile(folder / "tables" / "rc.bin", dtype="<f8"), tab.rc.ravel())
    assert np.array_equal(np.fromfile(folder / "tables" / "jac_stream0.bin", dtype="<u4"), tab.streams[128]["jt"].ravel())


def load(folder):
    handle = ctypes.c_void_p()
    err = ctypes.create_string_buffer(512)
    rc = abi.library().mx_create_from_export(str(folder).encode(), 0, ctypes.byref(handle), err, 512)
    return rc, err.value.decode(), handle


def test_a_missing_folder_is_refused(tmp_path):
    rc, msg, handle = load(tmp_path / "nothing")
    assert rc == 1 and "meta.txt cannot be read" in msg and handle.value is None


def test_a_short_table_is_refused_before_any_cuda_work(networks, tmp_path):
    _, _, folder = write(networks, tmp_path)
    f = folder / "tables" / "rc.bin"
    f.write_bytes(f.read_bytes()[:-8])
    rc, msg, handle = load(folder)
    assert rc == 3 and "rc.bin" in msg and "bytes expected" in msg and handle.value is None


def test_a_wrong_table_length_in_meta_is_refused(networks, tmp_path):
    _, tab, folder = write(networks, tmp_path)
    text = (folder / "meta.txt").read_text().replace(f"table perm int32 {tab.ns}", f"table perm int32 {tab.ns + 1}")
    (folder / "meta.txt").write_text(text)
    rc, msg, _ = load(folder)
    assert rc == 3 and "table perm" in msg


def test_a_missing_stream_is_refused(networks, tmp_path):
    _, _, folder = write(networks, tmp_path)
    text = "\n".join(line for line in (folder / "meta.txt").read_text().splitlines() if "jac_dst1" not in line)
    (folder / "meta.txt").write_text(text + "\n")
    rc, msg, _ = load(folder)
    assert rc == 3 and "jac_dst1" in msg


def compile_caller(out: Path) -> Path:
    """Build tests/cpp/call_export.cpp against the headers and the library (g++, no nvcc)."""
    lib = abi.LIBRARY.parent
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", str(ROOT / "include"), "-I", str(CUDA / "include"),
           str(ROOT / "tests" / "cpp" / "call_export.cpp"), "-o", str(out), "-L", str(lib), "-lmaxichem_b200",
           f"-Wl,-rpath,{lib}", "-L", str(CUDA / "lib64"), "-lcudart", f"-Wl,-rpath,{CUDA / 'lib64'}"]  # fmt: skip
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ is needed")
def test_the_cpp_caller_compiles(tmp_path):
    exe = compile_caller(tmp_path / "call_export")
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
