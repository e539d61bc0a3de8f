"""Build the CUDA library ``_build/libmaxichem_b200.so`` for sm_100a with nvcc (in-tree, no JIT cache)."""

from __future__ import annotations

import os
import subprocess
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
SOURCES = [PACKAGE / "csrc" / "maxichem_b200.cu", PACKAGE / "csrc" / "mixed.cu", PACKAGE / "csrc" / "surrogate.cu",
           PACKAGE / "csrc" / "derivatives.cu", PACKAGE / "csrc" / "coupling.cu", PACKAGE / "csrc" / "export.cpp"]
HEADERS = [PACKAGE / "csrc" / "device.cuh", PACKAGE / "csrc" / "solver.cuh", PACKAGE / "csrc" / "jvp.cuh",
           PACKAGE / "csrc" / "vjp.cuh", PACKAGE / "csrc" / "gemm.cuh", PACKAGE.parent / "include" / "maxichem_b200.h"]
OUTPUT = PACKAGE / "_build" / "libmaxichem_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [
    *ARCH, "-lineinfo", "-O3", "-std=c++17",
    "-fmad=false",  # every fused multiply-add in the kernels is an explicit fma(): the same bits as the oracle's
    "-Xptxas", "-v",
    "-Xcompiler", "-fPIC",
]  # fmt: skip


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if a source is newer than it (or force); return its path. Each source is its own
    translation unit (the call kernels' module does not see the derivative kernels), compiled in parallel."""
    OUTPUT.parent.mkdir(exist_ok=True)
    newest = max(p.stat().st_mtime for p in SOURCES + HEADERS)
    if force or not OUTPUT.exists() or OUTPUT.stat().st_mtime < newest:
        jobs = []
        for src in SOURCES:
            obj = OUTPUT.parent / (src.stem + ".o")
            cmd = [NVCC, *FLAGS, "-c", str(src), "-o", str(obj)]
            jobs.append((src, obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        logs = []
        for src, obj, proc in jobs:
            _, err = proc.communicate()
            if proc.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src.name}:\n{err}")
            logs.append(f"== {src.name}\n{err}")
        tmp = OUTPUT.with_suffix(".tmp.so")
        link = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *(str(o) for _, o, _ in jobs), "-o", str(tmp)]
        out = subprocess.run(link, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError(f"nvcc link failed:\n{out.stderr}")
        (OUTPUT.parent / "ptxas.log").write_text("".join(logs))
        if verbose:
            print("".join(logs))
        tmp.replace(OUTPUT)
    return OUTPUT


if __name__ == "__main__":
    build(force=True, verbose=True)
