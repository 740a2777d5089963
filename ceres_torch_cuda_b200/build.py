"""Build the sm_100a shared library ``lib/libceres_b200.so`` from ``csrc/`` with nvcc.

The library is built in-tree so that it travels with the source tree; nothing
is installed into site-packages. ``python -m ceres_torch_cuda_b200.build``
rebuilds it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIBDIR = PKG / "lib"
LIBNAME = "libceres_b200.so"
SOURCES = ["ba_kernels.cu", "ba_batch.cu"]
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def library_path() -> Path:
    return LIBDIR / LIBNAME


def _inputs() -> list[Path]:
    files = [CSRC / s for s in SOURCES]
    files += sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))
    return files


def is_stale() -> bool:
    lib = library_path()
    if not lib.exists():
        return True
    mtime = lib.stat().st_mtime
    return any(f.stat().st_mtime > mtime for f in _inputs())


def nvcc_command(output: Path, extra: list[str] | None = None) -> list[str]:
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return [nvcc, *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "--Werror", "all-warnings", "-Xcompiler", "-fPIC", "-shared",
            f"-I{INCLUDE}", "-o", str(output), *[str(CSRC / s) for s in SOURCES], *(extra or [])]


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if it is missing or older than its sources."""
    lib = library_path()
    if not force and not is_stale():
        return lib
    LIBDIR.mkdir(parents=True, exist_ok=True)
    tmp = lib.with_suffix(f".so.tmp{os.getpid()}")
    cmd = nvcc_command(tmp)
    if verbose:
        print(" ".join(cmd), flush=True)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"nvcc failed building {LIBNAME} (exit {proc.returncode})")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
