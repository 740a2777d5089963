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


OBJDIR = PKG / "_build"


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _inputs() -> list[Path]:
    return [CSRC / s for s in SOURCES] + _headers()


def is_stale() -> bool:
    lib = library_path()
    if not lib.exists():
        return True
    mtime = lib.stat().st_mtime
    return any(f.stat().st_mtime > mtime for f in _inputs())


def _object(src: str) -> Path:
    return OBJDIR / (Path(src).stem + ".o")


def _object_stale(src: str) -> bool:
    obj = _object(src)
    if not obj.exists():
        return True
    mtime = obj.stat().st_mtime
    return any(f.stat().st_mtime > mtime for f in [CSRC / src, *_headers()])


def _nvcc() -> str:
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _common_flags() -> list[str]:
    return [*ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "--Werror", "all-warnings", "-Xcompiler", "-fPIC",
            f"-I{INCLUDE}"]


def nvcc_command(output: Path, extra: list[str] | None = None) -> list[str]:
    """One nvcc line that compiles every source into ``output`` (a shared library)."""
    return [_nvcc(), *_common_flags(), "-shared", "-o", str(output), *[str(CSRC / s) for s in SOURCES],
            *(extra or [])]


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if it is missing or older than its sources. Each source is
    compiled to its own object (in parallel, only when it or a header changed), then
    the objects are linked."""
    lib = library_path()
    if not force and not is_stale():
        return lib
    LIBDIR.mkdir(parents=True, exist_ok=True)
    OBJDIR.mkdir(parents=True, exist_ok=True)
    procs = []
    for src in SOURCES:
        if not force and not _object_stale(src):
            continue
        tmp = _object(src).with_suffix(f".o.tmp{os.getpid()}")
        cmd = [_nvcc(), *_common_flags(), "-c", "-o", str(tmp), str(CSRC / src)]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, tmp, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for src, tmp, proc in procs:
        out, _ = proc.communicate()
        if proc.returncode != 0:
            sys.stderr.write(out)
            failed.append(src)
        else:
            os.replace(tmp, _object(src))
    if failed:
        raise RuntimeError(f"nvcc failed compiling {', '.join(failed)} for {LIBNAME}")
    tmp = lib.with_suffix(f".so.tmp{os.getpid()}")
    cmd = [_nvcc(), *ARCH_FLAGS, "-shared", "-o", str(tmp), *[str(_object(s)) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), flush=True)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"nvcc failed linking {LIBNAME} (exit {proc.returncode})")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
