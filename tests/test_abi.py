"""The C-ABI library loads and exports what include/ceres_b200.h declares, and the
ctypes mirror of ceres_b200_ba_t matches the C layout (no GPU needed)."""
from __future__ import annotations

import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from ceres_torch_cuda_b200 import _lib
from ceres_torch_cuda_b200 import build as B

HEADER = Path(__file__).resolve().parents[1] / "include" / "ceres_b200.h"


def _declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ceres_b200_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    B.build()
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    names = _declared_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.SIGNATURES), "ctypes signatures must cover exactly the header's functions"


def test_abi_version_and_struct_size(lib):
    assert lib.ceres_b200_abi_version() == _lib.ABI_VERSION
    assert lib.ceres_b200_ba_struct_bytes() == ctypes.sizeof(_lib.BAStruct)
    assert lib.ceres_b200_launch_count() >= 0


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
@pytest.mark.parametrize("ctype,mirror", [("ceres_b200_ba_t", _lib.BAStruct), ("ceres_b200_batch_t", _lib.BatchStruct),
                                         ("ceres_b200_clusters_t", _lib.ClusterStruct)])
def test_struct_field_offsets_match_c(tmp_path, ctype, mirror):
    fields = [f for f, _ in mirror._fields_]
    src = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {",
           f'printf("%zu\\n", sizeof({ctype}));']
    src += [f'printf("%zu\\n", offsetof({ctype}, {f}));' for f in fields]
    src += ["return 0; }"]
    c = tmp_path / "off.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "off"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(c)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == ctypes.sizeof(mirror)
    for f, off in zip(fields, out[1:]):
        assert getattr(mirror, f).offset == off, f


def test_stats_indices_match_header():
    text = HEADER.read_text()
    for name, idx in [("CERES_B200_STAT_COST", _lib.STAT_COST), ("CERES_B200_STAT_CAND_COST", _lib.STAT_CAND_COST),
                      ("CERES_B200_STAT_PCG_ITERS", _lib.STAT_PCG_ITERS), ("CERES_B200_STAT_ERROR", _lib.STAT_ERROR),
                      ("CERES_B200_STAT_CAND_STATE_SQ_C", _lib.STAT_CAND_STATE_SQ_C),
                      ("CERES_B200_NSTATS", _lib.NSTATS)]:
        m = re.search(rf"{name}\s*=\s*(\d+)", text)
        assert m and int(m.group(1)) == idx, name
    assert _lib.NSTATS * 8 <= _lib.CTL_COUNTERS and _lib.CTL_COUNTERS + 16 * 4 <= _lib.CTL_BYTES
    m = re.search(r"#define CERES_B200_CAM_ITEM (\d+)", text)
    assert m and int(m.group(1)) == _lib.CAM_ITEM


def test_invalid_arguments_are_rejected_without_a_gpu(lib):
    """Argument validation happens on the host before any CUDA call."""
    s = _lib.BAStruct()
    s.precision = 7  # not a precision
    assert lib.ceres_b200_ba_evaluate(ctypes.byref(s), 1, None) == _lib.EINVAL
    s.precision = _lib.FP64
    s.num_slices, s.num_points = 1, 31  # num_points must be 32 * num_slices
    assert lib.ceres_b200_ba_step(ctypes.byref(s), None) == _lib.EINVAL
    assert lib.ceres_b200_ba_pcg(None, 2, 0, 10, 0.1, 0, None) == _lib.EINVAL
    assert lib.ceres_b200_dense_cholesky_solve(None, None, None, 4, None, None) == _lib.EINVAL
    b = _lib.BatchStruct()
    b.num_problems = 3  # no arrays set
    assert lib.ceres_b200_batch_solve(ctypes.byref(b), 256, 1, 1, None) == _lib.EINVAL
    assert lib.ceres_b200_batch_solve(None, 256, 1, 1, None) == _lib.EINVAL
    assert lib.ceres_b200_batch_struct_bytes() == ctypes.sizeof(_lib.BatchStruct)
    # the cluster preconditioner's entry points check their struct before any CUDA call
    assert lib.ceres_b200_clusters_struct_bytes() == ctypes.sizeof(_lib.ClusterStruct)
    s = _lib.BAStruct()
    s.precision = _lib.FP64
    cl = _lib.ClusterStruct()  # no arrays, no components
    assert lib.ceres_b200_ba_cluster_factor(ctypes.byref(s), ctypes.byref(cl), None) == _lib.EINVAL
    assert lib.ceres_b200_ba_cluster_factor(ctypes.byref(s), None, None) == _lib.EINVAL
    assert lib.ceres_b200_ba_pcg_cluster(ctypes.byref(s), ctypes.byref(cl), 0, 10, 0.1, 0, None) == _lib.EINVAL
    # misaligned sources of the camera reduction's asynchronous copies (addresses only,
    # never dereferenced: the check comes first)
    for field, addr in (("res", 0x10008), ("winv", 0x10004), ("winv_ga", 0x10004), ("jac", 0x10010)):
        s = _lib.BAStruct()
        s.precision = _lib.FP32
        s.counters, s.stats = 0x10000, 0x10000
        s.jac, s.res, s.winv, s.winv_ga = 0x10000, 0x10000, 0x10000, 0x10000
        s.scratch, s.cand_cameras, s.cand_points, s.step_points = 0x10000, 0x10000, 0x10000, 0x10000
        setattr(s, field, addr)  # every other argument of the step passes its check
        assert lib.ceres_b200_ba_step(ctypes.byref(s), None) == _lib.EINVAL, field
