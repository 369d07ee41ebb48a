"""The LU-SGS sweep-record layout and launch shape on the CPU:
device/layout.cuh's diag_cells and sweep_slot and device/sweep.cuh's
sweep_shape, compiled by nvcc into a host program
(tests/sweep_layout_check.cu) and run without a GPU. The records of a case
are one slot per cell in anti-diagonal order, every chunk the sweep copies
is one contiguous range inside the case and its buffer; the sweep kernel and
the residual pass that writes the records index them through these two
functions."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _nvcc() -> str | None:
    cuda = Path("/usr/local/cuda/bin/nvcc")
    return str(cuda) if cuda.exists() else shutil.which("nvcc")


def test_records_are_one_slot_per_cell_by_anti_diagonal(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc is not installed")
    exe = tmp_path / "sweep_layout_check"
    # The device code of sweep.cuh is compiled for the B200 but never run: the
    # checks are the host-side layout and shape functions.
    subprocess.run([nvcc, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a", "-x", "cu",
                    "-I", str(ROOT / "bowshock_b200" / "csrc"),
                    "-I", str(ROOT / "include"), str(ROOT / "tests" / "sweep_layout_check.cu"), "-o", str(exe)],
                   check=True, capture_output=True, timeout=300)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
