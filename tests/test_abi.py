"""The C ABI without a GPU: the library loads, exports every entry point
include/bowshock.h declares, and rejects invalid input before touching the
device (the reference's RangeError checks, src/solver/config.ts:35-55)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from bowshock_b200 import _native, abi
from bowshock_b200.config import Boundary, Euler2DConfig, Primitive2D, grid_from_function, rectangular_grid

HEADER = Path(__file__).resolve().parent.parent / "include" / "bowshock.h"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^BS_API\s+[\w\s\*]+?\b(bs_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    names = declared_symbols()
    assert len(names) > 30
    for name in names:
        assert hasattr(lib, name), name


def test_python_bindings_cover_the_header():
    names = set(declared_symbols()) - {"bs_last_error", "bs_version"}
    assert names == set(_native.SIGNATURES), names ^ set(_native.SIGNATURES)


def test_struct_layouts_match_the_header():
    assert C.sizeof(abi.Config) == 208
    assert C.sizeof(abi.FaceFlux) == 72
    assert C.sizeof(abi.SolveResult) == 32
    assert C.sizeof(abi.Body) == 40
    assert C.sizeof(abi.BodyGridOptions) == 32  # nj, refinement, ni, flags, mach, gamma


def test_version_and_device_count_without_a_gpu():
    lib = _native.load()
    assert lib.bs_version().decode().startswith("bowshock_b200")
    n = C.c_int32(-1)
    assert lib.bs_device_count(C.byref(n)) == abi.BS_OK
    assert n.value >= 0


def outflow_config(grid, **kw) -> Euler2DConfig:
    base = dict(grid=grid, geometry="planar", gamma=1.4, flux="hllc", limiter="minmod",
                reconstruction="perVariable", time_integrator="ssprk2", cfl=0.5,
                time_stepping="local",
                boundaries={s: Boundary("outflow") for s in ("iMin", "iMax", "jMin", "jMax")})
    base.update(kw)
    return Euler2DConfig(**base)


@pytest.mark.parametrize("change,message", [
    (dict(cfl=0.0), "cfl must be in (0, 1]"),
    (dict(cfl=1.5), "cfl must be in (0, 1]"),
    (dict(reconstruction="shared"), "requires the 'vanAlbada' limiter"),
    (dict(boundaries={"iMin": Boundary("periodic"), "iMax": Boundary("outflow"),
                      "jMin": Boundary("outflow"), "jMax": Boundary("outflow")}), "periodic"),
    (dict(boundaries={"iMin": Boundary("inflow", Primitive2D(1, 1, 0, -1)), "iMax": Boundary("outflow"),
                      "jMin": Boundary("outflow"), "jMax": Boundary("outflow")}), "positive"),
])
def test_invalid_configurations_are_refused_before_the_gpu(change, message):
    lib = _native.load()
    cfg = outflow_config(rectangular_grid(4, 4, 0, 1, 0, 1), **change)
    h = C.c_void_p()
    a = cfg.to_abi()
    st = lib.bs_engine_create(C.byref(a), cfg.grid.x.ctypes.data_as(C.POINTER(C.c_double)),
                              cfg.grid.y.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h))
    assert st == abi.BS_INVALID_ARGUMENT
    assert message in lib.bs_last_error().decode()
    assert not h.value


def test_inverted_cells_and_axis_crossing_are_refused():
    lib = _native.load()
    flipped = grid_from_function(3, 3, lambda i, j: (-float(i), float(j)))
    cfg = outflow_config(flipped)
    a = cfg.to_abi()
    h = C.c_void_p()
    st = lib.bs_engine_create(C.byref(a), cfg.grid.x.ctypes.data_as(C.POINTER(C.c_double)),
                              cfg.grid.y.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h))
    assert st == abi.BS_INVALID_ARGUMENT
    assert "non-positive area" in lib.bs_last_error().decode()
    below = grid_from_function(3, 3, lambda i, j: (float(i), float(j) - 1.0))
    cfg = outflow_config(below, geometry="axisymmetric")
    a = cfg.to_abi()
    st = lib.bs_engine_create(C.byref(a), cfg.grid.x.ctypes.data_as(C.POINTER(C.c_double)),
                              cfg.grid.y.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h))
    assert st == abi.BS_INVALID_ARGUMENT
    assert "y >= 0" in lib.bs_last_error().decode()


def test_null_handles_are_errors_not_crashes():
    lib = _native.load()
    out = C.c_double()
    assert lib.bs_engine_density_residual_norm(None, C.byref(out)) == abi.BS_INVALID_ARGUMENT
    assert lib.bs_engine_destroy(None) == abi.BS_OK
    assert lib.bs_batch_destroy(None) == abi.BS_OK
    n = C.c_int32()
    assert lib.bs_batch_size(None, C.byref(n)) == abi.BS_INVALID_ARGUMENT
