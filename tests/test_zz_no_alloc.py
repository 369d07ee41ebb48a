"""The allocation-free LU-SGS step (bs_lusgs_step_static) against the
engine's own LU-SGS step (bs_engine_iterate_implicit), through the C ABI.

bs_lusgs_step_static is for callers that cannot let a library allocate
device memory - applications that give out all GPU memory from their own pool,
and solver loops that must not allocate once running - so here the test, as
such a caller, owns the device buffers (made with torch) and the entry point
uses only its static scratch. Two calls in a row must give the engine's state
after one and two steps. This file is collected last on purpose.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from bowshock_b200 import _native, abi
from bowshock_b200.engine import CudaEuler2D
from bowshock_b200.workloads import ogive_case
from oracle.oracle import OracleEuler2D

pytestmark = pytest.mark.gpu

CFL = 5.0
OMEGA = 1.5


def device_inputs(case, torch):
    """Grid metrics in the engine's device layout and the free-stream state,
    as device tensors owned by the caller."""
    o = OracleEuler2D(case.config)  # FP64 metrics by the reference's formulas
    i_faces, j_faces, cells = o.metrics()
    iface = np.zeros((i_faces.shape[0], 4), dtype=np.float32)
    iface[:, :3] = i_faces
    jface = np.zeros((j_faces.shape[0], 4), dtype=np.float32)
    jface[:, :3] = j_faces
    cell = cells[:, :2].astype(np.float32)
    n = case.config.grid.ni * case.config.grid.nj
    w = case.free.state
    g = case.config.gamma
    state = [np.full(n, w.rho), np.full(n, w.rho * w.u), np.full(n, w.rho * w.v),
             np.full(n, w.p / (g - 1) + 0.5 * w.rho * (w.u * w.u + w.v * w.v))]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    return dev(iface), dev(jface), dev(cell), [dev(s) for s in state]


def primitives_of(state, gamma) -> np.ndarray:
    rho, mu, mv, e = (s.cpu().numpy() for s in state)
    return np.stack([rho, mu / rho, mv / rho, (gamma - 1) * (e - 0.5 * (mu * mu + mv * mv) / rho)],
                    axis=1)


@pytest.mark.parametrize("ni, nj", [(96, 48), (512, 128)])
def test_static_step_matches_the_engine_step_twice_in_a_row(ni, nj):
    # 512 x 128 fills the scratch's cell limit (65,536), one sweep-record
    # slot per cell.
    torch = pytest.importorskip("torch")
    lib = _native.load()
    case = ogive_case(2.2, ni, nj)
    cfg = case.config.to_abi()
    iface, jface, cells, state = device_inputs(case, torch)
    stream = torch.cuda.current_stream()
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731

    with CudaEuler2D(case.config, 64) as engine:
        engine.set_uniform(case.free.state)
        for call in range(2):
            r_engine = engine.density_residual_norm()
            engine.iterate_implicit(1, CFL, OMEGA)
            torch.cuda.synchronize()
            residual = C.c_double()
            bad = C.c_int32()
            st = lib.bs_lusgs_step_static(C.byref(cfg), ptr(iface), ptr(jface), ptr(cells),
                                          *[ptr(s) for s in state], CFL, OMEGA,
                                          C.c_void_p(stream.cuda_stream), C.byref(residual),
                                          C.byref(bad))
            _native.check(st, lib)
            torch.cuda.synchronize()
            assert bad.value == 0
            assert abs(residual.value / r_engine - 1) < 1e-9, call
            w_static = primitives_of(state, case.config.gamma)
            w_engine = engine.primitives()
            assert np.max(np.abs(w_static - w_engine)) < 1e-10, call


def test_static_step_refuses_grids_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    lib = _native.load()
    case = ogive_case(2.0, 400, 200)  # 80000 cells > 65536
    cfg = case.config.to_abi()
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = C.c_void_p(dummy.data_ptr())
    residual = C.c_double()
    bad = C.c_int32()
    st = lib.bs_lusgs_step_static(C.byref(cfg), p, p, p, p, p, p, p, CFL, OMEGA, None,
                                  C.byref(residual), C.byref(bad))
    assert st == abi.BS_INVALID_ARGUMENT
    assert "at most 65536" in lib.bs_last_error().decode()
    # 64 x 513: within the cell limit, but wider than 512 cells across.
    from dataclasses import replace

    from bowshock_b200.config import grid_from_function

    wide = replace(case.config, grid=grid_from_function(64, 513, lambda i, j: (i / 64, 1 + j / 513)))
    cfg = wide.to_abi()
    st = lib.bs_lusgs_step_static(C.byref(cfg), p, p, p, p, p, p, p, CFL, OMEGA, None,
                                  C.byref(residual), C.byref(bad))
    assert st == abi.BS_INVALID_ARGUMENT
    assert "512 cells across" in lib.bs_last_error().decode()
