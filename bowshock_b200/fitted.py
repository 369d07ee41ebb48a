"""Host side of the fitted bow shock (src/solver/shock-fitting.ts,
src/analysis/fitted-flow.ts): the shock relations of a fitted shock, the
Taylor-Maccoll field on rays, and column placement by a density, over the
native library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native, abi
from .config import Primitive2D

_DENSITY = C.CFUNCTYPE(C.c_double, C.c_double, C.c_void_p)


def _prim(w) -> abi.Primitive:
    return abi.Primitive(float(w.rho), float(w.u), float(w.v), float(w.p))


def shock_state(free: Primitive2D, gamma: float, mach: float, nx: float, ny: float) -> abi.FittedShock:
    """shockState (src/solver/shock-fitting.ts:50-78): the state behind a
    shock of outward normal (nx, ny) met at relative normal Mach `mach`."""
    L = _native.load()
    out = abi.FittedShock()
    _native.check(L.bs_shock_state(C.byref(_prim(free)), gamma, mach, nx, ny, C.byref(out)), L)
    return out


def compatible_shock(free: Primitive2D, gamma: float, nx: float, ny: float, rho: float, a: float,
                     p: float, un: float) -> abi.FittedShock:
    """compatibleShock (src/solver/shock-fitting.ts:87-111): the shock whose
    post-shock state meets the u_n + a characteristic from behind."""
    L = _native.load()
    out = abi.FittedShock()
    _native.check(L.bs_compatible_shock(C.byref(_prim(free)), gamma, nx, ny, rho, a, p, un, C.byref(out)), L)
    return out


def cone_flow_field(mach: float, cone: float, gamma: float, polar, tolerance: float = 1e-13):
    """coneFlowField (src/validation/taylor-maccoll.ts:227-275) on the rays
    `polar`: (speed over the maximum speed, flow angle, the cone solution)."""
    L = _native.load()
    polar = np.ascontiguousarray(np.atleast_1d(polar), np.float64)
    speed = np.empty_like(polar)
    angle = np.empty_like(polar)
    flow = abi.ConeFlow()
    dp = C.POINTER(C.c_double)
    _native.check(L.bs_cone_flow_field(mach, cone, gamma, tolerance, len(polar), polar.ctypes.data_as(dp),
                                       speed.ctypes.data_as(dp), angle.ctypes.data_as(dp), C.byref(flow)), L)
    return speed, angle, flow


def column_positions(breakpoints, density, refinement: int = 1, total: int = 0) -> np.ndarray:
    """columnPositions (src/grid/spacing.ts:31-71): positions along a line
    of breakpoints with `density` nodes per unit length (a Python callable)."""
    L = _native.load()
    bp = np.ascontiguousarray(breakpoints, np.float64)
    cb = _DENSITY(lambda x, _user: float(density(x)))
    cap = 1 << 20
    out = np.empty(cap, np.float64)
    n = C.c_int32()
    dp = C.POINTER(C.c_double)
    _native.check(L.bs_column_positions(len(bp), bp.ctypes.data_as(dp), C.cast(cb, C.c_void_p), None,
                                        int(refinement), int(total), cap, out.ctypes.data_as(dp), C.byref(n)), L)
    return out[:n.value].copy()
