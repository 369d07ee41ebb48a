"""Grids and exact solutions from the native host code: `bodyGrid`
(src/grid/body-grid.ts:76-181), `bluntBodyGrid` (src/grid/blunt-grid.ts:159-540),
`rampGrid` (src/grid/shapes.ts:30-52),
`gridQuality` (src/grid/quality.ts:75-128), `taylorMaccoll`
(src/validation/taylor-maccoll.ts:153-216), `obliqueShock` / `normalShock`
(src/validation/gas-dynamics.ts:40-96)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native, abi
from .config import StructuredGrid


@dataclass(frozen=True)
class NoseShape:
    kind: str
    parameter: float = 0.0


@dataclass(frozen=True)
class Nose:
    shape: NoseShape
    length: float
    base_radius: float


@dataclass(frozen=True)
class Body:
    nose: Nose
    cylinder_length: float

    def to_abi(self) -> abi.Body:
        if self.nose.shape.kind not in abi.NOSE_KIND:
            raise ValueError(f"unknown nose shape {self.nose.shape.kind!r}")
        b = abi.Body()
        b.nose_kind = abi.NOSE_KIND[self.nose.shape.kind]
        b.parameter = self.nose.shape.parameter
        b.nose_length = self.nose.length
        b.base_radius = self.nose.base_radius
        b.cylinder_length = self.cylinder_length
        return b


@dataclass(frozen=True)
class BodyGrid:
    grid: StructuredGrid
    i_tip: int
    outer_angle: float
    two_scale: bool = False


def _take(handle: C.c_void_p, lib) -> tuple[StructuredGrid, int, float]:
    try:
        ni = C.c_int32()
        nj = C.c_int32()
        _native.check(lib.bs_grid_dims(handle, C.byref(ni), C.byref(nj)), lib)
        n = (ni.value + 1) * (nj.value + 1)
        x = np.empty(n)
        y = np.empty(n)
        _native.check(lib.bs_grid_nodes(handle, x.ctypes.data_as(C.POINTER(C.c_double)),
                                        y.ctypes.data_as(C.POINTER(C.c_double))), lib)
        tip = C.c_int32()
        angle = C.c_double()
        _native.check(lib.bs_grid_info(handle, C.byref(tip), C.byref(angle)), lib)
        return StructuredGrid(ni.value, nj.value, x, y), tip.value, angle.value
    finally:
        lib.bs_grid_destroy(handle)


def body_grid(body: Body, nj: int, mach: float, gamma: float = 1.4, refinement: int = 1,
              ni: int = 0, lib=None) -> BodyGrid:
    """bodyGrid: the H-topology grid of a sharp nose; `ni` > 0 asks for
    exactly that many columns."""
    L = lib or _native.load()
    o = abi.BodyGridOptions()
    o.nj = nj
    o.refinement = refinement
    o.ni = ni
    o.mach = mach
    o.gamma = gamma
    b = body.to_abi()
    h = C.c_void_p()
    _native.check(L.bs_body_grid(C.byref(b), C.byref(o), C.byref(h)), L)
    grid, tip, angle = _take(h, L)
    return BodyGrid(grid, tip, angle)


def blunt_body_grid(body: Body, nj: int, mach: float, refinement: int = 1, ni: int = 0,
                    gated: bool = True, outer_boundary=None, lib=None) -> BodyGrid:
    """bluntBodyGrid: the C-topology grid of a blunt nose (or of a sharp one
    whose shock detaches); iMin is the axis ahead of the tip. `gated=False`
    skips the quality gates, as for the reference's two-scale (Haack) noses.
    `outer_boundary` (n, 2) points (x, y), the first on the axis, y
    increasing, replaces the generator's arc and line."""
    L = lib or _native.load()
    o = abi.BodyGridOptions()
    o.nj = nj
    o.refinement = refinement
    o.ni = ni
    o.flags = 0 if gated else abi.GRID_UNGATED
    o.mach = mach
    o.gamma = 1.4
    b = body.to_abi()
    h = C.c_void_p()
    if outer_boundary is None:
        ox = oy = np.empty(0)
    else:
        pts = np.asarray(outer_boundary, dtype=np.float64).reshape(-1, 2)
        ox, oy = np.ascontiguousarray(pts[:, 0]), np.ascontiguousarray(pts[:, 1])
    dp = C.POINTER(C.c_double)
    _native.check(L.bs_blunt_body_grid_bounded(C.byref(b), C.byref(o), ox.ctypes.data_as(dp),
                                               oy.ctypes.data_as(dp), len(ox), C.byref(h)), L)
    two = C.c_int32()
    try:
        _native.check(L.bs_grid_two_scale(h, C.byref(two)), L)
    except BaseException:
        L.bs_grid_destroy(h)
        raise
    grid, tip, angle = _take(h, L)
    return BodyGrid(grid, tip, angle, bool(two.value))


@dataclass(frozen=True)
class TransonicGrid:
    """TransonicGrid (src/grid/transonic-grid.ts:84-101)."""

    grid: StructuredGrid
    i_tip: int
    i_shoulder: int
    far_radius: float
    x_upstream: float
    x_end: float
    base_nj: int
    topology: str = "H"


def transonic_grid(body: Body, refinement: int = 1, far_field: float = 100.0, cylinder: float = 10.0,
                   spacing: dict | None = None, nested: dict | None = None, lib=None) -> TransonicGrid:
    """transonicGrid (src/grid/transonic-grid.ts:128-460): the H grid of a
    sharp nose (the C grid of a blunt one) and `cylinder` calibers of
    cylinder, its far boundaries `far_field` body radii out (rounded up to
    whole base cells); `spacing` overrides TRANSONIC_SPACING's entries (wall,
    growth, tip, shoulder, nose, nose_growth); `nested` ({"far_field": ...,
    "cylinder": ...}) cuts the H grid back or continues it to that domain,
    every shared node the same."""
    L = lib or _native.load()
    o = abi.TransonicGridOptions()
    o.refinement = refinement
    o.far_field = far_field
    o.cylinder = cylinder
    if nested is not None:
        unknown = set(nested) - {"far_field", "cylinder"}
        if unknown:
            raise ValueError(f"unknown nested-domain entries {sorted(unknown)}")
        o.nested = 1
        o.nested_far_field = float(nested.get("far_field", 0.0))
        o.nested_cylinder = float(nested.get("cylinder", 0.0))
    for k, v in (spacing or {}).items():
        if k not in ("wall", "growth", "tip", "shoulder", "nose", "nose_growth"):
            raise ValueError(f"unknown transonic spacing {k!r}")
        if not v > 0:
            raise ValueError("the transonic grid's spacings must be positive")
        setattr(o, k, float(v))
    b = body.to_abi()
    h = C.c_void_p()
    _native.check(L.bs_transonic_grid(C.byref(b), C.byref(o), C.byref(h)), L)
    shoulder, base_nj, c_grid = C.c_int32(), C.c_int32(), C.c_int32()
    far, up, end = C.c_double(), C.c_double(), C.c_double()
    try:
        _native.check(L.bs_grid_transonic_info(h, C.byref(shoulder), C.byref(base_nj), C.byref(far), C.byref(up),
                                               C.byref(end), C.byref(c_grid)), L)
    except BaseException:
        L.bs_grid_destroy(h)
        raise
    grid, tip, _ = _take(h, L)
    return TransonicGrid(grid, tip, shoulder.value, far.value, up.value, end.value, base_nj.value,
                         "C" if c_grid.value else "H")


def ramp_grid(ni: int, nj: int, x_min: float, x_corner: float, x_max: float, height: float,
              angle: float, lib=None) -> StructuredGrid:
    L = lib or _native.load()
    h = C.c_void_p()
    _native.check(L.bs_ramp_grid(ni, nj, x_min, x_corner, x_max, height, angle, C.byref(h)), L)
    return _take(h, L)[0]


def grid_quality(grid: StructuredGrid, lib=None) -> abi.GridQuality:
    L = lib or _native.load()
    q = abi.GridQuality()
    _native.check(L.bs_grid_quality_of(grid.ni, grid.nj,
                                       grid.x.ctypes.data_as(C.POINTER(C.c_double)),
                                       grid.y.ctypes.data_as(C.POINTER(C.c_double)),
                                       C.byref(q)), L)
    return q


def taylor_maccoll(mach: float, cone_angle: float, gamma: float = 1.4,
                   tolerance: float = 1e-13, lib=None) -> abi.ConeFlow:
    L = lib or _native.load()
    f = abi.ConeFlow()
    _native.check(L.bs_taylor_maccoll(mach, cone_angle, gamma, tolerance, C.byref(f)), L)
    return f


def oblique_shock(mach: float, theta: float, gamma: float = 1.4, lib=None) -> abi.Shock:
    L = lib or _native.load()
    s = abi.Shock()
    _native.check(L.bs_oblique_shock(mach, theta, gamma, C.byref(s)), L)
    return s


def normal_shock(mach: float, gamma: float = 1.4, lib=None) -> abi.Shock:
    L = lib or _native.load()
    s = abi.Shock()
    _native.check(L.bs_normal_shock(mach, gamma, C.byref(s)), L)
    return s
