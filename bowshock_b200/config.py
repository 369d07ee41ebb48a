"""Solver configuration, mirroring the reference's `Euler2DConfig`
(src/engine-cpu/euler2d.ts:58-81) and `BoundaryCondition2D` (:34-56), and
the free stream of a verified-drag case (`freeStreamAt`,
src/analysis/verified-drag.ts:218-228)."""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Mapping

import numpy as np

from . import abi


@dataclass(frozen=True)
class Primitive2D:
    """Primitive state (rho, u, v, p) (src/scheme/flux.ts:331-336)."""

    rho: float
    u: float
    v: float
    p: float


@dataclass(frozen=True)
class StructuredGrid:
    """A block of ni x nj cells; node (i, j) at i + j (ni + 1)
    (src/grid/structured.ts:12-18)."""

    ni: int
    nj: int
    x: np.ndarray
    y: np.ndarray

    def __post_init__(self) -> None:
        n = (self.ni + 1) * (self.nj + 1)
        object.__setattr__(self, "x", np.ascontiguousarray(self.x, dtype=np.float64))
        object.__setattr__(self, "y", np.ascontiguousarray(self.y, dtype=np.float64))
        if self.x.shape != (n,) or self.y.shape != (n,):
            raise ValueError(f"a {self.ni} x {self.nj} grid needs {n} nodes")


def grid_from_function(ni: int, nj: int, node) -> StructuredGrid:
    """gridFromFunction (src/grid/structured.ts:57-77)."""
    if not (isinstance(ni, int) and isinstance(nj, int) and ni >= 1 and nj >= 1):
        raise ValueError("a grid needs at least one cell in each direction")
    x = np.empty((ni + 1) * (nj + 1))
    y = np.empty((ni + 1) * (nj + 1))
    for j in range(nj + 1):
        for i in range(ni + 1):
            px, py = node(i, j)
            x[i + j * (ni + 1)] = px
            y[i + j * (ni + 1)] = py
    return StructuredGrid(ni, nj, x, y)


def rectangular_grid(ni: int, nj: int, x0: float, x1: float, y0: float, y1: float) -> StructuredGrid:
    """rectangularGrid (src/grid/structured.ts:80-89)."""
    return grid_from_function(
        ni, nj, lambda i, j: (x0 + ((x1 - x0) * i) / ni, y0 + ((y1 - y0) * j) / nj)
    )


@dataclass(frozen=True)
class Boundary:
    """One side's condition: kind in inflow | outflow | wall | farField |
    periodic; `state` for inflow and farField."""

    kind: str
    state: Primitive2D | None = None

    def __post_init__(self) -> None:
        if self.kind not in abi.BC_KIND:
            raise ValueError(f"unknown boundary kind {self.kind!r}")
        if self.kind in ("inflow", "farField") and self.state is None:
            raise ValueError(f"a {self.kind} boundary needs a state")


@dataclass(frozen=True)
class Euler2DConfig:
    grid: StructuredGrid
    geometry: str = "axisymmetric"
    gamma: float = 1.4
    flux: str = "hllc"
    limiter: str = "vanAlbada"
    reconstruction: str = "sharedScaled"
    time_integrator: str = "ssprk2"
    cfl: float = 0.8
    time_stepping: str = "local"
    boundaries: Mapping[str, Boundary] = field(default_factory=dict)

    def to_abi(self) -> abi.Config:
        for name, table in (
            ("geometry", abi.GEOMETRY),
            ("flux", abi.FLUX),
            ("limiter", abi.LIMITER),
            ("reconstruction", abi.RECONSTRUCTION),
            ("time_integrator", abi.INTEGRATOR),
            ("time_stepping", abi.TIME_STEPPING),
        ):
            if getattr(self, name) not in table:
                raise ValueError(f"unknown {name} {getattr(self, name)!r}")
        c = abi.Config()
        c.ni = self.grid.ni
        c.nj = self.grid.nj
        c.geometry = abi.GEOMETRY[self.geometry]
        c.flux = abi.FLUX[self.flux]
        c.limiter = abi.LIMITER[self.limiter]
        c.reconstruction = abi.RECONSTRUCTION[self.reconstruction]
        c.integrator = abi.INTEGRATOR[self.time_integrator]
        c.time_stepping = abi.TIME_STEPPING[self.time_stepping]
        c.gamma = self.gamma
        c.cfl = self.cfl
        for side in abi.SIDES:
            if side not in self.boundaries:
                raise ValueError(f"no boundary condition on {side}")
            b = self.boundaries[side]
            c.boundaries[abi.SIDE[side]].kind = abi.BC_KIND[b.kind]
            if b.state is not None:
                s = b.state
                c.boundaries[abi.SIDE[side]].state = abi.Primitive(s.rho, s.u, s.v, s.p)
        return c


@dataclass(frozen=True)
class FreeStream:
    state: Primitive2D
    pressure: float
    dynamic_pressure: float


def fround(x: float) -> float:
    """Round to the nearest FP32 value (JavaScript's Math.fround)."""
    return float(np.float32(x))


def free_stream_at(mach: float, gamma: float) -> FreeStream:
    """freeStreamAt (src/analysis/verified-drag.ts:218-228): unit density and
    pressure, the speed rounded to FP32 so the FP32 field solves the same
    case, and the drag normalised by its own dynamic pressure."""
    u = fround(mach * math.sqrt(gamma))
    return FreeStream(Primitive2D(1.0, u, 0.0, 1.0), 1.0, 0.5 * u * u)


def steady_drag_config(grid: StructuredGrid, free: Primitive2D, gamma: float = 1.4, **overrides) -> Euler2DConfig:
    """The configuration `verifiedForebodyDrag` solves every grid with
    (src/analysis/verified-drag.ts:241-257): axisymmetric, HLLC, van Albada
    with the scaled shared factor, SSP-RK2 at CFL 0.8 with local steps;
    inflow upstream and outside, outflow downstream, the body a wall."""
    base = dict(
        grid=grid,
        geometry="axisymmetric",
        gamma=gamma,
        flux="hllc",
        limiter="vanAlbada",
        reconstruction="sharedScaled",
        time_integrator="ssprk2",
        cfl=0.8,
        time_stepping="local",
        boundaries={
            "iMin": Boundary("inflow", free),
            "iMax": Boundary("outflow"),
            "jMin": Boundary("wall"),
            "jMax": Boundary("inflow", free),
        },
    )
    base.update(overrides)
    return Euler2DConfig(**base)
