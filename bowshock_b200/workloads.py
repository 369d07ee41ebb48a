"""The benchmark workloads as cases: grid, configuration, free stream and
body, built from synthetic nose geometries (seeded where random).

- `cone_case`: the plain explicit case - a sharp 15 deg half-angle cone
  (nose 1.866 calibers long, so that the half-angle is exactly 15 deg), a
  2-caliber cylinder, Mach 2, 80 x 40 cells, minmod per-variable MUSCL + HLLC
  + SSP-RK3 at CFL 0.5 with local time steps.
- `drag_sweep_cases`: the drag curve - a tangent ogive of fineness 3 on a
  4-caliber cylinder at Mach 1.5, 1.6, ..., 3.0 (16 cases), 160 x 80 cells,
  the reference's steady scheme (van Albada with the scaled shared factor,
  HLLC; src/analysis/verified-drag.ts:241-257), marched by LU-SGS at CFL 5.

Lengths are in body diameters (base radius 0.5); the free stream is the
reference's nondimensional one (unit density and pressure, speed rounded to
FP32; src/analysis/verified-drag.ts:218-228), for which the drag coefficient
is the same as for the dimensional 101325 Pa / 288.15 K stream.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

from .config import Euler2DConfig, FreeStream, free_stream_at, steady_drag_config
from .grid import Body, Nose, NoseShape, body_grid

GAMMA = 1.4
DEG = math.pi / 180


@dataclass(frozen=True)
class Case:
    name: str
    config: Euler2DConfig
    free: FreeStream
    body: Body
    mach: float


def cone_body(half_angle_deg: float, cylinder: float, radius: float = 0.5) -> Body:
    return Body(Nose(NoseShape("conical"), radius / math.tan(half_angle_deg * DEG), radius), cylinder)


def ogive_body(fineness: float, cylinder: float, radius: float = 0.5) -> Body:
    """Tangent ogive (OpenRocket ogive parameter 1) `fineness` diameters long."""
    return Body(Nose(NoseShape("ogive", 1.0), 2 * radius * fineness, radius), cylinder)


def cone_case(ni: int = 80, nj: int = 40, mach: float = 2.0) -> Case:
    body = cone_body(15, 2.0)
    free = free_stream_at(mach, GAMMA)
    bg = body_grid(body, nj, mach, GAMMA, ni=ni)
    cfg = steady_drag_config(bg.grid, free.state, limiter="minmod", reconstruction="perVariable",
                             time_integrator="ssprk3", cfl=0.5)
    return Case(f"cone15-M{mach:g}-{ni}x{nj}", cfg, free, body, mach)


def ogive_case(mach: float, ni: int = 160, nj: int = 80) -> Case:
    body = ogive_body(3.0, 4.0)
    free = free_stream_at(mach, GAMMA)
    bg = body_grid(body, nj, mach, GAMMA, ni=ni)
    cfg = steady_drag_config(bg.grid, free.state)
    return Case(f"ogive3-cyl4-M{mach:.1f}-{ni}x{nj}", cfg, free, body, mach)


def drag_sweep_machs() -> list[float]:
    return [round(1.5 + 0.1 * k, 1) for k in range(16)]


def drag_sweep_cases(ni: int = 160, nj: int = 80) -> list[Case]:
    return [ogive_case(m, ni, nj) for m in drag_sweep_machs()]
