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


# ---- seeded batches of uneven cases ------------------------------------------

class SplitMix64:
    """SplitMix64 (Steele, Lea and Flood, 2014): a 64-bit seeded generator
    whose sequence any language can reproduce from the seed."""

    MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        self.state = seed & self.MASK

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & self.MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.MASK
        return z ^ (z >> 31)

    def uniform(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / (1 << 53)))

    def integer(self, n: int) -> int:
        return self.next_u64() % n


NOSE_FAMILIES = ("conical", "ogive", "parabolic", "ellipsoid", "haack")


@dataclass(frozen=True)
class NoseCase:
    """One seeded case: nose family, fineness (nose length in diameters),
    body length in diameters (nose + cylinder), Mach number and grid size."""

    seed: int
    family: str
    fineness: float
    body_length: float
    mach: float
    ni: int
    nj: int

    def body(self) -> Body:
        shape = {
            "conical": NoseShape("conical"),
            "ogive": NoseShape("ogive", 1.0),        # tangent ogive
            "parabolic": NoseShape("parabolic", 1.0),  # K = 1: tangent at the base
            "ellipsoid": NoseShape("ellipsoid"),
            "haack": NoseShape("haack", 0.0),        # Von Karman (LD-Haack)
        }[self.family]
        nose_length = 2 * 0.5 * self.fineness
        return Body(Nose(shape, nose_length, 0.5), max(0.0, self.body_length - nose_length))


def draw_nose_case(seed: int, levels: tuple[int, ...] = (0, 1, 2, 3), base_ni: int = 40,
                   machs: tuple[float, float] = (1.5, 5.0)) -> NoseCase:
    """A case drawn from the batched distribution: nose family uniform over
    NOSE_FAMILIES, fineness U[1, 5], body length U[2, 8] diameters, Mach
    U[1.5, 5.0], ni = base_ni 2^k with k uniform over `levels`, nj = ni / 2.
    The cylinder is the body length less the nose (none when the nose is
    longer)."""
    g = SplitMix64(seed)
    family = NOSE_FAMILIES[g.integer(len(NOSE_FAMILIES))]
    fineness = g.uniform(1.0, 5.0)
    body_length = g.uniform(2.0, 8.0)
    mach = g.uniform(*machs)
    k = levels[g.integer(len(levels))]
    ni = base_ni * 2**k
    return NoseCase(seed, family, fineness, body_length, mach, ni, ni // 2)


def case_from(nc: NoseCase) -> Case:
    """The grid and configuration of a seeded case: the H-topology grid where
    the tip is sharp and its shock attached, else the C-topology grid (the
    axis ahead of the tip a symmetry line), ungated for the two-scale Haack
    nose as the reference builds it. Raises if no grid can be made."""
    from . import _native
    from .config import Boundary
    from .grid import blunt_body_grid

    body = nc.body()
    free = free_stream_at(nc.mach, GAMMA)
    c_grid = False
    if nc.family in ("conical", "ogive", "parabolic"):
        try:
            grid = body_grid(body, nc.nj, nc.mach, GAMMA, ni=nc.ni).grid
        except _native.BowshockError:
            c_grid = True
    else:
        c_grid = True
    if c_grid:
        grid = blunt_body_grid(body, nc.nj, nc.mach, ni=nc.ni,
                               gated=nc.family not in ("haack", "conical", "ogive", "parabolic")).grid
        boundaries = {"iMin": Boundary("wall"), "iMax": Boundary("outflow"),
                      "jMin": Boundary("wall"), "jMax": Boundary("inflow", free.state)}
        cfg = steady_drag_config(grid, free.state, boundaries=boundaries)
    else:
        cfg = steady_drag_config(grid, free.state)
    name = f"{nc.family}-f{nc.fineness:.2f}-L{nc.body_length:.2f}-M{nc.mach:.2f}-{nc.ni}x{nc.nj}"
    return Case(name, cfg, free, body, nc.mach)


def make_cases(specs: list[NoseCase], threads: int | None = None) -> list[Case | None]:
    """The grid and configuration of every spec (case_from), made on
    `threads` host threads (the generator is native code that runs outside
    the interpreter lock); None where no grid can be made."""
    import os
    from concurrent.futures import ThreadPoolExecutor

    from . import _native

    def make(nc: NoseCase):
        try:
            return case_from(nc)
        except _native.BowshockError:
            return None

    with ThreadPoolExecutor(max_workers=threads or os.cpu_count() or 1) as pool:
        return list(pool.map(make, specs))


def seeded_cases(count: int, first_seed: int = 1, threads: int | None = None,
                 **draw) -> tuple[list[Case], list[NoseCase]]:
    """`count` consecutive seeds drawn as draw_nose_case, their grids made by
    make_cases; cases whose grid cannot be made are left out and returned
    second."""
    specs = [draw_nose_case(s, **draw) for s in range(first_seed, first_seed + count)]
    results = make_cases(specs, threads)
    made = [c for c in results if c is not None]
    refused = [nc for nc, c in zip(specs, results) if c is None]
    return made, refused


STREAM_MACHS = (1.5, 2.0, 3.0, 4.0)


def stream_specs(geometries: int, first_seed: int = 1, machs: tuple[float, ...] = STREAM_MACHS,
                 levels: tuple[int, ...] = (0, 1, 2, 3), base_ni: int = 80) -> list[NoseCase]:
    """The combined stream's cases: `geometries` seeded nose + body
    geometries of the batched distribution (draw_nose_case; the grid level
    is drawn per geometry, ni = base_ni 2^k), each at every Mach number of
    `machs`, geometry by geometry."""
    from dataclasses import replace

    out = []
    for s in range(first_seed, first_seed + geometries):
        g = draw_nose_case(s, levels=levels, base_ni=base_ni)
        out.extend(replace(g, mach=m) for m in machs)
    return out
