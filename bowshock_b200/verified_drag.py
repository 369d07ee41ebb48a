"""The forebody pressure drag with its measured discretisation error, from a
nested family of body grids (nj = 20, 40, 80, ...) each solved until the drag
itself settles: verifiedForebodyDrag (src/analysis/verified-drag.ts:230-319)
over any engine factory, and the same procedure for many cases at once, one
refinement level of every unverified case per GPU batch.

Each grid starts from the free stream and is iterated in checks of 500 r steps
(r the refinement) until its drag settles to `noise` (verification.
SettlingValue), at most 60 checks; a settled grid is refused if the flow
leaves the outflow plane subsonic or the bow shock reaches the outer boundary
(its outer row differs from the free stream by more than 1e-5). The values of
the family then give the error band (verification.refine_until_verified).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from .config import FreeStream, Primitive2D, free_stream_at, steady_drag_config
from .engine import cuda_engine, forebody_pressure_drag
from .grid import Body, body_grid
from .verification import (Estimate, SettlingValue, VerifiedValue, grid_convergence,
                           refine_until_verified)

BASE_NJ = 20
BATCH = 500
MAX_BATCHES = 60
OUTER_TOLERANCE = 1e-5
ORDER_TOLERANCE = 0.5
# Systematic error of the captured-shock forebody drag that refinement does
# not remove, relative (the reference's DRAG_FLOOR, measured against exact
# cone and ogive solutions; src/analysis/verified-drag.ts:108).
DRAG_FLOOR = 1e-3
# Settling threshold of this engine's drag, relative: its state and residual
# are FP64, and its drag settles far below the reference GPU engine's FP32
# noise (2e-6).
ENGINE_NOISE = 1e-9


class IterationStalled(Exception):
    pass


class InvalidCase(Exception):
    pass


@dataclass
class LevelReport:
    refinement: int
    ni: int
    nj: int
    iterations: int
    drag: float


@dataclass
class VerifiedDrag:
    """kind: 'solved' (result set), 'not-converged' or 'invalid' (reason)."""

    kind: str
    result: VerifiedValue | None = None
    reports: list[LevelReport] = field(default_factory=list)
    refinement: int | None = None
    reason: str | None = None
    column_density: float | None = None   # fitted families solved with more columns than usual
    floor: float | None = None            # the allowance in a fitted band, relative (fittedDragFloor)


def outflow_mach(gamma: float, ni: int, nj: int, cell) -> float:
    """Smallest u / a over the cells next to the outflow plane (iMax)."""
    return min(cell(ni - 1, j).u / math.sqrt(gamma * cell(ni - 1, j).p / cell(ni - 1, j).rho)
               for j in range(nj))


def outer_deviation(gamma: float, free, ni: int, nj: int, cell) -> float:
    """Largest deviation from the free stream over the outer row (jMax):
    density and pressure relative, velocity over the speed of sound."""
    a = math.sqrt(gamma * free.p / free.rho)
    worst = 0.0
    for i in range(ni):
        w = cell(i, nj - 1)
        worst = max(worst, abs(w.rho / free.rho - 1), abs(w.p / free.p - 1),
                    abs(w.u - free.u) / a, abs(w.v - free.v) / a)
    return worst


def _check_settled(gamma: float, free: FreeStream, ni: int, nj: int, cell) -> None:
    out = outflow_mach(gamma, ni, nj, cell)
    if not out > 1:
        raise InvalidCase(f"the flow leaves the grid at an axial Mach number of {out:.3f}, "
                          "where the outflow condition does not hold")
    dev = outer_deviation(gamma, free.state, ni, nj, cell)
    if not dev <= OUTER_TOLERANCE:
        raise InvalidCase(f"the flow along the outer boundary differs from the free stream by "
                          f"{dev:.1e}: the bow shock reaches it")


def verified_forebody_drag(body: Body, mach: float, gamma: float = 1.4, tolerance: float = 1e-4,
                           max_refinement: int = 8, noise: float = ENGINE_NOISE,
                           floor: float = DRAG_FLOOR, order_tolerance: float = ORDER_TOLERANCE,
                           engine_for: Callable | None = None,
                           on_level: Callable[[LevelReport], None] | None = None) -> VerifiedDrag:
    """verifiedForebodyDrag over an engine factory (default: this library's
    GPU engine), one grid at a time."""
    engine_for = engine_for or cuda_engine()
    free = free_stream_at(mach, gamma)
    reports: list[LevelReport] = []
    last = [1]

    def solve_at(r: int) -> float:
        last[0] = r
        grid = body_grid(body, BASE_NJ, mach, gamma, refinement=r).grid
        cfg = steady_drag_config(grid, free.state, gamma)
        engine = engine_for(cfg, free.state)
        try:
            settling = SettlingValue(noise)
            for k in range(1, MAX_BATCHES + 1):
                engine.iterate(BATCH * r)
                drag = forebody_pressure_drag(engine.wall_fluxes(), free, body.nose.base_radius)
                if not math.isfinite(drag):
                    raise IterationStalled("the solution is not finite")
                if settling.add(drag):
                    _check_settled(gamma, free, grid.ni, grid.nj, engine.cells())
                    rep = LevelReport(r, grid.ni, grid.nj, k * BATCH * r, drag)
                    reports.append(rep)
                    if on_level is not None:
                        on_level(rep)
                    return drag
            raise IterationStalled(f"the drag still changes by more than {noise} of its value "
                                   f"after {MAX_BATCHES * BATCH * r} iterations")
        finally:
            engine.destroy()

    try:
        result = refine_until_verified(solve_at, tolerance, floor, max_refinement, order_tolerance, noise)
        return VerifiedDrag("solved", result, reports)
    except IterationStalled as e:
        return VerifiedDrag("not-converged", None, reports, last[0], str(e))
    except InvalidCase as e:
        return VerifiedDrag("invalid", None, reports, last[0], str(e))


def verified_forebody_drags(cases: list[tuple[Body, float]], gamma: float = 1.4, tolerance: float = 1e-4,
                            max_refinement: int = 8, noise: float = ENGINE_NOISE,
                            floor: float = DRAG_FLOOR, order_tolerance: float = ORDER_TOLERANCE,
                            precision: int = 64, metric_bits: int = 32) -> list[VerifiedDrag]:
    """The same procedure for many (body, Mach) cases: each refinement level
    of every case not yet verified is one GPU batch, iterated in checks of
    500 r steps; a case whose drag has settled is frozen while the others go
    on. The outcome of every case is the one verified_forebody_drag gives.
    `metric_bits` 64 makes the residual read two-float metrics (the steady
    state of the FP64 CPU engine, at 24 more bytes per cell)."""
    from .batch import CudaBatch

    n = len(cases)
    frees = [free_stream_at(m, gamma) for _, m in cases]
    outcome: list[VerifiedDrag | None] = [None] * n
    levels: list[list[tuple[int, float]]] = [[] for _ in range(n)]
    reports: list[list[LevelReport]] = [[] for _ in range(n)]
    r = 1
    while r <= max_refinement:
        todo = [k for k in range(n) if outcome[k] is None]
        if not todo:
            break
        grids = [body_grid(cases[k][0], BASE_NJ, cases[k][1], gamma, refinement=r).grid for k in todo]
        batch = CudaBatch([steady_drag_config(g, frees[k].state, gamma) for g, k in zip(grids, todo)],
                          precision=precision)
        if metric_bits != 32:
            batch.set_metric_precision(metric_bits)
        try:
            batch.set_free_stream()
            settle = [SettlingValue(noise) for _ in todo]
            active = np.ones(len(todo), np.int32)
            for check in range(1, MAX_BATCHES + 1):
                batch.iterate(BATCH * r)
                for s, k in enumerate(todo):
                    if not active[s]:
                        continue
                    body = cases[k][0]
                    drag = batch.forebody_drag(s, frees[k], body.nose.base_radius)
                    if not math.isfinite(drag):
                        outcome[k] = VerifiedDrag("not-converged", None, reports[k], r, "the solution is not finite")
                        active[s] = 0
                    elif settle[s].add(drag):
                        active[s] = 0
                        g = grids[s]
                        w = batch.primitives(s).reshape(-1, 4)
                        cell = (lambda w_, ni_: (lambda i, j: Primitive2D(*map(float, w_[i + j * ni_]))))(w, g.ni)
                        try:
                            _check_settled(gamma, frees[k], g.ni, g.nj, cell)
                        except InvalidCase as e:
                            outcome[k] = VerifiedDrag("invalid", None, reports[k], r, str(e))
                            continue
                        reports[k].append(LevelReport(r, g.ni, g.nj, check * BATCH * r, drag))
                        levels[k].append((r, drag))
                if not active.any():
                    break
                batch.set_active(active)
            for s, k in enumerate(todo):
                if active[s] and outcome[k] is None:
                    outcome[k] = VerifiedDrag("not-converged", None, reports[k], r,
                                              f"the drag still changes by more than {noise} of its value "
                                              f"after {MAX_BATCHES * BATCH * r} iterations")
        finally:
            batch.destroy()
        # The error band of every case that solved this level.
        for k in todo:
            if outcome[k] is not None:
                continue
            est = grid_convergence([v for _, v in levels[k]], order_tolerance, noise)
            unc = None if est.kind == "unresolved" else est.uncertainty + floor * abs(est.value)
            verified = unc is not None and unc <= tolerance
            if verified or r * 2 > max_refinement:
                outcome[k] = VerifiedDrag("solved", VerifiedValue(est, unc, verified, list(levels[k])),
                                          reports[k])
        r *= 2
    return [o if o is not None else VerifiedDrag("solved", VerifiedValue(
        Estimate("unresolved", levels[k][-1][1] if levels[k] else math.nan, reason="no grid solved"),
        None, False, list(levels[k])), reports[k]) for k, o in enumerate(outcome)]
