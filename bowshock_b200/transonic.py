"""Transonic flow (Mach 1 to about 1.2) around a sharp nose followed by a
long cylinder standing for a wind-tunnel sting, with the bow shock captured
and far-field boundaries, and its forebody pressure (wave) drag
(src/analysis/transonic-flow.ts). The reference runs it on its FP64 CPU
engine and, on the GPU, in two-float arithmetic (euler2d-two-float.ts);
here every step runs on the GPU engine with an FP64 state and residual:
LU-SGS steps whose CFL number ramps from 1 by 1.2 a step, with Anderson
acceleration, until the drag settles."""
from __future__ import annotations

import math
import time
from dataclasses import dataclass

import numpy as np

from .config import Boundary, Euler2DConfig, FreeStream, free_stream_at
from .engine import CudaEuler2D
from .grid import Body, TransonicGrid, transonic_grid
from .verification import SettlingValue


@dataclass
class TransonicProblem:
    """TransonicProblem (transonic-flow.ts:48-56): the body, the grid, the
    engine's configuration and the free stream."""

    body: Body
    mach: float
    gamma: float
    refinement: int
    far_field: float
    cylinder: float
    grid: TransonicGrid
    config: Euler2DConfig
    free_stream: FreeStream

    def drag(self, engine: CudaEuler2D) -> float:
        """The forebody pressure drag coefficient over the jMin faces (the
        axis ahead of the tip adds nothing, the cylinder no axial force)."""
        return engine.forebody_drag(self.free_stream, self.body.nose.base_radius)


def transonic_problem(body: Body, mach: float, gamma: float = 1.4, refinement: int = 1, far_field: float = 100.0,
                      cylinder: float = 10.0, spacing: dict | None = None,
                      nested: dict | None = None) -> TransonicProblem:
    """transonicProblem (transonic-flow.ts:59-90): the transonic grid, far
    fields around it, the body (and the axis ahead of it) a wall: on the H
    grid of a sharp nose iMin is a far boundary upstream, on the C grid of a
    blunt one the axis ahead of the stagnation point; HLLC, van Albada with
    the scaled shared factor, axisymmetric."""
    grid = transonic_grid(body, refinement, far_field, cylinder, spacing, nested)
    free = free_stream_at(mach, gamma)
    far = Boundary("farField", free.state)
    config = Euler2DConfig(
        grid=grid.grid, geometry="axisymmetric", gamma=gamma, flux="hllc", limiter="vanAlbada",
        reconstruction="sharedScaled", time_integrator="ssprk2", cfl=0.8, time_stepping="local",
        boundaries={"iMin": far if grid.topology == "H" else Boundary("wall"), "iMax": far,
                    "jMin": Boundary("wall"), "jMax": far})
    return TransonicProblem(body, mach, gamma, refinement, far_field, cylinder, grid, config, free)


@dataclass
class TransonicSolution:
    """TransonicSolution (transonic-flow.ts:128-143); `primitives` (nj, ni, 4)
    of the last state, for starting the next grid of the family."""

    drag: float
    converged: bool
    steps: int
    seconds: float
    restarts: int
    rate: float
    stopped_by: str
    remaining_estimate: float
    primitives: np.ndarray


def geometric_remaining(values) -> float:
    """geometricRemaining (transonic-flow.ts:259-268): the remaining change of
    a geometrically converging sequence from its last three values,
    d2 r / (1 - r) with r the ratio of the last two changes; a last change at
    round-off (below 1e-12 of the value) is its own estimate; infinite if the
    changes do not fall."""
    if len(values) < 3:
        return math.inf
    a, b, c = values[-3:]
    d1, d2 = b - a, c - b
    if abs(d2) <= 1e-12 * abs(c):
        return abs(d2)
    if d1 == 0:
        return math.inf
    r = abs(d2 / d1)
    return abs(d2) * r / (1 - r) if r < 1 else math.inf


def solve_transonic(problem: TransonicProblem, noise: float = 1e-7, max_steps: int = 4000, check_every: int = 50,
                    cfl: float = 1000.0, depth: int = 8, plain_steps: int = 200, known_rate: float = math.nan,
                    geometric_noise: float | None = None, start: tuple[TransonicProblem, np.ndarray] | None = None,
                    on_check=None, metric_bits: int = 64) -> TransonicSolution:
    """solveTransonic (transonic-flow.ts:151-257) on the GPU engine: from the
    free stream (the CFL number ramped from 1 by 1.2 a step up to `cfl`) or
    from the solution on the coarser grid of the family (`start`: its
    problem and primitives (nj, ni, 4); each fine cell takes the coarse cell
    it lies in, at the full CFL number), LU-SGS steps with Anderson
    acceleration (`depth` differences after `plain_steps` plain steps; 0 for
    plain steps), the drag checked every `check_every` steps until it
    settles within `noise` (SettlingValue, with a rate known from the
    coarser grid) or, with `geometric_noise`, until its remaining change
    estimated from its last three checks is below that on two checks
    running. The residual reads two-float metrics (`metric_bits` 64), as the
    reference's two-float engine: with FP32 metrics the drag's fixed point
    moves by 1e-6 to 5e-6 of its value on these far-field domains."""
    g = problem.grid.grid
    w = None
    if start is not None:
        coarse, prims = start
        ratio = problem.refinement / coarse.refinement
        if not (ratio >= 1 and ratio == int(ratio)):
            raise ValueError("a start must come from a coarser grid of the family")
        r = int(ratio)
        w = np.asarray(prims, np.float64).reshape(coarse.grid.grid.nj, coarse.grid.grid.ni, 4)
        w = np.repeat(np.repeat(w, r, axis=0), r, axis=1)
        if w.shape[:2] != (g.nj, g.ni):
            raise ValueError("the start's grid is not the coarser grid of this family")
    t0 = time.perf_counter()
    with CudaEuler2D(problem.config) as engine:
        engine.set_metric_precision(metric_bits)
        if w is None:
            engine.set_uniform(problem.free_stream.state)
            engine.set_implicit_cfl(1.0)
        else:
            engine.set_primitives(w.reshape(-1, 4))
            engine.set_implicit_cfl(cfl)
        engine.set_anderson(depth, plain_steps)
        settling = SettlingValue(noise, known_rate)
        recent: list[float] = []
        estimate, geometric_passes, steps, drag = math.inf, 0, 0, math.nan
        stopped_by, converged = "steps", False
        while steps < max_steps:
            engine.iterate_accelerated(check_every, cfl, 1.5, 1.2)
            steps += check_every
            drag = problem.drag(engine)
            if not math.isfinite(drag):
                raise FloatingPointError("the drag is not finite")
            if on_check is not None:
                on_check(steps, drag, engine.density_residual_norm(), time.perf_counter() - t0)
            recent = (recent + [drag])[-3:]
            estimate = geometric_remaining(recent)
            geometric_passes = (geometric_passes + 1 if geometric_noise is not None
                                and estimate <= geometric_noise * abs(drag) else 0)
            settled = settling.add(drag)
            if settled or geometric_passes >= 2:
                stopped_by, converged = ("settling" if settled else "geometric"), True
                break
        restarts = engine.anderson_restarts()
        prims = engine.primitives().reshape(g.nj, g.ni, 4)
    return TransonicSolution(drag, converged, steps, time.perf_counter() - t0, restarts, settling.rate_to_pass_on,
                             stopped_by, estimate, prims)
