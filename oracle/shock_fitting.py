"""TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.

The fitted-shock iteration restated on the FP64 oracle, the checker of the
GPU's fitted solver: fitShock (src/solver/shock-fitting.ts:170-314) with
its shock relations (shockState and compatibleShock, :50-111) and
remapAlongLines (:324-358), step for step: the shock boundary from the flow
at the start of each step, one explicit step with those face states and
fluxes held, each shock node moved along its line by W dt / (n . line) (the
face on its axis side, dt half the top cell's height over its fastest
signal), the grid rebuilt on the new heights and the flow interpolated
along the lines. A problem is bowshock_b200.fitted.FitProblem (its lines,
fractions, heights, inflow states and start field).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .oracle import OracleEuler2D


def shock_states(free, gamma: float, mach: np.ndarray, nx: np.ndarray, ny: np.ndarray):
    """shockState (shock-fitting.ts:50-78) for arrays of faces: post-shock
    primitives (n, 4), speeds and post-shock normal velocities."""
    a = math.sqrt(gamma * free.p / free.rho)
    vn = free.u * nx + free.v * ny
    speed = mach * a + vn
    m2 = mach * mach
    density_ratio = (gamma + 1) * m2 / ((gamma - 1) * m2 + 2)
    pressure_ratio = 1 + 2 * gamma / (gamma + 1) * (m2 - 1)
    un = speed - mach * a / density_ratio
    w = np.stack([free.rho * density_ratio, free.u + (un - vn) * nx, free.v + (un - vn) * ny,
                  free.p * pressure_ratio], 1)
    return w, speed, un


def compatible_shocks(free, gamma: float, nx, ny, rho, a, p, un):
    """compatibleShock (shock-fitting.ts:87-111) for arrays of faces: the
    same bisection per face (bracket doubled from [1, 2], at most 100
    halvings, until the bracket is within 1e-15 of its top)."""
    impedance = rho * a
    target = p + impedance * un

    def mismatch(m):
        w, _, u = shock_states(free, gamma, m, nx, ny)
        return w[:, 3] + impedance * u - target

    n = len(nx)
    mach = np.ones(n)
    go = mismatch(np.ones(n)) < 0
    low, high = np.ones(n), np.full(n, 2.0)
    grow = go.copy()
    while grow.any():
        grow &= mismatch(high) < 0
        high = np.where(grow, 2 * high, high)
    active = go.copy()
    for _ in range(100):
        active &= high - low > 1e-15 * high
        if not active.any():
            break
        mid = 0.5 * (low + high)
        below = mismatch(mid) < 0
        low = np.where(active & below, mid, low)
        high = np.where(active & ~below, mid, high)
    mach = np.where(go, 0.5 * (low + high), 1.0)
    return shock_states(free, gamma, mach, nx, ny)


@dataclass
class OracleFit:
    engine: OracleEuler2D
    heights: np.ndarray
    max_speed: float
    iterations: int
    speeds: list


def _primitives(engine: OracleEuler2D, ni: int, nj: int) -> np.ndarray:
    return engine.primitives().reshape(nj, ni, 4)


def shock_boundary(engine: OracleEuler2D, problem):
    """The shock on every jMax face for the engine's flow and the flux
    through it (fitShock's shockBoundary, :184-214); applies both."""
    ni, nj, g = problem.ni, problem.nj, problem.gamma
    _, j_faces, _ = engine.metrics()
    f = j_faces.reshape(nj + 1, ni, 3)[nj]
    nx, ny = f[:, 0], f[:, 1]
    w = _primitives(engine, ni, nj)
    c1, c2 = w[nj - 1], w[nj - 2]
    states, speeds, _ = compatible_shocks(
        problem.free, g, nx, ny, c1[:, 0], np.sqrt(g * c1[:, 3] / c1[:, 0]), 1.5 * c1[:, 3] - 0.5 * c2[:, 3],
        1.5 * (c1[:, 1] * nx + c1[:, 2] * ny) - 0.5 * (c2[:, 1] * nx + c2[:, 2] * ny))
    rho, u, v, p = states.T
    energy = p / (g - 1) + 0.5 * rho * (u * u + v * v)
    un = u * nx + v * ny
    fluxes = np.stack([rho * un, rho * u * un + p * nx, rho * v * un + p * ny, un * (energy + p)], 1)
    engine.set_face_states("jMax", states)
    engine.set_face_fluxes("jMax", fluxes)
    return states, speeds, nx, ny


def remap_along_lines(problem, old_w: np.ndarray, old_h: np.ndarray, new_h: np.ndarray) -> np.ndarray:
    """remapAlongLines (:324-358): each new cell takes the primitives
    interpolated linearly between the old centres of its column (held at
    the end cells beyond them); distances along a column are the mean of
    its two lines' (a node's distance along its line is h times its
    fraction: the lines' directions are unit vectors)."""
    ni, nj = problem.ni, problem.nj
    fr = problem.fractions                                    # (ni + 1, nj + 1)

    def column_along(h):                                      # (ni, nj + 1)
        d = h[:, None] * fr
        return 0.5 * (d[:-1] + d[1:])

    old_c, new_c = column_along(old_h), column_along(new_h)
    centre = 0.5 * (old_c[:, :-1] + old_c[:, 1:])             # (ni, nj)
    out = np.empty((nj, ni, 4))
    for i in range(ni):
        d = 0.5 * (new_c[i, :-1] + new_c[i, 1:])
        for j in range(nj):
            jj = 0
            while jj < nj - 2 and centre[i, jj + 1] < d[j]:
                jj += 1
            t = min(max((d[j] - centre[i, jj]) / (centre[i, jj + 1] - centre[i, jj]), 0.0), 1.0)
            a, b = old_w[jj, i], old_w[jj + 1, i]
            out[j, i] = a + t * (b - a)
    return out.reshape(-1, 4)


def _engine(problem, heights, prims):
    e = OracleEuler2D(problem.config(heights))
    e.set_primitives(prims)
    if problem.inflow is not None:
        e.set_face_states("iMin", problem.inflow)
    return e


def fit_shock(problem, steps: int) -> OracleFit:
    """`steps` iterations of fitShock (one step per move)."""
    ni, nj, g = problem.ni, problem.nj, problem.gamma
    free = problem.free
    a_free = math.sqrt(g * free.p / free.rho)
    heights = problem.heights.copy()
    solver = _engine(problem, heights, problem.initial)
    max_speed = math.inf
    speeds_log = []
    for _ in range(steps):
        _, speeds, nx, ny = shock_boundary(solver, problem)
        solver.iterate(1)
        w = _primitives(solver, ni, nj)
        x, y = problem.nodes(heights)
        X, Y = x.reshape(nj + 1, ni + 1), y.reshape(nj + 1, ni + 1)
        nxt = heights.copy()
        for k in range(1, ni + 1):
            f = k - 1
            cell = w[nj - 1, min(k, ni - 1)]
            height = math.hypot(X[nj, k] - X[nj - 1, k], Y[nj, k] - Y[nj - 1, k])
            dt = 0.5 * height / (math.hypot(cell[1], cell[2]) + math.sqrt(g * cell[3] / cell[0]))
            nxt[k] = heights[k] + speeds[f] * dt / (problem.line_dx[k] * nx[f] + problem.line_dy[k] * ny[f])
        max_speed = float(np.max(np.abs(speeds)) / a_free)
        speeds_log.append(max_speed)
        if problem.first_node == "symmetry":
            def node(k):
                return (problem.line_x[k] + nxt[k] * problem.line_dx[k],
                        problem.line_y[k] + nxt[k] * problem.line_dy[k])
            (x1, y1), (x2, y2) = node(1), node(2)
            c = (x2 - x1) / (y2 * y2 - y1 * y1)
            nxt[0] = (x1 - c * y1 * y1 - problem.line_x[0]) / problem.line_dx[0]
        remapped = remap_along_lines(problem, w, heights, nxt)
        heights = nxt
        solver = _engine(problem, heights, remapped)
    shock_boundary(solver, problem)
    return OracleFit(solver, heights, max_speed, steps, speeds_log)
