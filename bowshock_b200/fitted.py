"""Host side of the fitted bow shock (src/solver/shock-fitting.ts,
src/analysis/fitted-flow.ts): the shock relations of a fitted shock, the
Taylor-Maccoll field on rays, and column placement by a density, over the
native library.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
from dataclasses import dataclass

import numpy as np

from . import _native, abi
from .config import (Boundary, Euler2DConfig, FreeStream, Primitive2D, StructuredGrid, free_stream_at,
                     steady_drag_config)
from .engine import forebody_pressure_drag
from .grid import Body, normal_shock, taylor_maccoll

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


# ---- the sharp-nose fit problem ----------------------------------------------

SHARP_START = 1e-3       # the solved domain starts at this fraction of the nose (fitted-flow.ts:79)
SHARP_ASPECT = 2.0       # cells along the body: this many times the across spacing (:84)
SOLVED_CYLINDER = 1.0    # shortest cylinder solved behind a nose, calibers (:131)
SPEED_TOLERANCE = 1e-12  # the fit stops when every shock face is slower than this times a_inf (:86)
RESIDUAL_TOLERANCE = 1e-12  # ... and the residual is below this, relative (:88)
MAX_ASPECT = 10.0        # the quality gates' largest aspect ratio (src/grid/quality.ts)


def line_strength(h, radius: float):
    """lineStrength (src/grid/blunt-grid.ts:560-562)."""
    return np.minimum(np.log1p(np.asarray(h) / radius), 2 * math.log(MAX_ASPECT))


def stretched_fraction(b, j, nj: int):
    """stretchedFraction (src/grid/blunt-grid.ts:565-567)."""
    return np.expm1(b * j / nj) / np.expm1(b)


@dataclass
class FitProblem:
    """What a fit needs (FitProblem, src/analysis/fitted-flow.ts:192-217):
    straight grid lines from the body with fixed node fractions, starting
    shock heights, the inflow plane's states (sharp noses), the start field
    and the drag of the part ahead of the solved domain."""

    line_x: np.ndarray       # (ni + 1,) line origins on the body
    line_y: np.ndarray
    line_dx: np.ndarray      # unit directions
    line_dy: np.ndarray
    fractions: np.ndarray    # (ni + 1, nj + 1) node fractions of each line's height
    heights: np.ndarray      # (ni + 1,) starting shock heights
    nj: int
    base_radius: float
    gamma: float
    mach: float
    free: Primitive2D
    inflow: np.ndarray | None   # (nj, 4) primitives outside the iMin faces, or None (axis)
    initial: np.ndarray      # (ni nj, 4) primitives, cell (i, j) at i + j ni
    first_node: str          # 'fixed' or 'symmetry'
    tip_drag: float          # drag coefficient of the nose ahead of the domain

    @property
    def ni(self) -> int:
        return len(self.line_x) - 1

    def nodes(self, heights=None) -> tuple[np.ndarray, np.ndarray]:
        """gridOnLines (src/grid/blunt-grid.ts:602-620): node (i, j) at
        i + j (ni + 1), each line cut at its own height."""
        h = self.heights if heights is None else np.asarray(heights, np.float64)
        d = h[None, :] * self.fractions.T                   # (nj + 1, ni + 1)
        x = self.line_x[None, :] + d * self.line_dx[None, :]
        y = self.line_y[None, :] + d * self.line_dy[None, :]
        return x.ravel(), y.ravel()

    def grid(self, heights=None) -> StructuredGrid:
        x, y = self.nodes(heights)
        return StructuredGrid(self.ni, self.nj, x, y)

    def config(self, heights=None) -> Euler2DConfig:
        """The engine on the grid (engineConfig, fitted-flow.ts:90-112): the
        steady scheme, iMin the inflow plane's face states (sharp) or a wall
        (the axis ahead of a blunt nose), iMax outflow, jMin the wall, jMax
        the fitted shock's face states."""
        i_min = Boundary("faceStates") if self.inflow is not None else Boundary("wall")
        return steady_drag_config(self.grid(heights), self.free, self.gamma, boundaries={
            "iMin": i_min, "iMax": Boundary("outflow"), "jMin": Boundary("wall"),
            "jMax": Boundary("faceStates")})

    def drag(self, wall) -> float:
        """The forebody drag from the wall's fluxes, with the tip's."""
        fs = FreeStream(self.free, 1.0, 0.5 * self.free.u ** 2)
        return forebody_pressure_drag(wall, fs, self.base_radius) + self.tip_drag


def _body_radius(body: Body, x) -> np.ndarray:
    L = _native.load()
    x = np.ascontiguousarray(np.atleast_1d(x), np.float64)
    r = np.empty_like(x)
    dp = C.POINTER(C.c_double)
    _native.check(L.bs_body_radius(C.byref(body.to_abi()), len(x), x.ctypes.data_as(dp), r.ctypes.data_as(dp)), L)
    return r


def _nose_slopes(body: Body) -> tuple[float, float]:
    L = _native.load()
    tip, base = C.c_double(), C.c_double()
    _native.check(L.bs_nose_slopes(C.byref(body.to_abi()), C.byref(tip), C.byref(base)), L)
    return tip.value, base.value


def sharp_fit_problem(asked: Body, mach: float, nj: int = 10, refinement: int = 1, gamma: float = 1.4,
                      column_density: float = 1.0) -> FitProblem:
    """sharpFitProblem (src/analysis/fitted-flow.ts:332-465): the flow between
    a sharp nose and its fitted shock, from a plane normal to the axis just
    behind the tip, where the tip cone's conical flow (Taylor-Maccoll) comes
    in, on vertical lines that keep the fractions of the tip shock's first
    guess. Raises ValueError where the reference refuses the nose."""
    R = asked.nose.base_radius
    body = Body(asked.nose, max(asked.cylinder_length, SOLVED_CYLINDER * 2 * R))
    L = body.nose.length
    x_end = L + body.cylinder_length
    free = free_stream_at(mach, gamma).state
    tip_slope, base_slope = _nose_slopes(body)
    if not math.isfinite(tip_slope):
        raise ValueError("the nose is blunt: it needs the blunt fit")
    tip_angle = math.atan(tip_slope)
    try:
        _, _, cone = cone_flow_field(mach, tip_angle, gamma, [tip_angle])
    except _native.BowshockError as e:
        raise ValueError(f"at Mach {_number(mach)} the bow shock cannot stay attached to a tip of "
                         f"{math.degrees(tip_angle):.1f} deg half-angle; this needs a sharper or longer nose, "
                         "or a higher Mach number") from e
    beta = cone.shock_angle
    enthalpy = gamma / (gamma - 1) + 0.5 * free.u * free.u
    v_max = math.sqrt(2 * enthalpy)
    jump = normal_shock(mach * math.sin(beta), gamma)
    entropy = jump.pressure_ratio / jump.density_ratio ** gamma

    def conical(polar) -> np.ndarray:
        rays = np.clip(np.atleast_1d(np.asarray(polar, np.float64)), tip_angle, beta)
        speed, angle, _ = cone_flow_field(mach, tip_angle, gamma, rays)
        v = speed * v_max
        a2 = (gamma - 1) * (enthalpy - 0.5 * v * v)
        rho = (a2 / gamma / entropy) ** (1 / (gamma - 1))
        return np.stack([rho, v * np.cos(angle), v * np.sin(angle), entropy * rho ** gamma], 1)

    nj = nj * refinement
    x0 = SHARP_START * L

    def guess(x):
        x = np.atleast_1d(np.asarray(x, np.float64))
        return np.maximum(x * math.tan(beta) - _body_radius(body, x), 1e-12 * L)

    L_ = _native.load()
    cap = 1 << 20
    xs = np.empty(cap, np.float64)
    count = C.c_int32()
    _native.check(L_.bs_sharp_fit_columns(C.byref(body.to_abi()), beta, x0, nj, refinement, SHARP_ASPECT,
                                          column_density, cap, xs.ctypes.data_as(C.POINTER(C.c_double)),
                                          C.byref(count)), L_)
    xs = xs[:count.value].copy()
    h = guess(xs)
    b = line_strength(h, R)
    fractions = stretched_fraction(b[:, None], np.arange(nj + 1)[None, :], nj)
    n = len(xs)
    problem = FitProblem(xs.copy(), _body_radius(body, xs), np.zeros(n), np.ones(n), fractions, h.copy(), nj, R,
                         gamma, mach, free, None, np.empty(0), "fixed", 0.0)
    X, Y = problem.nodes()
    X = X.reshape(nj + 1, n)
    Y = Y.reshape(nj + 1, n)
    # The inflow plane's faces take the conical flow at their midpoints.
    mx, my = 0.5 * (X[:-1, 0] + X[1:, 0]), 0.5 * (Y[:-1, 0] + Y[1:, 0])
    problem.inflow = conical(np.arctan2(my, mx))
    # The axial Mach number of the conical flow is least on the surface.
    surface = conical(tip_angle)[0]
    a_s = math.sqrt(gamma * surface[3] / surface[0])
    surface_mach = math.hypot(surface[1], surface[2]) / a_s
    axial_mach = surface[1] / a_s
    if not axial_mach > 1 and (not surface_mach > 1 or base_slope > 0):
        degrees = f"{math.degrees(tip_angle):.1f}"
        if surface_mach > 1:
            raise ValueError(
                f"at Mach {_number(mach)} the flow behind a tip of {degrees} deg half-angle crosses the solver's "
                f"starting plane, normal to the axis, at an axial Mach number of {axial_mach:.2f} at the surface, "
                "below 1, which this solver handles only where the nose meets the body without a corner: at a "
                "corner the drag converges too slowly to be verified; this needs a sharper or longer nose, a nose "
                "tangent to the body, or a higher Mach number")
        raise ValueError(
            f"at Mach {_number(mach)} the flow over a tip of {degrees} deg half-angle is subsonic at the surface "
            f"(Mach {surface_mach:.2f}), so the body behind the tip reaches it, which this solver does not handle "
            "yet; this needs a sharper or longer nose, or a higher Mach number")
    cx = 0.25 * (X[:-1, :-1] + X[:-1, 1:] + X[1:, :-1] + X[1:, 1:])
    cy = 0.25 * (Y[:-1, :-1] + Y[:-1, 1:] + Y[1:, :-1] + Y[1:, 1:])
    problem.initial = conical(np.arctan2(cy, cx).ravel())
    r0 = float(_body_radius(body, x0)[0])
    problem.tip_drag = taylor_maccoll(mach, tip_angle, gamma).surface_pressure_coefficient * (r0 / R) ** 2
    return problem


# ---- the fitted solve on the GPU -----------------------------------------------

class CudaFit:
    """A fit problem solved with its bow shock fitted, on the GPU (bs_fit_*):
    every step the shock boundary, an explicit step, the shock's move, the
    new grid and the remap, replayed from CUDA graphs."""

    def __init__(self, problem: FitProblem):
        self._lib = _native.load()
        self.problem = problem
        cfg = problem.config()
        dp = C.POINTER(C.c_double)
        arrays = [np.ascontiguousarray(a, np.float64) for a in (
            problem.line_x, problem.line_y, problem.line_dx, problem.line_dy, problem.fractions.reshape(-1),
            problem.heights)]
        inflow = None if problem.inflow is None else np.ascontiguousarray(problem.inflow, np.float64).reshape(-1)
        initial = np.ascontiguousarray(problem.initial, np.float64).reshape(-1)
        h = C.c_void_p()
        _native.check(self._lib.bs_fit_create(
            C.byref(cfg.to_abi()), *[a.ctypes.data_as(dp) for a in arrays], C.byref(_prim(problem.free)),
            None if inflow is None else inflow.ctypes.data_as(dp), 1 if problem.first_node == "symmetry" else 0,
            initial.ctypes.data_as(dp), C.byref(h)), self._lib)
        self._h = h
        self._keep = (arrays, inflow, initial)
        self.rate = math.nan   # the drag's convergence rate per check, once settled (settle)

    def destroy(self) -> None:
        if self._h:
            self._lib.bs_fit_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def _call(self, name: str, *args) -> None:
        _native.check(getattr(self._lib, name)(self._h, *args), self._lib)

    def iterate(self, steps: int) -> None:
        self._call("bs_fit_iterate", int(steps))

    def check(self) -> tuple[float, float]:
        """(largest shock speed of the last move over a_inf, relative residual)."""
        s, r = C.c_double(), C.c_double()
        self._call("bs_fit_check", C.byref(s), C.byref(r))
        return s.value, r.value

    def solve(self, max_iterations: int, speed_tolerance: float = SPEED_TOLERANCE,
              residual_tolerance: float = RESIDUAL_TOLERANCE, check_every: int = 100):
        """fitShock's loop (shock-fitting.ts:248-311): (converged, iterations,
        max speed, relative residual)."""
        it, conv = C.c_int32(), C.c_int32()
        s, r = C.c_double(), C.c_double()
        self._call("bs_fit_solve", speed_tolerance, residual_tolerance, int(max_iterations), int(check_every),
                   C.byref(it), C.byref(conv), C.byref(s), C.byref(r))
        return bool(conv.value), it.value, s.value, r.value

    def grid(self) -> StructuredGrid:
        """The fitted grid as it stands: its nodes on the current heights."""
        p = self.problem
        x = np.empty((p.ni + 1) * (p.nj + 1))
        y = np.empty_like(x)
        self._call("bs_fit_nodes", x.ctypes.data_as(C.POINTER(C.c_double)), y.ctypes.data_as(C.POINTER(C.c_double)))
        return StructuredGrid(p.ni, p.nj, x, y)

    def heights(self) -> np.ndarray:
        out = np.empty(self.problem.ni + 1)
        self._call("bs_fit_heights", out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def primitives(self) -> np.ndarray:
        out = np.empty(4 * self.problem.ni * self.problem.nj)
        self._call("bs_fit_read_primitives", out.ctypes.data_as(C.POINTER(C.c_double)))
        return out.reshape(-1, 4)

    def wall_fluxes(self) -> list:
        """The jMin wall's faces (boundaryFluxes('jMin')), FP64 on the GPU."""
        out = (abi.FaceFlux * self.problem.ni)()
        self._call("bs_fit_wall_fluxes", out)
        return list(out)

    def drag(self) -> float:
        """The problem's drag: the wall's forebody drag and the tip's."""
        f = self.problem.free
        d = C.c_double()
        self._call("bs_fit_forebody_drag", f.p, 0.5 * f.rho * (f.u ** 2 + f.v ** 2), self.problem.base_radius,
                   C.byref(d))
        return d.value + self.problem.tip_drag


def settle(fit: CudaFit, max_iterations: int, noise: float = 1e-7, speed_tolerance: float = 1e-6,
           check_every: int = 250, known_rate: float = math.nan):
    """The GPU fit's stopping rule (fitShockGpu, src/engine-gpu/shock-fitting-gpu.ts:
    135-170): every `check_every` steps the drag is added to a SettlingValue of
    `noise`; the fit has converged once the drag has settled and the shock
    moves slower than `speed_tolerance` times a_inf. The reference's all-FP32
    GPU fit settles its shock speeds at 1e-6 to 4e-6 (tolerance 3e-5) and its
    drag with a noise of 2e-6; here the state is FP64 and the residual reads
    two-float metrics, so a fit goes on converging to the FP64 floor (shock
    speeds near 1e-11 a_inf, relative residuals 1e-13, the drag within 1e-11
    of the reference's FP64 engine): the default noise of 1e-7 stops it
    where the drag is settled far below the digits the verified band keeps;
    noise 1e-11 with speed_tolerance 1e-10 settles it to the CPU engine's
    own limits. `known_rate`: the drag's rate of convergence per check on the grid
    before, for a fit started from that grid's (it may begin too close to
    its limit to show its own). Leaves the rate to pass on in fit.rate.
    Returns (converged, iterations, max speed, drag)."""
    from .verification import SettlingValue

    settling = SettlingValue(noise, known_rate)
    done, speed, drag = 0, math.inf, math.nan
    try:
        while done < max_iterations:
            n = min(check_every, max_iterations - done)
            fit.iterate(n)
            done += n
            speed, _ = fit.check()
            drag = fit.drag()
            if not math.isfinite(drag):
                break
            if settling.add(drag) and speed < speed_tolerance:
                return True, done, speed, drag
        return False, done, speed, drag
    finally:
        fit.rate = settling.rate_to_pass_on


def started_from(fine: FitProblem, coarse: FitProblem, heights: np.ndarray, cells: np.ndarray) -> FitProblem | None:
    """startedFrom (src/analysis/gpu-fitted-flow.ts:116-146): the problem on
    the grid refined by 2, started from the settled fit on `coarse` (its
    shock heights and its cells (nj, ni, 4)): on nested grids each fine cell
    lies inside one coarse cell, whose state it takes, and the heights of the
    new lines are interpolated in x between their neighbours. None where the
    grids do not nest (a line or node fraction of the coarse grid missing
    from the fine one, within 1e-12). The settled state does not depend on
    the start; only the steps to reach it do."""
    n, nj = coarse.ni, coarse.nj
    if fine.ni != 2 * n or fine.nj != 2 * nj:
        return None
    scale = abs(coarse.line_x[n] - coarse.line_x[0])
    if not (np.all(np.abs(fine.line_x[::2] - coarse.line_x) <= 1e-12 * scale)
            and np.all(np.abs(fine.line_y[::2] - coarse.line_y) <= 1e-12 * scale)
            and np.all(np.abs(fine.fractions[::2, ::2] - coarse.fractions) <= 1e-12)):
        return None
    h = np.asarray(heights, np.float64)
    new = np.empty(fine.ni + 1)
    new[::2] = h
    ax, bx = coarse.line_x[:-1], coarse.line_x[1:]
    t = (fine.line_x[1::2] - ax) / (bx - ax)
    new[1::2] = h[:-1] * (1 - t) + h[1:] * t
    c = np.asarray(cells, np.float64).reshape(nj, n, 4)
    initial = np.repeat(np.repeat(c, 2, axis=0), 2, axis=1)
    return dataclasses.replace(fine, heights=new, initial=initial.reshape(-1, 4))


# ---- the blunt-nose fit problem -------------------------------------------------

CAPTURED_START_STEPS = 3000   # captured steps that start a blunt family (fitted-flow.ts:943)
MAX_BLUNT_EXTENSION = 7       # calibers of cylinder the blunt body may gain (:163)
FITTED_MAX_SIZE_RATIO = 1.3   # the fitted grids' size-ratio gate (src/grid/quality.ts:64-68)
SMOOTHING_PASSES = 20         # 1-2-1 passes over a captured shock (shock-fitting.ts:389)


def captured_shock_heights(prims: np.ndarray, x: np.ndarray, y: np.ndarray, lines: np.ndarray,
                           free: Primitive2D) -> np.ndarray:
    """capturedShockHeights (src/solver/shock-fitting.ts:360-386): on each
    line the outer face of the outermost cell whose pressure rose by more
    than 5 % of its column's peak rise, smoothed by 20 passes of 1-2-1
    (mirrored at the ends). prims (nj, ni, 4); x, y (nj + 1, ni + 1); lines
    (ni + 1, 4) as (x, y, dx, dy)."""
    nj, ni = prims.shape[:2]
    h = np.empty(ni + 1)
    for i in range(ni + 1):
        c = min(i, ni - 1)
        p = prims[:, c, 3]
        peak = max(free.p, float(p.max()))
        threshold = max(0.05 * (peak - free.p), 1e-4 * free.p)
        above = np.nonzero(p - free.p > threshold)[0]
        top = int(above[-1]) if len(above) else 0
        lx, ly, dx, dy = lines[i]
        h[i] = (x[top + 1, i] - lx) * dx + (y[top + 1, i] - ly) * dy
    for _ in range(SMOOTHING_PASSES):
        c = h.copy()
        h[0] = 0.5 * (c[0] + c[1])
        h[1:-1] = 0.25 * c[:-2] + 0.5 * c[1:-1] + 0.25 * c[2:]
        h[-1] = 0.5 * (c[-1] + c[-2])
    return h


@dataclass
class BluntStart:
    """What starts a blunt family (BluntStart, fitted-flow.ts:472-490): the
    body solved, the base grid, its lines (x, y, dx, dy), the captured shock's
    heights along them and the captured solution (nj, ni, 4); on a two-scale
    nose the outer boundary (n, 2) the family's grids share."""

    body: Body
    asked_end: float
    grid: StructuredGrid
    lines: np.ndarray
    heights: np.ndarray
    captured: np.ndarray
    nj: int
    mach: float
    gamma: float
    outer_boundary: np.ndarray | None = None


def _grid_lines(grid: StructuredGrid) -> np.ndarray:
    """The lines of a C grid from the body node to the outer one: (ni + 1, 4)."""
    X = grid.x.reshape(grid.nj + 1, grid.ni + 1)
    Y = grid.y.reshape(grid.nj + 1, grid.ni + 1)
    ex, ey = X[grid.nj] - X[0], Y[grid.nj] - Y[0]
    length = np.hypot(ex, ey)
    return np.stack([X[0], Y[0], ex / length, ey / length], 1)


BOUNDARY_MARGIN = 0.5       # a two-scale boundary's margin over the first captured shock (fitted-flow.ts:951)
BOUNDARY_CELLS = 3          # ... and at least this many base-grid cells above it (:953)
BOUNDARY_SMOOTHING = 50     # 1-2-1 passes over that boundary's distances (:955)


def outer_cell_height(h, nj: int, radius: float):
    """outerCellHeight (src/grid/blunt-grid.ts:571-573): the outermost cell's
    height on a line of height h with nj cells."""
    return h * (1 - stretched_fraction(line_strength(h, radius), nj - 1, nj))


def two_scale_boundary(lines: np.ndarray, heights: np.ndarray, nj: int, radius: float) -> np.ndarray:
    """The outer boundary of a two-scale nose's family (secondCapture,
    fitted-flow.ts:624-672) from the shock captured on the generator's grid:
    on each line the captured height pushed out by half of itself and by at
    least three outer cells of the base grid, smoothed by 50 passes of 1-2-1
    (mirrored at the ends), the last point continuing the segment before it
    to the last line where that rises. Returns (ni + 1, 2) points."""
    d = (1 + BOUNDARY_MARGIN) * heights
    for _ in range(20):
        d = np.maximum(d, heights + BOUNDARY_CELLS * outer_cell_height(d, nj, radius))
    for _ in range(BOUNDARY_SMOOTHING):
        c = d.copy()
        d[0] = 0.5 * (c[0] + c[1])
        d[1:-1] = 0.25 * c[:-2] + 0.5 * c[1:-1] + 0.25 * c[2:]
        d[-1] = 0.5 * (c[-1] + c[-2])
    pts = np.stack([lines[:, 0] + d * lines[:, 2], lines[:, 1] + d * lines[:, 3]], 1)
    n = len(pts) - 1
    if n >= 2:
        (ax, ay), (bx, by) = pts[n - 2], pts[n - 1]
        y = by + (lines[n, 0] - bx) * (by - ay) / (bx - ax)
        if y > by:
            pts[n] = (lines[n, 0], y)
    return pts


def _capture(body: Body, grid: StructuredGrid, mach: float, gamma: float) -> np.ndarray:
    """bluntCapture (fitted-flow.ts:572-603): 3,000 explicit steps from the
    free stream on a C grid (the axis and the body walls, outflow behind,
    the free stream on the outer boundary), here on the GPU engine; the
    solution (nj, ni, 4)."""
    from .engine import CudaEuler2D

    free = free_stream_at(mach, gamma).state
    cfg = steady_drag_config(grid, free, gamma, boundaries={
        "iMin": Boundary("wall"), "iMax": Boundary("outflow"), "jMin": Boundary("wall"),
        "jMax": Boundary("inflow", free)})
    with CudaEuler2D(cfg) as e:
        e.set_uniform(free)
        e.iterate(CAPTURED_START_STEPS)
        return e.primitives().reshape(grid.nj, grid.ni, 4)


def solved_blunt_body(asked: Body, mach: float, nj: int = 20):
    """solvedBluntBody (fitted-flow.ts:154-222): the body a blunt nose's fit
    solves and its start grid (ungated). The cylinder is at least a caliber
    and is lengthened a caliber at a time, by at most seven, until the C
    grid's neighbouring cells differ in size by no more than the fitted
    grids' gate allows (1.3); if none passes, the shortest. A two-scale nose
    keeps the shortest, its family being built on its captured shock.
    Returns (body, grid.BodyGrid)."""
    from .grid import blunt_body_grid, grid_quality

    caliber = 2 * asked.nose.base_radius
    shortest = max(asked.cylinder_length, SOLVED_CYLINDER * caliber)
    first = None
    for extra in range(MAX_BLUNT_EXTENSION + 1):
        body = Body(asked.nose, shortest + extra * caliber)
        bg = blunt_body_grid(body, nj, mach, gated=False)
        if bg.two_scale or grid_quality(bg.grid).max_size_ratio <= FITTED_MAX_SIZE_RATIO:
            return body, bg
        if first is None:
            first = (body, bg)
    return first


def blunt_start(asked: Body, mach: float, nj: int = 20, gamma: float = 1.4) -> BluntStart:
    """bluntStart (fitted-flow.ts:498-508): the body's cylinder lengthened a
    caliber at a time until its C grid meets the fitted grids' size-ratio
    gate (solvedBluntBody, :140-185; a two-scale nose keeps the shortest);
    3,000 captured explicit steps from the free stream on it (here on the GPU
    engine) and the captured shock's heights (capturedShockHeights). On a
    two-scale nose (Haack, power series: the generator's boundary is sized
    for the tip) a second capture on the grid built on the first captured
    shock (two_scale_boundary), whose boundary the family then shares."""
    from .grid import blunt_body_grid

    R = asked.nose.base_radius
    body, bg = solved_blunt_body(asked, mach, nj)
    free = free_stream_at(mach, gamma).state

    def heights_of(grid: StructuredGrid, captured: np.ndarray):
        lines = _grid_lines(grid)
        X = grid.x.reshape(nj + 1, grid.ni + 1)
        Y = grid.y.reshape(nj + 1, grid.ni + 1)
        return lines, captured_shock_heights(captured, X, Y, lines, free)

    grid = bg.grid
    captured = _capture(body, grid, mach, gamma)
    lines, heights = heights_of(grid, captured)
    boundary = None
    if bg.two_scale:
        boundary = two_scale_boundary(lines, heights, nj, R)
        grid = blunt_body_grid(body, nj, mach, gated=False, outer_boundary=boundary).grid
        captured = _capture(body, grid, mach, gamma)
        lines, heights = heights_of(grid, captured)
    return BluntStart(body, asked.nose.length + asked.cylinder_length, grid, lines, heights, captured, nj, mach,
                      gamma, boundary)


def nested_heights(base_lines: np.ndarray, base_heights: np.ndarray, fine_lines: np.ndarray,
                   refinement: int) -> np.ndarray:
    """nestedHeights (fitted-flow.ts:788-812): the base heights on every
    refinement-th line, linear in the line's index between them (weights
    m / refinement, exact in binary, so every grid of the family nests in
    the next); refused if the fine grid lacks a base line."""
    n = len(base_lines) - 1
    if len(fine_lines) - 1 != refinement * n:
        raise ValueError("the refined grid does not have the lines of its base grid")
    scale = math.hypot(base_lines[n, 0] - base_lines[0, 0], base_lines[n, 1] - base_lines[0, 1])
    for k in range(n + 1):
        a, b = base_lines[k], fine_lines[refinement * k]
        if not math.hypot(a[0] - b[0], a[1] - b[1]) <= 1e-12 * scale:
            raise ValueError("the refined grid does not have the lines of its base grid")
    out = []
    for k in range(n):
        for m in range(refinement):
            t = m / refinement
            out.append(base_heights[k] * (1 - t) + base_heights[k + 1] * t)
    out.append(base_heights[n])
    return np.array(out)


def blunt_fit_family(start: BluntStart):
    """bluntFitFamily (fitted-flow.ts:683-730): the problem at each
    refinement from one captured start: the refined grid's lines (which
    keep every base line), the heights nested between the base ones, each
    line's node fractions fixed at its height, and the start field at the
    same fraction of the shock layer (shockLayerStart, :735-768) on the
    base grid's column; the first shock node normal to the axis."""
    from .grid import blunt_body_grid

    R = start.body.nose.base_radius
    free = free_stream_at(start.mach, start.gamma).state
    X0 = start.grid.x.reshape(start.nj + 1, start.grid.ni + 1)
    Y0 = start.grid.y.reshape(start.nj + 1, start.grid.ni + 1)
    along = (X0 - start.lines[:, 0]) * start.lines[:, 2] + (Y0 - start.lines[:, 1]) * start.lines[:, 3]
    frac = along / start.heights[None, :]
    centre = 0.25 * (frac[:-1, :-1] + frac[:-1, 1:] + frac[1:, :-1] + frac[1:, 1:])   # (nj, ni) of the base
    nj0 = start.nj

    def problem(refinement: int = 1) -> FitProblem:
        if refinement == 1:
            lines = start.lines
        else:
            lines = _grid_lines(blunt_body_grid(start.body, nj0, start.mach, refinement=refinement, gated=False,
                                                outer_boundary=start.outer_boundary).grid)
        heights = nested_heights(start.lines, start.heights, lines, refinement)
        nj = nj0 * refinement
        ni = len(lines) - 1
        fractions = stretched_fraction(line_strength(heights, R)[:, None], np.arange(nj + 1)[None, :], nj)
        fa = fractions.T
        s = 0.25 * (fa[:-1, :-1] + fa[1:, :-1] + fa[:-1, 1:] + fa[1:, 1:])              # (nj, ni)
        initial = np.empty((nj, ni, 4))
        for i in range(ni):
            column = i // refinement
            c = centre[:, column]
            w = start.captured[:, column]
            for j in range(nj):
                jj = 0
                while jj < nj0 - 2 and c[jj + 1] < s[j, i]:
                    jj += 1
                t = min(max((s[j, i] - c[jj]) / (c[jj + 1] - c[jj]), 0.0), 1.0)
                initial[j, i] = w[jj] + t * (w[jj + 1] - w[jj])
        return FitProblem(lines[:, 0].copy(), lines[:, 1].copy(), lines[:, 2].copy(), lines[:, 3].copy(), fractions,
                          heights, nj, R, start.gamma, start.mach, free, None, initial.reshape(-1, 4), "symmetry", 0.0)

    return problem


def blunt_fit_problem(asked: Body, mach: float, nj: int = 20, gamma: float = 1.4,
                      refinement: int = 1) -> FitProblem:
    """bluntFitProblem (src/analysis/fitted-flow.ts:467-469): the family's
    problem at `refinement` from a fresh captured start."""
    return blunt_fit_family(blunt_start(asked, mach, nj, gamma))(refinement)


# ---- verified fitted drag -------------------------------------------------------

FITTED_BASE_NJ = 20            # base grid cells across (fitted-flow.ts:1003)
FALLBACK_COLUMN_DENSITY = 1.5  # a sharp family whose grid fails only the gates, solved again (:70)
FITTED_DRAG_FLOOR = 7e-5       # systematic error of the fitted drag, relative (src/analysis/verified-drag.ts:132)
FITTED_NOISE = 1e-7            # the verified fitted drag's settling noise by default, relative (settle)
FITTED_MIN_ANGLE = 12.0        # the fitted grids' quality gates (src/grid/quality.ts:24-38, 64-68), degrees
FITTED_MIN_WALL_ANGLE = 50.0
FITTED_MAX_ASPECT = 13.0
TWO_SCALE_DRAG_FLOOR = 8e-4    # a two-scale family's allowance, relative (src/analysis/verified-drag.ts:159)
# The Von Karman noses checked against a reference: length in calibers, Mach
# number (VON_KARMAN_REFERENCES, fitted-flow.ts:890-900).
VON_KARMAN_REFERENCES = ((1, 1.5), (1, 2), (1, 3), (3, 2), (3, 3), (5, 1.5), (5, 2), (5, 3), (6, 3))


def _number(x: float) -> str:
    """A number as the reference's messages print it (shortest form, no '.0')."""
    x = float(x)
    return str(int(x)) if x.is_integer() else repr(x)


def inside_outline(points, point, tolerance: float = 1e-9) -> bool:
    """insideOutline (fitted-flow.ts:903-940): whether `point` lies in the
    convex hull of `points` (a point, a segment or a polygon) or on it,
    within `tolerance` after scaling each coordinate by the points' extent in
    it. The hull by the monotone chain (A. M. Andrew, 1979), counterclockwise,
    dropping turns within the tolerance."""
    pts = [(float(a), float(b)) for a, b in points]
    sx = (max(p[0] for p in pts) - min(p[0] for p in pts)) or 1.0
    sy = (max(p[1] for p in pts) - min(p[1] for p in pts)) or 1.0
    scaled = sorted((a / sx, b / sy) for a, b in pts)
    q = (float(point[0]) / sx, float(point[1]) / sy)

    def cross(o, a, b):
        return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])

    def chain(seq):
        h: list = []
        for c in seq:
            while len(h) >= 2 and cross(h[-2], h[-1], c) <= tolerance:
                h.pop()
            h.append(c)
        return h[:-1]

    hull = chain(scaled) + chain(scaled[::-1])
    if len(hull) <= 2:
        a = hull[0] if hull else scaled[0]
        b = hull[1] if len(hull) > 1 else a
        dx, dy = b[0] - a[0], b[1] - a[1]
        n2 = dx * dx + dy * dy
        t = ((q[0] - a[0]) * dx + (q[1] - a[1]) * dy) / n2 if n2 > 0 else 0.0
        u = min(max(t, 0.0), 1.0)
        return math.hypot(q[0] - a[0] - u * dx, q[1] - a[1] - u * dy) <= tolerance
    return all(cross(hull[k], hull[(k + 1) % len(hull)], q) >= -tolerance for k in range(len(hull)))


def blunt_nose_refusal(body: Body, mach: float) -> str | None:
    """bluntNoseRefusal (fitted-flow.ts:863-876): why a nose the fitted
    solver could solve is not served, or None. Sharp tips and ellipsoids are
    served; of the noses with unbounded tip curvature only the Von Karman
    (LD-Haack, C = 0) nose, inside the outline of the lengths and Mach
    numbers checked against a reference."""
    shape = body.nose.shape
    if math.isfinite(_nose_slopes(body)[0]) or shape.kind == "ellipsoid":
        return None
    if not (shape.kind == "haack" and shape.parameter == 0):
        return ("of the blunt noses whose tip curvature is unbounded, only the Von Karman (LD-Haack) nose has "
                "been checked against a reference so far")
    calibers = body.nose.length / (2 * body.nose.base_radius)
    if inside_outline(VON_KARMAN_REFERENCES, (calibers, mach)):
        return None
    checked = ", ".join(f"{_number(c)} at Mach {_number(m)}" for c, m in VON_KARMAN_REFERENCES)
    unit = "caliber" if calibers == 1 else "calibers"
    return (f"a Von Karman nose of {_number(calibers)} {unit} at Mach {_number(mach)} lies outside the referenced "
            f"range (the outline of the noses checked against a reference, in calibers: {checked})")


def fitted_drag_floor(floor: float, start: BluntStart | None) -> float:
    """fittedDragFloor (fitted-flow.ts:964-966): the caller's allowance,
    raised to TWO_SCALE_DRAG_FLOOR for a two-scale start (one with its own
    outer boundary)."""
    if start is not None and start.outer_boundary is not None:
        return max(floor, TWO_SCALE_DRAG_FLOOR)
    return floor


class FitNotConverged(Exception):
    def __init__(self, refinement: int, reason: str):
        super().__init__(reason)
        self.refinement = refinement


class FitRefused(FitNotConverged):
    pass


class GridRefused(FitRefused):
    pass


def fitted_grid_failure(grid: StructuredGrid) -> str | None:
    """fittedGridFailure (fitted-flow.ts:293-306): the fitted grids' gates."""
    from .grid import grid_quality

    q = grid_quality(grid)
    f = []
    if not q.min_area > 0:
        f.append("a cell has non-positive area")
    if not q.min_angle >= FITTED_MIN_ANGLE * math.pi / 180:
        f.append(f"cell angle {math.degrees(q.min_angle):.1f} deg below {FITTED_MIN_ANGLE:.1f} deg")
    if not q.min_wall_angle >= FITTED_MIN_WALL_ANGLE * math.pi / 180:
        f.append(f"wall cell angle {math.degrees(q.min_wall_angle):.1f} deg below {FITTED_MIN_WALL_ANGLE:.1f} deg")
    if not q.max_size_ratio <= FITTED_MAX_SIZE_RATIO:
        f.append(f"neighbouring cells differ in size by {q.max_size_ratio:.2f} (limit {FITTED_MAX_SIZE_RATIO:g})")
    if not q.max_aspect_ratio <= FITTED_MAX_ASPECT:
        f.append(f"cell aspect ratio {q.max_aspect_ratio:.1f} above {FITTED_MAX_ASPECT:g}")
    if not f:
        return None
    return f"the grid on the fitted shock fails its quality checks ({'; '.join(f)}): a limit of the present grids"


def base_mach(problem: FitProblem, asked_end: float, prims: np.ndarray) -> float:
    """baseMach (fitted-flow.ts:262-291): the smallest axial Mach number
    across the layer at the end of the body asked for (infinite if the
    domain ends there). prims (nj, ni, 4)."""
    x = problem.line_x
    n = len(x) - 1
    tol = 1e-12 * abs(asked_end)
    if not x[n] > asked_end + tol:
        return math.inf
    g = problem.gamma
    axial = prims[:, :, 1] / np.sqrt(g * prims[:, :, 3] / prims[:, :, 0])     # (nj, ni)
    hit = np.nonzero(np.abs(x - asked_end) <= tol)[0]
    if len(hit) and hit[0] > 0:
        return float(axial[:, hit[0] - 1].min())
    centre = 0.5 * (x[:-1] + x[1:])
    a = 0
    while a + 2 < n and centre[a + 1] <= asked_end:
        a += 1
    t = min(max((asked_end - centre[a]) / (centre[a + 1] - centre[a]), 0.0), 1.0)
    return float(((1 - t) * axial[:, a] + t * axial[:, a + 1]).min())


def fitted_case_failure(problem: FitProblem, asked_end: float, grid: StructuredGrid, prims: np.ndarray) -> str | None:
    """fittedCaseFailure (fitted-flow.ts:308-330): the grid's gates, a
    supersonic outflow and a supersonic flow at the end of the body asked for."""
    e = fitted_grid_failure(grid)
    if e is not None:
        return e
    g = problem.gamma
    last = prims[:, -1]
    outflow = float((last[:, 1] / np.sqrt(g * last[:, 3] / last[:, 0])).min())
    if not outflow > 1:
        return f"the flow leaves the grid at an axial Mach number of {outflow:.3f}, where the outflow condition does not hold"
    base = base_mach(problem, asked_end, prims)
    if not base > 1:
        return f"the flow at the end of the body is subsonic (axial Mach number {base:.3f}), so what lies behind it could reach the body"
    return None


def verified_fitted_drag(body: Body, mach: float, gamma: float = 1.4, tolerance: float = 1e-4,
                         max_refinement: int = 8, floor: float = FITTED_DRAG_FLOOR,
                         iterations_per_refinement: int = 200000, on_level=None, on_fallback=None,
                         noise: float = FITTED_NOISE, speed_tolerance: float = 1e-6):
    """The verified fitted drag as the reference's GPU driver computes it
    (verifiedFittedDragGpu, src/analysis/gpu-fitted-flow.ts:197-338, the
    procedure of verifiedFittedDrag, fitted-flow.ts:1011-1080), for sharp
    noses and for blunt ones (one captured start for the family; two
    captures and a shared outer boundary on a two-scale nose): noses the
    reference does not serve refused (blunt_nose_refusal); grids refined by 2
    from 20 cells across until the drag's band (grid convergence index plus
    the allowance, `floor` raised to TWO_SCALE_DRAG_FLOOR on a two-scale
    family) is within `tolerance`, each finer grid started from the settled
    fit before it (started_from) with that fit's rate of convergence. A
    first grid whose fit does not settle stops the run without a value; on a
    finer grid (or one too large for the GPU) the band of the grids before it
    stands (result.stopped). A flow failing the checks is refused, but a
    sharp family whose grid fails only the quality gates is solved again with
    1.5 times as many columns. Each fit settles when its drag changes by less
    than `noise` (relative) and its shock by less than `speed_tolerance`
    a_inf; the same noise is the band's. Returns a
    verified_drag.VerifiedDrag."""
    from .verification import refine_until_verified
    from .verified_drag import LevelReport, VerifiedDrag

    asked_end = body.nose.length + body.cylinder_length
    reports: list = []
    refusal = blunt_nose_refusal(body, mach)
    if refusal is not None:
        return VerifiedDrag("invalid", None, reports, 1, refusal)
    blunt = None
    start = None
    if not math.isfinite(_nose_slopes(body)[0]):
        # Blunt: one captured start for the whole family (bluntFitFamily).
        try:
            start = blunt_start(body, mach, FITTED_BASE_NJ, gamma)
            blunt = blunt_fit_family(start)
        except ValueError as e:
            return VerifiedDrag("invalid", None, reports, 1, str(e))
    floor = fitted_drag_floor(floor, start)

    def family(density: float):
        # The last grid's problem, its settled fit and its rate, to start the next from.
        previous: list = []

        def solve_at(r: int) -> float:
            if blunt is not None:
                fresh = blunt(r)
            else:
                fresh = sharp_fit_problem(body, mach, nj=FITTED_BASE_NJ, refinement=r, gamma=gamma,
                                          column_density=density)
            p, rate = fresh, math.nan
            if previous:
                coarse, heights, cells, rate = previous[-1]
                p = started_from(fresh, coarse, heights, cells) or fresh
            with CudaFit(p) as g:
                converged, it, speed, drag = settle(g, iterations_per_refinement * r, noise=noise,
                                                    speed_tolerance=speed_tolerance, check_every=250 * r,
                                                    known_rate=rate)
                if not converged:
                    raise FitNotConverged(r, f"the fit stopped after {it} iterations with the shock moving at "
                                             f"{speed:.1e} of the sound speed or the drag still changing")
                grid = g.grid()
                prims = g.primitives().reshape(p.nj, p.ni, 4)
                settled = (p, g.heights(), prims, g.rate)
            e = fitted_grid_failure(grid)
            if e is not None:
                raise GridRefused(r, e)
            e = fitted_case_failure(p, asked_end, grid, prims)
            if e is not None:
                raise FitRefused(r, e)
            previous[:] = [settled]
            rep = LevelReport(r, p.ni, p.nj, it, drag)
            reports.append(rep)
            if on_level is not None:
                on_level(rep)
            return drag

        def stop_on(e: Exception) -> str | None:
            # A finer grid too large for the GPU, or whose fit does not
            # settle, leaves the band of the grids before it; a case refused
            # on any grid stays refused (verifiedFittedDragGpu's stopOn).
            if isinstance(e, FitRefused):
                return None
            if isinstance(e, FitNotConverged):
                return f"its fit did not converge ({e})"
            if isinstance(e, _native.BowshockError) and e.status == abi.BS_MEMORY_LIMIT:
                return str(e)
            return None

        return refine_until_verified(solve_at, tolerance, floor, max_refinement, 0.5, noise, stop_on)

    try:
        try:
            return VerifiedDrag("solved", family(1.0), reports, floor=floor)
        except GridRefused as e:
            if blunt is not None:
                raise
            if on_fallback is not None:
                on_fallback(e.refinement, str(e))
            reports.clear()
            return VerifiedDrag("solved", family(FALLBACK_COLUMN_DENSITY), reports,
                                column_density=FALLBACK_COLUMN_DENSITY, floor=floor)
    except FitRefused as e:
        return VerifiedDrag("invalid", None, reports, e.refinement, str(e))
    except FitNotConverged as e:
        return VerifiedDrag("not-converged", None, reports, e.refinement, str(e))
    except ValueError as e:
        return VerifiedDrag("invalid", None, reports, 1, str(e))


def settle_many(fits: list[CudaFit], max_iterations: int, noise: float = 1e-7, speed_tolerance: float = 1e-6,
                check_every: int = 250) -> list:
    """settle() for many fits at once, one host thread each: every fit has
    its own stream and its calls release the interpreter lock, so their
    small, launch-bound steps overlap on the GPU."""
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=max(1, len(fits))) as pool:
        return list(pool.map(lambda f: settle(f, max_iterations, noise, speed_tolerance, check_every), fits))
