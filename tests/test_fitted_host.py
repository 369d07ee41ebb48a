"""Host pieces of the fitted bow shock against the reference's own tests
(tests/solver/shock-fitting.test.ts:9-121): the Rankine-Hugoniot state
behind a fitted shock, the shock compatible with the flow behind it, and
the Taylor-Maccoll field on rays that starts a fit on a sharp nose."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

from bowshock_b200.config import Primitive2D
from bowshock_b200.fitted import column_positions, compatible_shock, cone_flow_field, shock_state
from bowshock_b200.grid import normal_shock, oblique_shock

GOLDEN_DIR = Path(__file__).parent / "golden"

GAMMA = 1.4
DEG = math.pi / 180


def free_at(mach: float) -> Primitive2D:
    return Primitive2D(1.0, mach * math.sqrt(GAMMA), 0.0, 1.0)


@pytest.mark.parametrize("mach", [1.2, 2, 3, 5])
def test_a_normal_shock_at_the_free_stream_mach_stands_still(mach):
    s = shock_state(free_at(mach), GAMMA, mach, -1.0, 0.0)
    exact = normal_shock(mach, GAMMA)
    assert abs(s.speed) < 1e-13
    assert abs(s.state.p - exact.pressure_ratio) < 1e-12
    assert abs(s.state.rho - exact.density_ratio) < 1e-12
    a2 = math.sqrt(GAMMA * s.state.p / s.state.rho)
    assert abs(math.hypot(s.state.u, s.state.v) / a2 - exact.downstream_mach) < 1e-12


@pytest.mark.parametrize("mach,theta", [(2, 10), (3, 20), (5, 8)])
def test_an_oblique_shock_at_the_wave_angle_turns_the_flow_by_the_wedge(mach, theta):
    exact = oblique_shock(mach, theta * DEG, GAMMA)
    b = exact.beta
    s = shock_state(free_at(mach), GAMMA, mach * math.sin(b), -math.sin(b), math.cos(b))
    assert abs(s.speed) < 1e-13
    assert abs(s.state.p - exact.pressure_ratio) < 1e-12
    assert abs(math.atan2(s.state.v, s.state.u) - theta * DEG) < 1e-12


def test_fluxes_are_continuous_across_the_shock_in_its_own_frame():
    rng = np.random.default_rng(71)
    for _ in range(300):
        mach_free, mach_rel, angle = rng.uniform(1.05, 6), rng.uniform(1, 4), rng.uniform(0, 2 * math.pi)
        free = free_at(mach_free)
        nx, ny = math.cos(angle), math.sin(angle)
        s = shock_state(free, GAMMA, mach_rel, nx, ny)

        def flux(w):
            un = w.u * nx + w.v * ny - s.speed
            ut = -w.u * ny + w.v * nx
            h = GAMMA / (GAMMA - 1) * w.p / w.rho + 0.5 * (un * un + ut * ut)
            return [w.rho * un, w.rho * un * un + w.p, w.rho * un * ut, w.rho * un * h]

        before, after = flux(free), flux(s.state)
        scale = [before[0], before[1], abs(before[0]) * 10 + 1, abs(before[3])]
        for k in range(4):
            assert abs(after[k] - before[k]) < 1e-12 * max(abs(scale[k]), 1)


def _behind(w, p=None):
    return dict(rho=w.rho, a=math.sqrt(GAMMA * w.p / w.rho), p=w.p if p is None else p, un=-w.u)


def test_the_exact_post_shock_state_behind_gives_a_standing_shock():
    free = free_at(3)
    w = shock_state(free, GAMMA, 3, -1, 0).state
    b = _behind(w)
    assert abs(compatible_shock(free, GAMMA, -1, 0, b["rho"], b["a"], b["p"], b["un"]).speed) < 1e-12


def test_higher_pressure_behind_moves_the_shock_out_and_lower_moves_it_in():
    free = free_at(3)
    w = shock_state(free, GAMMA, 3, -1, 0).state
    up = _behind(w, 1.05 * w.p)
    down = _behind(w, 0.95 * w.p)
    assert compatible_shock(free, GAMMA, -1, 0, up["rho"], up["a"], up["p"], up["un"]).speed > 0
    assert compatible_shock(free, GAMMA, -1, 0, down["rho"], down["a"], down["p"], down["un"]).speed < 0


def test_where_no_shock_fits_it_is_a_mach_wave():
    free = free_at(2)
    nx, ny = -math.sin(45 * DEG), math.cos(45 * DEG)
    s = compatible_shock(free, GAMMA, nx, ny, 1.0, math.sqrt(GAMMA), 1.0, free.u * nx + free.v * ny)
    assert abs(s.state.p - 1) < 1e-14 and abs(s.state.rho - 1) < 1e-14 and s.mach == 1.0


def test_cone_field_meets_the_shock_and_the_cone():
    cone = 20 * DEG
    speed, angle, flow = cone_flow_field(3.0, cone, GAMMA, [cone])
    # On the cone the flow runs along the surface at the surface Mach number.
    assert abs(angle[0] - cone) < 1e-10
    mach_surface = math.sqrt(2 / ((GAMMA - 1) * (1 / speed[0] ** 2 - 1)))
    assert abs(mach_surface - flow.surface_mach) < 1e-9
    # Just behind the shock the flow is turned by the oblique shock's deflection.
    beta = flow.shock_angle
    _, behind, _ = cone_flow_field(3.0, cone, GAMMA, [beta])
    tan_d = 2 / math.tan(beta) * (9 * math.sin(beta) ** 2 - 1) / (9 * (GAMMA + math.cos(2 * beta)) + 2)
    assert abs(behind[0] - math.atan(tan_d)) < 1e-10
    # Between them the flow angle falls monotonically from the deflection to the cone.
    rays = np.linspace(cone, beta, 50)
    _, angles, _ = cone_flow_field(3.0, cone, GAMMA, rays)
    assert np.all(np.diff(angles) < 0)


def test_column_positions_follow_the_density():
    xs = column_positions([0.0, 1.0, 3.0], lambda x: 10.0, 1)
    assert xs[0] == 0.0 and xs[-1] == 3.0 and 1.0 in xs
    assert len(xs) == 31 and np.allclose(np.diff(xs), 0.1)
    exact = column_positions([0.0, 2.0], lambda x: 1.0 + x, 1, total=12)
    assert len(exact) == 13


def test_sharp_fit_problem_lays_lines_under_the_tip_cone_shock():
    from bowshock_b200.fitted import sharp_fit_problem
    from bowshock_b200.workloads import cone_body

    p = sharp_fit_problem(cone_body(20, 4.0), 3.0, nj=10)
    assert p.nj == 10 and p.ni > 100 and p.first_node == "fixed"
    assert np.all(np.diff(p.line_x) > 0) and np.all(p.line_dx == 0) and np.all(p.line_dy == 1)
    assert np.allclose(p.fractions[:, 0], 0) and np.allclose(p.fractions[:, -1], 1)
    beta = cone_flow_field(3.0, 20 * DEG, GAMMA, [20 * DEG])[2].shock_angle
    on_nose = p.line_x < 0.5 / math.tan(20 * DEG)
    assert np.allclose((p.line_y + p.heights)[on_nose], p.line_x[on_nose] * math.tan(beta), rtol=1e-12)
    assert p.inflow.shape == (10, 4) and p.initial.shape == (p.ni * 10, 4)
    with pytest.raises(ValueError):
        sharp_fit_problem(cone_body(45, 4.0), 1.5, nj=10)


def test_oracle_face_states_keep_a_uniform_stream():
    from bowshock_b200.config import Boundary, grid_from_function, steady_drag_config
    from oracle.oracle import OracleEuler2D

    free = free_at(2.0)
    grid = grid_from_function(12, 8, lambda i, j: (0.1 * i, 0.05 + 0.1 * j + 0.01 * i))
    cfg = steady_drag_config(grid, free, boundaries={
        "iMin": Boundary("faceStates"), "iMax": Boundary("outflow"), "jMin": Boundary("outflow"),
        "jMax": Boundary("faceStates")})
    o = OracleEuler2D(cfg)
    o.set_uniform(free)
    w = np.array([free.rho, free.u, free.v, free.p])
    o.set_face_states("iMin", np.tile(w, (8, 1)))
    o.set_face_states("jMax", np.tile(w, (12, 1)))
    o.iterate(20)
    assert np.allclose(o.primitives().reshape(-1, 4), w, atol=1e-12)


def test_oracle_fit_moves_the_shock_towards_rest_and_the_conical_drag():
    # A few hundred fitted steps on the Mach 3, 20 deg cone (nj = 10): the
    # shock slows by orders of magnitude and the drag is already within a few
    # 1e-3 of Taylor-Maccoll (the reference measured +0.1017 % converged).
    from bowshock_b200.fitted import sharp_fit_problem
    from bowshock_b200.grid import taylor_maccoll
    from bowshock_b200.workloads import cone_body
    from oracle.shock_fitting import fit_shock

    p = sharp_fit_problem(cone_body(20, 4.0), 3.0, nj=10)
    f = fit_shock(p, 150)
    assert f.speeds[-1] < 0.02 * f.speeds[0]
    exact = taylor_maccoll(3.0, 20 * DEG, GAMMA).surface_pressure_coefficient
    assert abs(p.drag(f.engine.boundary_fluxes("jMin")) / exact - 1) < 3e-3


def _fit_create(p, cfg=None, **change):
    """bs_fit_create on a fit problem with some inputs changed; returns
    (status, message). Its argument checks run before any CUDA call."""
    import ctypes as C

    from bowshock_b200 import _native, abi

    cfg = cfg or p.config()
    L = _native.load()
    dp = C.POINTER(C.c_double)
    arrays = {k: np.ascontiguousarray(change.get(k, getattr(p, k)), np.float64).reshape(-1)
              for k in ("line_x", "line_y", "line_dx", "line_dy", "fractions", "heights")}
    inflow = change.get("inflow", p.inflow)
    inflow = None if inflow is None else np.ascontiguousarray(inflow, np.float64).reshape(-1)
    initial = np.ascontiguousarray(p.initial, np.float64).reshape(-1)
    h = C.c_void_p()
    st = L.bs_fit_create(C.byref(cfg.to_abi()), *[arrays[k].ctypes.data_as(dp) for k in
                                                  ("line_x", "line_y", "line_dx", "line_dy", "fractions", "heights")],
                         C.byref(abi.Primitive(p.free.rho, p.free.u, p.free.v, p.free.p)),
                         None if inflow is None else inflow.ctypes.data_as(dp), change.get("first_node", 0),
                         initial.ctypes.data_as(dp), C.byref(h))
    return st, L.bs_last_error().decode()


def test_fit_create_refuses_bad_problems_before_touching_the_gpu():
    from bowshock_b200 import abi
    from bowshock_b200.config import Boundary
    from bowshock_b200.fitted import sharp_fit_problem
    from bowshock_b200.workloads import cone_body

    p = sharp_fit_problem(cone_body(20, 4.0), 3.0, nj=10)
    cfg = p.config()
    cfg.boundaries["jMax"] = Boundary("outflow")
    st, msg = _fit_create(p, cfg)
    assert st == abi.BS_INVALID_ARGUMENT and "jMax" in msg
    cfg = p.config()
    cfg.boundaries["iMin"] = Boundary("outflow")
    st, msg = _fit_create(p, cfg)
    assert st == abi.BS_INVALID_ARGUMENT and "iMin" in msg
    st, msg = _fit_create(p, inflow=None)
    assert st == abi.BS_INVALID_ARGUMENT and "inflow" in msg
    st, msg = _fit_create(p, line_dx=p.line_dx + 0.1)
    assert st == abi.BS_INVALID_ARGUMENT and "unit" in msg
    st, msg = _fit_create(p, heights=np.where(np.arange(len(p.heights)) == 3, -1.0, p.heights))
    assert st == abi.BS_INVALID_ARGUMENT and "heights" in msg
    st, msg = _fit_create(p, fractions=p.fractions * 2)
    assert st == abi.BS_INVALID_ARGUMENT and "fractions" in msg
    st, msg = _fit_create(p, first_node=2)
    assert st == abi.BS_INVALID_ARGUMENT and "first_node" in msg
    import dataclasses

    cfg = dataclasses.replace(p.config(), time_integrator="forwardEuler")
    st, msg = _fit_create(p, cfg)
    assert st == abi.BS_INVALID_ARGUMENT and "SSP-RK" in msg


def test_blunt_grid_families_nest():
    # tests/analysis/fitted-flow.test.ts:76-114: the refined C grid keeps
    # every line of the base grid; nested heights keep the base heights on
    # them, and the node fractions fixed at those heights nest too.
    from bowshock_b200.fitted import _grid_lines, line_strength, nested_heights, stretched_fraction
    from bowshock_b200.grid import Body, Nose, NoseShape, blunt_body_grid

    body = Body(Nose(NoseShape("ellipsoid"), 1.5, 0.5), 2.0)
    coarse = _grid_lines(blunt_body_grid(body, 20, 2.0, gated=False).grid)
    rng = np.random.default_rng(3)
    h1 = 0.3 + 0.1 * rng.random(len(coarse))
    for r in (2, 4):
        fine = _grid_lines(blunt_body_grid(body, 20, 2.0, refinement=r, gated=False).grid)
        assert len(fine) - 1 == r * (len(coarse) - 1)
        assert np.max(np.hypot(*(fine[::r, :2] - coarse[:, :2]).T)) < 1e-13
        h = nested_heights(coarse, h1, fine, r)
        assert np.array_equal(h[::r], h1)
        f1 = stretched_fraction(line_strength(h1, 0.5)[:, None], np.arange(21)[None, :], 20)
        fr = stretched_fraction(line_strength(h, 0.5)[:, None], np.arange(20 * r + 1)[None, :], 20 * r)
        assert np.max(np.abs(fr[::r, ::r] - f1)) < 1e-14
    with pytest.raises(ValueError):
        nested_heights(coarse, h1, coarse[:-1], 1)


# ---- two-scale noses (no GPU: grids, outline, allowance) ---------------------------

def test_two_scale_family_nests_on_its_outer_boundary():
    # tests/analysis/fitted-flow.test.ts:179-225: a 3-caliber Haack nose at
    # Mach 2 is two-scale and keeps its cylinder; every grid of a family on
    # an outer boundary (here 0.4 of the generator's lines, heights 0.6 of
    # the base grid's, made up) keeps the base lines, heights and node
    # fractions at refinements 2, 4 and 8.
    from bowshock_b200.config import free_stream_at
    from bowshock_b200.fitted import BluntStart, _grid_lines, blunt_fit_family, started_from
    from bowshock_b200.grid import Body, Nose, NoseShape, blunt_body_grid

    body = Body(Nose(NoseShape("haack", 0.0), 3.0, 0.5), 2.0)
    first = blunt_body_grid(body, 20, 2.0, gated=False)
    assert first.two_scale
    X = first.grid.x.reshape(21, -1)
    Y = first.grid.y.reshape(21, -1)
    lines = _grid_lines(first.grid)
    h = np.hypot(X[20] - X[0], Y[20] - Y[0])
    boundary = np.stack([lines[:, 0] + 0.4 * h * lines[:, 2], lines[:, 1] + 0.4 * h * lines[:, 3]], 1)
    base = blunt_body_grid(body, 20, 2.0, gated=False, outer_boundary=boundary).grid
    bl = _grid_lines(base)
    Xb = base.x.reshape(21, -1)
    Yb = base.y.reshape(21, -1)
    free = free_stream_at(2.0, 1.4).state
    captured = np.tile([free.rho, free.u, free.v, free.p], (20, base.ni, 1))
    start = BluntStart(body, 5.0, base, bl, 0.6 * np.hypot(Xb[20] - Xb[0], Yb[20] - Yb[0]), captured, 20, 2.0,
                       1.4, boundary)
    family = blunt_fit_family(start)
    coarse = family(1)
    assert coarse.ni == base.ni
    for r in (2, 4, 8):
        fine = family(r)
        assert fine.ni == 2 * coarse.ni and fine.nj == 2 * coarse.nj
        assert np.array_equal(fine.line_x[::2], coarse.line_x) and np.array_equal(fine.line_y[::2], coarse.line_y)
        assert np.array_equal(fine.heights[::2], coarse.heights)
        assert np.array_equal(fine.fractions[::2, ::2], coarse.fractions)
        # startedFrom (src/analysis/gpu-fitted-flow.ts:116-146) takes the
        # nested grid: the coarse heights on the shared lines, each fine cell
        # the coarse cell it lies in.
        cells = np.arange(coarse.nj * coarse.ni * 4, dtype=np.float64).reshape(coarse.nj, coarse.ni, 4)
        moved = 1.01 * coarse.heights
        s = started_from(fine, coarse, moved, cells)
        assert s is not None and np.array_equal(s.heights[::2], moved)
        assert np.all((s.heights[1::2] - moved[:-1]) * (s.heights[1::2] - moved[1:]) <= 0)
        w = s.initial.reshape(fine.nj, fine.ni, 4)
        assert np.array_equal(w[1::2, 1::2], cells) and np.array_equal(w[::2, 1::2], cells)
        coarse = fine
    assert started_from(family(4), family(1), family(1).heights, cells[:20, :base.ni]) is None


def test_outer_boundary_refusals_and_the_sphere_is_one_scale():
    from bowshock_b200._native import BowshockError
    from bowshock_b200.grid import Body, Nose, NoseShape, blunt_body_grid

    sphere = Body(Nose(NoseShape("ellipsoid"), 0.5, 0.5), 1.0)
    assert not blunt_body_grid(sphere, 20, 2.0, gated=False).two_scale
    for bad in ([[-1.0, 0.0]], [[-1.0, 0.1], [0.0, 2.0]], [[-1.0, 0.0], [0.0, 2.0], [1.0, 1.0]]):
        with pytest.raises(BowshockError, match="outer boundary"):
            blunt_body_grid(sphere, 20, 2.0, gated=False, outer_boundary=bad)


def test_von_karman_outline_and_allowance():
    # tests/analysis/fitted-flow.test.ts:227-297: ellipsoids and sharp tips
    # served; Von Karman noses inside the outline of the lengths and Mach
    # numbers checked; other two-scale noses refused; the allowance raised
    # on a two-scale start only.
    from bowshock_b200.fitted import (FITTED_DRAG_FLOOR, TWO_SCALE_DRAG_FLOOR, VON_KARMAN_REFERENCES, BluntStart,
                                      blunt_nose_refusal, fitted_drag_floor, inside_outline)
    from bowshock_b200.grid import Body, Nose, NoseShape

    known = json.loads((GOLDEN_DIR / "reference_known_answers.json").read_text())
    assert TWO_SCALE_DRAG_FLOOR == known["two_scale_drag_floor"]["value"]

    def nose(shape, calibers):
        return Body(Nose(shape, calibers, 0.5), 1.0)

    vk = NoseShape("haack", 0.0)
    assert blunt_nose_refusal(nose(NoseShape("ellipsoid"), 6), 1.2) is None
    for c, m in VON_KARMAN_REFERENCES:
        assert blunt_nose_refusal(nose(vk, c), m) is None
    assert "outside the referenced range" in blunt_nose_refusal(nose(vk, 8), 1.2)
    for c, m in ((5, 3), (6, 3), (4.1, 2.5), (5.6, 2.5), (5.3, 2)):
        assert blunt_nose_refusal(nose(vk, c), m) is None, (c, m)
    for c, m in ((5.7, 2.5), (5.4, 2), (6, 2), (6, 1.5), (5.1, 1.5), (6.1, 3)):
        assert "outside the referenced range" in blunt_nose_refusal(nose(vk, c), m), (c, m)
    assert "only the Von Karman" in blunt_nose_refusal(nose(NoseShape("haack", 1 / 3), 3), 2)
    assert "only the Von Karman" in blunt_nose_refusal(nose(NoseShape("power", 0.75), 3), 2)
    assert blunt_nose_refusal(nose(NoseShape("ogive", 1.0), 1), 1.2) is None
    assert inside_outline([[3, 2]], [3, 2]) and not inside_outline([[3, 2]], [3, 2.1])
    assert inside_outline([[1, 2], [3, 2]], [2, 2]) and not inside_outline([[1, 2], [3, 2]], [2, 2.01])
    quad = [[1, 2], [3, 2], [3, 3], [5, 1.5]]
    assert all(inside_outline(quad, p) for p in ([3, 2], [4, 2], [5, 1.5]))
    assert not inside_outline(quad, [5, 2]) and not inside_outline(quad, [1, 1.5])
    assert not inside_outline(VON_KARMAN_REFERENCES, [6, 1.5]) and not inside_outline(VON_KARMAN_REFERENCES, [6, 2])

    def start(boundary):
        return BluntStart(None, 0.0, None, None, None, None, 20, 2.0, 1.4, boundary)

    assert fitted_drag_floor(FITTED_DRAG_FLOOR, None) == FITTED_DRAG_FLOOR
    assert fitted_drag_floor(FITTED_DRAG_FLOOR, start(None)) == FITTED_DRAG_FLOOR
    assert fitted_drag_floor(FITTED_DRAG_FLOOR, start(np.array([[-1.0, 0.0]]))) == TWO_SCALE_DRAG_FLOOR


# ---- the fitted problems' refusals and bodies (tests/analysis/fitted-flow.test.ts:115-178, 361-488) --------

def _ogive_body(length: float, cylinder: float, parameter: float = 1.0):
    from bowshock_b200.grid import Body, Nose, NoseShape

    return Body(Nose(NoseShape("ogive", parameter), length, 0.5), cylinder)


def _cone(angle_deg: float, cylinder: float):
    from bowshock_b200.grid import Body, Nose, NoseShape

    return Body(Nose(NoseShape("conical"), 0.5 / math.tan(angle_deg * DEG), 0.5), cylinder)


def test_sharp_tips_refused_with_their_angle_and_what_to_change():
    from bowshock_b200.fitted import sharp_fit_problem

    with pytest.raises(ValueError, match=r"at Mach 1.2 the bow shock cannot stay attached to a tip of 45.0 deg "
                                         r"half-angle; this needs a sharper or longer nose"):
        sharp_fit_problem(_cone(45, 2.0), 1.2, nj=20)
    ogive = _ogive_body(3.0, 2.0)
    with pytest.raises(ValueError, match=r"at Mach 1.2 the flow over a tip of 18.9 deg half-angle is subsonic at "
                                         r"the surface \(Mach 0.85\)"):
        sharp_fit_problem(ogive, 1.2, nj=20)
    sharp_fit_problem(ogive, 1.5, nj=20)
    for r in (1, 8):
        sharp_fit_problem(ogive, 1.35, nj=20, refinement=r)
    short = _ogive_body(2.0, 2.0)
    sharp_fit_problem(short, 1.6, nj=20)
    with pytest.raises(ValueError, match=r"is subsonic at the surface \(Mach 0.99\)"):
        sharp_fit_problem(short, 1.59, nj=20)
    for r in (1, 8):
        with pytest.raises(ValueError, match=r"crosses the solver's starting plane, normal to the axis, at an axial "
                                             r"Mach number of 0.95 at the surface, below 1, which this solver "
                                             r"handles only where the nose meets the body without a corner"):
            sharp_fit_problem(_cone(24, 2.0), 1.5, nj=20, refinement=r)


def test_a_36_deg_tip_passes_the_fitted_gates_but_not_the_generated_ones():
    # The secant ogive (0.5) of 1 caliber at Mach 3: wall cells near 53 deg,
    # below the generated grids' 60 deg, above the fitted grids' 50.
    from bowshock_b200.fitted import fitted_grid_failure, sharp_fit_problem
    from bowshock_b200.grid import grid_quality

    p = sharp_fit_problem(_ogive_body(1.0, 2.0, 0.5), 3.0, nj=20)
    g = p.grid()
    q = grid_quality(g)
    assert 50 * DEG < q.min_wall_angle < 60 * DEG
    assert fitted_grid_failure(g) is None


def test_base_flow_is_tested_at_the_end_of_the_body_asked_for():
    # A cylinder shorter than the caliber always solved ends inside a column:
    # the axial Mach number there, interpolated between the columns; a bare
    # nose ends on a grid line, the column just ahead of it tested.
    from bowshock_b200.fitted import base_mach, sharp_fit_problem

    g = 1.4
    cone = _cone(20, 0.3)
    p = sharp_fit_problem(cone, 3.0, nj=20)
    end = cone.nose.length + 0.3
    assert not np.any(np.abs(p.line_x - end) < 1e-9)

    def mach(x):
        return 0.5 + 0.2 * x

    def flow(problem):
        xc = 0.5 * (problem.line_x[:-1] + problem.line_x[1:])
        w = np.zeros((problem.nj, problem.ni, 4))
        w[..., 0] = 1
        w[..., 1] = math.sqrt(g) * mach(xc)[None, :]
        w[..., 3] = 1
        return w

    assert abs(base_mach(p, end, flow(p)) - mach(end)) < 1e-12
    bare = _cone(20, 0.0)
    p0 = sharp_fit_problem(bare, 3.0, nj=20)
    corner = int(np.nonzero(p0.line_x == bare.nose.length)[0][0])
    assert corner > 0
    ahead = mach(0.5 * (p0.line_x[corner - 1] + p0.line_x[corner]))
    assert abs(base_mach(p0, bare.nose.length, flow(p0)) - ahead) < 1e-12


def test_a_blunt_nose_cylinder_is_lengthened_until_its_start_grid_meets_the_size_ratio_gate():
    # The 1.5-caliber ellipsoid at Mach 1.2 on one caliber of cylinder: its
    # start grid passes on three; the 3:1 ellipsoid with two calibers at
    # Mach 2 keeps its cylinder; a bare nose gets the caliber always solved.
    from bowshock_b200.fitted import FITTED_MAX_SIZE_RATIO, solved_blunt_body
    from bowshock_b200.grid import Body, Nose, NoseShape, grid_quality

    asked = Body(Nose(NoseShape("ellipsoid"), 1.5, 0.5), 1.0)
    body, bg = solved_blunt_body(asked, 1.2, 20)
    assert body.cylinder_length == 3.0 and body.nose == asked.nose
    assert grid_quality(bg.grid).max_size_ratio <= FITTED_MAX_SIZE_RATIO
    e3 = Body(Nose(NoseShape("ellipsoid"), 3.0, 0.5), 2.0)
    assert solved_blunt_body(e3, 2.0, 20)[0].cylinder_length == 2.0
    assert solved_blunt_body(Body(e3.nose, 0.0), 3.0, 20)[0].cylinder_length == 1.0


def test_a_lengthened_blunt_family_nests_at_mach_1_2():
    # What started_from and nested_heights need, on a family whose cylinder
    # is lengthened; the start's heights are made up (0.4 of each line).
    from bowshock_b200.config import free_stream_at
    from bowshock_b200.fitted import BluntStart, _grid_lines, blunt_fit_family, solved_blunt_body, started_from
    from bowshock_b200.grid import Body, Nose, NoseShape

    asked = Body(Nose(NoseShape("ellipsoid"), 1.5, 0.5), 1.0)
    body, bg = solved_blunt_body(asked, 1.2, 20)
    lines = _grid_lines(bg.grid)
    X = bg.grid.x.reshape(21, -1)
    Y = bg.grid.y.reshape(21, -1)
    free = free_stream_at(1.2, 1.4).state
    captured = np.tile([free.rho, free.u, free.v, free.p], (20, bg.grid.ni, 1))
    start = BluntStart(body, 2.5, bg.grid, lines, 0.4 * np.hypot(X[20] - X[0], Y[20] - Y[0]), captured, 20, 1.2, 1.4)
    family = blunt_fit_family(start)
    coarse = family(1)
    assert coarse.line_x[-1] == body.nose.length + body.cylinder_length
    for r in (2, 4, 8):
        fine = family(r)
        assert fine.ni == 2 * coarse.ni and fine.nj == 2 * coarse.nj
        assert np.array_equal(fine.line_x[::2], coarse.line_x) and np.array_equal(fine.line_y[::2], coarse.line_y)
        assert np.array_equal(fine.heights[::2], coarse.heights)
        assert np.array_equal(fine.fractions[::2, ::2], coarse.fractions)
        assert started_from(fine, coarse, coarse.heights, coarse.initial) is not None
        coarse = fine


def test_two_scale_boundary_keeps_its_margin_and_continues_the_last_segment():
    # secondCapture's boundary (fitted-flow.ts:624-672) on made-up lines: at
    # least 1.5 times the captured height and three outer cells above it
    # before smoothing, smoothed by 50 passes of 1-2-1, its first point on the
    # axis, and the last point continuing the segment before it where that
    # rises.
    from bowshock_b200.fitted import (BOUNDARY_CELLS, BOUNDARY_MARGIN, BOUNDARY_SMOOTHING, outer_cell_height,
                                      two_scale_boundary)

    n = 40
    s = np.linspace(0, 1, n + 1)
    angle = 0.5 * math.pi * np.minimum(s / 0.5, 1.0)
    lines = np.stack([2.0 * s, 0.5 * np.sin(angle), -np.cos(angle), np.sin(angle)], 1)
    lines[0, 1] = 0.0
    heights = 0.2 + 0.3 * s
    pts = two_scale_boundary(lines, heights, 20, 0.5)
    assert pts.shape == (n + 1, 2) and pts[0, 1] == 0.0
    d = (1 + BOUNDARY_MARGIN) * heights
    for _ in range(20):
        d = np.maximum(d, heights + BOUNDARY_CELLS * outer_cell_height(d, 20, 0.5))
    assert np.all(d >= 1.5 * heights)
    for _ in range(BOUNDARY_SMOOTHING):
        c = d.copy()
        d[0], d[-1] = 0.5 * (c[0] + c[1]), 0.5 * (c[-1] + c[-2])
        d[1:-1] = 0.25 * c[:-2] + 0.5 * c[1:-1] + 0.25 * c[2:]
    expected = lines[:, :2] + d[:, None] * lines[:, 2:]
    assert np.array_equal(pts[:-1], expected[:-1])
    (ax, ay), (bx, by) = expected[-3], expected[-2]
    y = by + (lines[-1, 0] - bx) * (by - ay) / (bx - ax)
    assert (pts[-1] == (lines[-1, 0], y)).all() if y > by else np.array_equal(pts[-1], expected[-1])
    assert np.all(np.diff(pts[:, 1]) > 0)
