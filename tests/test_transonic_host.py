"""The transonic grid and driver without a GPU: the H grid of a sharp nose and
its cylinder (src/grid/transonic-grid.ts), its nesting and refusals, and the
oracle's restatement of solveTransonic on it reproducing the drag the
reference measured on the 7 deg cone of NACA TN 4233 at Mach 1.2
(tests/analysis/transonic-flow.test.ts:14-39)."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

from bowshock_b200.grid import Body, Nose, NoseShape, taylor_maccoll, transonic_grid
from bowshock_b200.transonic import geometric_remaining, transonic_problem

TN = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())[
    "transonic_cone_tn4233_mach1_2"]
HALF = TN["cone_half_angle_deg"] * math.pi / 180


def _cone() -> Body:
    R = TN["base_radius"]
    return Body(Nose(NoseShape("conical"), R / math.tan(HALF), R), 0.0)


def test_transonic_grid_reaches_the_far_field_in_geometric_cells_and_nests():
    body = _cone()
    L = body.nose.length
    t1 = transonic_grid(body, 1, TN["far_field"], TN["cylinder"])
    g = t1.grid
    # 30 cells across reach 100 radii from a wall cell of 0.05 growing by e^0.2.
    assert t1.base_nj == 30 == g.nj
    assert t1.far_radius == pytest.approx(0.05 / 0.2 * math.expm1(0.2 * 30), rel=1e-15)
    assert t1.x_upstream == -t1.far_radius and t1.x_end == pytest.approx(L + 2 * TN["cylinder"], rel=1e-15)
    X = g.x.reshape(g.nj + 1, g.ni + 1)
    Y = g.y.reshape(g.nj + 1, g.ni + 1)
    assert X[0, t1.i_tip] == 0.0 and X[0, t1.i_shoulder] == L
    assert np.all(np.diff(X[0]) > 0) and np.all(Y[0, : t1.i_tip + 1] == 0)
    assert np.allclose(Y[-1], t1.far_radius, rtol=0, atol=1e-12 * t1.far_radius)
    # Spacing near 0.05 radii at the tip and 0.02 at the shoulder (each
    # interval's column count rounded to whole cells).
    assert X[0, t1.i_tip + 1] - X[0, t1.i_tip] == pytest.approx(0.05, rel=0.1)
    assert X[0, t1.i_shoulder] - X[0, t1.i_shoulder - 1] == pytest.approx(0.02, rel=0.1)
    for r in (2, 4):
        tr = transonic_grid(body, r, TN["far_field"], TN["cylinder"])
        Xr = tr.grid.x.reshape(tr.grid.nj + 1, tr.grid.ni + 1)
        Yr = tr.grid.y.reshape(tr.grid.nj + 1, tr.grid.ni + 1)
        assert tr.grid.ni == r * g.ni and tr.grid.nj == r * g.nj
        assert np.array_equal(Xr[::r, ::r], X) and np.array_equal(Yr[::r, ::r], Y)
        assert tr.i_tip == r * t1.i_tip and tr.i_shoulder == r * t1.i_shoulder


def test_transonic_grid_refusals():
    from bowshock_b200._native import BowshockError

    body = _cone()
    with pytest.raises(BowshockError, match="needs a cylinder"):
        transonic_grid(body, 1, 100, 0.0)
    with pytest.raises(BowshockError, match="beyond four nose lengths"):
        transonic_grid(body, 1, 20, 10)
    with pytest.raises(BowshockError, match="refinement"):
        transonic_grid(body, 3, 100, 10)
    with pytest.raises(ValueError, match="positive"):
        transonic_grid(body, 1, 100, 10, spacing={"wall": -1})
    # tests/grid/transonic-grid.test.ts:239-251: a blunt nose meeting the
    # cylinder at an angle; nested domains on a blunt nose (:150-176).
    corner = Body(Nose(NoseShape("power", 0.5), 2.0, 1.0), 0.0)
    with pytest.raises(BowshockError, match="tangentially"):
        transonic_grid(corner, 1, 100, 10)
    with pytest.raises(BowshockError, match="blunt"):
        transonic_grid(Body(Nose(NoseShape("ellipsoid"), 2.0, 1.0), 0.0), 1, 100, 10, nested={"far_field": 200})


# ---- tests/grid/transonic-grid.test.ts ---------------------------------------------

DEG = math.pi / 180
CONE7 = Body(Nose(NoseShape("conical"), 1 / math.tan(7 * DEG), 1.0), 0.0)
OGIVE6 = Body(Nose(NoseShape("ogive", 1.0), 6.0, 1.0), 0.0)


def _nodes(tg):
    g = tg.grid
    return g.x.reshape(g.nj + 1, g.ni + 1), g.y.reshape(g.nj + 1, g.ni + 1)


def _radius(body, x):
    from bowshock_b200.fitted import _body_radius

    return _body_radius(body, np.asarray(x, np.float64))


@pytest.mark.parametrize("body", [CONE7, OGIVE6], ids=["cone", "ogive"])
def test_sharp_grids_reach_the_far_boundaries_with_tip_and_shoulder_on_lines(body):
    from bowshock_b200.grid import grid_quality

    tg = transonic_grid(body, 1, 100, 10)
    X, Y = _nodes(tg)
    assert 100 <= tg.far_radius < 125 and tg.x_upstream == -tg.far_radius and tg.topology == "H"
    assert tg.x_end == pytest.approx(body.nose.length + 20, abs=1e-12)
    assert X[0, tg.i_tip] == 0 and X[0, tg.i_shoulder] == body.nose.length
    assert np.allclose(Y[0], _radius(body, X[0]), rtol=0, atol=1e-12)
    assert np.allclose(Y[-1], tg.far_radius, rtol=0, atol=1e-9)
    q = grid_quality(tg.grid)
    assert q.min_area > 0
    assert q.min_wall_angle > 60 * DEG and q.min_angle > 30 * DEG and q.max_size_ratio < 1.4


def test_sharp_grids_keep_the_near_body_rows_when_the_far_boundaries_move():
    near, far = transonic_grid(CONE7, 1, 50, 10), transonic_grid(CONE7, 1, 400, 10)
    assert far.grid.nj > near.grid.nj
    Yn, Yf = _nodes(near)[1], _nodes(far)[1]
    for j in range(1, 6):
        assert abs(Yf[j, far.i_shoulder] / Yn[j, near.i_shoulder] - 1) < 0.05


@pytest.mark.parametrize("nested", [{"far_field": 50}, {"far_field": 200}, {"cylinder": 5}, {"cylinder": 20}],
                         ids=["far-50", "far-200", "cylinder-5", "cylinder-20"])
def test_nested_domains_share_every_node_and_nest_under_refinement(nested):
    from bowshock_b200.grid import grid_quality

    for r in (1, 2):
        plain = transonic_grid(CONE7, r, 100, 10)
        g = transonic_grid(CONE7, r, 100, 10, nested=nested)
        far = nested.get("far_field", 100)
        assert g.far_radius >= far and -g.x_upstream >= far
        assert g.x_end >= CONE7.nose.length + 2 * nested.get("cylinder", 10)
        assert g.grid.nj % r == 0 and g.i_tip % r == 0
        Xg, Yg = _nodes(g)
        Xp, Yp = _nodes(plain)
        assert Xg[0, g.i_tip] == 0
        off = plain.i_tip - g.i_tip
        nj = min(plain.grid.nj, g.grid.nj)
        lo, hi = max(0, -off), min(g.grid.ni, plain.grid.ni - off)
        assert np.array_equal(Xg[: nj + 1, lo: hi + 1], Xp[: nj + 1, lo + off: hi + off + 1])
        assert np.array_equal(Yg[: nj + 1, lo: hi + 1], Yp[: nj + 1, lo + off: hi + off + 1])
        assert hi - lo + 1 == min(plain.grid.ni, g.grid.ni) + 1
        q = grid_quality(g.grid)
        assert q.min_area > 0 and q.min_wall_angle > 60 * DEG and q.min_angle > 30 * DEG
    c = transonic_grid(CONE7, 1, 100, 10, nested=nested)
    f = transonic_grid(CONE7, 2, 100, 10, nested=nested)
    assert f.grid.ni == 2 * c.grid.ni and f.grid.nj == 2 * c.grid.nj
    Xc, Yc = _nodes(c)
    Xf, Yf = _nodes(f)
    assert max(np.abs(Xf[::2, ::2] - Xc).max(), np.abs(Yf[::2, ::2] - Yc).max()) < 1e-9


def test_a_nested_domain_equal_to_the_grids_own_is_the_grid():
    plain = transonic_grid(CONE7, 1, 100, 10)
    same = transonic_grid(CONE7, 1, 100, 10, nested={"far_field": 100, "cylinder": 10})
    assert np.array_equal(same.grid.x, plain.grid.x) and np.array_equal(same.grid.y, plain.grid.y)
    assert same.far_radius == plain.far_radius


@pytest.mark.parametrize("length", [1.0, 2.0, 3.0])
def test_blunt_noses_get_a_c_grid_from_the_axis_ahead_to_the_end_of_the_cylinder(length):
    from bowshock_b200.grid import grid_quality

    body = Body(Nose(NoseShape("ellipsoid"), length, 1.0), 0.0)
    tg = transonic_grid(body, 1, 100, 10)
    X, Y = _nodes(tg)
    assert tg.topology == "C" and tg.i_tip == 0
    assert X[0, tg.i_shoulder] == pytest.approx(length, abs=1e-12)
    assert np.allclose(Y[0], _radius(body, X[0]), rtol=0, atol=1e-9)
    xf, yf = X[-1], Y[-1]
    assert np.allclose(np.where(xf <= 0, np.hypot(xf, yf), yf), tg.far_radius, rtol=0, atol=1e-9)
    assert np.all(Y[:, 0] == 0) and np.all(X[:, 0] <= 0)
    assert np.allclose(X[:, -1], tg.x_end, rtol=0, atol=1e-12)
    assert X[-1, 0] == pytest.approx(-tg.far_radius, abs=1e-9)
    # The reference measured wall cells at 85.3 deg or more, corners at 51 deg
    # or more, neighbours within 1.92 (hemisphere) and 1.43 in size.
    q = grid_quality(tg.grid)
    assert q.min_area > 0
    assert q.min_wall_angle > 80 * DEG and q.min_angle > 45 * DEG
    assert q.max_size_ratio < (2 if length == 1 else 1.5)


def test_blunt_c_grids_nest():
    body = Body(Nose(NoseShape("ellipsoid"), 2.0, 1.0), 0.0)
    c, f = transonic_grid(body, 1, 100, 10), transonic_grid(body, 2, 100, 10)
    assert f.grid.ni == 2 * c.grid.ni and f.grid.nj == 2 * c.grid.nj
    Xc, Yc = _nodes(c)
    Xf, Yf = _nodes(f)
    assert max(np.abs(Xf[::2, ::2] - Xc).max(), np.abs(Yf[::2, ::2] - Yc).max()) < 1e-9


def test_geometric_remaining():
    assert geometric_remaining([1.0, 2.0]) == math.inf
    # Changes 1, 0.5: r = 0.5, remaining 0.5 r / (1 - r) = 0.5.
    assert geometric_remaining([0.0, 1.0, 1.5]) == pytest.approx(0.5)
    assert geometric_remaining([0.0, 1.0, 3.0]) == math.inf
    assert geometric_remaining([1.0, 1.0, 1.0 + 1e-14]) == pytest.approx(1e-14, rel=1e-3)
    assert geometric_remaining([1.0, 1.0, 2.0]) == math.inf


def test_oracle_solve_reproduces_the_measured_drag_on_the_base_grid():
    # The oracle's FP64 restatement of solveTransonic on the base grid (3,540
    # cells) settles in 550 steps to 0.08321842; the reference measured
    # 0.0832184, within 0.3 % of Taylor-Maccoll (the cone's surface flow is
    # supersonic at Mach 1.2).
    from oracle.transonic import solve_transonic

    p = transonic_problem(_cone(), TN["mach"], refinement=1, far_field=TN["far_field"], cylinder=TN["cylinder"])
    s = TN["solve"]
    out = solve_transonic(p, s["noise"], s["max_steps"], s["check_every"], s["cfl"], s["depth"], s["plain_steps"])
    assert out.converged
    assert abs(out.drag - TN["drags"][0]) <= 5e-8
    exact = taylor_maccoll(TN["mach"], HALF, 1.4).surface_pressure_coefficient
    assert abs(out.drag / exact - 1) < TN["within_taylor_maccoll"]


def test_a_start_must_come_from_a_coarser_grid_of_the_family():
    # solveTransonic's refusal (transonic-flow.ts:162-166), before any GPU work.
    from bowshock_b200.transonic import solve_transonic

    coarse = transonic_problem(_cone(), TN["mach"], refinement=2)
    fine = transonic_problem(_cone(), TN["mach"], refinement=1)
    prims = np.ones((coarse.grid.grid.nj, coarse.grid.grid.ni, 4))
    with pytest.raises(ValueError, match="coarser grid of the family"):
        solve_transonic(fine, start=(coarse, prims))
    other = transonic_problem(_cone(), TN["mach"], refinement=1, far_field=50)
    with pytest.raises(ValueError, match="not the coarser grid"):
        solve_transonic(transonic_problem(_cone(), TN["mach"], refinement=2),
                        start=(other, np.ones((other.grid.grid.nj, other.grid.grid.ni, 4))))
