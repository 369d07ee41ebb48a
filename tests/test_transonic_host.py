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
    with pytest.raises(BowshockError, match="sharp noses"):
        transonic_grid(Body(Nose(NoseShape("ellipsoid"), 1.0, 1.0), 0.0), 1, 100, 10)
    with pytest.raises(ValueError, match="positive"):
        transonic_grid(body, 1, 100, 10, spacing={"wall": -1})


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
