"""bluntBodyGrid (src/grid/blunt-grid.ts:159-540), the C-topology grid of
blunt noses, checked the way tests/grid/blunt-grid.test.ts checks it: quality
gates over random blunt rockets, nodes on the wall, the axis and the outflow
plane, the outer line at twice Billig's standoff, nested refinement, and the
shapes it refuses. Host code only: no GPU."""
from __future__ import annotations

import math

import numpy as np
import pytest

from bowshock_b200 import _native
from bowshock_b200.grid import Body, Nose, NoseShape, blunt_body_grid, grid_quality
from bowshock_b200.workloads import SplitMix64

HEMISPHERE_CYLINDER = Body(Nose(NoseShape("ellipsoid"), 0.5, 0.5), 4.0)


def billig_standoff(mach: float, radius: float) -> float:
    """Billig's sphere standoff correlation, delta / R = 0.143 exp(3.24 / M^2)."""
    return radius * 0.143 * math.exp(3.24 / (mach * mach))


def ellipsoid_radius(body: Body, x: np.ndarray) -> np.ndarray:
    L, R = body.nose.length, body.nose.base_radius
    s = np.clip(1.0 - x / L, 0.0, 1.0)
    return np.where(x < L, R * np.sqrt(np.maximum(0.0, 1.0 - s * s)), R)


def nodes(grid):
    n1 = grid.ni + 1
    return grid.x.reshape(grid.nj + 1, n1), grid.y.reshape(grid.nj + 1, n1)


def test_random_blunt_rockets_pass_every_quality_gate():
    """40 seeded ellipsoid-nosed rockets (nose 0.5-1.5 long, cylinder 2-15)
    at Mach 1.5-5 pass the gates, with lines leaving the wall within 10 deg
    of normal (tests/grid/blunt-grid.test.ts:37-49)."""
    g = SplitMix64(7)
    for _ in range(40):
        body = Body(Nose(NoseShape("ellipsoid"), g.uniform(0.5, 1.5), 0.5), g.uniform(2.0, 15.0))
        mach = g.uniform(1.5, 5.0)
        q = grid_quality(blunt_body_grid(body, 20, mach).grid)
        assert q.min_wall_angle > 80 * math.pi / 180, (body, mach)


def test_nodes_on_wall_axis_outflow_and_the_outer_line_at_twice_billig():
    """tests/grid/blunt-grid.test.ts:50-64."""
    grid = blunt_body_grid(HEMISPHERE_CYLINDER, 20, 3.0).grid
    X, Y = nodes(grid)
    body_length = 0.5 + 4.0
    assert np.max(np.abs(Y[0] - ellipsoid_radius(HEMISPHERE_CYLINDER, X[0]))) < 1e-12
    assert np.all(Y[:, 0] == 0.0)
    assert np.max(np.abs(X[:, -1] - body_length)) < 1e-12
    assert abs(-X[-1, 0] - 2 * billig_standoff(3.0, 0.5)) < 1e-12


def test_refinement_keeps_every_coarse_node():
    """tests/grid/blunt-grid.test.ts:65-86."""
    coarse = blunt_body_grid(HEMISPHERE_CYLINDER, 20, 2.0).grid
    Xc, Yc = nodes(coarse)
    for r in (2, 4):
        fine = blunt_body_grid(HEMISPHERE_CYLINDER, 20, 2.0, refinement=r).grid
        assert (fine.ni, fine.nj) == (r * coarse.ni, r * coarse.nj)
        Xf, Yf = nodes(fine)
        assert np.max(np.abs(Xf[::r, ::r] - Xc)) < 1e-12
        assert np.max(np.abs(Yf[::r, ::r] - Yc)) < 1e-12


def test_exact_column_count():
    for ni in (40, 80, 160):
        grid = blunt_body_grid(HEMISPHERE_CYLINDER, ni // 2, 2.5, ni=ni).grid
        assert (grid.ni, grid.nj) == (ni, ni // 2)


def test_refused_shapes():
    """A paraboloid half as long as its radius meets the cylinder too steeply;
    a hemisphere with no cylinder at Mach 1.5 fails the gates
    (tests/grid/blunt-grid.test.ts:198-210)."""
    power = Body(Nose(NoseShape("power", 0.5), 0.5, 0.5), 4.0)
    with pytest.raises(_native.BowshockError, match="more than"):
        blunt_body_grid(power, 20, 3.0)
    stub = Body(Nose(NoseShape("ellipsoid"), 0.5, 0.5), 0.0)
    with pytest.raises(_native.GridQualityError):
        blunt_body_grid(stub, 20, 1.5)


def test_two_scale_haack_nose_builds_ungated():
    """The reference builds the Haack nose's grid without the gates
    (tests/grid/blunt-grid.test.ts:133-137)."""
    haack = Body(Nose(NoseShape("haack", 0.0), 3.0, 0.5), 2.0)
    grid = blunt_body_grid(haack, 20, 2.0, gated=False).grid
    X, Y = nodes(grid)
    assert np.all(Y[:, 0] == 0.0) and np.all(np.isfinite(X)) and np.all(np.isfinite(Y))
