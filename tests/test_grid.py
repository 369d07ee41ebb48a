"""The grid generator against the reference's body-grid properties
(tests/grid/body-grid.test.ts) and the engine's metrics conventions
(src/grid/structured.ts)."""
from __future__ import annotations

import math
import random

import numpy as np
import pytest

from bowshock_b200 import _native
from bowshock_b200.grid import Body, Nose, NoseShape, body_grid, grid_quality, ramp_grid
from oracle.oracle import OracleEuler2D

from cases import GAMMA, cone_body, ogive_body
from bowshock_b200.config import Boundary, Euler2DConfig


def random_rockets(seed: int, n: int, mach_range: tuple[float, float]):
    """Sharp-nosed rockets as the reference's property tests draw them: noses
    of 2 to 8 calibers (cone, ogive of parameter 0.2-1, parabolic), no
    cylinder or one of 1 to 25 calibers."""
    rng = random.Random(seed)
    for _ in range(n):
        kind = rng.choice(["conical", "ogive", "parabolic"])
        param = {"conical": 0.0, "ogive": rng.uniform(0.2, 1), "parabolic": rng.uniform(0, 1)}[kind]
        length = rng.uniform(2, 8)
        cyl = 0.0 if rng.random() < 0.3 else rng.uniform(1, 25)
        yield Body(Nose(NoseShape(kind, param), length, 0.5), cyl), rng.uniform(*mach_range)


@pytest.mark.parametrize("seed,mach_range", [(121, (2, 5)), (123, (1.5, 2))])
def test_generated_grids_pass_every_quality_gate(seed, mach_range):
    for body, mach in random_rockets(seed, 25, mach_range):
        g = body_grid(body, 20, mach, GAMMA).grid
        q = grid_quality(g)
        assert q.min_area > 0
        assert q.min_angle >= 12 * math.pi / 180 - 1e-12
        assert q.min_wall_angle >= 60 * math.pi / 180 - 1e-12
        assert q.max_size_ratio <= 1.3 + 1e-12
        assert q.max_aspect_ratio <= 10 + 1e-12


def test_wall_nodes_lie_on_the_profile_with_tip_and_shoulder_on_grid_lines():
    body = ogive_body(3.0, 4.0)
    bg = body_grid(body, 20, 2.0, GAMMA)
    g = bg.grid
    xs = g.x[: g.ni + 1]
    ys = g.y[: g.ni + 1]
    assert xs[bg.i_tip] == 0.0
    assert np.any(xs == body.nose.length)
    assert abs(xs[-1] - 7.0) < 1e-12
    assert np.all(np.diff(xs) > 0)
    assert np.all(ys[: bg.i_tip + 1] == 0.0)
    assert np.all(np.abs(ys[xs >= body.nose.length] - 0.5) < 1e-12)


def test_refined_grids_are_nested():
    body = cone_body(12, 3.0)
    coarse = body_grid(body, 20, 2.5, GAMMA).grid
    fine = body_grid(body, 20, 2.5, GAMMA, refinement=2).grid
    assert fine.ni == 2 * coarse.ni and fine.nj == 2 * coarse.nj
    cx = coarse.x.reshape(coarse.nj + 1, coarse.ni + 1)
    fx = fine.x.reshape(fine.nj + 1, fine.ni + 1)
    cy = coarse.y.reshape(coarse.nj + 1, coarse.ni + 1)
    fy = fine.y.reshape(fine.nj + 1, fine.ni + 1)
    assert np.allclose(fx[::2, ::2], cx, atol=1e-12)
    assert np.allclose(fy[::2, ::2], cy, atol=1e-12)


@pytest.mark.parametrize("ni,nj", [(80, 40), (160, 80), (40, 20), (320, 160)])
def test_exact_column_counts(ni, nj):
    g = body_grid(ogive_body(3.0, 4.0), nj, 2.0, GAMMA, ni=ni).grid
    assert (g.ni, g.nj) == (ni, nj)
    assert grid_quality(g).min_area > 0


def test_blunt_and_steep_tips_are_refused_by_the_h_grid():
    with pytest.raises(_native.BowshockError, match="blunt"):
        body_grid(Body(Nose(NoseShape("ellipsoid"), 2.0, 0.5), 2.0), 20, 2.0, GAMMA)
    with pytest.raises(_native.BowshockError, match="tip half-angles"):
        body_grid(cone_body(40, 2.0), 20, 3.0, GAMMA)


def test_metrics_conventions_on_a_ramp():
    g = ramp_grid(6, 4, -1.0, 0.0, 1.0, 1.0, 10 * math.pi / 180)
    cfg = Euler2DConfig(grid=g, geometry="axisymmetric",
                        boundaries={s: Boundary("outflow") for s in ("iMin", "iMax", "jMin", "jMax")})
    i_faces, j_faces, cells = OracleEuler2D(cfg).metrics()
    # unit normals, i-faces towards +i, j-faces towards +j
    assert np.allclose(np.hypot(i_faces[:, 0], i_faces[:, 1]), 1.0)
    assert np.all(i_faces[:, 0] > 0) and np.all(j_faces[:, 1] > 0)
    # axisymmetric volume = planar area x centroid radius
    assert np.allclose(cells[:, 0], cells[:, 1] * cells[:, 3])
