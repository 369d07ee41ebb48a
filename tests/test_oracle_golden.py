"""The CPU oracle (C++ restatement of src/engine-cpu/euler2d.ts) pinned to the
reference's own known answers (tests/golden/reference_known_answers.json,
extracted from the reference's test files by extract_known_answers.py)."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

from bowshock_b200.config import Boundary, Euler2DConfig, Primitive2D, free_stream_at, steady_drag_config
from bowshock_b200.grid import body_grid
from oracle.oracle import OracleEuler2D

from cases import GAMMA, cone_body, lcg_random
from bowshock_b200.config import grid_from_function

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())


@pytest.mark.parametrize("level", [0, 1])
def test_verified_drag_of_the_20_degree_cone(level):
    # tests/gpu/verified-drag-gpu.test.ts:16-46 pins the CPU engine's drag on
    # the family's first two grids; the oracle converged to round-off must be
    # within the reference's own 2e-6 (it lands within 1e-8).
    g = GOLDEN["verified_drag_cone20_mach3"]
    refinement = g["refinements"][level]
    body = cone_body(g["body"]["half_angle_deg"], g["body"]["cylinder"])
    free = free_stream_at(g["mach"], GAMMA)
    bg = body_grid(body, g["nj"], g["mach"], GAMMA, refinement=refinement)
    o = OracleEuler2D(steady_drag_config(bg.grid, free.state))
    o.set_uniform(free.state)
    o.iterate(600 * refinement)
    assert o.density_residual_norm() < 1e-11
    cd = o.forebody_drag(free.pressure, free.dynamic_pressure, 0.5)
    assert abs(cd / g["drag"][level] - 1) < 1e-7


def implicit_case():
    g = GOLDEN["implicit_equals_explicit"]
    body = cone_body(g["body"]["half_angle_deg"], g["body"]["cylinder"])
    free = free_stream_at(g["mach"], GAMMA)
    bg = body_grid(body, g["nj"], g["mach"], GAMMA)
    cfg = steady_drag_config(bg.grid, free.state, boundaries={
        "iMin": Boundary("inflow", free.state), "iMax": Boundary("outflow"),
        "jMin": Boundary("wall"), "jMax": Boundary("farField", free.state)})
    return g, cfg, free


def test_lusgs_reaches_the_explicit_drag_within_1e12():
    # tests/engine-cpu/implicit.test.ts:201-240
    g, cfg, free = implicit_case()
    explicit = OracleEuler2D(cfg)
    explicit.set_uniform(free.state)
    explicit.iterate(g["explicit_steps"])
    assert explicit.density_residual_norm() < g["residual_below"]
    s = OracleEuler2D(cfg)
    s.set_uniform(free.state)
    cfl = 1.0
    for _ in range(600):
        if s.density_residual_norm() <= 1e-13:
            break
        s.iterate_implicit(1, cfl)
        cfl = min(1000.0, cfl * 1.2)
    assert s.density_residual_norm() < 1e-12
    d_exp = explicit.forebody_drag(free.pressure, free.dynamic_pressure, 0.5)
    d_imp = s.forebody_drag(free.pressure, free.dynamic_pressure, 0.5)
    assert abs(d_imp / d_exp - 1) < g["drag_equal_within"]


@pytest.mark.parametrize("mach", [0.8, 1.0, 1.5])
def test_uniform_flow_stays_uniform_with_far_field_boundaries(mach):
    # tests/engine-cpu/implicit.test.ts:67-101: implicit then explicit steps
    # on a distorted axisymmetric grid keep a free stream to 1e-12.
    random = lcg_random(7)

    def node(i, j):
        interior = 0 < i < 14 and 0 < j < 10
        return (i + (0.5 * random() if interior else 0.0), 1 + j + (0.5 * random() if interior else 0.0))

    grid = grid_from_function(14, 10, node)
    w = Primitive2D(1.0, mach * math.sqrt(GAMMA), 0.0, 1.0)
    far = Boundary("farField", w)
    cfg = Euler2DConfig(grid=grid, geometry="axisymmetric", gamma=GAMMA, flux="hllc",
                        limiter="vanAlbada", reconstruction="sharedScaled", time_integrator="ssprk2",
                        cfl=0.8, time_stepping="local",
                        boundaries={"iMin": far, "iMax": far, "jMin": far, "jMax": far})
    s = OracleEuler2D(cfg)
    s.set_uniform(w)
    s.iterate_implicit(20, 100)
    s.iterate(20)
    p = s.primitives().reshape(-1, 4)
    assert np.max(np.abs(p[:, 0] - 1)) < 1e-12
    assert np.max(np.abs(p[:, 1] - w.u)) < 1e-12
    assert np.max(np.abs(p[:, 2])) < 1e-12
    assert np.max(np.abs(p[:, 3] - 1)) < 1e-12


def test_time_step_formula():
    # tests/engine-cpu/euler2d.test.ts:141-175: on a uniform Cartesian grid
    # dt = CFL dx dy / ((|u| + a) dy + (|v| + a) dx).
    grid = grid_from_function(5, 4, lambda i, j: (0.2 * i, 0.5 * j))
    w = Primitive2D(1.2, 0.4, -0.3, 0.9)
    cfg = Euler2DConfig(grid=grid, geometry="planar", gamma=GAMMA, flux="hllc", limiter="minmod",
                        reconstruction="perVariable", time_integrator="ssprk2", cfl=0.7,
                        time_stepping="local",
                        boundaries={s: Boundary("outflow") for s in ("iMin", "iMax", "jMin", "jMax")})
    s = OracleEuler2D(cfg)
    s.set_uniform(w)
    a = math.sqrt(GAMMA * w.p / w.rho)
    expect = 0.7 * 0.2 * 0.5 / ((abs(w.u) + a) * 0.5 + (abs(w.v) + a) * 0.2)
    assert np.allclose(s.time_steps(), expect, rtol=1e-14)


def test_oracle_rejects_invalid_configurations():
    from oracle.oracle import OracleError

    grid = grid_from_function(4, 4, lambda i, j: (i, j))
    base = dict(grid=grid, geometry="planar", gamma=GAMMA, flux="hllc", limiter="minmod",
                reconstruction="shared", time_integrator="ssprk2", cfl=0.5, time_stepping="local",
                boundaries={s: Boundary("outflow") for s in ("iMin", "iMax", "jMin", "jMax")})
    with pytest.raises(OracleError):
        OracleEuler2D(Euler2DConfig(**base))
    with pytest.raises(OracleError):
        OracleEuler2D(Euler2DConfig(**{**base, "reconstruction": "perVariable", "cfl": 1.5}))


def test_non_physical_state_is_rejected():
    from oracle.oracle import OracleError

    grid = grid_from_function(4, 4, lambda i, j: (i, j))
    cfg = Euler2DConfig(grid=grid, geometry="planar", gamma=GAMMA, flux="hllc", limiter="minmod",
                        reconstruction="perVariable", time_integrator="ssprk2", cfl=0.5,
                        time_stepping="local",
                        boundaries={s: Boundary("outflow") for s in ("iMin", "iMax", "jMin", "jMax")})
    s = OracleEuler2D(cfg)
    with pytest.raises(OracleError):
        s.set_uniform(Primitive2D(1.0, 0.0, 0.0, -1.0))
