"""Captured-shock cones on the GPU against the exact conical solution.

The reference holds its CPU engine's cones to Taylor-Maccoll: on 60 x 30 ramp
grids the mean cone-surface pressure over x = 1.0 to 1.4 within 1e-3 (Mach
2.35, 10 deg; Mach 2, 15 deg) or 4e-3 (Mach 3, 20 deg), the residual to
1e-10 of its start, and the captured shock within half a cell of the exact
one on every grid line with x in (0.6, 1.3)
(tests/engine-cpu/euler2d-cone.test.ts:95-124); and cone-cylinders on its
generated grids within 1e-3 over 0.5 to 0.95 of the cone length
(tests/engine-cpu/body-validation.test.ts:72-116). The same checks here run
on the FP64 GPU engine, and on the plain explicit configuration (a 15 deg
cone of 1 caliber on a 2-caliber cylinder at Mach 2, 80 x 40, minmod,
SSP-RK3 at CFL 0.5, marched from the free stream to an RMS density
residual of 1e-6), whose oracle solve sits 4.6e-4 below Taylor-Maccoll.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from bowshock_b200.config import Boundary, Euler2DConfig, Primitive2D
from bowshock_b200.engine import CudaEuler2D
from bowshock_b200.grid import ramp_grid, taylor_maccoll

from cases import DEG, GAMMA, config1

pytestmark = pytest.mark.gpu


def wall_pressure(faces) -> list[tuple[float, float]]:
    """(x, p) of each wall face: the x-momentum and y-momentum fluxes of a
    wall face are p n."""
    return [(f.x, f.flux[1] * f.nx + f.flux[2] * f.ny) for f in faces]


def test_config1_cone_surface_pressure_matches_taylor_maccoll():
    cfg, free, body = config1()
    exact = taylor_maccoll(2.0, 15 * DEG, GAMMA)
    with CudaEuler2D(cfg, 64) as e:
        e.set_uniform(free.state)
        res = e.solve("explicit", tolerance=1e-6, max_steps=20000, check_every=50)
        assert res.status == 0 and res.residual <= 1e-6
        faces = wall_pressure(e.boundary_fluxes("jMin"))
    L = body.nose.length
    values = [p for x, p in faces if 0.5 * L < x < 0.95 * L]
    assert len(values) >= 10
    dev = float(np.mean(values)) / exact.surface_pressure_ratio - 1
    assert abs(dev) < 1e-3
    assert abs(dev - (-4.56e-4)) < 5e-6  # the oracle's own figure on this grid


def ramp_cone(mach: float, cone_deg: float) -> tuple[Euler2DConfig, Primitive2D]:
    free = Primitive2D(1.0, mach * math.sqrt(GAMMA), 0.0, 1.0)
    grid = ramp_grid(60, 30, -0.5, 0.0, 1.5, 1.2, cone_deg * DEG)
    cfg = Euler2DConfig(grid=grid, geometry="axisymmetric", gamma=GAMMA, flux="hllc",
                        limiter="vanAlbada", reconstruction="sharedScaled",
                        time_integrator="ssprk2", cfl=0.8, time_stepping="local",
                        boundaries={"iMin": Boundary("inflow", free), "iMax": Boundary("outflow"),
                                    "jMin": Boundary("wall"), "jMax": Boundary("outflow")})
    return cfg, free


@pytest.mark.parametrize("mach, cone, tolerance", [(2.35, 10, 1e-3), (2.0, 15, 1e-3), (3.0, 20, 4e-3)])
def test_ramp_cones_meet_taylor_maccoll_and_capture_the_shock_within_half_a_cell(mach, cone, tolerance):
    cfg, free = ramp_cone(mach, cone)
    exact = taylor_maccoll(mach, cone * DEG, GAMMA)
    with CudaEuler2D(cfg, 64) as e:
        e.set_uniform(free)
        r0 = e.density_residual_norm()
        e.iterate(2000)
        assert e.density_residual_norm() < 1e-10 * r0
        faces = wall_pressure(e.boundary_fluxes("jMin"))
        w = e.primitives()
        cx, cy = e.centroids()
    p = np.mean([pw for x, pw in faces if 1.0 < x < 1.4])
    assert abs(p / exact.surface_pressure_ratio - 1) < tolerance
    # The captured shock: where the pressure crosses the mean of its
    # free-stream and post-shock values, on each vertical grid line.
    ni, nj = cfg.grid.ni, cfg.grid.nj
    p_mid = 0.5 * (1 + exact.post_shock_pressure_ratio)
    pr = w[:, 3].reshape(nj, ni)
    offsets = []
    for i in range(ni):
        x = cx[i]
        if x < 0.6 or x > 1.3:
            continue
        for j in range(nj - 2, -1, -1):
            p0, p1 = pr[j, i], pr[j + 1, i]
            if p0 > p_mid and p1 <= p_mid:
                y0, y1 = cy[i + j * ni], cy[i + (j + 1) * ni]
                y = y0 + (y1 - y0) * (p0 - p_mid) / (p0 - p1)
                offsets.append((y - x * math.tan(exact.shock_angle)) / (y1 - y0))
                break
    assert len(offsets) > 10
    assert max(abs(o) for o in offsets) < 0.5
