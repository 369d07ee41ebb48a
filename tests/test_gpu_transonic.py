"""Transonic flow on the GPU (bowshock_b200.transonic): the 7 deg cone of NACA
TN 4233 at Mach 1.2 with its far-field domain, LU-SGS steps at a CFL number
ramped to 1000 with Anderson acceleration, on three grids of the family,
each finer one started from the coarser solution. The reference measured
0.0832184, 0.0830547 and 0.0830207 on its FP64 CPU engine
(tests/analysis/transonic-flow.test.ts:14-39); the GPU solves (FP64 state
and residual, FP32 metrics and operator) meet them to their printed digits
and the oracle's restatement of the same steps."""
from __future__ import annotations

import json
import math
import time
from pathlib import Path

import pytest

from bowshock_b200.grid import Body, Nose, NoseShape, taylor_maccoll
from bowshock_b200.transonic import solve_transonic, transonic_problem

pytestmark = pytest.mark.gpu

TN = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())[
    "transonic_cone_tn4233_mach1_2"]
HALF = TN["cone_half_angle_deg"] * math.pi / 180


def _problem(refinement: int):
    R = TN["base_radius"]
    cone = Body(Nose(NoseShape("conical"), R / math.tan(HALF), R), 0.0)
    return transonic_problem(cone, TN["mach"], refinement=refinement, far_field=TN["far_field"],
                             cylinder=TN["cylinder"])


def test_transonic_cone_drags_are_the_measured_ones_on_three_grids():
    s = TN["solve"]
    exact = taylor_maccoll(TN["mach"], HALF, 1.4).surface_pressure_coefficient
    previous = None
    drags = []
    for k, r in enumerate((1, 2, 4)):
        p = _problem(r)
        t0 = time.perf_counter()
        out = solve_transonic(p, s["noise"], s["max_steps"] * r, s["check_every"], s["cfl"], s["depth"],
                              s["plain_steps"], known_rate=previous[1].rate if previous else math.nan,
                              start=(previous[0], previous[1].primitives) if previous else None)
        print(f"transonic r={r}: {p.grid.grid.ni} x {p.grid.grid.nj} cells, {out.steps} steps, "
              f"{time.perf_counter() - t0:.2f} s, restarts {out.restarts}, drag {out.drag:.10f} "
              f"(measured {TN['drags'][k]})")
        assert out.converged and out.stopped_by == "settling"
        assert abs(out.drag - TN["drags"][k]) <= 1e-7
        drags.append(out.drag)
        previous = (p, out)
    assert abs(drags[0] / exact - 1) < TN["within_taylor_maccoll"]
    # Converging towards Taylor-Maccoll under refinement.
    assert abs(drags[2] - exact) < abs(drags[1] - exact) < abs(drags[0] - exact)


def test_two_float_metrics_put_the_steady_state_on_the_oracle():
    # 3,000 steps on the base grid (residual at its round-off floor): with
    # two-float metrics the GPU's drag is the FP64 oracle's; with FP32
    # metrics it wanders by about 1e-6 of its value (the reference's reason
    # for its two-float engine near Mach 1).
    from oracle.transonic import solve_transonic as oracle_solve

    s = TN["solve"]
    p = _problem(1)
    deep = dict(noise=1e-15, max_steps=3000, check_every=s["check_every"], cfl=s["cfl"], depth=s["depth"],
                plain_steps=s["plain_steps"])
    gpu64 = solve_transonic(p, **deep, metric_bits=64)
    gpu32 = solve_transonic(p, **deep, metric_bits=32)
    ora = oracle_solve(p, **deep)
    print(f"deep: oracle {ora.drag:.13f}, two-float {gpu64.drag:.13f} ({gpu64.drag / ora.drag - 1:+.1e}), "
          f"FP32 {gpu32.drag:.13f} ({gpu32.drag / ora.drag - 1:+.1e})")
    assert abs(gpu64.drag / ora.drag - 1) < 1e-9
    assert abs(gpu32.drag / ora.drag - 1) > 3e-7
    settled_gpu = solve_transonic(p, s["noise"], s["max_steps"], s["check_every"], s["cfl"], s["depth"],
                                  s["plain_steps"])
    settled_ora = oracle_solve(p, s["noise"], s["max_steps"], s["check_every"], s["cfl"], s["depth"],
                               s["plain_steps"])
    # Each settled run stops within its settling noise (1e-7 of the drag) of
    # the steady state, on either side.
    assert settled_gpu.converged and settled_ora.converged
    assert abs(settled_gpu.drag / ora.drag - 1) < 5 * s["noise"]
    assert abs(settled_ora.drag / ora.drag - 1) < 5 * s["noise"]


def test_blunt_nose_on_its_c_grid_follows_the_oracle():
    # A 2:1 ellipsoid at Mach 1.1 on its transonic C grid (the axis ahead of
    # the stagnation point a wall): 2,000 accelerated steps on the GPU with
    # two-float metrics and on the FP64 oracle give the same drag.
    from oracle.transonic import solve_transonic as oracle_solve

    body = Body(Nose(NoseShape("ellipsoid"), 2.0, 1.0), 0.0)
    p = transonic_problem(body, 1.1)
    assert p.grid.topology == "C" and p.config.boundaries["iMin"].kind == "wall"
    deep = dict(noise=1e-15, max_steps=2000, check_every=50, cfl=1000.0, depth=8, plain_steps=200)
    gpu = solve_transonic(p, **deep)
    ora = oracle_solve(p, **deep)
    print(f"ellipsoid M1.1: {p.grid.grid.ni} x {p.grid.grid.nj} cells, oracle {ora.drag:.12f}, "
          f"GPU {gpu.drag:.12f} ({gpu.drag / ora.drag - 1:+.1e})")
    assert math.isfinite(gpu.drag) and gpu.drag > 0
    assert abs(gpu.drag / ora.drag - 1) < 1e-8
