"""Two-scale noses on the GPU fit: a Von Karman nose, whose tip curvature is
unbounded, so its C grid's boundary is sized for the tip. The family's
outer boundary is the shock captured on that grid pushed out by a margin, a
second capture on the grid built on it starts the family, and the fitted
drags on nj = 20 and 40 are the ones the reference measured on its FP64 CPU
engine (tests/analysis/two-scale-fit.test.ts:24-80)."""
from __future__ import annotations

import json
import time
from pathlib import Path

import numpy as np
import pytest

from bowshock_b200.fitted import (CudaFit, TWO_SCALE_DRAG_FLOOR, blunt_fit_family, blunt_start,
                                  fitted_case_failure, fitted_grid_failure, settle)
from bowshock_b200.grid import Body, Nose, NoseShape

pytestmark = pytest.mark.gpu

_ALL = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())
VK = _ALL["fitted_von_karman_mach2"]


def _body() -> Body:
    b = VK["body"]
    return Body(Nose(NoseShape(b["shape"], float(b["parameter"])), b["length"], b["base_radius"]), b["cylinder"])


def _settled(p, cap: int, r: int, noise: float = 1e-7, speed_tolerance: float = 1e-6):
    with CudaFit(p) as g:
        converged, it, speed, drag = settle(g, cap, noise=noise, speed_tolerance=speed_tolerance,
                                            check_every=250 * r)
        return converged, it, speed, drag, g.grid(), g.primitives().reshape(p.nj, p.ni, 4)


def _oracle_capture(body, grid, mach, gamma):
    # bluntCapture on the FP64 oracle: the reference's CPU engine for the start.
    from bowshock_b200.config import Boundary, free_stream_at, steady_drag_config
    from bowshock_b200.fitted import CAPTURED_START_STEPS
    from oracle.oracle import OracleEuler2D

    free = free_stream_at(mach, gamma).state
    cfg = steady_drag_config(grid, free, gamma, boundaries={
        "iMin": Boundary("wall"), "iMax": Boundary("outflow"), "jMin": Boundary("wall"),
        "jMax": Boundary("inflow", free)})
    e = OracleEuler2D(cfg)
    e.set_primitives(np.tile([free.rho, free.u, free.v, free.p], grid.ni * grid.nj))
    e.iterate(CAPTURED_START_STEPS)
    return e.primitives().reshape(grid.nj, grid.ni, 4)


def test_two_scale_start_follows_the_oracle(monkeypatch):
    # Both captures (67 and 113 columns) on the GPU engine against the
    # oracle's: the same captured shock, so the same outer boundary, grid and
    # starting heights; the flow within the FP32-metric floor.
    import bowshock_b200.fitted as fitted

    gpu = blunt_start(_body(), VK["mach"], VK["nj"])
    monkeypatch.setattr(fitted, "_capture", _oracle_capture)
    ora = blunt_start(_body(), VK["mach"], VK["nj"])
    assert gpu.grid.ni == ora.grid.ni == 113
    assert np.array_equal(gpu.outer_boundary, ora.outer_boundary)
    assert np.array_equal(gpu.heights, ora.heights)
    scale = np.abs(ora.captured).max(axis=(0, 1))
    assert np.max(np.abs(gpu.captured - ora.captured) / scale) < 1e-4


def test_von_karman_fitted_drags_are_the_measured_ones():
    # nj = 20 and its refinement, each settled from the family's shock-layer
    # start (the reference starts the finer from the coarser fit: the same
    # fixed point) until the drag changes by less than 1e-11 and the shock by
    # less than 1e-10 a_inf. The reference's FP64 fits agree with its measured
    # drags to 1e-9; so does the GPU fit, whose residual reads two-float
    # metrics (about 1e-11 here).
    t0 = time.perf_counter()
    start = blunt_start(_body(), VK["mach"], VK["nj"])
    t_start = time.perf_counter() - t0
    assert start.outer_boundary is not None and start.outer_boundary[0, 1] == 0.0
    family = blunt_fit_family(start)
    asked_end = VK["body"]["length"] + VK["body"]["cylinder"]
    for r, want in ((1, VK["drag_nj20"]), (2, VK["drag_nj40"])):
        p = family(r)
        t0 = time.perf_counter()
        converged, it, speed, drag, grid, prims = _settled(p, 40000 * r, r, noise=1e-11, speed_tolerance=1e-10)
        print(f"two-scale r={r}: {p.ni} x {p.nj} cells, {it} steps, {time.perf_counter() - t0:.2f} s "
              f"(start {t_start:.2f} s), speed {speed:.1e}, drag {drag:.12f}, rel {drag / want - 1:+.2e}")
        assert converged
        assert fitted_grid_failure(grid) is None
        assert fitted_case_failure(p, asked_end, grid, prims) is None
        assert abs(drag / want - 1) < VK["within"]


def test_verified_fitted_drag_of_a_von_karman_nose_carries_the_two_scale_allowance():
    # Four grids (nj = 20 to 160) confirm the order; the band holds the
    # two-scale allowance of 8e-4 of the drag.
    from bowshock_b200.fitted import verified_fitted_drag

    t0 = time.perf_counter()
    out = verified_fitted_drag(_body(), VK["mach"], tolerance=1e-3, max_refinement=8)
    print(f"verified two-scale: {out.kind} {out.reason} {time.perf_counter() - t0:.2f} s "
          f"{[(l.refinement, l.ni, l.nj, l.iterations, l.drag) for l in out.reports]}")
    assert out.kind == "solved", out.reason
    assert out.floor == TWO_SCALE_DRAG_FLOOR == _ALL["two_scale_drag_floor"]["value"]
    v = out.result
    assert v.verified and v.uncertainty <= 1e-3 and len(v.levels) == 4
    assert v.uncertainty >= TWO_SCALE_DRAG_FLOOR * abs(v.estimate.value)
    assert abs(v.levels[0][1] / VK["drag_nj20"] - 1) < 3e-7
    assert abs(v.levels[1][1] / VK["drag_nj40"] - 1) < 3e-7
