"""The fitted bow shock on the GPU (bs_fit_*): step for step against the
oracle's restatement of fitShock (oracle/shock_fitting.py), and the
reference's own test of the method (tests/analysis/fitted-flow.test.ts:36-59):
on the Mach 3, 20 deg cone the drag is within 0.03 % of Taylor-Maccoll on the
grid refined once and converges at second order, to the values the
reference measured (+0.1017 % and +0.0251 %)."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

from bowshock_b200.fitted import CudaFit, settle, sharp_fit_problem
from bowshock_b200.grid import taylor_maccoll
from bowshock_b200.workloads import cone_body

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())[
    "fitted_cone_mach3"]


def _problem(refinement: int = 1):
    b = GOLDEN["body"]
    return sharp_fit_problem(cone_body(b["half_angle_deg"], b["cylinder"]), GOLDEN["mach"], nj=GOLDEN["nj"],
                             refinement=refinement)


def test_fitted_steps_follow_the_oracle():
    # 150 steps from the conical start: the GPU (FP64 state, FP32 metrics
    # rebuilt after every move) and the FP64 oracle agree on the shock's
    # heights, the flow and the drag.
    from oracle.shock_fitting import fit_shock

    p = _problem()
    with CudaFit(p) as g:
        g.iterate(150)
        h, w, d = g.heights(), g.primitives(), g.drag()
        speed, _ = g.check()
    o = fit_shock(p, 150)
    wo = o.engine.primitives().reshape(-1, 4)
    assert np.max(np.abs(h - o.heights)) < 1e-7 * np.max(o.heights)
    assert np.max(np.abs(w - wo) / np.abs(wo).max(axis=0)) < 1e-5
    assert abs(d / p.drag(o.engine.boundary_fluxes("jMin")) - 1) < 1e-6
    assert abs(speed / o.speeds[-1] - 1) < 2e-3


def test_fitted_cone_drag_converges_at_second_order_to_taylor_maccoll():
    exact = taylor_maccoll(GOLDEN["mach"], GOLDEN["body"]["half_angle_deg"] * math.pi / 180, 1.4) \
        .surface_pressure_coefficient
    errors = []
    for r in GOLDEN["refinements"]:
        with CudaFit(_problem(r)) as g:
            converged, _, speed, drag = settle(g, 60000 * r, check_every=250 * r)
        assert converged and speed < 1e-6
        errors.append(drag / exact - 1)
    coarse, fine = errors
    assert abs(fine) < GOLDEN["fine_below"]
    assert GOLDEN["ratio_above"] < coarse / fine < GOLDEN["ratio_below"]
    assert abs(fine - (coarse - fine) / 3) < GOLDEN["extrapolated_within"]
    # The values the reference measured, to the digits it gives.
    for e, measured in zip(errors, GOLDEN["measured_rel_err"]):
        assert abs(e - measured) < 5e-7


HEMI = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())[
    "fitted_hemisphere_mach2"]


def _hemisphere():
    from bowshock_b200.fitted import blunt_fit_problem
    from bowshock_b200.grid import Body, Nose, NoseShape

    b = HEMI["body"]
    body = Body(Nose(NoseShape(b["shape"]), b["length"], b["base_radius"]), b["cylinder"])
    return blunt_fit_problem(body, HEMI["mach"], nj=HEMI["nj"])


def test_blunt_fit_follows_the_oracle():
    # The hemisphere-cylinder from its captured start: the shock's axis node
    # kept normal to the axis; GPU and oracle agree after 100 steps.
    from oracle.shock_fitting import fit_shock

    p = _hemisphere()
    assert p.first_node == "symmetry" and p.inflow is None
    with CudaFit(p) as g:
        g.iterate(100)
        h, w, d = g.heights(), g.primitives(), g.drag()
    o = fit_shock(p, 100)
    wo = o.engine.primitives().reshape(-1, 4)
    assert np.max(np.abs(h - o.heights)) < 1e-6 * np.max(o.heights)
    assert np.max(np.abs(w - wo) / np.abs(wo).max(axis=0)) < 1e-4
    assert abs(d / p.drag(o.engine.boundary_fluxes("jMin")) - 1) < 1e-5


def test_hemisphere_stagnation_pressure_is_the_pitot_value():
    # tests/analysis/fitted-flow.test.ts:61-74: the wall pressure at the
    # stagnation point, behind the fitted normal shock, within 1e-4 of the
    # pitot pressure (the reference measured +0.0076 %; captured, +9.7 %).
    from bowshock_b200.grid import normal_shock

    p = _hemisphere()
    with CudaFit(p) as g:
        converged, _, speed, _ = settle(g, 60000, check_every=250)
        face = g.wall_fluxes()[0]
    assert converged and speed < 1e-6
    g_ = p.gamma
    shock = normal_shock(HEMI["mach"], g_)
    m2 = shock.downstream_mach
    pitot = shock.pressure_ratio * (1 + 0.5 * (g_ - 1) * m2 * m2) ** (g_ / (g_ - 1))
    wall = face.flux[1] * face.nx + face.flux[2] * face.ny
    assert abs(wall / pitot - 1) < HEMI["within"]


def test_verified_fitted_drag_of_the_cone_contains_the_exact_drag():
    # verifiedFittedDrag (src/analysis/fitted-flow.ts:1005-1075) on the GPU
    # fit: grids of 20 cells across refined by 2 until the band is within
    # 1e-4; the Taylor-Maccoll drag of the cone lies inside the band.
    from bowshock_b200.fitted import verified_fitted_drag

    b = GOLDEN["body"]
    exact = taylor_maccoll(GOLDEN["mach"], b["half_angle_deg"] * math.pi / 180, 1.4).surface_pressure_coefficient
    out = verified_fitted_drag(cone_body(b["half_angle_deg"], b["cylinder"]), GOLDEN["mach"], tolerance=1e-4,
                               max_refinement=8)
    assert out.kind == "solved", out.reason
    v = out.result
    assert v.verified and v.uncertainty <= 1e-4
    assert abs(v.estimate.value - exact) <= v.uncertainty
    assert [r for r, _ in v.levels] == [1, 2, 4, 8][:len(v.levels)] and len(v.levels) >= 4
    assert abs(v.estimate.extrapolated - exact) < 2e-5 * exact


_ALL = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())
OGIVE = _ALL["fitted_ogive_mach1_35"]
FALLBACK = _ALL["fitted_ogive_fallback_mach1_5"]


def _ogive(cylinder: float):
    from bowshock_b200.grid import Body, Nose, NoseShape

    return Body(Nose(NoseShape("ogive", 1.0), 3.0, 0.5), cylinder)


def test_ogive_with_an_axially_subsonic_tip_converges_as_measured():
    # tests/analysis/fitted-flow.test.ts:490-534: the 3-caliber tangent ogive
    # at Mach 1.35, on 10 cells across refined once, against the page's
    # extrapolated drag; the reference measured +2.075e-2 and +4.730e-3.
    ref = OGIVE["extrapolated"]
    errors = []
    for r in (1, 2):
        p = sharp_fit_problem(_ogive(OGIVE["body"]["cylinder"]), OGIVE["mach"], nj=10, refinement=r)
        with CudaFit(p) as g:
            _, _, speed, drag = settle(g, 80000 * r, check_every=250 * r)
        assert speed < 1e-6
        errors.append(drag / ref - 1)
    coarse, fine = errors
    assert 0 < fine < OGIVE["fine_below"]
    assert OGIVE["ratio_above"] < coarse / fine < OGIVE["ratio_below"]
    assert abs(coarse - OGIVE["coarse_family_nj10_rel"][0]) < 5e-6
    assert abs(fine - OGIVE["coarse_family_nj10_rel"][1]) < 5e-7


def test_ogive_base_grid_drag_is_the_measured_one():
    # The page's base grid (nj = 20): 0.1081856017 on the reference's FP64
    # engine. Settled until the drag changes by less than 1e-11 and the shock
    # by less than 1e-10 a_inf, the GPU fit (two-float metrics) meets it to
    # the digits given.
    p = sharp_fit_problem(_ogive(OGIVE["body"]["cylinder"]), OGIVE["mach"], nj=20)
    with CudaFit(p) as g:
        converged, _, speed, drag = settle(g, 120000, noise=1e-11, speed_tolerance=1e-10, check_every=250)
    assert converged and speed < 1e-10
    assert abs(drag / OGIVE["verified_nj20_value"] - 1) < 1e-9


def test_a_grid_failing_only_the_gates_is_solved_again_with_more_columns():
    # tests/analysis/fitted-flow.test.ts:536-566: on 30 calibers of cylinder
    # at Mach 1.5 the usual grid's wall cells reach an aspect ratio of 18.0;
    # the family is solved again with 1.5 times the columns (184), whose drag
    # the reference measured as 0.10583491196235459.
    from bowshock_b200.fitted import FALLBACK_COLUMN_DENSITY, verified_fitted_drag

    fallbacks = []
    out = verified_fitted_drag(_ogive(FALLBACK["body"]["cylinder"]), FALLBACK["mach"], tolerance=0.0, floor=0.0,
                               max_refinement=1, on_fallback=lambda r, why: fallbacks.append((r, why)),
                               noise=1e-11, speed_tolerance=1e-10)
    assert len(fallbacks) == 1 and fallbacks[0][0] == 1
    assert f"cell aspect ratio {FALLBACK['aspect_ratio']:.1f} above {FALLBACK['aspect_limit']}" in fallbacks[0][1]
    assert out.kind == "solved" and out.column_density == FALLBACK_COLUMN_DENSITY
    assert out.reports[0].ni == FALLBACK["columns"]
    assert abs(out.result.levels[0][1] / FALLBACK["value"] - 1) < 1e-9


def test_verified_fitted_drag_of_a_blunt_nose():
    # The hemisphere-cylinder at Mach 2 through the verified procedure: one
    # captured start for the family, grids of 20 cells across refined by 2,
    # the nested heights of the refined grids keeping the base heights.
    from bowshock_b200.fitted import blunt_fit_family, blunt_start, verified_fitted_drag
    from bowshock_b200.grid import Body, Nose, NoseShape

    b = HEMI["body"]
    body = Body(Nose(NoseShape(b["shape"]), b["length"], b["base_radius"]), b["cylinder"])
    family = blunt_fit_family(blunt_start(body, HEMI["mach"], 20))
    p1, p2 = family(1), family(2)
    assert np.array_equal(p2.heights[::2], p1.heights) and p2.nj == 40
    out = verified_fitted_drag(body, HEMI["mach"], tolerance=1e-3, max_refinement=8)
    assert out.kind == "solved", out.reason
    v = out.result
    assert v.verified and v.uncertainty <= 1e-3 and len(v.levels) >= 2
    assert abs(v.levels[0][1] - out.reports[0].drag) == 0.0


def test_a_bare_nose_is_solved_with_a_cylinder_only_where_its_base_flow_is_supersonic():
    # tests/analysis/fitted-flow.test.ts:413-426: the bare 20 deg cone at
    # Mach 3, solved on a caliber of cylinder, leaves its base at Mach 2; the
    # same grid with the flow slowed to Mach 0.42 is refused.
    from bowshock_b200.fitted import base_mach
    from bowshock_b200.grid import Body, Nose, NoseShape

    bare = Body(Nose(NoseShape("conical"), 0.5 / math.tan(20 * math.pi / 180), 0.5), 0.0)
    p = sharp_fit_problem(bare, 3.0, nj=20)
    with CudaFit(p) as g:
        converged, _, _, _ = settle(g, 20000, check_every=250)
        prims = g.primitives().reshape(p.nj, p.ni, 4)
    assert converged
    assert base_mach(p, bare.nose.length, prims) > 1
    slow = np.tile([1.0, 0.5, 0.0, 1.0], (p.nj, p.ni, 1))
    assert base_mach(p, bare.nose.length, slow) < 1


def test_verified_fitted_drag_without_convergence_gives_only_the_reason():
    # tests/analysis/fitted-flow.test.ts:569-588: ten steps per grid.
    from bowshock_b200.fitted import verified_fitted_drag

    out = verified_fitted_drag(cone_body(20, 1.0), 3.0, tolerance=0.0, floor=0.0, max_refinement=8,
                               iterations_per_refinement=10)
    assert out.kind == "not-converged" and out.refinement == 1 and out.result is None
    assert "the fit stopped after 10 iterations" in out.reason
