"""Solution verification (bowshock_b200.verification) and the verified-drag
driver's refusals, on the cases the reference tests them with
(tests/verification/grid-convergence.test.ts, iterative-convergence.test.ts,
tests/analysis/verified-drag.test.ts). No GPU: the driver runs over fake
engines here."""
from __future__ import annotations

import json
import math
from pathlib import Path

import pytest

from bowshock_b200.config import Primitive2D
from bowshock_b200.engine import BoundaryFaceFlux
from bowshock_b200.grid import Body, Nose, NoseShape
from bowshock_b200.verification import SettlingValue, grid_convergence, refine_until_verified
from bowshock_b200.verified_drag import verified_forebody_drag

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())
OPT = dict(order_tolerance=0.3, noise=1e-12)


def family(phi, grids=4):
    return [phi(2.0 ** -k) for k in range(grids)]


def test_second_order_family_recovers_order_limit_and_band():
    e = grid_convergence(family(lambda h: 0.3 + 0.04 * h * h), **OPT)
    assert e.kind == "monotone"
    assert e.order == pytest.approx(2, abs=1e-12)
    assert e.extrapolated == pytest.approx(0.3, abs=1e-14)
    assert e.uncertainty / abs(e.value - 0.3) == pytest.approx(1.25, abs=1e-10)


def test_first_order_band_and_order_cap():
    e = grid_convergence(family(lambda h: -1 + 0.2 * h), **OPT)
    assert e.order == pytest.approx(1, abs=1e-12)
    assert e.uncertainty / abs(e.value + 1) == pytest.approx(1.25, abs=1e-10)
    e = grid_convergence(family(lambda h: 2 + 0.5 * h ** 3), **OPT)
    assert e.order == pytest.approx(3, abs=1e-12)
    assert e.uncertainty > 1.25 * abs(e.value - 2)


def test_asymptotic_range_oscillation_and_unresolved_cases():
    phi = lambda h: 1 + 0.1 * h + 5 * h ** 4  # noqa: E731
    e = grid_convergence(family(phi), **OPT)
    assert e.kind == "unresolved" and "orders of the two finest triples differ" in e.reason
    assert grid_convergence(family(phi, 9), **OPT).kind == "monotone"
    e = grid_convergence([1, 1.1, 1.05, 1.07], **OPT)
    assert e.kind == "oscillatory" and e.uncertainty == pytest.approx(0.05, abs=1e-12)
    for values, reason in (([1, 1.001, 1.003, 1.007], "do not shrink"),
                           ([1, 1, 1, 1], "too small to measure"), ([1.2, 1.1, 1.05], "four grids")):
        e = grid_convergence(values, **OPT)
        assert e.kind == "unresolved" and reason in e.reason


def test_finest_change_below_noise_is_bounded_by_the_coarser_order():
    noise = 1e-6
    exact = family(lambda h: 1 + 1e-4 * h * h)
    e = grid_convergence(exact, order_tolerance=0.3, noise=noise)
    assert e.kind == "monotone" and e.order == pytest.approx(2, abs=1e-6)
    assert e.uncertainty == pytest.approx(1.25 * (1e-4 * (0.25 ** 2 - 0.125 ** 2) + 2e-6) / 3, abs=1e-9)
    e = grid_convergence([1.0005, 1.0001, 1, 1], order_tolerance=0.3, noise=1e-6)
    assert e.kind == "unresolved" and "below the noise but not the one" in e.reason


@pytest.mark.parametrize("fam", GOLDEN["grid_convergence_cone_families"]["families"], ids=lambda f: f["name"])
def test_measured_cone_families_band_contains_the_true_error(fam):
    o = GOLDEN["grid_convergence_cone_families"]["options"]
    values = fam["values"]
    res = refine_until_verified(lambda r: values[int(math.log2(r))], tolerance=math.inf, floor=o["floor"],
                                max_refinement=o["max_refinement"], order_tolerance=o["order_tolerance"],
                                noise=o["noise"])
    if res.uncertainty is not None:
        assert abs(res.estimate.value - fam["exact"]) <= res.uncertainty


def test_a_finer_grid_that_fails_keeps_the_coarser_result_where_allowed():
    values = [1.04, 1.01, 1.0025]

    def solve_at(r):
        if r == 8:
            raise RuntimeError("too large for this GPU")
        return values[int(math.log2(r))]

    base = dict(tolerance=0, floor=0, order_tolerance=0.5, noise=1e-12)
    coarser = refine_until_verified(solve_at, max_refinement=4, **base)
    stopped = refine_until_verified(solve_at, max_refinement=8, stop_on=lambda e: str(e), **base)
    assert stopped.stopped == (8, "too large for this GPU")
    assert stopped.levels == coarser.levels and stopped.uncertainty == coarser.uncertainty
    with pytest.raises(RuntimeError):
        refine_until_verified(solve_at, max_refinement=8, **base)


def test_settling_value_settles_near_the_limit_of_a_geometric_iteration():
    for rate in (0.1, 0.5, 0.85):
        s, limit, noise = SettlingValue(1e-8), 2.0, 1e-8
        for n in range(400):
            v = limit + 1e4 * noise * limit * rate ** n
            if s.add(v):
                break
        assert n < 399 and abs(v - limit) <= 2 * noise * limit


def test_settling_value_never_settles_on_a_drift():
    s = SettlingValue(1e-8)
    assert not any(s.add(1 + 1e-3 * k) for k in range(100))


# ---- the driver's refusals (fake engines, no GPU) ------------------------------

CONE = Body(Nose(NoseShape("conical"), 0.5 / math.tan(20 * math.pi / 180), 0.5), 2.0)
FREE = Primitive2D(1.0, 3 * math.sqrt(1.4), 0.0, 1.0)


class FakeEngine:
    def __init__(self, wall, cell):
        self.calls, self._wall, self._cell = 0, wall, cell

    def iterate(self, steps):
        self.calls += 1

    def wall_fluxes(self):
        return self._wall(self.calls)

    def cells(self):
        return self._cell

    def destroy(self):
        pass


def _face(fx):
    return [BoundaryFaceFlux(1.0, 0.5, 0.3, -0.95, 0.5, (0.0, fx, 0.0, 0.0))]


def test_a_drag_that_never_settles_is_not_converged():
    res = verified_forebody_drag(CONE, 3.0, max_refinement=8, noise=1e-12,
                                 engine_for=lambda cfg, free: FakeEngine(lambda k: _face(1 + k * 1e-3),
                                                                         lambda i, j: FREE))
    assert res.kind == "not-converged" and "still changes" in res.reason


def test_subsonic_outflow_and_a_shock_at_the_outer_boundary_are_invalid():
    sub = Primitive2D(1.0, 0.93 * math.sqrt(1.4), 0.0, 1.0)
    res = verified_forebody_drag(CONE, 3.0, max_refinement=8, noise=1e-12,
                                 engine_for=lambda cfg, free: FakeEngine(lambda k: _face(1.2), lambda i, j: sub))
    assert res.kind == "invalid" and "outflow condition does not hold" in res.reason

    def factory(cfg, free):
        nj = cfg.grid.nj
        return FakeEngine(lambda k: _face(1.2),
                          lambda i, j: Primitive2D(1.2, FREE.u, 0.0, 1.3) if (i, j) == (7, nj - 1) else FREE)

    res = verified_forebody_drag(CONE, 3.0, max_refinement=8, noise=1e-12, engine_for=factory)
    assert res.kind == "invalid" and "bow shock reaches it" in res.reason
