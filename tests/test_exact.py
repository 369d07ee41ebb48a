"""Exact solutions in the library's host code against the reference's known
answers: Taylor-Maccoll cones vs NASA SP-3004 and the NPARC case
(tests/validation/taylor-maccoll.test.ts:12-70), shock relations
(tests/validation/gas-dynamics.test.ts)."""
from __future__ import annotations

import json
import math
from pathlib import Path

import pytest

from bowshock_b200 import _native
from bowshock_b200.grid import normal_shock, oblique_shock, taylor_maccoll

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())
DEG = math.pi / 180


@pytest.mark.parametrize("row", GOLDEN["taylor_maccoll_sp3004"]["rows"])
def test_taylor_maccoll_against_sp3004(row):
    cone, mach, shock, surface_mach, cp = row
    tol = GOLDEN["taylor_maccoll_sp3004"]["tolerance"]
    f = taylor_maccoll(mach, cone * DEG)
    assert abs(f.shock_angle - shock) < tol["shock_angle_abs"]
    assert abs(f.surface_mach / surface_mach - 1) < tol["surface_mach_rel"]
    assert abs(f.surface_pressure_coefficient - cp) < tol["cp_abs"]


def test_taylor_maccoll_nparc_case():
    g = GOLDEN["taylor_maccoll_nparc"]
    f = taylor_maccoll(g["mach"], g["cone_deg"] * DEG)
    assert abs(f.post_shock_mach - g["post_shock_mach"]) < 5e-4
    assert abs(f.surface_mach - g["surface_mach"]) < 5e-4
    assert abs(f.surface_mach - g["surface_mach_cfd"]) < 2e-4
    assert abs(f.surface_pressure_ratio - g["surface_pressure_ratio"]) < 5e-4


def test_taylor_maccoll_compresses_isentropically_behind_the_shock():
    for mach, cone in ((1.5, 10), (2, 20), (4, 30)):
        f = taylor_maccoll(mach, cone * DEG)
        assert f.surface_pressure_ratio > f.post_shock_pressure_ratio
        assert f.surface_mach < f.post_shock_mach
        assert f.shock_angle > cone * DEG


def test_detached_cone_is_refused():
    with pytest.raises(_native.BowshockError):
        taylor_maccoll(1.5, 40 * DEG)


def test_oblique_shock_is_consistent():
    s = oblique_shock(2.5, 10 * DEG)
    # the deflection of the found wave angle is the wedge angle
    m2s2 = (2.5 * math.sin(s.beta)) ** 2
    theta = math.atan(2 * (m2s2 - 1) / (math.tan(s.beta) * (2.5**2 * (1.4 + math.cos(2 * s.beta)) + 2)))
    assert abs(theta - 10 * DEG) < 1e-12
    n = normal_shock(2.5 * math.sin(s.beta))
    assert abs(n.pressure_ratio - s.pressure_ratio) < 1e-12
    with pytest.raises(_native.BowshockError):
        oblique_shock(1.5, 30 * DEG)


def test_normal_shock_limits():
    n = normal_shock(1.0)
    assert abs(n.pressure_ratio - 1) < 1e-15 and abs(n.downstream_mach - 1) < 1e-15
    strong = normal_shock(1e4)
    assert abs(strong.density_ratio - 6) < 1e-6  # (gamma + 1) / (gamma - 1)
