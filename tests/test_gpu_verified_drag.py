"""The verified-drag driver on the GPU engine: each grid of the family solved
until its drag settles gives the drag the reference's FP64 CPU engine gives
on the same grid (tests/gpu/verified-drag-gpu.test.ts:16-46 pins r = 1 and
2), and the batched driver gives every case what the single one gives."""
from __future__ import annotations

import json
import math
from pathlib import Path

import pytest

from bowshock_b200.grid import Body, Nose, NoseShape
from bowshock_b200.verified_drag import verified_forebody_drag, verified_forebody_drags

pytestmark = pytest.mark.gpu

PIN = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())[
    "verified_drag_cone20_mach3"]


def _cone(cylinder):
    b = PIN["body"]
    half = b["half_angle_deg"] * math.pi / 180
    return Body(Nose(NoseShape("conical"), b["base_radius"] / math.tan(half), b["base_radius"]), cylinder)


def test_settled_drags_match_the_reference_pins():
    res = verified_forebody_drag(_cone(PIN["body"]["cylinder"]), PIN["mach"], max_refinement=2)
    assert res.kind == "solved"
    drags = [r.drag for r in res.reports]
    assert [r.refinement for r in res.reports] == PIN["refinements"]
    for got, want in zip(drags, PIN["drag"]):
        assert abs(got / want - 1) < PIN["tolerance_relative"]
    # Two grids give no band yet (four are needed).
    assert res.result.estimate.kind == "unresolved" and not res.result.verified


def test_batched_driver_gives_each_case_what_the_single_driver_gives():
    cases = [(_cone(2.0), 3.0), (_cone(4.0), 2.5)]
    batched = verified_forebody_drags(cases, max_refinement=2)
    for (body, mach), got in zip(cases, batched):
        one = verified_forebody_drag(body, mach, max_refinement=2)
        assert got.kind == one.kind == "solved"
        assert [r.refinement for r in got.reports] == [r.refinement for r in one.reports]
        for a, b in zip(got.reports, one.reports):
            assert a.drag == pytest.approx(b.drag, rel=1e-12)
            assert a.iterations == b.iterations
