"""Host logic of the combined stream (no GPU): the cases it draws and the
waves it plans within a device-memory budget."""
from __future__ import annotations

from bowshock_b200.stream import sweep_slots, by_grid_size, case_device_bytes, plan_waves
from bowshock_b200.workloads import STREAM_MACHS, stream_specs


def test_every_geometry_runs_at_every_mach_on_one_grid_level():
    specs = stream_specs(50, first_seed=2_000_001)
    assert len(specs) == 50 * len(STREAM_MACHS)
    for g in range(50):
        four = specs[4 * g:4 * g + 4]
        assert [s.mach for s in four] == list(STREAM_MACHS)
        assert len({(s.seed, s.family, s.fineness, s.body_length, s.ni, s.nj) for s in four}) == 1
    assert {s.ni for s in specs} <= {80, 160, 320, 640}
    assert all(s.nj * 2 == s.ni for s in specs)


def test_waves_are_consecutive_and_within_the_budget():
    specs = stream_specs(200, first_seed=2_000_001)
    budget = 3 * case_device_bytes(640, 320)
    waves = plan_waves(specs, budget)
    assert [k for w in waves for k in w] == list(range(len(specs)))
    for w in waves:
        used = sum(case_device_bytes(specs[k].ni, specs[k].nj) for k in w)
        assert used <= budget or len(w) == 1
    # A wave closes only when the next case would not fit.
    for a, b in zip(waves, waves[1:]):
        used = sum(case_device_bytes(specs[k].ni, specs[k].nj) for k in a)
        nxt = case_device_bytes(specs[b[0]].ni, specs[b[0]].nj)
        assert used + nxt > budget


def test_a_case_larger_than_the_budget_is_a_wave_of_its_own():
    specs = stream_specs(20, first_seed=2_000_001)
    waves = plan_waves(specs, 1)
    assert waves == [[k] for k in range(len(specs))]


def test_device_bytes_grow_with_the_sweep_record_slots():
    # One record slot per cell: 80 x 40 has 3,200 cells.
    assert sweep_slots(80, 40) == 3200
    assert sweep_slots(160, 80) == 12800
    b = case_device_bytes(80, 40)
    assert b == 3200 * 124 + 120 * 16 + 3200 * 160 + 64 * 120
    assert case_device_bytes(640, 320) > 60 * b


def test_waves_by_grid_size_hold_one_size_where_the_budget_allows():
    specs = stream_specs(100, first_seed=2_000_001)
    order = by_grid_size(specs)
    assert sorted(order) == list(range(len(specs)))
    sizes = [specs[k].ni for k in order]
    assert sizes == sorted(sizes)
    waves = plan_waves(specs, 40 * case_device_bytes(640, 320), order)
    assert [k for w in waves for k in w] == order
    mixed = [w for w in waves if len({specs[k].ni for k in w}) > 1]
    assert len(mixed) <= 3     # only where one size ends and the next begins
