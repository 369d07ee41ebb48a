"""The seeded batch of uneven cases: SplitMix64 draws, the case distribution
(nose family, fineness, body length, Mach number, grid level) and grid
construction on the host threads. No GPU."""
from __future__ import annotations

from bowshock_b200.workloads import (NOSE_FAMILIES, SplitMix64, case_from, draw_nose_case,
                                     seeded_cases)


def test_splitmix64_is_a_pure_function_of_the_seed():
    a, b = SplitMix64(42), SplitMix64(42)
    xs = [a.next_u64() for _ in range(8)]
    assert xs == [b.next_u64() for _ in range(8)]
    assert len(set(xs)) == 8 and all(0 <= x < 2**64 for x in xs)
    assert xs != [SplitMix64(43).next_u64() for _ in range(8)]


def test_draws_follow_the_distribution():
    specs = [draw_nose_case(s) for s in range(1, 401)]
    assert {s.family for s in specs} == set(NOSE_FAMILIES)
    assert all(1.0 <= s.fineness <= 5.0 and 2.0 <= s.body_length <= 8.0 for s in specs)
    assert all(1.5 <= s.mach <= 5.0 for s in specs)
    assert {s.ni for s in specs} == {40, 80, 160, 320}
    assert all(s.nj == s.ni // 2 for s in specs)
    assert draw_nose_case(17) == draw_nose_case(17)


def test_cylinder_is_body_length_less_the_nose():
    for seed in range(1, 50):
        nc = draw_nose_case(seed)
        body = nc.body()
        assert body.nose.length == 2 * 0.5 * nc.fineness
        assert body.cylinder_length == max(0.0, nc.body_length - body.nose.length)


def test_seeded_cases_build_grids_on_host_threads():
    made, refused = seeded_cases(12, first_seed=1, levels=(0,))
    assert len(made) + len(refused) == 12
    assert len(made) >= 10
    for case in made:
        cfg = case.config
        assert (cfg.grid.ni, cfg.grid.nj) == (40, 20)
    # The same seed builds the same grid.
    first = next(s for s in range(1, 13) if draw_nose_case(s, levels=(0,)).family != "ellipsoid")
    a = case_from(draw_nose_case(first, levels=(0,)))
    b = case_from(draw_nose_case(first, levels=(0,)))
    assert a.name == b.name
    assert (a.config.grid.x == b.config.grid.x).all() and (a.config.grid.y == b.config.grid.y).all()
