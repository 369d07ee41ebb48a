"""Every tile shape of the residual pass computes the same steps.

The autotuner picks the tile shape the residual pass and the explicit stages
run with (bs_batch_set_tile_shape); the shape only decides which CTA
computes which cell, so the state after any number of steps must be the
same bit for bit whatever the shape, on grids whose sizes are multiples of
no tile size and in a batch of uneven cases. The same holds for the LU-SGS
update mode the autotuner also picks: the update applied inside the next
residual pass or by a separate kernel after each sweep.
"""
from __future__ import annotations

import numpy as np
import pytest

from bowshock_b200.batch import CudaBatch
from bowshock_b200.workloads import ogive_case

pytestmark = pytest.mark.gpu

SHAPES = [-1, 0, 1, 2, 3, 4, 5, 6, 7]


def cases():
    return [ogive_case(2.2, 40, 20), ogive_case(1.7, 58, 27), ogive_case(3.1, 100, 45)]


def states_after(shape: int, method: str, fused: bool = True) -> list[np.ndarray]:
    cs = cases()
    b = CudaBatch([c.config for c in cs], precision=64)
    try:
        b.set_tile_shape(shape)
        b.set_update_mode(fused)
        t = b.tuning()
        assert t["tile_shape"] == shape and t["fused_update"] == fused
        b.set_free_stream()
        if method == "lusgs":
            # 40 steps: tolerance out of reach, so every case takes them all.
            res = b.solve("lusgs", 1e-14, max_steps=40, check_every=20)
            assert all(r.steps == 40 for r in res)
        else:
            b.iterate(30)
        return [b.primitives(k) for k in range(len(cs))]
    finally:
        b.destroy()


@pytest.mark.parametrize("method", ["lusgs", "explicit"])
def test_every_tile_shape_takes_the_same_steps(method):
    ref = states_after(-1, method)
    for shape in SHAPES[1:]:
        got = states_after(shape, method)
        for a, b in zip(ref, got):
            assert np.array_equal(a, b), (method, shape)


@pytest.mark.parametrize("shape", [-1, 2])
def test_the_update_applied_in_the_residual_pass_or_after_the_sweep_gives_the_same_steps(shape):
    # The fused residual pass applies the previous step's correction to every
    # cell it reads with the update kernel's own arithmetic, so 40 steps end
    # on the same state either way, bit for bit.
    fused = states_after(shape, "lusgs", True)
    separate = states_after(shape, "lusgs", False)
    for a, b in zip(fused, separate):
        assert np.array_equal(a, b), shape


@pytest.mark.parametrize("env", [{"BOWSHOCK_NO_PDL": "1"}, {"BOWSHOCK_SWEEP_CHUNK": "16"},
                                 {"BOWSHOCK_SWEEP_CHUNK": "2"}])
def test_launch_modes_leave_the_steps_unchanged(env, monkeypatch):
    # The launch switches (read when a batch is created) change how the
    # residual pass and the sweep are launched and how many diagonals one
    # bulk copy brings, not what they compute: 40 steps end on the same state.
    ref = states_after(-1, "lusgs")
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    got = states_after(-1, "lusgs")
    for a, b in zip(ref, got):
        assert np.array_equal(a, b), env


def test_one_diagonal_chunks_reach_the_same_steady_state(monkeypatch):
    # Chunks of one diagonal leave the sweep's step loop without unrolling, and
    # its FP32 operator then rounds a little differently (about 1e-8 after two
    # steps, the same in every run): the path to the steady state moves at
    # that level, the steady state and its drag do not.
    def drags():
        cs = cases()
        b = CudaBatch([c.config for c in cs], precision=64)
        try:
            b.set_free_stream()
            res = b.solve("lusgs", 1e-10, max_steps=4000)
            assert all(r.status == 0 for r in res)
            return [b.forebody_drag(k, c.free, c.body.nose.base_radius) for k, c in enumerate(cs)]
        finally:
            b.destroy()

    ref = drags()
    monkeypatch.setenv("BOWSHOCK_SWEEP_CHUNK", "1")
    for a, b in zip(ref, drags()):
        assert abs(b / a - 1) < 1e-12


def test_autotune_picks_a_shape_and_keeps_the_state():
    cs = cases()
    b = CudaBatch([c.config for c in cs], precision=64)
    try:
        b.set_free_stream()
        b.solve("lusgs", 1e-14, max_steps=20, check_every=20)
        before = [b.primitives(k) for k in range(len(cs))]
        lanes, ms = b.autotune("lusgs", 10)
        t = b.tuning()
        assert t["lanes"] == lanes and -1 <= t["tile_shape"] < 8 and ms > 0
        for k in range(len(cs)):
            assert np.array_equal(b.primitives(k), before[k])
    finally:
        b.destroy()


def test_autotune_cache_applies_a_grid_size_class_choice():
    # A batch of a class tuned before takes the stored lanes, tile shape and
    # update mode instead of timing them, and steps to the same state as an
    # untuned batch.
    from bowshock_b200 import abi, batch as batch_module

    cs = cases()
    first = CudaBatch([c.config for c in cs], precision=64)
    try:
        first.set_free_stream()
        batch_module._TUNED.pop(first.size_class("lusgs"), None)
        first.autotune("lusgs", 20, cache=True)
        chosen = first.tuning()
    finally:
        first.destroy()
    assert first.size_class("lusgs") in batch_module._TUNED
    ref = states_after(-1, "lusgs")
    second = CudaBatch([c.config for c in cs], precision=64)
    try:
        second.set_free_stream()
        second.autotune("lusgs", 20, cache=True)
        assert second.tuning() == chosen
        res = second.solve("lusgs", 1e-14, max_steps=40, check_every=20)
        assert all(r.steps == 40 for r in res)
        for k in range(len(cs)):
            assert np.array_equal(second.primitives(k), ref[k])
        for bad in (0, len(cs) + 1):
            assert second._lib.bs_batch_set_lanes(second._h, bad) == abi.BS_INVALID_ARGUMENT
    finally:
        second.destroy()
