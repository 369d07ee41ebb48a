"""Failure detection on the device, through the C ABI, without a GPU fault.

A step that turns a cell non-physical is flagged by the kernel that wrote it
(the per-case status word the reference's update shader sets with atomicOr,
src/engine-gpu/shaders/euler2d.wgsl:265-269, 486-490) and surfaces as
NonPhysicalStateError, as the CPU engine's checkPhysical raises it
(src/engine-cpu/euler2d.ts:1471-1483). An LU-SGS sweep whose bounded wait
runs out (made to run out here by a wait limit of zero polls, while the
drain of its copies keeps the full bound) leaves the state as it was, the
call returns BS_EXECUTION and the engine goes on working.
"""
from __future__ import annotations

import numpy as np
import pytest

from bowshock_b200 import abi
from bowshock_b200._native import BowshockError, NonPhysicalStateError
from bowshock_b200.config import Boundary, Euler2DConfig, grid_from_function
from bowshock_b200.engine import CudaEuler2D
from bowshock_b200.workloads import ogive_case
from oracle.oracle import OracleEuler2D, OracleError

pytestmark = pytest.mark.gpu


def emptied_cell_case():
    """A cold cell at rest (p = 1e-10) between flows leaving it at speed 10
    on both sides. Its local time step, set by its own tiny sound speed, is
    far too long for the fluxes of its neighbours: one explicit step takes
    more mass out of it than it holds. The start itself is physical."""
    ni, nj = 9, 3
    grid = grid_from_function(ni, nj, lambda i, j: (i / ni, j / nj))
    b = Boundary("outflow")
    cfg = Euler2DConfig(grid=grid, geometry="planar", gamma=1.4, flux="hllc", limiter="minmod",
                        reconstruction="perVariable", time_integrator="forwardEuler", cfl=0.5,
                        time_stepping="local", boundaries={"iMin": b, "iMax": b, "jMin": b, "jMax": b})
    w = np.zeros((nj, ni, 4))
    w[..., 0] = 1.0
    w[..., 3] = 1.0
    w[:, :4, 1] = -10.0
    w[:, 5:, 1] = 10.0
    w[:, 4, 3] = 1e-10
    return cfg, w.reshape(-1)


@pytest.mark.parametrize("precision", [64, 32])
def test_a_step_that_empties_a_cell_is_flagged_on_the_device(precision):
    cfg, w = emptied_cell_case()
    o = OracleEuler2D(cfg)
    o.set_primitives(w)
    with pytest.raises(OracleError, match="NON_PHYSICAL"):
        o.iterate(1)
    with CudaEuler2D(cfg, precision) as e:
        e.set_primitives(w)  # passes the host's check
        with pytest.raises(NonPhysicalStateError):
            e.iterate(1)
        # The engine goes on: a fresh physical start steps cleanly.
        e.set_primitives(np.tile([1.0, 0.1, 0.0, 1.0], cfg.grid.ni * cfg.grid.nj))
        e.iterate(3)
        assert np.all(np.isfinite(e.primitives()))


def test_a_sweep_that_gives_up_waiting_leaves_the_state_and_the_engine_usable():
    case = ogive_case(2.0, 40, 20)
    with CudaEuler2D(case.config, 64) as e:
        e.set_uniform(case.free.state)
        e.iterate_implicit(5, 5.0)
        before = e.primitives()
        e.set_sweep_wait_limit(0)   # every sweep gives up at its first wait
        with pytest.raises(BowshockError) as info:
            e.iterate_implicit(1, 5.0)
        assert info.value.status == abi.BS_EXECUTION
        assert "gave up waiting" in str(info.value)
        assert np.array_equal(e.primitives(), before)
        e.set_sweep_wait_limit(-1)
        e.iterate_implicit(3, 5.0)
        after = e.primitives()
    # The same 5 + 3 steps without the failed one.
    with CudaEuler2D(case.config, 64) as ref:
        ref.set_uniform(case.free.state)
        ref.iterate_implicit(5, 5.0)
        ref.iterate_implicit(3, 5.0)
        assert np.array_equal(after, ref.primitives())


def test_a_solve_whose_sweep_gives_up_reports_an_execution_error():
    from bowshock_b200.batch import CudaBatch

    cases = [ogive_case(m, 40, 20) for m in (1.8, 2.4)]
    b = CudaBatch([c.config for c in cases], precision=64)
    try:
        b.set_free_stream()
        b.set_sweep_wait_limit(0)
        res = b.solve("lusgs", 1e-6, max_steps=40, check_every=20)
        assert [r.status for r in res] == [abi.BS_EXECUTION] * 2
        b.set_sweep_wait_limit(-1)
        res = b.solve("lusgs", 1e-6, max_steps=20000, check_every=20)
        assert all(r.status == 0 for r in res)
    finally:
        b.destroy()
