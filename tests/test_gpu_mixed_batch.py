"""One batch of uneven cases against the FP64 oracle, case by case.

The batched path packs cases of every grid level (40 x 20 to 640 x 320),
H grids of sharp noses and C grids of blunt and two-scale ones, into shared
arenas at per-case offsets and runs them as lanes of concurrent step chains.
A packing or offset mistake that shows only with mixed sizes would leave
some case with the wrong answer, so every case is held to the oracle:

  - with two-float metrics (the residual's metrics to about 48 bits), each
    converged GPU field is a steady state of the oracle's own FP64 discrete
    equations: the oracle's RMS density residual of that field is at most
    the 1e-6 the GPU marched to, and the oracle's FP64 wall-pressure drag of
    it equals the GPU's to 1e-9;
  - the two smaller levels are also solved by the oracle from the free
    stream: drag within 1e-4 relative, density and pressure within an L1
    distance of 1e-5 of their mean;
  - with FP32 metrics (the production setting) the same batch's drags stay
    within 1e-4 of the oracle's solves.
The reference's CPU engine is the oracle (src/engine-cpu/euler2d.ts); the
cases are drawn from the batched distribution's families (nose shapes of
src/geometry/nose.ts on the generated grids of src/grid/body-grid.ts and
src/grid/blunt-grid.ts).
"""
from __future__ import annotations

import numpy as np
import pytest

from bowshock_b200.batch import CudaBatch
from bowshock_b200.workloads import NoseCase, case_from
from oracle.oracle import OracleEuler2D, parallel_solve

pytestmark = pytest.mark.gpu

# (family, fineness, body length, Mach, ni): H grids for the sharp noses whose
# shock stays attached, C grids for the ellipsoids and the Haack nose.
SPECS = [
    ("ogive", 3.0, 6.0, 2.0, 40),
    ("ellipsoid", 1.5, 4.0, 2.5, 40),
    ("conical", 2.0, 5.0, 3.0, 80),
    ("haack", 3.0, 6.0, 2.0, 80),
    ("parabolic", 3.0, 6.0, 2.2, 160),
    ("ellipsoid", 2.0, 5.0, 2.0, 160),
    ("ogive", 4.0, 7.0, 2.5, 320),
    ("conical", 3.0, 6.0, 2.0, 640),
]
TOL = 1e-6


@pytest.fixture(scope="module")
def cases():
    out = [case_from(NoseCase(k, fam, f, L, m, ni, ni // 2)) for k, (fam, f, L, m, ni) in enumerate(SPECS)]
    kinds = {c.config.boundaries["iMin"].kind for c in out}
    assert kinds == {"inflow", "wall"}  # both grid topologies are in the batch
    return out


def solve_batch(cases, metric_bits: int):
    b = CudaBatch([c.config for c in cases], precision=64)
    try:
        b.set_metric_precision(metric_bits)
        b.set_free_stream()
        res = b.solve("lusgs", TOL, relative=False, max_steps=40000, check_every=20, cfl=5.0, omega=1.5)
        prims = [b.primitives(k) for k in range(len(cases))]
        drags = [b.forebody_drag(k, c.free, c.body.nose.base_radius) for k, c in enumerate(cases)]
        return res, prims, drags
    finally:
        b.destroy()


@pytest.fixture(scope="module")
def small_oracle(cases):
    """The oracle's own solves of the two smaller levels, from the free stream."""
    small = [k for k, c in enumerate(cases) if c.config.grid.ni <= 80]
    engines = []
    for k in small:
        o = OracleEuler2D(cases[k].config)
        o.set_uniform(cases[k].free.state)
        engines.append(o)
    status, steps, res, init = parallel_solve(engines, "lusgs", TOL, 40000, 20, cfl=5.0, omega=1.5,
                                              relative=False, threads=len(engines))
    assert all(s == 0 for s in status)
    out = {}
    for k, o in zip(small, engines):
        c = cases[k]
        out[k] = (o.primitives().reshape(-1, 4),
                  o.forebody_drag(c.free.pressure, c.free.dynamic_pressure, c.body.nose.base_radius))
    return out


def test_every_case_of_a_mixed_batch_is_a_steady_state_of_the_oracle(cases, small_oracle):
    res, prims, drags = solve_batch(cases, 64)
    for k, (c, r) in enumerate(zip(cases, res)):
        assert r.status == 0, (c.name, r.status, r.residual)
        assert r.residual <= TOL, c.name
        o = OracleEuler2D(c.config)
        o.set_primitives(prims[k].reshape(-1))
        r_oracle = o.density_residual_norm()
        assert r_oracle <= TOL * (1 + 1e-3), (c.name, r_oracle)
        cd_oracle = o.forebody_drag(c.free.pressure, c.free.dynamic_pressure, c.body.nose.base_radius)
        assert abs(drags[k] / cd_oracle - 1) < 1e-9, (c.name, drags[k], cd_oracle)
        if k in small_oracle:
            w_ref, cd_ref = small_oracle[k]
            assert abs(drags[k] / cd_ref - 1) < 1e-4, (c.name, drags[k], cd_ref)
            for v in (0, 3):  # density, pressure
                l1 = np.mean(np.abs(prims[k][:, v] - w_ref[:, v])) / np.mean(np.abs(w_ref[:, v]))
                assert l1 < 1e-5, (c.name, v, l1)


def test_the_production_batch_meets_the_oracle_drags(cases, small_oracle):
    res, prims, drags = solve_batch(cases, 32)
    for k, (c, r) in enumerate(zip(cases, res)):
        assert r.status == 0, (c.name, r.status, r.residual)
        assert r.residual <= TOL, c.name
        if k in small_oracle:
            assert abs(drags[k] / small_oracle[k][1] - 1) < 1e-4, c.name
        else:
            # The oracle's FP64 drag of the GPU's own field: the wall fluxes of
            # the batch's packed boundary geometry, case by case.
            o = OracleEuler2D(c.config)
            o.set_primitives(prims[k].reshape(-1))
            cd = o.forebody_drag(c.free.pressure, c.free.dynamic_pressure, c.body.nose.base_radius)
            assert abs(drags[k] / cd - 1) < 1e-6, c.name
