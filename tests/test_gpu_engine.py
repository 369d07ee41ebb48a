"""GPU engine against the FP64 CPU oracle, through the C ABI.

Modelled on the reference's GPU-vs-CPU twin tests (tests/gpu/euler2d-gpu.test.ts)
and its verified-drag pin (tests/gpu/verified-drag-gpu.test.ts). The FP64
engine (FP64 state and residual, FP32 metrics and LU-SGS operator) is held to
tolerances set by its FP32 metrics (about 1e-7 relative); the FP32 engine to
the reference GPU engine's own tolerances.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from bowshock_b200.config import Boundary, Euler2DConfig, Primitive2D, free_stream_at, steady_drag_config
from bowshock_b200.engine import CudaEuler2D, NonPhysicalStateError, cuda_engine, forebody_pressure_drag
from bowshock_b200.grid import body_grid
from oracle.oracle import OracleEuler2D

from cases import GAMMA, cone_body, config1, distorted_grid, uniform_primitives

pytestmark = pytest.mark.gpu


def all_sides(b: Boundary) -> dict:
    return {"iMin": b, "iMax": b, "jMin": b, "jMax": b}


def pulse_config(precision_tag: str = "") -> Euler2DConfig:
    """A smooth pressure pulse on a randomly distorted grid (the reference's
    local-stepping twin test, tests/gpu/euler2d-gpu.test.ts:421-449)."""
    grid = distorted_grid(16, 12, 0, 2, 0, 1.5)
    return Euler2DConfig(grid=grid, geometry="planar", gamma=GAMMA, flux="hllc", limiter="vanLeer",
                         reconstruction="perVariable", time_integrator="ssprk2", cfl=0.6,
                         time_stepping="local", boundaries=all_sides(Boundary("outflow")))


def pulse(x: float, y: float) -> Primitive2D:
    return Primitive2D(1.0, 0.3, 0.1, 1 + 0.3 * math.exp(-8 * ((x - 1) ** 2 + (y - 0.75) ** 2)))


def field_primitives(engine, field) -> np.ndarray:
    cx, cy = engine.centroids()
    return np.array([tuple(field(x, y).__dict__.values()) for x, y in zip(cx, cy)])


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("geometry", ["planar", "axisymmetric"])
def test_uniform_flow_is_preserved_on_a_distorted_grid(precision, geometry):
    # tests/gpu/euler2d-gpu.test.ts:90-115
    w = Primitive2D(1.2, 0.7, -0.4 if geometry == "planar" else 0.0, 0.9)
    grid = distorted_grid(12, 10, 0, 2, 0.5, 1.5)
    cfg = Euler2DConfig(grid=grid, geometry=geometry, gamma=GAMMA, flux="hllc", limiter="vanLeer",
                        reconstruction="perVariable", time_integrator="ssprk2", cfl=0.5,
                        time_stepping="global", boundaries=all_sides(Boundary("inflow", w)))
    with CudaEuler2D(cfg, precision) as e:
        e.set_uniform(w)
        e.iterate(60)
        p = e.primitives()
    tol = 1e-5
    assert np.max(np.abs(p[:, 0] - w.rho)) < tol
    assert np.max(np.abs(p[:, 1] - w.u)) < tol
    assert np.max(np.abs(p[:, 2] - w.v)) < tol
    assert np.max(np.abs(p[:, 3] - w.p)) < tol


def test_residual_and_time_steps_match_the_oracle():
    cfg = pulse_config()
    o = OracleEuler2D(cfg)
    with CudaEuler2D(cfg, 64) as e:
        w = field_primitives(e, pulse)
        e.set_primitives(w)
        o.set_primitives(w)
        r_gpu = e.residual_vector()
        dt_gpu = e.time_steps()
        norm_gpu = e.density_residual_norm()
    r_cpu = o.residual()
    # The residual is a sum of O(p A) face fluxes; the GPU's FP32 metrics
    # perturb each by about 1e-7 of itself.
    i_faces, j_faces, _ = o.metrics()
    flux_scale = np.max(w[:, 3]) * max(np.max(i_faces[:, 2]), np.max(j_faces[:, 2]))
    assert np.max(np.abs(r_gpu - r_cpu)) < 1e-6 * flux_scale
    dt_cpu = o.time_steps()
    assert np.max(np.abs(dt_gpu / dt_cpu - 1)) < 1e-6
    assert abs(norm_gpu / o.density_residual_norm() - 1) < 1e-6


@pytest.mark.parametrize("precision,tol", [(64, 1e-6), (32, 1e-5)])
def test_local_time_stepping_matches_the_oracle_step_by_step(precision, tol):
    # tests/gpu/euler2d-gpu.test.ts:421-449: 20 local steps, p within 1e-5.
    cfg = pulse_config()
    o = OracleEuler2D(cfg)
    with CudaEuler2D(cfg, precision) as e:
        w = field_primitives(e, pulse)
        e.set_primitives(w)
        o.set_primitives(w)
        e.iterate(20)
        o.iterate(20)
        assert e.steps == 20
        p_gpu = e.primitives()[:, 3]
    p_cpu = o.primitives()[3::4]
    assert np.max(np.abs(p_gpu - p_cpu)) < tol


@pytest.mark.parametrize("integrator", ["forwardEuler", "ssprk2", "ssprk3"])
@pytest.mark.parametrize("recon,limiter", [("perVariable", "minmod"), ("shared", "vanAlbada"),
                                           ("sharedScaled", "vanAlbada"),
                                           ("perVariable", "monotonizedCentral")])
def test_schemes_match_the_oracle(integrator, recon, limiter):
    cfg, free, _ = config1(40, 20)
    cfg = Euler2DConfig(**{**cfg.__dict__, "time_integrator": integrator, "reconstruction": recon,
                           "limiter": limiter, "cfl": 0.5})
    o = OracleEuler2D(cfg)
    o.set_uniform(free.state)
    o.iterate(30)
    with CudaEuler2D(cfg, 64) as e:
        e.set_uniform(free.state)
        e.iterate(30)
        w = e.primitives()
    wc = o.primitives().reshape(-1, 4)
    assert np.max(np.abs(w - wc)) < 1e-6


def test_wall_fluxes_match_the_oracle_on_the_same_state():
    cfg, free, body = config1(40, 20)
    with CudaEuler2D(cfg, 64) as e:
        e.set_uniform(free.state)
        e.iterate(200)
        q = e.read_state().astype(np.float64)
        wall = e.boundary_fluxes("jMin")
        inflow = e.boundary_fluxes("iMin")
        cd = e.forebody_drag(free, body.nose.base_radius)
        w = e.primitives()
    o = OracleEuler2D(cfg)
    o.set_primitives(w)
    ref = o.boundary_fluxes("jMin")
    for a, b in zip(wall, ref):
        assert abs(a.x - b.x) < 1e-15 and abs(a.area - b.area) < 1e-15
        assert abs(a.nx - b.nx) < 1e-15 and abs(a.ny - b.ny) < 1e-15
        for k in range(4):
            assert abs(a.flux[k] - b.flux[k]) < 1e-9 * (1 + abs(b.flux[k]))
        assert abs(a.flux[0]) < 1e-12  # no mass through the wall
    ref_in = o.boundary_fluxes("iMin")
    for a, b in zip(inflow, ref_in):
        for k in range(4):
            assert abs(a.flux[k] - b.flux[k]) < 1e-9 * (1 + abs(b.flux[k]))
    cd_ref = o.forebody_drag(free.pressure, free.dynamic_pressure, body.nose.base_radius)
    assert abs(cd / cd_ref - 1) < 1e-9
    assert abs(forebody_pressure_drag(wall, free, body.nose.base_radius) / cd_ref - 1) < 1e-9
    del q


def test_verified_drag_pin_on_the_gpu():
    # tests/gpu/verified-drag-gpu.test.ts:16-46: the CPU engine's drag on the
    # 20 deg cone at Mach 3 (cylinder 4, nj = 20, refinement 1) is
    # 0.283146976102; the GPU must be within 2e-6 of it.
    body = cone_body(20, 4.0)
    free = free_stream_at(3.0, GAMMA)
    bg = body_grid(body, 20, 3.0, GAMMA)
    cfg = steady_drag_config(bg.grid, free.state)
    engine = cuda_engine()(cfg, free.state)
    try:
        engine.iterate(1500)
        cd = forebody_pressure_drag(engine.wall_fluxes(), free, 0.5)
        assert abs(cd / 0.283146976102 - 1) < 2e-6
        assert engine.engine.density_residual_norm() < 1e-11
        cells = engine.cells()
        assert cells(0, 0).rho > 0
    finally:
        engine.destroy()


def test_verified_drag_pin_with_two_float_metrics_is_the_cpu_engines():
    # The same steady state with two-float metrics in the residual: the GPU
    # drag meets the reference CPU engine's 0.283146976102 as the FP64
    # oracle does (4.2e-9), where the FP32 metrics leave it near 1e-7.
    body = cone_body(20, 4.0)
    free = free_stream_at(3.0, GAMMA)
    bg = body_grid(body, 20, 3.0, GAMMA)
    cfg = steady_drag_config(bg.grid, free.state)
    drags = {}
    for bits in (32, 64):
        with CudaEuler2D(cfg) as e:
            e.set_metric_precision(bits)
            e.set_uniform(free.state)
            e.iterate(1500)
            assert e.density_residual_norm() < 1e-11
            drags[bits] = forebody_pressure_drag(e.boundary_fluxes("jMin"), free, 0.5)
    print(f"cone pin: FP32 metrics {drags[32] / 0.283146976102 - 1:+.2e}, "
          f"two-float {drags[64] / 0.283146976102 - 1:+.2e}")
    assert abs(drags[64] / 0.283146976102 - 1) < 1e-8
    assert abs(drags[32] / 0.283146976102 - 1) < 2e-6


def test_lusgs_reaches_the_explicit_steady_state():
    # tests/engine-cpu/implicit.test.ts:201-240: LU-SGS from CFL 1 up to 1000
    # reaches the explicit scheme's drag; the GPU's FP32 operator changes only
    # the path.
    body = cone_body(15, 1.0)
    free = free_stream_at(2.0, GAMMA)
    bg = body_grid(body, 12, 2.0, GAMMA)
    cfg = steady_drag_config(bg.grid, free.state, boundaries={
        "iMin": Boundary("inflow", free.state), "iMax": Boundary("outflow"),
        "jMin": Boundary("wall"), "jMax": Boundary("farField", free.state)})
    explicit = OracleEuler2D(cfg)
    explicit.set_uniform(free.state)
    explicit.iterate(6000)
    assert explicit.density_residual_norm() < 1e-12
    cd_ref = explicit.forebody_drag(free.pressure, free.dynamic_pressure, 0.5)
    with CudaEuler2D(cfg, 64) as e:
        e.set_uniform(free.state)
        e.set_implicit_cfl(1.0)
        e.iterate_implicit(400, 1000.0, 1.5, 1.2)
        r = e.density_residual_norm()
        cd = e.forebody_drag(free, 0.5)
    assert r < 1e-10
    assert abs(cd / cd_ref - 1) < 1e-7


def test_lusgs_step_matches_the_oracle_early_on():
    cfg, free, _ = config1(40, 20)
    cfg = Euler2DConfig(**{**cfg.__dict__, "limiter": "vanAlbada", "reconstruction": "sharedScaled"})
    o = OracleEuler2D(cfg)
    o.set_uniform(free.state)
    o.iterate_implicit(5, 5.0)
    with CudaEuler2D(cfg, 64) as e:
        e.set_uniform(free.state)
        e.iterate_implicit(5, 5.0)
        w = e.primitives()
    wc = o.primitives().reshape(-1, 4)
    assert np.max(np.abs(w - wc)) < 1e-5


def test_fp32_engine_lusgs_steps_match_the_fp32_oracle():
    # The all-FP32 engine (the reference GPU engine's arithmetic) through the
    # same residual pass, records and sweep: five LU-SGS steps against the
    # oracle's FP32 instantiation, to FP32 rounding.
    cfg, free, _ = config1(40, 20)
    o = OracleEuler2D(cfg, 32)
    o.set_uniform(free.state)
    o.iterate_implicit(5, 5.0)
    with CudaEuler2D(cfg, 32) as e:
        e.set_uniform(free.state)
        e.iterate_implicit(5, 5.0)
        w = e.primitives()
    wc = o.primitives().reshape(-1, 4)
    assert np.max(np.abs(w - wc)) < 1e-4


@pytest.mark.parametrize("ni, nj", [(48, 512), (40, 481)])
def test_lusgs_steps_on_grids_512_rows_wide_match_the_oracle(ni, nj):
    # The widest cases the sweep takes: 16 consumer warps (512 rows), and 15
    # full warps and one of a single row (481), with a pulse and a variation
    # along j so that every row's residual is not zero.
    height = 2.0 * nj / ni
    grid = distorted_grid(ni, nj, 0, 2, 0, height)
    cfg = Euler2DConfig(grid=grid, geometry="planar", gamma=GAMMA, flux="hllc", limiter="vanAlbada",
                        reconstruction="perVariable", time_integrator="ssprk2", cfl=0.6,
                        time_stepping="local", boundaries=all_sides(Boundary("outflow")))

    def field(x, y):
        return Primitive2D(1.0 + 0.05 * math.sin(6 * y / height), 0.3, 0.1,
                           1 + 0.3 * math.exp(-8 * ((x - 1) ** 2 + (y - height / 2) ** 2)))

    o = OracleEuler2D(cfg)
    o.set_initial_condition(lambda x, y: tuple(field(x, y).__dict__.values()))
    o.iterate_implicit(5, 5.0)
    with CudaEuler2D(cfg, 64) as e:
        e.set_primitives(field_primitives(e, field))
        e.iterate_implicit(5, 5.0)
        w = e.primitives()
    wc = o.primitives().reshape(-1, 4)
    assert np.max(np.abs(w - wc)) < 1e-5


def test_config1_converges_to_1e6_with_the_oracle_drag():
    cfg, free, body = config1()
    with CudaEuler2D(cfg, 64) as e:
        e.set_uniform(free.state)
        res = e.solve("explicit", tolerance=1e-6, max_steps=20000, check_every=50)
        assert res.status == 0
        assert res.residual <= 1e-6
        cd = e.forebody_drag(free, body.nose.base_radius)
    o = OracleEuler2D(cfg)
    o.set_uniform(free.state)
    st, steps, r, r0 = o.solve("explicit", 1e-6, 20000, 50, relative=False)
    assert st == 0
    cd_ref = o.forebody_drag(free.pressure, free.dynamic_pressure, body.nose.base_radius)
    assert abs(cd / cd_ref - 1) < 1e-4


def test_non_physical_initial_state_is_rejected():
    cfg, free, _ = config1(40, 20)
    with CudaEuler2D(cfg, 64) as e:
        w = uniform_primitives(cfg, Primitive2D(1.0, 0.0, 0.0, -1.0))
        with pytest.raises(NonPhysicalStateError):
            e.set_primitives(w)


def test_overlapping_calls_on_one_engine_return_busy():
    """One operation at a time per engine (ExclusiveRunner,
    src/engine-gpu/gpu-common.ts:122-140): a call made while another thread's
    call runs gets BS_BUSY, and the engine works again afterwards."""
    import threading
    import time

    from bowshock_b200._native import BusyError

    cfg, free, _ = config1()
    with CudaEuler2D(cfg, 64) as e:
        e.set_uniform(free.state)
        worker = threading.Thread(target=e.iterate, args=(6000,))
        worker.start()
        seen = False
        for _ in range(4000):
            try:
                e.density_residual_norm()
            except BusyError:
                seen = True
                break
            time.sleep(0.0002)
        worker.join()
        assert seen
        assert e.steps == 6000
        assert math.isfinite(e.density_residual_norm())


def test_autotune_keeps_the_state_and_the_answer():
    from bowshock_b200.batch import CudaBatch
    from bowshock_b200.workloads import ogive_case

    cases = [ogive_case(m, 40, 20) for m in (1.6, 2.0, 2.4, 2.8, 3.2)]
    results = []
    for tune in (False, True):
        b = CudaBatch([c.config for c in cases], precision=64)
        b.set_free_stream()
        b.solve("lusgs", 1e-6, max_steps=60, check_every=20)  # a state away from the free stream
        before = b.residual_norms()
        if tune:
            lanes, ms = b.autotune("lusgs", 10)
            assert lanes in (1, 2, 4) and ms > 0
            # The state comes back exactly; the norm's FP64 atomic sums may be
            # added in another order.
            assert np.allclose(b.residual_norms(), before, rtol=1e-12, atol=0)
        res = b.solve("lusgs", 1e-6, max_steps=20000, check_every=20)
        assert all(r.status == 0 for r in res)
        results.append([b.forebody_drag(k, c.free, 0.5) for k, c in enumerate(cases)])
        b.destroy()
    assert np.allclose(results[0], results[1], rtol=1e-6, atol=0)


def test_metric_precision_and_accelerated_steps_refuse_and_reduce_as_documented():
    # bs_engine_set_metric_precision takes 32 or 64 bits, and 64 only on the
    # FP64 engine; bs_engine_iterate_accelerated without acceleration (depth
    # 0) is bs_engine_iterate_implicit, state for state.
    from bowshock_b200._native import BowshockError

    body = cone_body(20, 4.0)
    free = free_stream_at(3.0, GAMMA)
    cfg = steady_drag_config(body_grid(body, 10, 3.0, GAMMA).grid, free.state)
    with CudaEuler2D(cfg) as e:
        with pytest.raises(BowshockError, match="32 or 64"):
            e.set_metric_precision(48)
        e.set_metric_precision(64)
        e.set_metric_precision(32)
    with CudaEuler2D(cfg, precision=32) as e:
        with pytest.raises(BowshockError, match="FP32 metrics"):
            e.set_metric_precision(64)
    states = []
    for accelerated in (False, True):
        with CudaEuler2D(cfg) as e:
            e.set_uniform(free.state)
            e.set_implicit_cfl(1.0)
            if accelerated:
                e.set_anderson(0)
                e.iterate_accelerated(40, 50.0, 1.5, 1.2)
            else:
                e.iterate_implicit(40, 50.0, 1.5, 1.2)
            states.append(e.primitives())
    assert np.array_equal(states[0], states[1])
