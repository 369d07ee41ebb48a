"""The GPU engine behind the reference's plug-in boundary.

`CudaEuler2D` mirrors the method surface of the reference's engines
(`Euler2D`, src/engine-cpu/euler2d.ts:290-1484; `GpuEuler2D`,
src/engine-gpu/euler2d-gpu.ts:183-723) over the C ABI of include/bowshock.h,
and `cuda_engine()` is an `EngineFactory` (src/analysis/verified-drag.ts:33-37)
like `cpuEngine` (:322-332) and `gpuEngine` (src/analysis/gpu-engine.ts:14-41):
it returns a `SteadyEngine` with `iterate`, `wall_fluxes`, `cells` and
`destroy`. Everything runs in the CUDA library; there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Iterable

import numpy as np

from . import _native, abi
from ._native import BowshockError, NonPhysicalStateError  # noqa: F401
from .config import Euler2DConfig, FreeStream, Primitive2D

_dp = C.POINTER(C.c_double)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


@dataclass(frozen=True)
class BoundaryFaceFlux:
    """BoundaryFaceFlux (src/engine-cpu/euler2d.ts:99-113)."""

    x: float
    y: float
    nx: float
    ny: float
    area: float
    flux: tuple[float, float, float, float]


def forebody_pressure_drag(wall: Iterable[BoundaryFaceFlux], free: FreeStream,
                           base_radius: float) -> float:
    """forebodyPressureDrag (src/analysis/forces.ts:19-30), on the host in FP64."""
    force = 0.0
    for face in wall:
        force += (face.flux[1] - free.pressure * face.nx) * face.area
    return (2 * force) / (free.dynamic_pressure * base_radius * base_radius)


class CudaEuler2D:
    """One grid on the GPU. `precision` is 64 (FP64 state and residual,
    FP32 LU-SGS operator; the default) or 32 (all-FP32 field with gamma rounded
    to FP32, the reference GPU engine's arithmetic)."""

    def __init__(self, config: Euler2DConfig, precision: int = 64):
        self._lib = _native.load()
        self.config = config
        self._abi = config.to_abi()
        self.ni = config.grid.ni
        self.nj = config.grid.nj
        self.precision = precision
        h = C.c_void_p()
        _native.check(self._lib.bs_engine_create_ex(C.byref(self._abi), _ptr(config.grid.x),
                                                    _ptr(config.grid.y), precision, C.byref(h)),
                      self._lib)
        self._h = h

    # -- lifetime -----------------------------------------------------------
    def destroy(self) -> None:
        """destroy (src/engine-gpu/euler2d-gpu.ts:673-675)."""
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _native.check(self._lib.bs_engine_destroy(h), self._lib)
        self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def _handle(self) -> C.c_void_p:
        if self._h is None:
            raise RuntimeError("the engine has been destroyed")
        return self._h

    def _call(self, name: str, *args) -> None:
        _native.check(getattr(self._lib, name)(self._handle(), *args), self._lib)

    @property
    def n_cells(self) -> int:
        return self.ni * self.nj

    # -- state ----------------------------------------------------------------
    def centroids(self) -> tuple[np.ndarray, np.ndarray]:
        cx = np.empty(self.n_cells)
        cy = np.empty(self.n_cells)
        self._call("bs_engine_centroids", _ptr(cx), _ptr(cy))
        return cx, cy

    def set_primitives(self, w: np.ndarray) -> None:
        """Four primitives (rho, u, v, p) per cell, cell (i, j) at 4 (i + j ni)."""
        w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
        if w.size != 4 * self.n_cells:
            raise ValueError(f"four values per cell are needed ({4 * self.n_cells})")
        self._call("bs_engine_set_primitives", _ptr(w))

    def set_initial_condition(self, field: Callable[[float, float], Primitive2D]) -> None:
        """setInitialCondition (src/engine-gpu/euler2d-gpu.ts:412-431): the
        field's value at every centroid."""
        cx, cy = self.centroids()
        w = np.empty((self.n_cells, 4))
        for k, (x, y) in enumerate(zip(cx, cy)):
            s = field(x, y)
            w[k] = (s.rho, s.u, s.v, s.p)
        self.set_primitives(w)

    def set_uniform(self, s: Primitive2D) -> None:
        self.set_primitives(np.tile(np.array([s.rho, s.u, s.v, s.p], dtype=np.float64), self.n_cells))

    def set_cell_primitives(self, cell: Callable[[int, int], Primitive2D]) -> None:
        """setCellPrimitives (src/engine-gpu/euler2d-gpu.ts:437-459)."""
        w = np.empty((self.n_cells, 4))
        for j in range(self.nj):
            for i in range(self.ni):
                s = cell(i, j)
                w[i + j * self.ni] = (s.rho, s.u, s.v, s.p)
        self.set_primitives(w)

    def read_state(self) -> np.ndarray:
        """readState (src/engine-gpu/euler2d-gpu.ts:549-571): FP32 conserved
        variables, shape (ni nj, 4)."""
        q = np.empty(4 * self.n_cells, dtype=np.float32)
        self._call("bs_engine_read_state", q.ctypes.data_as(C.POINTER(C.c_float)))
        return q.reshape(-1, 4)

    def primitives(self) -> np.ndarray:
        """Primitives of every cell in FP64 (gpuPrimitive2D,
        src/engine-gpu/euler2d-gpu.ts:136-146), shape (ni nj, 4)."""
        w = np.empty(4 * self.n_cells)
        self._call("bs_engine_read_primitives", _ptr(w))
        return w.reshape(-1, 4)

    def primitive(self, i: int, j: int) -> Primitive2D:
        """primitive(i, j) (src/engine-cpu/euler2d.ts:447-454)."""
        if not (0 <= i < self.ni and 0 <= j < self.nj):
            raise IndexError(f"cell ({i}, {j}) is outside the {self.ni} x {self.nj} grid")
        w = self.primitives()[i + j * self.ni]
        return Primitive2D(*map(float, w))

    @property
    def steps(self) -> int:
        s = C.c_int64()
        self._call("bs_engine_steps", C.byref(s))
        return s.value

    # -- marching -------------------------------------------------------------
    def iterate(self, count: int) -> None:
        """iterate (src/engine-cpu/euler2d.ts:554-560): explicit steps."""
        self._call("bs_engine_iterate", int(count))

    def set_implicit_cfl(self, cfl: float) -> None:
        self._call("bs_engine_set_implicit_cfl", float(cfl))

    def iterate_implicit(self, count: int, cfl: float, omega: float = 1.5,
                         growth: float = 1.0) -> None:
        """LU-SGS steps (iterateImplicit, src/engine-cpu/euler2d.ts:581-589). With
        growth = 1 the CFL number is `cfl` throughout, as on the CPU engine;
        otherwise it ramps from the value set by set_implicit_cfl."""
        if growth == 1.0:
            self.set_implicit_cfl(cfl)
        self._call("bs_engine_iterate_implicit", int(count), float(cfl), float(omega), float(growth))

    def iterate_accelerated(self, count: int, cfl: float, omega: float = 1.5, growth: float = 1.0) -> None:
        """LU-SGS steps with the Anderson acceleration of set_anderson, its
        history kept from call to call (solveTransonic's steps,
        src/analysis/transonic-flow.ts:151-245): plain steps until
        `plain_steps` have been taken since the state or the settings were set,
        accelerated ones after. The CFL number grows by `growth` per step up to
        `cfl` from its current value (set_implicit_cfl)."""
        self._call("bs_engine_iterate_accelerated", int(count), float(cfl), float(omega), float(growth))

    def set_metric_precision(self, bits: int) -> None:
        """64: two-float metrics in the residual (FP32 values plus their FP32
        low parts, as the reference's two-float engine); 32: FP32 metrics."""
        self._call("bs_engine_set_metric_precision", int(bits))

    def set_sweep_wait_limit(self, polls: int) -> None:
        """Polls each bounded wait of later LU-SGS sweeps makes before it
        gives up (-1: the default bound). A sweep that gives up leaves the
        state as it was and the call raises BS_EXECUTION; for tests."""
        self._call("bs_engine_set_sweep_wait_limit", int(polls))

    def anderson_restarts(self) -> int:
        """The times the acceleration forgot its history since its last reset."""
        r = C.c_int32()
        self._call("bs_engine_anderson_restarts", C.byref(r))
        return r.value

    def set_anderson(self, depth: int, plain_steps: int = 30) -> None:
        """Anderson acceleration of later LU-SGS solves (AndersonMixing,
        src/solver/anderson.ts): `depth` differences kept, 0 for plain steps,
        after `plain_steps` plain steps."""
        self._call("bs_engine_set_anderson", int(depth), int(plain_steps))

    def solve(self, method: str = "lusgs", tolerance: float = 1e-6, relative: bool = False,
              max_steps: int = 100000, check_every: int = 20, cfl: float = 5.0,
              omega: float = 1.5) -> abi.SolveResult:
        """March to a steady state: until the FP64 RMS density residual is at
        most `tolerance` (times the starting residual when `relative`)."""
        r = abi.SolveResult()
        st = self._lib.bs_engine_solve(self._handle(), 1 if method == "lusgs" else 0, cfl, omega,
                                       tolerance, 1 if relative else 0, max_steps, check_every,
                                       C.byref(r))
        if st not in (abi.BS_OK, abi.BS_NOT_CONVERGED):
            _native.check(st, self._lib)
        return r

    # -- evaluations ----------------------------------------------------------
    def density_residual_norm(self) -> float:
        """densityResidualNorm (src/engine-cpu/euler2d.ts:480-491), FP64 on the GPU."""
        out = C.c_double()
        self._call("bs_engine_density_residual_norm", C.byref(out))
        return out.value

    def residual_vector(self) -> np.ndarray:
        """residualVector (src/engine-cpu/euler2d.ts:456-472)."""
        r = np.empty(4 * self.n_cells)
        self._call("bs_engine_residual", _ptr(r))
        return r

    def time_steps(self) -> np.ndarray:
        dt = np.empty(self.n_cells)
        self._call("bs_engine_time_steps", _ptr(dt))
        return dt

    def boundary_fluxes(self, side: str = "jMin") -> list[BoundaryFaceFlux]:
        """boundaryFluxes (src/engine-cpu/euler2d.ts:499-525), FP64 on the GPU."""
        n = self.nj if side in ("iMin", "iMax") else self.ni
        out = (abi.FaceFlux * n)()
        self._call("bs_engine_boundary_fluxes", abi.SIDE[side], out)
        return [BoundaryFaceFlux(f.x, f.y, f.nx, f.ny, f.area, tuple(f.flux)) for f in out]

    def forebody_drag(self, free: FreeStream, base_radius: float) -> float:
        """forebodyPressureDrag over the jMin wall (src/analysis/forces.ts:19-30),
        evaluated and reduced in FP64 on the GPU."""
        cd = C.c_double()
        self._call("bs_engine_forebody_drag", free.pressure, free.dynamic_pressure,
                   float(base_radius), C.byref(cd))
        return cd.value


class SteadyEngine:
    """SteadyEngine (src/analysis/verified-drag.ts:22-29) over a CudaEuler2D."""

    def __init__(self, engine: CudaEuler2D):
        self.engine = engine

    def iterate(self, steps: int) -> None:
        self.engine.iterate(steps)

    def wall_fluxes(self) -> list[BoundaryFaceFlux]:
        return self.engine.boundary_fluxes("jMin")

    def cells(self) -> Callable[[int, int], Primitive2D]:
        w = self.engine.primitives()
        ni = self.engine.ni
        return lambda i, j: Primitive2D(*map(float, w[i + j * ni]))

    def destroy(self) -> None:
        self.engine.destroy()


def cuda_engine(precision: int = 64) -> Callable[[Euler2DConfig, Primitive2D], SteadyEngine]:
    """The GPU engine as an EngineFactory, like gpuEngine
    (src/analysis/gpu-engine.ts:14-41): started from the free stream."""

    def factory(config: Euler2DConfig, free_stream: Primitive2D) -> SteadyEngine:
        if config.flux not in ("hllc", "rusanov"):
            raise ValueError(f"the GPU engine has no {config.flux} flux (only hllc and rusanov)")
        e = CudaEuler2D(config, precision)
        e.set_uniform(free_stream)
        return SteadyEngine(e)

    return factory
