"""TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.

ctypes harness over oracle/_build/libbsoracle.so, the C++ restatement of the
reference's FP64 CPU engine (src/engine-cpu/euler2d.ts). Only the tests,
`__graft_entry__.smoke()` and bench.py's CPU-baseline leg use it, as the
checker or as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from bowshock_b200 import abi
from bowshock_b200.config import Euler2DConfig

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libbsoracle.so"

_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (plain IEEE arithmetic)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        dp = C.POINTER(C.c_double)
        vp = C.c_void_p
        L.bso_last_error.restype = C.c_char_p
        L.bso_create.argtypes = [C.POINTER(abi.Config), dp, dp, C.c_int, C.POINTER(vp)]
        L.bso_destroy.argtypes = [vp]
        L.bso_destroy.restype = None
        for name, args in {
            "bso_centroids": [vp, dp, dp],
            "bso_metrics": [vp, dp, dp, dp],
            "bso_set_primitives": [vp, dp],
            "bso_set_conserved": [vp, dp],
            "bso_set_face_states": [vp, C.c_int, dp],
            "bso_set_face_fluxes": [vp, C.c_int, dp],
            "bso_set_quantize": [vp, C.c_int],
            "bso_iterate": [vp, C.c_int],
            "bso_iterate_implicit": [vp, C.c_int, C.c_double, C.c_double],
            "bso_implicit_correction": [vp, C.c_double, C.c_double, dp],
            "bso_density_residual_norm": [vp, dp],
            "bso_residual": [vp, dp],
            "bso_time_steps": [vp, dp],
            "bso_boundary_fluxes": [vp, C.c_int, C.POINTER(abi.FaceFlux)],
            "bso_forebody_drag": [vp, C.c_double, C.c_double, C.c_double, dp],
            "bso_conserved": [vp, dp],
            "bso_primitives": [vp, dp],
            "bso_solve": [vp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                          C.c_int, C.POINTER(C.c_int), dp, dp],
            "bso_parallel_solve": [C.c_int, C.POINTER(vp), C.c_int, C.c_double, C.c_double,
                                   C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.POINTER(C.c_int), dp, dp, C.POINTER(C.c_int)],
        }.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.bso_steps.argtypes = [vp]
        L.bso_steps.restype = C.c_int64
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _check(status: int) -> None:
    if status != abi.BS_OK:
        raise OracleError(status, lib().bso_last_error().decode())


class OracleEuler2D:
    """The FP64 CPU engine (precision=64), or the same code in FP32
    (precision=32, only to predict rounding floors)."""

    def __init__(self, config: Euler2DConfig, precision: int = 64):
        self.config = config
        self._abi = config.to_abi()
        self.ni = config.grid.ni
        self.nj = config.grid.nj
        h = C.c_void_p()
        _check(lib().bso_create(C.byref(self._abi), _dp(config.grid.x), _dp(config.grid.y),
                                precision, C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().bso_destroy(h)
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def n_cells(self) -> int:
        return self.ni * self.nj

    def centroids(self) -> tuple[np.ndarray, np.ndarray]:
        cx = np.empty(self.n_cells)
        cy = np.empty(self.n_cells)
        _check(lib().bso_centroids(self._h, _dp(cx), _dp(cy)))
        return cx, cy

    def metrics(self):
        ni, nj = self.ni, self.nj
        i_faces = np.empty(3 * (ni + 1) * nj)
        j_faces = np.empty(3 * ni * (nj + 1))
        cells = np.empty(4 * ni * nj)
        _check(lib().bso_metrics(self._h, _dp(i_faces), _dp(j_faces), _dp(cells)))
        return i_faces.reshape(-1, 3), j_faces.reshape(-1, 3), cells.reshape(-1, 4)

    def set_primitives(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
        assert w.size == 4 * self.n_cells
        _check(lib().bso_set_primitives(self._h, _dp(w)))

    def set_initial_condition(self, field) -> None:
        """setInitialCondition (euler2d.ts:406-425): field(x, y) -> (rho, u, v, p) at centroids."""
        cx, cy = self.centroids()
        w = np.array([tuple(field(x, y)) for x, y in zip(cx, cy)], dtype=np.float64)
        self.set_primitives(w)

    def set_uniform(self, s) -> None:
        w = np.tile(np.array([s.rho, s.u, s.v, s.p], dtype=np.float64), self.n_cells)
        self.set_primitives(w)

    def set_face_states(self, side: str, prims: np.ndarray) -> None:
        """setFaceStates (src/engine-cpu/euler2d.ts:356-366): primitives
        outside each face of a 'faceStates' side."""
        p = np.ascontiguousarray(prims, dtype=np.float64).reshape(-1)
        _check(lib().bso_set_face_states(self._h, abi.SIDE[side], _dp(p)))

    def set_face_fluxes(self, side: str, fluxes: np.ndarray | None) -> None:
        """setFaceFluxes (:368-390): fluxes per unit area imposed on each face
        of a 'faceStates' side, or None for the Riemann flux."""
        if fluxes is None:
            _check(lib().bso_set_face_fluxes(self._h, abi.SIDE[side], None))
            return
        f = np.ascontiguousarray(fluxes, dtype=np.float64).reshape(-1)
        _check(lib().bso_set_face_fluxes(self._h, abi.SIDE[side], _dp(f)))

    def set_conserved(self, q: np.ndarray) -> None:
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
        _check(lib().bso_set_conserved(self._h, _dp(q)))

    def set_quantize(self, on: bool) -> None:
        """FP64 engine only: round the stored state to FP32 after every update
        (FP32 storage, FP64 arithmetic) - a probe of what an FP32 field
        loses, not a mode of the reference."""
        _check(lib().bso_set_quantize(self._h, 1 if on else 0))

    def iterate(self, steps: int) -> None:
        _check(lib().bso_iterate(self._h, steps))

    def iterate_implicit(self, steps: int, cfl: float, omega: float = 1.5) -> None:
        _check(lib().bso_iterate_implicit(self._h, steps, cfl, omega))

    def implicit_correction(self, cfl: float, omega: float = 1.5) -> np.ndarray:
        dq = np.empty(4 * self.n_cells)
        _check(lib().bso_implicit_correction(self._h, cfl, omega, _dp(dq)))
        return dq

    def density_residual_norm(self) -> float:
        out = C.c_double()
        _check(lib().bso_density_residual_norm(self._h, C.byref(out)))
        return out.value

    def residual(self) -> np.ndarray:
        r = np.empty(4 * self.n_cells)
        _check(lib().bso_residual(self._h, _dp(r)))
        return r

    def time_steps(self) -> np.ndarray:
        dt = np.empty(self.n_cells)
        _check(lib().bso_time_steps(self._h, _dp(dt)))
        return dt

    def boundary_fluxes(self, side: str = "jMin") -> list[abi.FaceFlux]:
        n = self.nj if side in ("iMin", "iMax") else self.ni
        out = (abi.FaceFlux * n)()
        _check(lib().bso_boundary_fluxes(self._h, abi.SIDE[side], out))
        return list(out)

    def forebody_drag(self, p_inf: float, q_inf: float, base_radius: float) -> float:
        cd = C.c_double()
        _check(lib().bso_forebody_drag(self._h, p_inf, q_inf, base_radius, C.byref(cd)))
        return cd.value

    def conserved(self) -> np.ndarray:
        q = np.empty(4 * self.n_cells)
        _check(lib().bso_conserved(self._h, _dp(q)))
        return q

    def primitives(self) -> np.ndarray:
        w = np.empty(4 * self.n_cells)
        _check(lib().bso_primitives(self._h, _dp(w)))
        return w

    @property
    def steps(self) -> int:
        return int(lib().bso_steps(self._h))

    def solve(self, method: str, tol: float, max_steps: int, check_every: int = 10,
              cfl: float = 5.0, omega: float = 1.5, relative: bool = True):
        """Steady solve: (status, steps, residual, initial residual)."""
        steps = C.c_int()
        res = C.c_double()
        init = C.c_double()
        st = lib().bso_solve(self._h, 1 if method == "lusgs" else 0, cfl, omega, tol,
                             1 if relative else 0, max_steps, check_every, C.byref(steps),
                             C.byref(res), C.byref(init))
        return st, steps.value, res.value, init.value


def parallel_solve(engines: list[OracleEuler2D], method: str, tol: float, max_steps: int,
                   check_every: int = 10, cfl: float = 5.0, omega: float = 1.5,
                   relative: bool = True, threads: int | None = None):
    """Solve independent cases on `threads` host threads (one case per thread
    at a time). Returns arrays (status, steps, residual, initial)."""
    n = len(engines)
    threads = threads or os.cpu_count() or 1
    handles = (C.c_void_p * n)(*[e.handle.value for e in engines])
    steps = (C.c_int * n)()
    status = (C.c_int * n)()
    res = np.empty(n)
    init = np.empty(n)
    lib().bso_parallel_solve(n, handles, 1 if method == "lusgs" else 0, cfl, omega, tol,
                             1 if relative else 0, max_steps, check_every, threads, steps,
                             _dp(res), _dp(init), status)
    return np.array(status), np.array(steps), res, init
