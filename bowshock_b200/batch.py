"""Many cases of uneven size solved together on one GPU: every launch covers
all active cases, and each case stops at its own tolerance."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native, abi
from .config import Euler2DConfig, FreeStream

_dp = C.POINTER(C.c_double)


# The autotuner's choices per grid-size class (CudaBatch.size_class), kept for
# the life of the process: a later batch of the same class applies them
# instead of timing its candidates again.
_TUNED: dict[tuple, tuple[dict, float]] = {}


class CudaBatch:
    def __init__(self, configs: list[Euler2DConfig], precision: int = 64):
        self._lib = _native.load()
        self.configs = list(configs)
        n = len(self.configs)
        self._abi = (abi.Config * n)(*[c.to_abi() for c in self.configs])
        self._xs = [c.grid.x for c in self.configs]
        self._ys = [c.grid.y for c in self.configs]
        xs = (_dp * n)(*[x.ctypes.data_as(_dp) for x in self._xs])
        ys = (_dp * n)(*[y.ctypes.data_as(_dp) for y in self._ys])
        h = C.c_void_p()
        _native.check(self._lib.bs_batch_create(n, self._abi, xs, ys, precision, C.byref(h)), self._lib)
        self._h = h
        self.n = n

    def destroy(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _native.check(self._lib.bs_batch_destroy(h), self._lib)
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

    def _call(self, name: str, *args) -> None:
        if self._h is None:
            raise RuntimeError("the batch has been destroyed")
        _native.check(getattr(self._lib, name)(self._h, *args), self._lib)

    def set_free_stream(self) -> None:
        self._call("bs_batch_set_free_stream")

    def set_primitives(self, c: int, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
        g = self.configs[c].grid
        if w.size != 4 * g.ni * g.nj:
            raise ValueError("four values per cell are needed")
        self._call("bs_batch_set_primitives", c, w.ctypes.data_as(_dp))

    def solve(self, method: str = "lusgs", tolerance: float = 1e-6, relative: bool = False,
              max_steps: int = 100000, check_every: int = 20, cfl: float = 5.0,
              omega: float = 1.5) -> list[abi.SolveResult]:
        out = (abi.SolveResult * self.n)()
        self._call("bs_batch_solve", 1 if method == "lusgs" else 0, cfl, omega, tolerance,
                   1 if relative else 0, max_steps, check_every, out)
        return list(out)

    def set_metric_precision(self, bits: int) -> None:
        """64: two-float metrics in the residual; 32: FP32 metrics (default)."""
        self._call("bs_batch_set_metric_precision", int(bits))

    def set_tile_shape(self, shape: int) -> None:
        """The residual pass's tile shape: -1 the default, 0 .. 7 the
        autotuner's choices (bs_batch_set_tile_shape)."""
        self._call("bs_batch_set_tile_shape", int(shape))

    def set_update_mode(self, fused: bool) -> None:
        """LU-SGS steps apply their update inside the next residual pass
        (True, the default) or by a separate kernel after each sweep
        (bs_batch_set_update_mode); the autotuner chooses."""
        self._call("bs_batch_set_update_mode", 1 if fused else 0)

    def tuning(self) -> dict:
        """Lanes, tile shape and update mode as set or tuned."""
        v = [C.c_int32() for _ in range(5)]
        self._call("bs_batch_tuning", *[C.byref(x) for x in v])
        lanes, shape, ti, tj, threads = (x.value for x in v)
        fused = C.c_int32()
        self._call("bs_batch_update_mode", C.byref(fused))
        return {"lanes": lanes, "tile_shape": shape, "tile": f"{ti}x{tj}", "threads": threads,
                "fused_update": bool(fused.value)}

    def set_sweep_wait_limit(self, polls: int) -> None:
        """As CudaEuler2D.set_sweep_wait_limit, for the batch's sweeps."""
        self._call("bs_batch_set_sweep_wait_limit", int(polls))

    def set_anderson(self, depth: int, plain_steps: int = 30) -> None:
        """Anderson acceleration of later LU-SGS solves: `depth` differences
        kept (0: plain steps), after `plain_steps` plain steps."""
        self._call("bs_batch_set_anderson", int(depth), int(plain_steps))

    def anderson_restarts(self) -> np.ndarray:
        """Per case, the times the last solve's acceleration forgot its history."""
        out = np.zeros(self.n, np.int32)
        self._call("bs_batch_anderson_restarts", out.ctypes.data_as(C.POINTER(C.c_int32)))
        return out

    def forebody_drag(self, c: int, free: FreeStream, base_radius: float) -> float:
        cd = C.c_double()
        self._call("bs_batch_forebody_drag", c, free.pressure, free.dynamic_pressure,
                   float(base_radius), C.byref(cd))
        return cd.value

    def primitives(self, c: int) -> np.ndarray:
        g = self.configs[c].grid
        w = np.empty(4 * g.ni * g.nj)
        self._call("bs_batch_read_primitives", c, w.ctypes.data_as(_dp))
        return w.reshape(-1, 4)

    def residual_norms(self) -> np.ndarray:
        r = np.empty(self.n)
        self._call("bs_batch_density_residual_norms", r.ctypes.data_as(_dp))
        return r

    def last_solve_timing(self) -> tuple[float, int]:
        ms = C.c_double()
        launches = C.c_int64()
        self._call("bs_batch_last_solve_timing", C.byref(ms), C.byref(launches))
        return ms.value, launches.value

    FIELDS = {"schlieren": 0, "mach": 1, "cp": 2, "density": 3}

    def flow_field(self, c: int, field: str, free: FreeStream, length: float = 0.5) -> np.ndarray:
        """Case c's display field per cell (i fastest), computed on the GPU:
        'schlieren' (|grad rho| x length / rho_inf), 'mach', 'cp', 'density'."""
        g = self.configs[c].grid
        out = np.empty(g.ni * g.nj)
        st = free.state
        w = abi.Primitive(st.rho, st.u, st.v, st.p)
        self._call("bs_batch_flow_field", c, self.FIELDS[field], C.byref(w), float(length), out.ctypes.data_as(_dp))
        return out

    def iterate(self, steps: int) -> None:
        """Explicit steps of the active cases."""
        self._call("bs_batch_iterate", steps)

    def set_active(self, flags) -> None:
        f = np.ascontiguousarray(np.asarray(flags, dtype=np.int32))
        if f.size != self.n:
            raise ValueError("one flag per case")
        self._call("bs_batch_set_active", f.ctypes.data_as(C.POINTER(C.c_int32)))

    def size_class(self, method: str = "lusgs") -> tuple:
        """The batch's grid-size class for the autotuner's cache: the method,
        the widest case's ni and nj, and the case count rounded up to a power
        of two."""
        ni = max(c.grid.ni for c in self.configs)
        nj = max(c.grid.nj for c in self.configs)
        return (method, ni, nj, 1 << max(0, (self.n - 1).bit_length()))

    def autotune(self, method: str = "lusgs", steps: int = 40, cfl: float = 5.0,
                 omega: float = 1.5, cache: bool = False) -> tuple[int, float]:
        """Chooses the number of lanes, the residual pass's tile shape and
        (LU-SGS) the update mode by timing `steps` steps with each candidate
        (the state is unchanged); returns (lanes, ms per step). With `cache`,
        a batch of a grid-size class tuned before in this process takes the
        stored choice without timing (ms per step is then the stored one)."""
        key = self.size_class(method)
        if cache and key in _TUNED:
            t, ms_stored = _TUNED[key]
            self.set_lanes(t["lanes"])
            self.set_tile_shape(t["tile_shape"])
            if method == "lusgs":
                self.set_update_mode(t["fused_update"])
            return t["lanes"], ms_stored
        lanes = C.c_int32()
        ms = C.c_double()
        self._call("bs_batch_autotune", 1 if method == "lusgs" else 0, steps, cfl, omega,
                   C.byref(lanes), C.byref(ms))
        if cache:
            _TUNED[key] = (self.tuning(), ms.value)
        return lanes.value, ms.value

    def set_lanes(self, lanes: int) -> None:
        """The number of lanes, as the autotuner would set it
        (bs_batch_set_lanes)."""
        self._call("bs_batch_set_lanes", int(lanes))

    def kernel_times(self, method: str = "lusgs", cfl: float = 5.0, omega: float = 1.5,
                     iterations: int = 20) -> tuple[float, float, float]:
        ms = np.empty(3)
        self._call("bs_batch_kernel_times", 1 if method == "lusgs" else 0, cfl, omega, iterations,
                   ms.ctypes.data_as(_dp))
        return float(ms[0]), float(ms[1]), float(ms[2])
