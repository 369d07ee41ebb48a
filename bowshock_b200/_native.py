"""Loads lib/libbowshock_b200.so and declares its C entry points
(include/bowshock.h). Raises if the library has not been built: there is no
fallback implementation."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

from . import abi

LIB_DIR = Path(__file__).resolve().parent / "lib"
LIB_PATH = LIB_DIR / "libbowshock_b200.so"


class NativeLibraryMissing(ImportError):
    pass


class BowshockError(RuntimeError):
    """A failed C entry point: `status` is its bs_status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class NonPhysicalStateError(BowshockError):
    """The reference's NonPhysicalStateError (src/solver/errors.ts:2)."""


class GridQualityError(BowshockError):
    """The reference's GridQualityError (src/grid/body-grid.ts:57-59)."""


class BusyError(BowshockError):
    """An overlapping call on the same engine (ExclusiveRunner,
    src/engine-gpu/gpu-common.ts:122-140)."""


class NotConvergedError(BowshockError):
    pass


_ERRORS = {
    abi.BS_NON_PHYSICAL: NonPhysicalStateError,
    abi.BS_GRID_QUALITY: GridQualityError,
    abi.BS_BUSY: BusyError,
    abi.BS_NOT_CONVERGED: NotConvergedError,
}

_lib: C.CDLL | None = None

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_vp = C.c_void_p

# name -> argument types; every one returns bs_status.
SIGNATURES: dict[str, list] = {
    "bs_device_count": [_ip],
    "bs_set_device": [C.c_int32],
    "bs_engine_create": [C.POINTER(abi.Config), _dp, _dp, C.POINTER(_vp)],
    "bs_engine_create_ex": [C.POINTER(abi.Config), _dp, _dp, C.c_int32, C.POINTER(_vp)],
    "bs_engine_time_steps": [_vp, _dp],
    "bs_engine_destroy": [_vp],
    "bs_engine_centroids": [_vp, _dp, _dp],
    "bs_engine_set_primitives": [_vp, _dp],
    "bs_engine_iterate": [_vp, C.c_int32],
    "bs_engine_set_implicit_cfl": [_vp, C.c_double],
    "bs_engine_iterate_implicit": [_vp, C.c_int32, C.c_double, C.c_double, C.c_double],
    "bs_engine_density_residual_norm": [_vp, _dp],
    "bs_engine_residual": [_vp, _dp],
    "bs_engine_boundary_fluxes": [_vp, C.c_int32, C.POINTER(abi.FaceFlux)],
    "bs_engine_forebody_drag": [_vp, C.c_double, C.c_double, C.c_double, _dp],
    "bs_engine_read_state": [_vp, _fp],
    "bs_engine_read_primitives": [_vp, _dp],
    "bs_engine_steps": [_vp, C.POINTER(C.c_int64)],
    "bs_engine_solve": [_vp, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_int32,
                        C.c_int32, C.c_int32, C.POINTER(abi.SolveResult)],
    "bs_batch_create": [C.c_int32, C.POINTER(abi.Config), C.POINTER(_dp), C.POINTER(_dp),
                        C.c_int32, C.POINTER(_vp)],
    "bs_batch_destroy": [_vp],
    "bs_batch_size": [_vp, _ip],
    "bs_batch_set_primitives": [_vp, C.c_int32, _dp],
    "bs_batch_set_free_stream": [_vp],
    "bs_batch_solve": [_vp, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32,
                       C.c_int32, C.POINTER(abi.SolveResult)],
    "bs_batch_set_anderson": [_vp, C.c_int32, C.c_int32],
    "bs_batch_anderson_restarts": [_vp, _ip],
    "bs_engine_set_anderson": [_vp, C.c_int32, C.c_int32],
    "bs_engine_iterate_accelerated": [_vp, C.c_int32, C.c_double, C.c_double, C.c_double],
    "bs_engine_anderson_restarts": [_vp, _ip],
    "bs_engine_set_metric_precision": [_vp, C.c_int32],
    "bs_engine_set_sweep_wait_limit": [_vp, C.c_int32],
    "bs_fp64_fma_rate": [C.c_int32, _dp, _dp],
    "bs_batch_set_sweep_wait_limit": [_vp, C.c_int32],
    "bs_batch_set_tile_shape": [_vp, C.c_int32],
    "bs_batch_tuning": [_vp, _ip, _ip, _ip, _ip, _ip],
    "bs_batch_set_update_mode": [_vp, C.c_int32],
    "bs_batch_set_lanes": [_vp, C.c_int32],
    "bs_batch_update_mode": [_vp, _ip],
    "bs_batch_set_metric_precision": [_vp, C.c_int32],
    "bs_batch_forebody_drag": [_vp, C.c_int32, C.c_double, C.c_double, C.c_double, _dp],
    "bs_batch_read_primitives": [_vp, C.c_int32, _dp],
    "bs_batch_density_residual_norms": [_vp, _dp],
    "bs_batch_last_solve_timing": [_vp, _dp, C.POINTER(C.c_int64)],
    "bs_batch_kernel_times": [_vp, C.c_int32, C.c_double, C.c_double, C.c_int32, _dp],
    "bs_lusgs_step_static": [C.POINTER(abi.Config), _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_double,
                             C.c_double, _vp, _dp, _ip],
    "bs_body_grid": [C.POINTER(abi.Body), C.POINTER(abi.BodyGridOptions), C.POINTER(_vp)],
    "bs_blunt_body_grid": [C.POINTER(abi.Body), C.POINTER(abi.BodyGridOptions), C.POINTER(_vp)],
    "bs_blunt_body_grid_bounded": [C.POINTER(abi.Body), C.POINTER(abi.BodyGridOptions), _dp, _dp, C.c_int32,
                                   C.POINTER(_vp)],
    "bs_ramp_grid": [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                     C.c_double, C.POINTER(_vp)],
    "bs_grid_dims": [_vp, _ip, _ip],
    "bs_grid_nodes": [_vp, _dp, _dp],
    "bs_grid_info": [_vp, _ip, _dp],
    "bs_grid_two_scale": [_vp, _ip],
    "bs_transonic_grid": [C.POINTER(abi.Body), C.POINTER(abi.TransonicGridOptions), C.POINTER(_vp)],
    "bs_grid_transonic_info": [_vp, _ip, _ip, _dp, _dp, _dp, _ip],
    "bs_grid_destroy": [_vp],
    "bs_grid_quality_of": [C.c_int32, C.c_int32, _dp, _dp, C.POINTER(abi.GridQuality)],
    "bs_taylor_maccoll": [C.c_double, C.c_double, C.c_double, C.c_double,
                          C.POINTER(abi.ConeFlow)],
    "bs_oblique_shock": [C.c_double, C.c_double, C.c_double, C.POINTER(abi.Shock)],
    "bs_normal_shock": [C.c_double, C.c_double, C.POINTER(abi.Shock)],
    "bs_cone_flow_field": [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32, _dp, _dp, _dp,
                           C.POINTER(abi.ConeFlow)],
    "bs_shock_state": [C.POINTER(abi.Primitive), C.c_double, C.c_double, C.c_double, C.c_double,
                       C.POINTER(abi.FittedShock)],
    "bs_compatible_shock": [C.POINTER(abi.Primitive), C.c_double, C.c_double, C.c_double, C.c_double,
                            C.c_double, C.c_double, C.c_double, C.POINTER(abi.FittedShock)],
    "bs_body_radius": [C.POINTER(abi.Body), C.c_int32, _dp, _dp],
    "bs_nose_slopes": [C.POINTER(abi.Body), _dp, _dp],
    "bs_fit_create": [C.POINTER(abi.Config), _dp, _dp, _dp, _dp, _dp, _dp, C.POINTER(abi.Primitive), _dp,
                      C.c_int32, _dp, C.POINTER(_vp)],
    "bs_fit_destroy": [_vp],
    "bs_fit_iterate": [_vp, C.c_int32],
    "bs_fit_check": [_vp, _dp, _dp],
    "bs_fit_solve": [_vp, C.c_double, C.c_double, C.c_int32, C.c_int32, _ip, _ip, _dp, _dp],
    "bs_fit_heights": [_vp, _dp],
    "bs_fit_nodes": [_vp, _dp, _dp],
    "bs_fit_read_primitives": [_vp, _dp],
    "bs_fit_wall_fluxes": [_vp, C.POINTER(abi.FaceFlux)],
    "bs_fit_forebody_drag": [_vp, C.c_double, C.c_double, C.c_double, _dp],
    "bs_sharp_fit_columns": [C.POINTER(abi.Body), C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_double,
                             C.c_double, C.c_int32, _dp, _ip],
    "bs_column_positions": [C.c_int32, _dp, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, _dp,
                            _ip],
    "bs_batch_iterate": [_vp, C.c_int32],
    "bs_batch_flow_field": [_vp, C.c_int32, C.c_int32, C.POINTER(abi.Primitive), C.c_double, _dp],
    "bs_batch_set_active": [_vp, _ip],
    "bs_batch_autotune": [_vp, C.c_int32, C.c_int32, C.c_double, C.c_double, _ip, _dp],
    "bs_gemm_bf16": [_vp, _vp, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _vp],
    "bs_gemm_bf16_time": [_vp, _vp, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_float)],
    "bs_mlp_create": [C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(_vp)],
    "bs_mlp_destroy": [_vp],
    "bs_mlp_param_count": [_vp, C.POINTER(C.c_int64)],
    "bs_mlp_get_params": [_vp, _vp],
    "bs_mlp_set_params": [_vp, _vp],
    "bs_mlp_set_data": [_vp, C.c_int64, _vp, _vp],
    "bs_mlp_train": [_vp, C.c_int32, C.c_float, C.c_uint64, _vp],
    "bs_mlp_loss_grad": [_vp, C.c_int32, _vp, _vp, _vp, _vp],
    "bs_mlp_predict": [_vp, C.c_int64, _vp, _vp],
}


def _declare(lib: C.CDLL) -> None:
    lib.bs_last_error.restype = C.c_char_p
    lib.bs_last_error.argtypes = []
    lib.bs_version.restype = C.c_char_p
    lib.bs_version.argtypes = []
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int


def load(path: Path | str | None = None) -> C.CDLL:
    """The native library, loaded once. Raises NativeLibraryMissing if it has
    not been built (python -c 'import __graft_entry__; __graft_entry__.build()')."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise NativeLibraryMissing(
            f"{p} is missing: build the CUDA library first (bowshock_b200.build.build())"
        )
    lib = C.CDLL(str(p))
    _declare(lib)
    if path is None:
        _lib = lib
    return lib


def check(status: int, lib: C.CDLL | None = None) -> None:
    if status != abi.BS_OK:
        L = lib or load()
        message = L.bs_last_error().decode()
        raise _ERRORS.get(status, BowshockError)(status, message)
