"""ctypes mirror of include/bowshock.h: enums, structs and status codes.

Only type definitions live here; `bowshock_b200._native` loads the library
and declares the entry points.
"""
from __future__ import annotations

import ctypes as C

# bs_status
BS_OK = 0
BS_INVALID_ARGUMENT = 1
BS_NON_PHYSICAL = 2
BS_MEMORY_LIMIT = 3
BS_EXECUTION = 4
BS_NOT_CONVERGED = 5
BS_BUSY = 6
BS_GRID_QUALITY = 7

STATUS_NAMES = {
    BS_OK: "BS_OK",
    BS_INVALID_ARGUMENT: "BS_INVALID_ARGUMENT",
    BS_NON_PHYSICAL: "BS_NON_PHYSICAL",
    BS_MEMORY_LIMIT: "BS_MEMORY_LIMIT",
    BS_EXECUTION: "BS_EXECUTION",
    BS_NOT_CONVERGED: "BS_NOT_CONVERGED",
    BS_BUSY: "BS_BUSY",
    BS_GRID_QUALITY: "BS_GRID_QUALITY",
}

GEOMETRY = {"planar": 0, "axisymmetric": 1}
FLUX = {"hllc": 0, "rusanov": 1}
LIMITER = {
    "firstOrder": 0,
    "minmod": 1,
    "vanLeer": 2,
    "vanAlbada": 3,
    "monotonizedCentral": 4,
    "unlimitedCentral": 5,
}
RECONSTRUCTION = {"perVariable": 0, "shared": 1, "sharedScaled": 2}
INTEGRATOR = {"forwardEuler": 0, "ssprk2": 1, "ssprk3": 2}
TIME_STEPPING = {"local": 0, "global": 1}
BC_KIND = {"inflow": 0, "outflow": 1, "wall": 2, "farField": 3, "periodic": 4, "faceStates": 5}
SIDES = ("iMin", "iMax", "jMin", "jMax")
SIDE = {name: k for k, name in enumerate(SIDES)}
GRID_UNGATED = 1
NOSE_KIND = {"conical": 0, "ogive": 1, "ellipsoid": 2, "power": 3, "parabolic": 4, "haack": 5}


class Primitive(C.Structure):
    _fields_ = [("rho", C.c_double), ("u", C.c_double), ("v", C.c_double), ("p", C.c_double)]


class Boundary(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("state", Primitive)]


class Config(C.Structure):
    _fields_ = [
        ("ni", C.c_int32),
        ("nj", C.c_int32),
        ("geometry", C.c_int32),
        ("flux", C.c_int32),
        ("limiter", C.c_int32),
        ("reconstruction", C.c_int32),
        ("integrator", C.c_int32),
        ("time_stepping", C.c_int32),
        ("gamma", C.c_double),
        ("cfl", C.c_double),
        ("boundaries", Boundary * 4),
    ]


class FaceFlux(C.Structure):
    _fields_ = [
        ("x", C.c_double),
        ("y", C.c_double),
        ("nx", C.c_double),
        ("ny", C.c_double),
        ("area", C.c_double),
        ("flux", C.c_double * 4),
    ]


class SolveResult(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("steps", C.c_int32),
        ("residual", C.c_double),
        ("initial_residual", C.c_double),
        ("drag", C.c_double),
    ]


class Body(C.Structure):
    _fields_ = [
        ("nose_kind", C.c_int32),
        ("reserved", C.c_int32),
        ("parameter", C.c_double),
        ("nose_length", C.c_double),
        ("base_radius", C.c_double),
        ("cylinder_length", C.c_double),
    ]


class BodyGridOptions(C.Structure):
    _fields_ = [
        ("nj", C.c_int32),
        ("refinement", C.c_int32),
        ("ni", C.c_int32),
        ("flags", C.c_int32),
        ("mach", C.c_double),
        ("gamma", C.c_double),
    ]


class TransonicGridOptions(C.Structure):
    _fields_ = [
        ("refinement", C.c_int32),
        ("nested", C.c_int32),
        ("far_field", C.c_double),
        ("cylinder", C.c_double),
        ("wall", C.c_double),
        ("growth", C.c_double),
        ("tip", C.c_double),
        ("shoulder", C.c_double),
        ("nose", C.c_double),
        ("nose_growth", C.c_double),
        ("nested_far_field", C.c_double),
        ("nested_cylinder", C.c_double),
    ]


class GridQuality(C.Structure):
    _fields_ = [
        ("min_angle", C.c_double),
        ("min_wall_angle", C.c_double),
        ("max_size_ratio", C.c_double),
        ("max_aspect_ratio", C.c_double),
        ("min_area", C.c_double),
    ]


class ConeFlow(C.Structure):
    _fields_ = [
        ("shock_angle", C.c_double),
        ("post_shock_mach", C.c_double),
        ("post_shock_pressure_ratio", C.c_double),
        ("surface_mach", C.c_double),
        ("surface_pressure_ratio", C.c_double),
        ("surface_pressure_coefficient", C.c_double),
    ]


class FittedShock(C.Structure):
    _fields_ = [
        ("state", Primitive),
        ("speed", C.c_double),
        ("normal_velocity", C.c_double),
        ("mach", C.c_double),
    ]


class Shock(C.Structure):
    _fields_ = [
        ("beta", C.c_double),
        ("pressure_ratio", C.c_double),
        ("density_ratio", C.c_double),
        ("downstream_mach", C.c_double),
    ]
