"""Grids and configurations shared by the tests, built as the reference's
own tests build them (tests/engine-cpu/*.test.ts, tests/gpu/*.test.ts)."""
from __future__ import annotations

import math

import numpy as np

from bowshock_b200.config import (
    Boundary,
    Euler2DConfig,
    Primitive2D,
    free_stream_at,
    grid_from_function,
    steady_drag_config,
)

GAMMA = 1.4
DEG = math.pi / 180


def lcg_random(seed: int):
    """The reference tests' linear congruential generator
    (tests/gpu/euler2d-gpu.test.ts:78-83)."""
    state = seed

    def random() -> float:
        nonlocal state
        state = (state * 1664525 + 1013904223) % 2**32
        return state / 2**32 - 0.5

    return random


def distorted_grid(ni: int, nj: int, x0: float, x1: float, y0: float, y1: float, seed: int = 2024,
                   amount: float = 0.6):
    """Random interior node displacements (distortedGrid,
    tests/gpu/euler2d-gpu.test.ts:76-88)."""
    random = lcg_random(seed)

    def node(i, j):
        interior = 0 < i < ni and 0 < j < nj
        di = amount * random() if interior else 0.0
        dj = amount * random() if interior else 0.0
        return (x0 + ((x1 - x0) * (i + di)) / ni, y0 + ((y1 - y0) * (j + dj)) / nj)

    return grid_from_function(ni, nj, node)


from bowshock_b200.workloads import cone_body, cone_case, ogive_body, ogive_case  # noqa: E402,F401


def config1(ni: int = 80, nj: int = 40):
    """The plain explicit case (bowshock_b200.workloads.cone_case)."""
    c = cone_case(ni, nj)
    return c.config, c.free, c.body


def config2(mach: float, ni: int = 160, nj: int = 80):
    """One case of the drag-curve sweep (bowshock_b200.workloads.ogive_case)."""
    c = ogive_case(mach, ni, nj)
    return c.config, c.free, c.body


def uniform_primitives(cfg: Euler2DConfig, s: Primitive2D) -> np.ndarray:
    return np.tile(np.array([s.rho, s.u, s.v, s.p]), cfg.grid.ni * cfg.grid.nj)
