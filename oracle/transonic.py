"""TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.

solveTransonic (src/analysis/transonic-flow.ts:151-257) restated on the FP64
oracle, the checker of the GPU's transonic solve: from the free stream, LU-SGS
steps at a CFL number ramped from 1 by 1.2 a step, Anderson acceleration
(oracle/anderson.py) after the plain steps, its history forgotten when |f|^2
exceeds 100 times its least value (:183-206), the drag checked every
`check_every` steps until it settles (SettlingValue). A problem is
bowshock_b200.transonic.TransonicProblem (its configuration and free stream).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from bowshock_b200.verification import SettlingValue

from .anderson import AndersonMixing
from .oracle import OracleEuler2D


@dataclass
class OracleTransonic:
    engine: OracleEuler2D
    drag: float
    steps: int
    converged: bool


def solve_transonic(problem, noise: float = 1e-7, max_steps: int = 4000, check_every: int = 50,
                    cfl: float = 1000.0, depth: int = 8, plain_steps: int = 200) -> OracleTransonic:
    o = OracleEuler2D(problem.config)
    o.set_uniform(problem.free_stream.state)
    mixing = AndersonMixing(4 * o.n_cells, depth) if depth > 0 else None
    f = problem.free_stream
    radius = problem.body.nose.base_radius
    settling = SettlingValue(noise)
    best, c, n, drag = np.inf, 1.0, 0, float("nan")
    while n < max_steps:
        for _ in range(check_every):
            if mixing is None or n < plain_steps:
                o.iterate_implicit(1, c)
            else:
                x = o.conserved()
                fc = o.implicit_correction(c)
                nf = float(fc @ fc)
                if nf > 100 * best:
                    mixing.reset()
                    best = nf
                best = min(best, nf)
                o.set_conserved(mixing.next(x, fc))
            n += 1
            c = min(cfl, c * 1.2)
        drag = o.forebody_drag(f.pressure, f.dynamic_pressure, radius)
        if settling.add(drag):
            return OracleTransonic(o, drag, n, True)
    return OracleTransonic(o, drag, n, False)
