"""Anderson acceleration on the CPU: the oracle's restatement of
src/solver/anderson.ts pinned to the reference's own known answers
(tests/engine-cpu/implicit.test.ts:285-331), including accelerated LU-SGS
steps of the FP64 oracle that reach the explicit scheme's drag."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

from oracle.anderson import AndersonMixing
from oracle.oracle import OracleEuler2D
from test_oracle_golden import implicit_case

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())["anderson"]


def test_without_history_the_step_is_the_plain_one():
    g = GOLDEN["plain_step"]
    a = AndersonMixing(3, g["depth"])
    assert a.next(np.array(g["x"]), np.array(g["f"])).tolist() == g["next"]


def test_a_slow_linear_iteration_converges_far_faster():
    g = GOLDEN["linear"]
    n = g["n"]
    diag = np.array([1 / (1 + g["stiffness"] * k / (n - 1)) for k in range(n)])
    b = np.sin(np.arange(1, n + 1, dtype=np.float64))

    def correction(x):
        return (b - diag * x) / 4

    def error(x):
        return float(np.max(np.abs(x - b / diag)))

    plain = np.zeros(n)
    accelerated = np.zeros(n)
    anderson = AndersonMixing(n, g["depth"])
    for _ in range(g["steps"]):
        plain = plain + correction(plain)
        accelerated = anderson.next(accelerated, correction(accelerated))
    start = error(np.zeros(n))
    assert error(accelerated) < g["accelerated_below"] * start
    assert error(plain) > g["plain_above"] * start


def test_dependent_differences_are_dropped_oldest_first():
    # Two equal corrections in a row make the first difference zero: the
    # least-squares problem drops it and the step uses the others.
    a = AndersonMixing(2, 3)
    a.next(np.array([0.0, 0.0]), np.array([1.0, 1.0]))
    a.next(np.array([1.0, 1.0]), np.array([1.0, 1.0]))
    out = a.next(np.array([2.0, 2.0]), np.array([0.5, 0.25]))
    assert np.all(np.isfinite(out))


def test_accelerated_lusgs_reaches_the_explicit_drag():
    g, cfg, free = implicit_case()
    ga = GOLDEN["lusgs"]
    explicit = OracleEuler2D(cfg)
    explicit.set_uniform(free.state)
    explicit.iterate(g["explicit_steps"])
    s = OracleEuler2D(cfg)
    s.set_uniform(free.state)
    s.iterate_implicit(ga["plain_steps"], ga["plain_cfl"])
    anderson = AndersonMixing(4 * s.n_cells, ga["depth"])
    steps = 0
    for _ in range(ga["max_steps"]):
        if s.density_residual_norm() <= 1e-13:
            break
        x = s.conserved().ravel()
        f = s.implicit_correction(ga["cfl"]).ravel()
        s.set_conserved(anderson.next(x, f))
        steps += 1
    assert s.density_residual_norm() < ga["residual_below"]
    d_exp = explicit.forebody_drag(free.pressure, free.dynamic_pressure, 0.5)
    d_acc = s.forebody_drag(free.pressure, free.dynamic_pressure, 0.5)
    assert abs(d_acc / d_exp - 1) < ga["drag_equal_within"]
    assert math.isfinite(d_acc) and steps < ga["max_steps"]
