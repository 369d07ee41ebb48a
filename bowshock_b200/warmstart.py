"""Warm-started batched solves: solved cases train the network
(bowshock_b200.mlp), whose prediction of a new case's steady field replaces
the free stream as the starting state. The solver's own FP64 residual still
decides convergence, so the drag is the solver's; a case whose warm start
fails (non-physical state, or no convergence within its budget) is solved
again from the free stream.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .batch import CudaBatch
from .mlp import WarmStartNet, case_samples, primitives_from_prediction, targets_from_primitives

TOLERANCE = 1e-6
CFL = 5.0
OMEGA = 1.5


@dataclass
class BatchSolve:
    status: list[int]
    steps: list[int]
    initial_residual: list[float]
    drags: list[float]
    device_ms: float
    fields: list[np.ndarray] | None


def solve_cases(cases, starts: list[np.ndarray] | None = None, max_steps: int = 5000,
                keep_fields: bool = False) -> BatchSolve:
    """All `cases` in one batch by LU-SGS CFL 5 to RMS d(rho)/dt <= 1e-6,
    from the free stream or from `starts` (primitives per case)."""
    batch = CudaBatch([c.config for c in cases], precision=64)
    try:
        if starts is None:
            batch.set_free_stream()
        else:
            for k, w in enumerate(starts):
                batch.set_primitives(k, w)
        res = batch.solve("lusgs", TOLERANCE, relative=False, max_steps=max_steps, check_every=20,
                          cfl=CFL, omega=OMEGA)
        ms, _ = batch.last_solve_timing()
        drags = [batch.forebody_drag(k, c.free, c.body.nose.base_radius) for k, c in enumerate(cases)]
        fields = [batch.primitives(k) for k in range(len(cases))] if keep_fields else None
        return BatchSolve([r.status for r in res], [r.steps for r in res], [r.initial_residual for r in res],
                          drags, ms, fields)
    finally:
        batch.destroy()


def training_set(cases, fields, cells_per_case: int, seed: int = 1) -> tuple[np.ndarray, np.ndarray]:
    """Samples and targets of up to `cells_per_case` random cells of each
    solved case."""
    rng = np.random.default_rng(seed)
    samples, targets = [], []
    for case, w in zip(cases, fields):
        s = case_samples(case)
        t = targets_from_primitives(w, case.free)
        pick = rng.choice(len(s), size=min(cells_per_case, len(s)), replace=False)
        samples.append(s[pick])
        targets.append(t[pick])
    return np.concatenate(samples), np.concatenate(targets)


def predicted_starts(net: WarmStartNet, cases) -> list[np.ndarray]:
    """The network's field of every case, as primitives per cell."""
    samples = [case_samples(c) for c in cases]
    pred = net.predict(np.concatenate(samples))
    starts, k = [], 0
    for c, s in zip(cases, samples):
        starts.append(primitives_from_prediction(pred[k:k + len(s)], c.free))
        k += len(s)
    return starts


def warm_solve(net: WarmStartNet, cases, max_steps: int = 5000,
               warm_steps: int = 2500) -> tuple[BatchSolve, list[int]]:
    """Warm-started batch; cases whose warm start fails (non-physical, or not
    converged within `warm_steps`, about three times a typical cold solve
    here) are solved again from the free stream within `max_steps` (their
    steps and time are added). Returns the combined result and the indices
    that fell back."""
    warm = solve_cases(cases, predicted_starts(net, cases), max_steps=min(warm_steps, max_steps))
    failed = [k for k, s in enumerate(warm.status) if s != 0]
    if failed:
        cold = solve_cases([cases[k] for k in failed], max_steps=max_steps)
        for j, k in enumerate(failed):
            warm.status[k] = cold.status[j]
            warm.steps[k] += cold.steps[j]
            warm.drags[k] = cold.drags[j]
        warm.device_ms += cold.device_ms
    return warm, failed
