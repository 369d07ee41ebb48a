"""Warm-started batched solves: solved cases train the network
(bowshock_b200.mlp), whose prediction of a new case's steady field replaces
the free stream as the starting state. The solver's own FP64 residual still
decides convergence, so the drag is the solver's; a case whose warm start
fails (non-physical state, or no convergence within its budget) is solved
again from the free stream.
"""
from __future__ import annotations

import time
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
    predict_s: float = 0.0    # warm starts: the network's prediction and its host transforms, wall
    launches: int = 0         # solver kernels launched


def solve_cases(cases, starts: list[np.ndarray] | None = None, max_steps: int = 5000,
                keep_fields: bool = False, tolerance: float = TOLERANCE, anderson: int = 0) -> BatchSolve:
    """All `cases` in one batch by LU-SGS CFL 5 to RMS d(rho)/dt <= `tolerance`
    (1e-6), from the free stream or from `starts` (primitives per case);
    `anderson` > 0 accelerates the steps with that many differences."""
    batch = CudaBatch([c.config for c in cases], precision=64)
    try:
        if anderson:
            batch.set_anderson(anderson, 30)
        if starts is None:
            batch.set_free_stream()
        else:
            for k, w in enumerate(starts):
                batch.set_primitives(k, w)
        res = batch.solve("lusgs", tolerance, relative=False, max_steps=max_steps, check_every=20,
                          cfl=CFL, omega=OMEGA)
        ms, launches = batch.last_solve_timing()
        drags = [batch.forebody_drag(k, c.free, c.body.nose.base_radius) for k, c in enumerate(cases)]
        fields = [batch.primitives(k) for k in range(len(cases))] if keep_fields else None
        return BatchSolve([r.status for r in res], [r.steps for r in res], [r.initial_residual for r in res],
                          drags, ms, fields, launches=launches)
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


@dataclass
class Training:
    net: WarmStartNet
    solved: int              # converged cases whose fields were sampled
    samples: int
    solve_device_ms: float
    seconds: float           # Adam steps, wall time
    steps: int
    loss_first: float        # mean of the first and last 10 steps' losses
    loss_last: float


def train_on_solves(cases, cells_per_case: int = 4096, train_steps: int = 3000, max_steps: int = 5000,
                    batch: int = 16384, seed: int = 1) -> Training:
    """Solves `cases` cold in one batch and trains a 5 x 256 network on
    `cells_per_case` random cells of each converged one: Adam with the
    learning rate 1e-3, 3e-4 and 1e-4 over the three thirds of the steps."""
    solved = solve_cases(cases, max_steps=max_steps, keep_fields=True)
    ok = [k for k, s in enumerate(solved.status) if s == 0]
    samples, targets = training_set([cases[k] for k in ok], [solved.fields[k] for k in ok], cells_per_case)
    solved.fields = None
    net = WarmStartNet(hidden_layers=5, batch=batch, seed=seed)
    net.set_data(samples, targets)
    t0 = time.perf_counter()
    losses: list[float] = []
    third = max(1, train_steps // 3)
    for phase, lr in enumerate((1e-3, 3e-4, 1e-4)):
        losses.extend(net.train(third, lr, seed=101 + phase).tolist())
    return Training(net, len(ok), len(samples), solved.device_ms, time.perf_counter() - t0, 3 * third,
                    float(np.mean(losses[:10])), float(np.mean(losses[-10:])))


def predicted_starts(net: WarmStartNet, cases) -> list[np.ndarray]:
    """The network's field of every case, as primitives per cell."""
    samples = [case_samples(c) for c in cases]
    pred = net.predict(np.concatenate(samples))
    starts, k = [], 0
    for c, s in zip(cases, samples):
        starts.append(primitives_from_prediction(pred[k:k + len(s)], c.free))
        k += len(s)
    return starts


def warm_solve(net: WarmStartNet, cases, max_steps: int = 5000, warm_steps: int = 2500,
               tolerance: float = TOLERANCE, fallback_anderson: int = 0) -> tuple[BatchSolve, list[int]]:
    """Warm-started batch; cases whose warm start fails (non-physical, or not
    converged within `warm_steps`, about three times a typical cold solve
    here) are solved again from the free stream within `max_steps` (their
    steps and time are added), by plain LU-SGS steps or, with
    `fallback_anderson` > 0, Anderson-accelerated ones (which converge the
    cases whose plain steps settle into a cycle but slow most others).
    Returns the combined result and the indices that fell back."""
    t0 = time.perf_counter()
    starts = predicted_starts(net, cases)
    predict_s = time.perf_counter() - t0
    warm = solve_cases(cases, starts, max_steps=min(warm_steps, max_steps), tolerance=tolerance)
    del starts
    warm.predict_s = predict_s
    failed = [k for k, s in enumerate(warm.status) if s != 0]
    if failed:
        cold = solve_cases([cases[k] for k in failed], max_steps=max_steps, tolerance=tolerance,
                           anderson=fallback_anderson)
        for j, k in enumerate(failed):
            warm.status[k] = cold.status[j]
            warm.steps[k] += cold.steps[j]
            warm.drags[k] = cold.drags[j]
        warm.device_ms += cold.device_ms
        warm.launches += cold.launches
    return warm, failed
