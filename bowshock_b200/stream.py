"""The combined warm-started stream: many seeded cases on grids of up to
640 x 320, more than one batch can hold at once, solved wave by wave. Each
wave's grids are made on the host threads while the GPU solves the wave
before it; the network predicts every cell of the wave, the wave is solved
by LU-SGS from those fields (warmstart.warm_solve: a case whose warm start
fails is solved again from the free stream), and the next wave follows.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

from .mlp import WarmStartNet
from .warmstart import warm_solve
from .workloads import Case, NoseCase, make_cases

# Device bytes per cell of a case in an FP64 LU-SGS batch: the state and
# the other buffer it alternates with over a run of steps, 2 x 4 x 8; time
# step 4, cell metrics 8, the i- and j-face metrics 16 each (one face of each
# per cell, the extra row and column counted separately) and the correction
# dQ 16; forward and backward sweep records 5 x 16 each per slot, of which a
# case has sweep_slots(ni, nj).
CELL_BYTES = 64 + 4 + 8 + 16 + 16 + 16
SLOT_BYTES = 160


def sweep_slots(ni: int, nj: int) -> int:
    """Record slots of a case: one per cell, stored by anti-diagonal with no
    slot off the grid, as the device layout (sweep_slots in
    device/layout.cuh)."""
    return ni * nj


def case_device_bytes(ni: int, nj: int) -> int:
    """Device memory one case takes in an FP64 LU-SGS batch (the network's
    buffers and the batch's per-case words aside)."""
    return ni * nj * CELL_BYTES + (ni + nj) * 16 + sweep_slots(ni, nj) * SLOT_BYTES + 64 * (ni + nj)


def plan_waves(specs: list[NoseCase], budget_bytes: int, order: list[int] | None = None) -> list[list[int]]:
    """Consecutive runs of specs (in `order`, by default as given) whose
    cases fit in `budget_bytes` of device memory together (a case larger
    than the budget is a wave of its own)."""
    waves: list[list[int]] = []
    current: list[int] = []
    used = 0
    for k in (range(len(specs)) if order is None else order):
        s = specs[k]
        b = case_device_bytes(s.ni, s.nj)
        if current and used + b > budget_bytes:
            waves.append(current)
            current, used = [], 0
        current.append(k)
        used += b
    if current:
        waves.append(current)
    return waves


def by_grid_size(specs: list[NoseCase]) -> list[int]:
    """Spec indices, smallest grids first (stable)."""
    return sorted(range(len(specs)), key=lambda k: (specs[k].ni * specs[k].nj, k))


@dataclass
class WaveReport:
    ni: int                   # largest grid of the wave, cells along
    cases: int
    refused: int
    cells: int
    device_ms: float          # warm solves and free-stream re-solves
    predict_s: float          # network prediction and its host transforms, wall
    fell_back: int
    converged: int
    cell_steps: int
    launches: int = 0         # solver kernels


@dataclass
class StreamResult:
    status: list[int | None]   # per spec: 0 converged, else a bs_status; None: no grid
    steps: list[int]
    drags: list[float]
    fell_back: list[int]       # spec indices whose warm start failed
    waves: list[WaveReport]
    wall_s: float              # the whole stream, first grid to last solve
    first_build_s: float       # grids of the first wave (not overlapped)
    kept: dict[int, Case] = field(default_factory=dict)


def run_stream(net: WarmStartNet, specs: list[NoseCase], budget_bytes: int, threads: int,
               max_steps: int = 2500, warm_steps: int = 1250, base_ni: int = 80,
               keep: set[int] | None = None, tolerance: float = 1e-6) -> StreamResult:
    """Solves every spec, wave by wave: smallest grids first, each wave
    within `budget_bytes` (plan_waves), the next wave's grids made on
    `threads` host threads while the current one solves. The step budgets
    are those of a grid `base_ni` cells along, scaled by the wave's largest
    ni (the LU-SGS steps a case needs grow about as fast): `warm_steps`
    before a warm start falls back, `max_steps` from the free stream. The
    cases of `keep` (spec indices) are returned with their grids."""
    keep = keep or set()
    waves = plan_waves(specs, budget_bytes, by_grid_size(specs))
    n = len(specs)
    status: list[int | None] = [None] * n
    steps = [0] * n
    drags = [float("nan")] * n
    fell: list[int] = []
    reports: list[WaveReport] = []
    kept: dict[int, Case] = {}

    def build(idx: list[int]) -> list[Case | None]:
        return make_cases([specs[k] for k in idx], threads)

    t_start = time.perf_counter()
    with ThreadPoolExecutor(max_workers=1) as builder:
        future = builder.submit(build, waves[0])
        first_build_s = 0.0
        for w, idx in enumerate(waves):
            built = future.result()
            if w == 0:
                first_build_s = time.perf_counter() - t_start
            if w + 1 < len(waves):
                future = builder.submit(build, waves[w + 1])
            pairs = [(k, c) for k, c in zip(idx, built) if c is not None]
            del built
            for k, c in pairs:
                if k in keep:
                    kept[k] = c
            if not pairs:
                reports.append(WaveReport(max(specs[k].ni for k in idx), len(idx), len(idx), 0, 0.0, 0.0, 0, 0, 0))
                continue
            cases = [c for _, c in pairs]
            scale = max(specs[k].ni for k in idx) / base_ni
            res, failed = warm_solve(net, cases, max_steps=int(max_steps * scale),
                                     warm_steps=int(warm_steps * scale), tolerance=tolerance)
            cells = [c.config.grid.ni * c.config.grid.nj for c in cases]
            for j, (k, _) in enumerate(pairs):
                status[k] = res.status[j]
                steps[k] = res.steps[j]
                drags[k] = res.drags[j]
            fell.extend(pairs[j][0] for j in failed)
            reports.append(WaveReport(
                max(specs[k].ni for k in idx), len(idx), len(idx) - len(pairs), sum(cells), res.device_ms, res.predict_s, len(failed),
                sum(1 for s in res.status if s == 0), sum(c * s for c, s in zip(cells, res.steps)),
                res.launches))
            del cases, pairs, res
    return StreamResult(status, steps, drags, fell, reports, time.perf_counter() - t_start, first_build_s, kept)
