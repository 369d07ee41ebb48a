"""Solution verification of a computed quantity: iterative convergence of the
value on one grid, and its discretisation error from a nested family of grids
refined by 2. Restates src/verification/iterative-convergence.ts:54-121
(SettlingValue) and src/verification/grid-convergence.ts:109-283
(gridConvergence, refineUntilVerified).

Grid convergence index: I. B. Celik, U. Ghia, P. J. Roache and C. J. Freitas,
"Procedure for estimation and reporting of uncertainty due to discretization in
CFD applications", J. Fluids Eng. editorial policy (2008), steps 3 to 5, with
ratio 2: p = |ln|e32/e21|| / ln 2, phi_ext = (2^p phi1 - phi2) / (2^p - 1),
GCI = 1.25 |e21| / (2^p - 1) (absolute). As in the reference, the order is
capped at the scheme's formal order 2, the asymptotic range is judged by the
agreement of the two finest triples' orders (four grids), a finest change
under the noise is bounded by the coarser triple's prediction, and an
oscillation is bounded by the range of the three finest values (F. Stern et
al., J. Fluids Eng. 123 (2001) 793-802, with the full range).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable

FORMAL_ORDER = 2.0
SAFETY_FACTOR = 1.25
RATIO = 2.0
GRID_MEASURABLE = 10.0      # a change between grids carries an order above this x noise
SETTLE_MEASURABLE = 10.0    # a change between checks gives a rate above this x noise
RATE_POINTS = 8


class SettlingValue:
    """Whether an iterated value has stopped changing by more than its noise
    (relative). It approaches its limit geometrically at a rate r per check,
    so what remains after the last k checks is |v_n - v_(n-k)| r^k / (1 - r^k);
    r is the slope of a least-squares line through the logarithms of the last
    eight changes of ten times the noise or more, or a rate known from a
    coarser grid (the larger of the usable ones); k is the number of checks
    over which the error halves. The change and what remains must both be
    within the noise on two successive checks."""

    def __init__(self, noise: float, known_rate: float = math.nan):
        self.noise = noise
        self.known_rate = known_rate
        self.values: list[float] = []
        self.measurable: list[tuple[int, float]] = []
        self.passes = 0

    @property
    def measured_rate(self) -> float:
        pts = self.measurable[-RATE_POINTS:]
        if len(pts) < 2:
            return math.nan
        mx = sum(x for x, _ in pts) / len(pts)
        my = sum(y for _, y in pts) / len(pts)
        sxy = sum((x - mx) * (y - my) for x, y in pts)
        sxx = sum((x - mx) ** 2 for x, _ in pts)
        return math.exp(sxy / sxx)

    @property
    def rate(self) -> float:
        usable = [r for r in (self.measured_rate, self.known_rate) if r < 1]
        return max(usable) if usable else math.nan

    @property
    def rate_to_pass_on(self) -> float:
        m = self.measured_rate
        return m if m < 1 else self.known_rate

    def add(self, value: float) -> bool:
        """Records the value after the next check; True once settled."""
        n = len(self.values)
        change = abs(value - self.values[-1]) if n > 0 else math.nan
        self.values.append(value)
        allowed = self.noise * abs(value)
        if change > SETTLE_MEASURABLE * allowed:
            self.measurable.append((n, math.log(change)))
        rate = self.rate
        remaining = 0.0
        if rate < 1:
            k = max(1, math.ceil(math.log(0.5) / math.log(rate)))
            if n < k:
                remaining = math.inf
            else:
                f = rate ** k
                remaining = abs(value - self.values[n - k]) * f / (1 - f)
        passed = change <= allowed and remaining <= allowed
        self.passes = self.passes + 1 if passed else 0
        return self.passes >= 2


@dataclass(frozen=True)
class Estimate:
    """kind: 'monotone' (value, extrapolated, order, uncertainty),
    'oscillatory' (value, uncertainty) or 'unresolved' (value, reason)."""

    kind: str
    value: float
    uncertainty: float | None = None
    extrapolated: float | None = None
    order: float | None = None
    reason: str | None = None


_OSCILLATES = "the values oscillate under refinement"
_TOO_SMALL = "the changes between grids are too small to measure"


def _unmeasurable(values, noise: float) -> float:
    return GRID_MEASURABLE * noise * max(abs(v) for v in values)


def _observed_order(coarse: float, medium: float, fine: float, noise: float):
    e21 = medium - fine
    e32 = coarse - medium
    lim = _unmeasurable((coarse, medium, fine), noise)
    if abs(e21) <= lim or abs(e32) <= lim:
        return _TOO_SMALL
    if e32 / e21 < 0:
        return _OSCILLATES
    if abs(e32 / e21) <= 1:
        return "the changes do not shrink under refinement"
    return math.log(abs(e32 / e21)) / math.log(RATIO)


def _within_noise(values, coarse_order: float, noise: float) -> Estimate:
    value = values[3]
    e21 = values[2] - value
    predicted = (values[1] - values[2]) / RATIO ** coarse_order
    if not abs(e21 - predicted) <= _unmeasurable(values, noise):
        return Estimate("unresolved", value, reason=(
            f"the finest change ({e21:.2e}) is below the noise but not the one the coarser "
            f"grids predict ({predicted:.2e})"))
    gain = RATIO ** min(coarse_order, FORMAL_ORDER) - 1
    scale = noise * max(abs(v) for v in values)
    bound = max(abs(e21), abs(predicted)) + 2 * scale
    return Estimate("monotone", value, uncertainty=SAFETY_FACTOR * bound / gain,
                    extrapolated=value - predicted / gain, order=coarse_order)


def grid_convergence(values, order_tolerance: float, noise: float) -> Estimate:
    """Error estimate of values on grids refined successively by 2, coarsest
    first (gridConvergence, src/verification/grid-convergence.ts:109-149)."""
    values = [float(v) for v in values]
    if not all(math.isfinite(v) for v in values):
        raise ValueError("the values must be finite")
    n = len(values)
    value = values[-1]
    if n < 4:
        return Estimate("unresolved", value, reason="four grids are needed to confirm the order")
    finest = values[-3:]
    fine = _observed_order(finest[0], finest[1], value, noise)
    if fine == _OSCILLATES:
        return Estimate("oscillatory", value, uncertainty=max(finest) - min(finest))
    coarse = _observed_order(values[-4], values[-3], values[-2], noise)
    if fine == _TOO_SMALL and not isinstance(coarse, str):
        return _within_noise(values[-4:], coarse, noise)
    for triple in (fine, coarse):
        if isinstance(triple, str):
            return Estimate("unresolved", value, reason=triple)
    if not abs(fine - coarse) <= order_tolerance:
        return Estimate("unresolved", value, reason=(
            f"the observed orders of the two finest triples differ ({coarse:.2f} and {fine:.2f})"))
    p = min(fine, FORMAL_ORDER)
    e21 = values[-2] - value
    gain = RATIO ** p - 1
    return Estimate("monotone", value, uncertainty=SAFETY_FACTOR * abs(e21) / gain,
                    extrapolated=value - e21 / gain, order=fine)


@dataclass
class VerifiedValue:
    estimate: Estimate
    uncertainty: float | None      # discretisation estimate + floor |value|, absolute
    verified: bool                 # the band is known and within the tolerance
    levels: list[tuple[int, float]] = field(default_factory=list)
    stopped: tuple[int, str] | None = None


def refine_until_verified(solve_at: Callable[[int], float], tolerance: float, floor: float,
                          max_refinement: int, order_tolerance: float, noise: float,
                          stop_on: Callable[[Exception], str | None] | None = None) -> VerifiedValue:
    """Solves on grids refined by 2 until the value's error band is known and
    within `tolerance` or `max_refinement` is reached (refineUntilVerified,
    src/verification/grid-convergence.ts:253-283)."""
    levels: list[tuple[int, float]] = []
    result: VerifiedValue | None = None
    r = 1
    while r <= max_refinement:
        try:
            value = solve_at(r)
        except Exception as e:  # a finer grid that cannot be solved
            reason = stop_on(e) if (result is not None and stop_on is not None) else None
            if result is None or reason is None:
                raise
            result.stopped = (r, reason)
            return result
        levels.append((r, value))
        est = grid_convergence([v for _, v in levels], order_tolerance, noise)
        unc = None if est.kind == "unresolved" else est.uncertainty + floor * abs(est.value)
        result = VerifiedValue(est, unc, unc is not None and unc <= tolerance, list(levels))
        if result.verified:
            break
        r *= 2
    if result is None:
        raise ValueError("the finest refinement must be at least 1")
    return result
