"""TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.

Anderson acceleration of a fixed-point iteration x <- x + f(x), restated
from src/solver/anderson.ts:20-123 (AndersonMixing): Walker and Ni's type II
form (SIAM J. Numer. Anal. 49 (2011) 1715-1735) without damping. With the
last `depth` differences of the iterates, dX, and of their corrections, dF,

    gamma = argmin |f - dF gamma|,   x_next = x + f - (dX + dF) gamma,

the least-squares problem solved by modified Gram-Schmidt, the oldest
columns dropped while a column keeps less than 1e-10 of its norm after
orthogonalisation (anderson.ts:78-114). The tests use it as the checker of
the GPU's accelerated LU-SGS steps and pin it to the reference's own known
answers.
"""
from __future__ import annotations

import numpy as np


class AndersonMixing:
    def __init__(self, size: int, depth: int):
        if depth < 1:
            raise ValueError("depth must be at least 1")
        self.size = size
        self.depth = depth
        self.reset()

    def reset(self) -> None:
        """Forgets the history (anderson.ts:35-41)."""
        self.dx: list[np.ndarray] = []
        self.df: list[np.ndarray] = []
        self.last_x: np.ndarray | None = None
        self.last_f: np.ndarray | None = None

    def next(self, x: np.ndarray, f: np.ndarray) -> np.ndarray:
        """The next iterate from x and its correction f (anderson.ts:44-71)."""
        x = np.asarray(x, np.float64)
        f = np.asarray(f, np.float64)
        if x.shape != (self.size,) or f.shape != (self.size,):
            raise ValueError("wrong vector size")
        if self.last_x is not None:
            self.dx.append(x - self.last_x)
            self.df.append(f - self.last_f)
            if len(self.dx) > self.depth:
                self.dx.pop(0)
                self.df.pop(0)
        self.last_x = x.copy()
        self.last_f = f.copy()
        out = x + f
        for g, dx, df in zip(self._least_squares(f), self.dx, self.df):
            if g != 0.0:
                out -= g * (dx + df)
        return out

    def _least_squares(self, f: np.ndarray) -> np.ndarray:
        m = len(self.df)
        gamma = np.zeros(m)
        for first in range(m):
            cols = m - first
            q: list[np.ndarray] = []
            r = np.zeros((cols, cols))
            ok = True
            for c in range(cols):
                v = self.df[first + c].copy()
                norm0 = float(np.sqrt(v @ v))
                for p in range(c):
                    proj = float(q[p] @ v)
                    r[p, c] = proj
                    v -= proj * q[p]
                norm = float(np.sqrt(v @ v))
                if not norm > 1e-10 * norm0 or norm0 == 0.0:
                    ok = False
                    break
                r[c, c] = norm
                q.append(v / norm)
            if not ok:
                continue
            rhs = [float(qc @ f) for qc in q]
            for c in range(cols - 1, -1, -1):
                s = rhs[c] - sum(r[c, p] * gamma[first + p] for p in range(c + 1, cols))
                gamma[first + c] = s / r[c, c]
            return gamma
        return gamma
