"""Display fields (schlieren, Mach, Cp, density) computed on the GPU against
the reference's cell formulas (src/render/flow-fields.ts:36-117) restated
here in numpy on the same state."""
from __future__ import annotations

import numpy as np
import pytest

from bowshock_b200.batch import CudaBatch
from bowshock_b200.workloads import ogive_case

pytestmark = pytest.mark.gpu
GAMMA = 1.4


def _reference_fields(grid, w, free, length):
    ni, nj = grid.ni, grid.nj
    rho, u, v, p = (w[:, k].reshape(nj, ni) for k in range(4))
    st = free.state
    mach = np.hypot(u, v) / np.sqrt(GAMMA * p / rho)
    cp = (p - st.p) / (0.5 * st.rho * (st.u ** 2 + st.v ** 2))
    X = grid.x.reshape(nj + 1, ni + 1)
    Y = grid.y.reshape(nj + 1, ni + 1)
    sch = np.empty((nj, ni))
    for j in range(nj):
        for i in range(ni):
            corners = [(i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)]
            across = [(i, j - 1), (i + 1, j), (i, j + 1), (i - 1, j)]
            gx = gy = area = 0.0
            for e in range(4):
                (ai, aj), (bi, bj) = corners[e], corners[(e + 1) % 4]
                ci, cj = across[e]
                inside = 0 <= ci < ni and 0 <= cj < nj
                q = 0.5 * (rho[j, i] + rho[cj, ci]) if inside else rho[j, i]
                dx = X[bj, bi] - X[aj, ai]
                dy = Y[bj, bi] - Y[aj, ai]
                gx += q * dy
                gy -= q * dx
                area += 0.5 * (X[aj, ai] * Y[bj, bi] - X[bj, bi] * Y[aj, ai])
            sch[j, i] = np.hypot(gx, gy) / abs(area) * length / st.rho
    return {"schlieren": sch.ravel(), "mach": mach.ravel(), "cp": cp.ravel(), "density": (rho / st.rho).ravel()}


def test_display_fields_match_the_reference_formulas():
    case = ogive_case(2.5, 40, 20)
    b = CudaBatch([case.config], precision=64)
    b.set_free_stream()
    b.solve("lusgs", 1e-6, max_steps=200, check_every=20)
    w = b.primitives(0).reshape(-1, 4)
    ref = _reference_fields(case.config.grid, w, case.free, 0.5)
    for name, want in ref.items():
        got = b.flow_field(0, name, case.free, 0.5)
        assert np.allclose(got, want, rtol=1e-10, atol=1e-12), name
    # The flow is not uniform after 200 steps: the fields vary.
    assert ref["mach"].std() > 0.05 and ref["schlieren"].max() > 0.1
    b.destroy()
