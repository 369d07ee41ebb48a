"""Host-side pieces of the learned warm start: case values, cell samples and
the target transforms (no GPU)."""
from __future__ import annotations

import numpy as np

from bowshock_b200.config import free_stream_at
from bowshock_b200.mlp import (case_samples, case_values, primitives_from_prediction,
                               targets_from_primitives)
from bowshock_b200.workloads import case_from, draw_nose_case, ogive_case


def test_case_values_encode_family_fineness_length_and_mach():
    case = ogive_case(2.5, 40, 20)
    v = case_values(case)
    assert v.shape == (8,) and v[1] == 1.0 and v[[0, 2, 3, 4]].sum() == 0.0
    assert np.isclose(v[5], 3.0 / 5) and np.isclose(v[6], 7.0 / 8) and np.isclose(v[7], 2.5 / 5)


def test_samples_cover_every_cell_inside_the_grid():
    case = case_from(draw_nose_case(3, levels=(0,)))
    s = case_samples(case)
    g = case.config.grid
    assert s.shape == (g.ni * g.nj, 10)
    assert s[:, 0].min() >= g.x.min() and s[:, 0].max() <= g.x.max()
    assert s[:, 1].min() >= 0.0 and s[:, 1].max() <= g.y.max()
    assert np.all(s[:, 2:] == case_values(case))


def test_targets_and_predictions_are_inverse_transforms():
    free = free_stream_at(3.0, 1.4)
    rng = np.random.default_rng(0)
    w = np.stack([rng.uniform(0.5, 5, 100), rng.uniform(-1, 3, 100), rng.uniform(-1, 1, 100),
                  rng.uniform(0.5, 20, 100)], 1)
    t = targets_from_primitives(w, free)
    assert np.allclose(t[:, 0], np.log(w[:, 0]), atol=1e-6)
    back = primitives_from_prediction(t, free).reshape(-1, 4)
    assert np.allclose(back, w, rtol=1e-5, atol=1e-5)
