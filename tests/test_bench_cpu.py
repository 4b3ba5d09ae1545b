"""Host-side helpers of bench.py, on the CPU.

neighbour_work counts, at one particle state, the candidates a query tests
(the particles of the 27 cells around its own cell of size h) and the
in-range pairs (r <= h, self excluded); both are checked here against brute
force on a small seeded point set.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), ".."))
import bench  # noqa: E402


def test_neighbour_work_matches_brute_force():
    pytest.importorskip("scipy")
    rng = np.random.default_rng(11)
    h = 0.1
    x = rng.uniform(0.0, 0.8, size=(1500, 3)).astype(np.float32)
    w = bench.neighbour_work(x, h, step_ms=2.0, passes=10, sample=len(x))
    x64 = x.astype(np.float64)
    c = np.floor(x64 / h).astype(np.int64)
    near = (np.abs(c[:, None, :] - c[None, :, :]) <= 1).all(axis=2)
    cand = near.sum(axis=1).mean()
    r2 = ((x64[:, None, :] - x64[None, :, :]) ** 2).sum(axis=2)
    pairs = (r2 <= h * h).sum(axis=1).mean() - 1.0
    assert w["candidates_per_particle"] == pytest.approx(cand, abs=0.05)
    assert w["in_range_pairs_per_particle"] == pytest.approx(pairs, abs=0.01)
    assert w["pair_evaluations_per_s"] == pytest.approx(w["in_range_pairs_per_particle"] * len(x) * 10 / 2e-3,
                                                        rel=1e-3)
