"""Serving host logic without a GPU: the Poisson arrival process."""

from __future__ import annotations

import numpy as np


def test_poisson_arrivals():
    from vfhe_b200.serve import poisson_arrivals

    t = poisson_arrivals(1000.0, 20000, np.random.default_rng(0))
    gaps = np.diff(t)
    assert (gaps >= 0).all()
    assert abs(gaps.mean() - 1e-3) < 5e-5  # mean gap 1/rate
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.05  # exponential: coefficient of variation 1
    assert (poisson_arrivals(0.0, 5, np.random.default_rng(0)) == 0).all()
