"""Pins the CPU oracle to the reference: the arith cases of test_gpu_arith.py run
with the oracle as the engine under test and the reference library (built from the
reference's own sources by oracle/build_ref.sh) as the checker."""

from __future__ import annotations

import pytest

from .test_gpu_arith import (  # noqa: F401  (re-collected here with other engines)
    test_elementwise,
    test_forward_inverse,
    test_mod_reduce_lifted_and_division,
    test_mul_by_xai,
    test_permute,
    test_round_trip_identity,
    test_scaled_lift_and_base_extension,
    test_transform_prime_sizes_and_extremes,
)

CPU_RINGS = [
    (16, [50, 50], 1),
    (256, [50, 50, 50], None),
    (1024, [20, 20], 8),
    (4096, [50, 50, 50], None),
    (4096, [50, 50, 50], 1),
    (2**12, [50] + [40] * 3 + [50], 1),
]


@pytest.fixture
def engines(oracle_engine, ref_portable):
    return [oracle_engine, ref_portable]


@pytest.fixture(params=CPU_RINGS, ids=lambda p: f"N{p[0]}-s{p[2]}-L{len(p[1])}")
def rings(request, engines):
    from .helpers import twin_rings

    N, sizes, split = request.param
    return twin_rings(engines, N, sizes, split)
