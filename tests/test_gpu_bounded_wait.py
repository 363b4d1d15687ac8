"""The bounded waits of the bulk-copy kernels end, flag the fault and keep the context.

Every kernel that waits on an mbarrier for a bulk copy (the persistent transforms, the
staged key-switch MAC) bounds the wait; a wait that gives up raises a device flag the
host reads through vfhe_cuda_device_faults.  Here a one-thread kernel waits on a barrier
that no copy will ever complete, with a short limit: it must return, the flag must be
set and then clear, and the engine must keep computing correct results afterwards.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_survives(cuda, oracle_engine):
    lib = cuda.lib
    assert lib.vfhe_cuda_device_faults() == 0
    assert lib.vfhe_cuda_selfcheck_bounded_wait(4096) == 1
    assert lib.vfhe_cuda_device_faults() != 0
    assert lib.vfhe_cuda_clear_device_faults() == 0
    assert lib.vfhe_cuda_device_faults() == 0

    # the context is still usable: a transform matches the oracle
    from .helpers import poly_from_rows, same, twin_rings, uniform_rows

    rings = twin_rings([cuda, oracle_engine], 2**12, [50] * 3, 1)
    rows = uniform_rows(rings[0], np.random.default_rng(5))
    g, o = poly_from_rows(rings[0], rows), poly_from_rows(rings[1], rows)
    g.to_NTT()
    o.to_NTT()
    same(g, o)
