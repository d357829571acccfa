"""Host logic of the batched consumers: dedup grouping of identical cross-sections."""

from __future__ import annotations

import numpy as np

from omb200.consumers import dedup_groups


def test_dedup_groups():
    a = np.ones((3, 3, 4, 4))
    b = 2 * a
    reps, gid = dedup_groups([a, b, a.copy(), b, 3 * a])
    assert reps == [0, 1, 4]
    assert gid == [0, 1, 0, 1, 2]
