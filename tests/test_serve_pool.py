"""Host logic of the serving loop that needs no GPU: the device-memory pool's
first-fit allocation and coalescing, and the batch item layout."""
import ctypes as C
import random

import numpy as np

from sleek_b200 import _capi
from sleek_b200.serve import GRANULE, ITEM_DTYPE, DevicePool


def test_item_layout_matches_the_c_struct():
    assert ITEM_DTYPE.itemsize == C.sizeof(_capi.BatchItem)
    for name, _ in _capi.BatchItem._fields_:
        assert ITEM_DTYPE.fields[name][1] == getattr(_capi.BatchItem, name).offset


def test_pool_first_fit_and_coalescing():
    p = DevicePool(64 * GRANULE, device="cpu")
    a = p.alloc(10 * GRANULE)
    b = p.alloc(1)
    c = p.alloc(20 * GRANULE)
    assert (a, b, c) == (0, 10 * GRANULE, 11 * GRANULE)
    assert p.free_bytes == 33 * GRANULE
    assert p.alloc(40 * GRANULE) is None
    p.free(b, 1)
    p.free(a, 10 * GRANULE)
    assert p.alloc(11 * GRANULE) == 0  # a and b merged
    p.free(0, 11 * GRANULE)
    p.free(c, 20 * GRANULE)
    assert p.free_bytes == 64 * GRANULE
    assert p.alloc(64 * GRANULE) == 0  # everything merged back


def test_pool_random_alloc_free_keeps_accounting():
    rng = random.Random(3)
    p = DevicePool(1 << 20, device="cpu")
    live = []
    for _ in range(3000):
        if live and rng.random() < 0.45:
            off, n = live.pop(rng.randrange(len(live)))
            p.free(off, n)
        else:
            n = rng.randint(1, 40000)
            off = p.alloc(n)
            if off is not None:
                live.append((off, n))
        spans = sorted((o, o + max(GRANULE, (n + GRANULE - 1) // GRANULE * GRANULE)) for o, n in live)
        assert all(e <= s2 for (_, e), (s2, _) in zip(spans, spans[1:]))  # no overlap
    for off, n in live:
        p.free(off, n)
    assert p.free_bytes == p.size and p.alloc(p.size) == 0
