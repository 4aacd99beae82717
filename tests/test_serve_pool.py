"""Host logic of the serving loop that needs no GPU: the device-memory pool's
next-fit allocation and coalescing, the batch item layout, and the loop's
refusal of requests that can never be admitted (it must end, not spin)."""
import ctypes as C
import random
import time

import numpy as np
import pytest
import torch

from sleek_b200 import _capi
from sleek_b200.serve import GRANULE, ITEM_DTYPE, DevicePool, Request, Server


def test_item_layout_matches_the_c_struct():
    assert ITEM_DTYPE.itemsize == C.sizeof(_capi.BatchItem)
    for name, _ in _capi.BatchItem._fields_:
        assert ITEM_DTYPE.fields[name][1] == getattr(_capi.BatchItem, name).offset


def test_pool_next_fit_and_coalescing():
    p = DevicePool(64 * GRANULE, device="cpu")
    a = p.alloc(10 * GRANULE)
    b = p.alloc(1)
    c = p.alloc(20 * GRANULE)
    assert (a, b, c) == (0, 10 * GRANULE, 11 * GRANULE)
    assert p.free_bytes == 33 * GRANULE
    assert p.alloc(40 * GRANULE) is None
    p.free(b, 1)
    p.free(a, 10 * GRANULE)
    t = p.alloc(33 * GRANULE)  # next fit: the search starts after c
    assert t == 31 * GRANULE
    assert p.alloc(11 * GRANULE) == 0  # wraps around to a and b, merged
    p.free(0, 11 * GRANULE)
    p.free(c, 20 * GRANULE)
    p.free(t, 33 * GRANULE)
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


def _bare_server(pool_bytes, max_batch_chunks=1 << 10):
    """A server without CUDA streams or plans: admission and the loop's exit
    conditions only (with no slot nothing is ever launched)."""
    srv = Server.__new__(Server)
    srv.pool = DevicePool(pool_bytes, device="cpu")
    srv.max_batch, srv.max_batch_chunks = 8, max_batch_chunks
    srv.slots, srv.queue, srv.completed = [], [], []
    srv.t0 = time.perf_counter()
    return srv


def test_server_fails_what_can_never_be_admitted_and_ends():
    srv = _bare_server(1 << 20, max_batch_chunks=16)
    x = torch.zeros(1 << 20, dtype=torch.float32)  # 4 MB: its stream cannot fit a 1 MB pool
    y = torch.zeros(1 << 17, dtype=torch.float32)  # 512 KB = 32 chunks: more than a launch holds
    z = torch.zeros(1 << 10, dtype=torch.float32)  # fits, but no slot will ever run it
    reqs = [Request("compress", t, np.dtype(np.float32), None, arrival=0.0, rid=i) for i, t in enumerate((x, y, z))]
    stats = srv.serve(reqs)
    assert stats["requests"] == 3 and stats["errors"] == 3
    for r in reqs:
        assert r.result_bytes == -_capi.SLEEK_ERR_CAPACITY
        with pytest.raises(_capi.SleekError):
            srv.result(r)
    assert srv.pool.free_bytes == srv.pool.size and not srv.queue


def _take_by_walking(srv):
    """The admission rule written as a walk over the whole queue (every request
    after a full launch is kept unchanged)."""
    take, chunks, keep = [], 0, []
    for r in srv.queue:
        ch = (r.raw_bytes + 16383) // 16384
        if len(take) < srv.max_batch and chunks + ch <= srv.max_batch_chunks:
            n = srv._out_bytes(r)
            off = srv.pool.alloc(n)
            if off is not None:
                r.out_off, r.out_bytes = off, n
                take.append(r)
                chunks += ch
                continue
        keep.append(r)
    srv.queue = keep
    return take


def test_take_equals_the_full_walk():
    rng = random.Random(5)
    src = torch.zeros(1 << 18, dtype=torch.float32)
    for trial in range(40):
        sizes = [rng.choice([1, 100, 5000, 40000, 200000]) for _ in range(rng.randint(1, 60))]
        a = _bare_server(rng.choice([1 << 20, 4 << 20, 64 << 20]), max_batch_chunks=rng.choice([8, 64, 1024]))
        b = _bare_server(a.pool.size, a.max_batch_chunks)
        a.max_batch = b.max_batch = rng.choice([1, 3, 8, 100])
        for srv in (a, b):
            srv.queue = [Request("compress", src[:n], np.dtype(np.float32), None, rid=i) for i, n in enumerate(sizes)]
        for _ in range(4):  # successive launches from the same queue and pool
            got = [(r.rid, r.out_off) for r in a._take()]
            want = [(r.rid, r.out_off) for r in _take_by_walking(b)]
            assert got == want, trial
            assert [r.rid for r in a.queue] == [r.rid for r in b.queue]
