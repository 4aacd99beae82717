"""The serving loop (continuous batching over several streams, outputs in a
device pool admitted by free memory), in Python (Server) and in a thread of the
library (NativeServer): every request's result is bit-identical to the same
request run alone through the single-buffer entry points, and the loop reports
latency percentiles and throughput."""
import time

import numpy as np
import pytest
import torch

from oracle import oracle as O
from sleek_b200 import api
from sleek_b200 import _capi
from sleek_b200.serve import NativeServer, Request, Server

pytestmark = pytest.mark.gpu


def _requests(n, seed):
    rng = np.random.default_rng(seed)
    src32 = torch.cumsum(torch.randn(1 << 22, device="cuda", dtype=torch.float64), 0).float() * 0.01
    src64 = torch.cumsum(torch.randn(1 << 21, device="cuda", dtype=torch.float64), 0) * 0.01
    bank = []
    for i in range(8):  # streams for the decompress requests
        dt = np.float32 if i % 2 else np.float64
        src = src32 if dt == np.float32 else src64
        cnt = int(rng.integers(1, 300_000))
        eb = None if i % 3 == 0 else 1e-3
        bank.append((api.compress(src[:cnt].contiguous(), eb), dt, eb, cnt))
    reqs, t = [], 0.0
    for k in range(n):
        t += rng.exponential(2e-4)
        if rng.random() < 0.6:
            dt = np.float32 if rng.random() < 0.5 else np.float64
            src = src32 if dt == np.float32 else src64
            cnt = int(np.exp(rng.uniform(np.log(256), np.log(2_000_000))))
            off = int(rng.integers(0, src.numel() - cnt))
            eb = None if rng.random() < 0.5 else float(10 ** rng.uniform(-6, -2))
            reqs.append(Request("compress", src[off:off + cnt], np.dtype(dt), eb, arrival=t, rid=k))
        else:
            s, dt, eb, cnt = bank[int(rng.integers(0, len(bank)))]
            reqs.append(Request("decompress", s, np.dtype(dt), eb, num_elements=cnt, arrival=t, rid=k))
    return reqs


def test_serving_results_equal_alone_runs(cuda):
    reqs = _requests(300, 1)
    srv = Server(hbm_budget=2 << 30, slots=3, max_batch=64)
    stats = srv.serve(reqs, keep=lambda r: True)
    assert stats["requests"] == len(reqs) and stats["errors"] == 0
    assert stats["p50_ms"] > 0 and stats["p99_ms"] >= stats["p50_ms"]
    for r in reqs:
        got = srv.result(r)
        if r.op == "compress":
            alone = api.compress(r.src, r.eb)
            assert torch.equal(got, alone)
        else:
            alone = api.decompress(r.src, r.dtype, r.eb)
            assert torch.equal(got, alone.view(torch.uint8))
        srv.release(r)
    assert srv.pool.free_bytes == srv.pool.size
    srv.close()


def test_serving_admits_by_free_memory(cuda):
    # a pool that holds only a few outputs at a time: everything still completes
    reqs = _requests(60, 2)
    srv = Server(hbm_budget=64 << 20, slots=2, max_batch=16)
    stats = srv.serve(reqs)
    assert stats["requests"] == len(reqs) and stats["errors"] == 0
    assert srv.pool.free_bytes == srv.pool.size
    srv.close()


def test_serving_sample_matches_oracle(cuda):
    reqs = [r for r in _requests(40, 3) if r.raw_bytes < (1 << 20)][:10]
    srv = Server(hbm_budget=1 << 30, slots=2, max_batch=8)
    srv.serve(reqs, keep=lambda r: True)
    for r in reqs:
        got = srv.result(r).cpu().numpy().tobytes()
        if r.op == "compress":
            assert got == O.encode(r.src.cpu().numpy(), r.eb)
        else:
            assert got == O.decode(r.src.cpu().numpy().tobytes(), r.dtype, r.eb).tobytes()
        srv.release(r)
    srv.close()


def _alone(r):
    if r.op == "compress":
        return api.compress(r.src, r.eb)
    return api.decompress(r.src, r.dtype, r.eb).view(torch.uint8)


def test_native_serving_results_equal_alone_runs(cuda):
    reqs = _requests(300, 1)
    srv = NativeServer(hbm_budget=2 << 30, slots=3, max_batch=64)
    stats = srv.serve(reqs, keep=lambda r: True)
    assert stats["requests"] == len(reqs) and stats["errors"] == 0
    assert stats["p50_ms"] > 0 and stats["p99_ms"] >= stats["p50_ms"]
    assert all(r.done >= r.arrival for r in reqs)
    for r in reqs:
        assert torch.equal(srv.result(r), _alone(r)), (r.rid, r.op)
        srv.release(r)
    torch.cuda.synchronize()
    for _ in range(100):  # the loop applies releases on its next pass
        free, size = srv.arena_info()
        if free == size:
            break
        time.sleep(0.01)
    assert free == size
    srv.close()


def test_native_serving_admits_by_free_memory(cuda):
    # an arena that holds only a few outputs at a time: everything still completes
    reqs = _requests(60, 2)
    srv = NativeServer(hbm_budget=64 << 20, slots=2, max_batch=16)
    stats = srv.serve(reqs)
    assert stats["requests"] == len(reqs) and stats["errors"] == 0
    srv.close()


def test_native_serving_sample_matches_oracle(cuda):
    reqs = [r for r in _requests(40, 3) if r.raw_bytes < (1 << 20)][:10]
    srv = NativeServer(hbm_budget=1 << 30, slots=2, max_batch=8)
    srv.serve(reqs, keep=lambda r: True)
    for r in reqs:
        got = srv.result(r).cpu().numpy().tobytes()
        if r.op == "compress":
            assert got == O.encode(r.src.cpu().numpy(), r.eb)
        else:
            assert got == O.decode(r.src.cpu().numpy().tobytes(), r.dtype, r.eb).tobytes()
        srv.release(r)
    srv.close()


def test_native_serving_fails_impossible_requests_at_once(cuda):
    x = torch.zeros(3 << 20, dtype=torch.float32, device="cuda")  # 12 MB, output larger than the arena
    small = torch.zeros(1000, dtype=torch.float32, device="cuda")
    reqs = [Request("compress", x, np.dtype(np.float32), None, arrival=0.0, rid=0),
            Request("compress", small, np.dtype(np.float32), None, arrival=0.0, rid=1)]
    srv = NativeServer(hbm_budget=8 << 20, slots=1, max_batch=4)
    stats = srv.serve(reqs, keep=lambda r: True)
    assert stats["requests"] == 2 and stats["errors"] == 1
    assert reqs[0].result_bytes == -_capi.SLEEK_ERR_CAPACITY
    assert torch.equal(srv.result(reqs[1]), api.compress(small, None))
    srv.release(reqs[1])
    srv.close()


def test_native_serving_replays_arrival_times(cuda):
    # requests spaced 20 ms apart are not completed before they arrive
    src = torch.cumsum(torch.randn(1 << 16, device="cuda"), 0)
    reqs = [Request("compress", src, np.dtype(np.float32), 1e-3, arrival=0.02 * k, rid=k) for k in range(5)]
    srv = NativeServer(hbm_budget=256 << 20, slots=2, max_batch=8)
    stats = srv.serve(reqs)
    assert stats["errors"] == 0
    for r in reqs:
        assert r.done >= r.arrival
        assert r.done - r.arrival < 0.015  # served alone, promptly
    assert stats["span_s"] >= 0.08
    srv.close()



def _native_requests(xs, tag0):
    arr = (_capi.ServerRequest * len(xs))()
    for i, x in enumerate(xs):
        q = arr[i]
        q.input = x.data_ptr()
        q.num_elements = x.numel()
        q.tag = tag0 + i
        q.op = 0
        q.elem_bytes = 4
        q.keep = 1
    return arr


def _drain(srv, n):
    L = _capi.lib()
    buf = (_capi.ServerCompletion * 256)()
    got, k = {}, _capi.C.c_longlong()
    while len(got) < n:
        _capi.check(L.sleek_server_poll(srv._h, buf, 256, _capi.C.byref(k), 200))
        for i in range(k.value):
            got[buf[i].tag] = (buf[i].result_bytes, buf[i].output)
    return got


def test_native_server_takes_requests_from_several_threads(cuda):
    import threading

    L = _capi.lib()
    srv = NativeServer(hbm_budget=1 << 30, slots=3, max_batch=32, max_batch_chunks=1 << 14)
    src = torch.cumsum(torch.randn(1 << 22, device="cuda"), 0) * 0.01
    groups = [[src[k * 1000 + j * 7: k * 1000 + j * 7 + 5000 + 300 * j] for j in range(40)] for k in range(4)]
    arrays = [_native_requests(g, 1000 * k) for k, g in enumerate(groups)]
    ths = [threading.Thread(target=lambda a=a: _capi.check(L.sleek_server_submit(srv._h, a, len(a))))
           for a in arrays]
    [t.start() for t in ths]
    [t.join() for t in ths]
    got = _drain(srv, 160)
    for k, g in enumerate(groups):
        for i, x in enumerate(g):
            res, ptr = got[1000 * k + i]
            off = ptr - srv.base
            assert torch.equal(srv.arena[off:off + res], api.compress(x, None))
            assert L.sleek_server_release(srv._h, _capi.C.c_void_p(ptr)) == 0
    n = _capi.C.c_longlong()
    _capi.check(L.sleek_server_outstanding(srv._h, _capi.C.byref(n)))
    assert n.value == 0
    srv.close()


def test_native_server_destroy_with_launches_in_flight(cuda):
    # destroy finishes what was admitted and returns; releases of unknown
    # addresses are ignored
    L = _capi.lib()
    srv = NativeServer(hbm_budget=4 << 30, slots=2, max_batch=16)
    src = torch.cumsum(torch.randn(1 << 26, device="cuda"), 0) * 0.01
    xs = [src[j << 20: (j << 20) + (8 << 20)] for j in range(20)]
    a = _native_requests(xs, 0)
    _capi.check(L.sleek_server_submit(srv._h, a, len(a)))
    assert L.sleek_server_release(srv._h, _capi.C.c_void_p(srv.base + 12345 * 256)) == 0
    srv.close()  # returns once the admitted work is done
    torch.cuda.synchronize()
