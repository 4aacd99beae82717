"""The serving loop (continuous batching over several streams, outputs in a
device pool admitted by free memory): every request's result is bit-identical to
the same request run alone through the single-buffer entry points, and the loop
reports latency percentiles and throughput."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sleek_b200 import api
from sleek_b200.serve import Request, Server

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
