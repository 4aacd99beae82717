"""Compressed transfers (sleek_compress_to_host / sleek_decompress_from_host):
the stream assembled in host memory from independently encoded segments is
byte-identical to the oracle's (and to a one-shot device compress) for one
segment, many segments, ragged ends and empty arrays; decompressing from host
memory reproduces the oracle's decode; malformed tables and short buffers are
statuses raised before any device work, malformed chunks statuses from the
device decoder."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sleek_b200 import api

pytestmark = pytest.mark.gpu

CS = 16384


def _data(dtype, n, seed):
    rng = np.random.default_rng(seed)
    x = (np.cumsum(rng.normal(0, 1, n)) * 0.25).astype(dtype)
    if n > 50:
        x[rng.integers(0, n, n // 50)] = np.nan
    return x


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("eb", [None, 1e-4])
@pytest.mark.parametrize("nbytes,seg", [(0, 0), (1000, 0), (5 * CS + 24, 0), (37 * CS + 8, 3 * CS),
                                        (64 * CS, 4 * CS), (41 * CS + 16, CS), (9 * CS, 1)])
def test_round_trip_matches_oracle(cuda, dtype, eb, nbytes, seg):
    w = np.dtype(dtype).itemsize
    x = _data(dtype, nbytes // w, nbytes + w)
    want = O.encode(x, eb)
    t = torch.from_numpy(x).cuda() if x.size else torch.empty(0, dtype=torch.from_numpy(x).dtype, device="cuda")
    h = api.compress_to_host(t, eb, segment_bytes=seg)
    assert not h.is_cuda
    assert h.numpy().tobytes() == want
    if x.size:
        assert api.compress(t, eb).cpu().numpy().tobytes() == want
    y = api.decompress_from_host(h, dtype, eb, segment_bytes=seg)
    assert y.is_cuda
    assert y.cpu().numpy().tobytes() == O.decode(want, dtype, eb).tobytes()


def test_pageable_host_buffers(cuda):
    x = _data(np.float32, 20 * CS // 4 + 3, 9)
    want = O.encode(x)
    out = torch.empty(api.sleek_upper_bound_size(x.nbytes), dtype=torch.uint8)  # not pinned
    h = api.compress_to_host(torch.from_numpy(x).cuda(), out=out, segment_bytes=4 * CS)
    assert h.numpy().tobytes() == want
    y = api.decompress_from_host(torch.frombuffer(bytearray(want), dtype=torch.uint8), np.float32,
                                 segment_bytes=4 * CS)
    assert y.cpu().numpy().tobytes() == x.tobytes()


def test_errors_before_device_work(cuda):
    x = _data(np.float64, 10 * CS // 8, 3)
    s = bytearray(O.encode(x, 1e-3))
    s[8], s[9] = 0, 0  # first csize 0
    with pytest.raises(api.SleekError) as e:
        api.decompress_from_host(torch.frombuffer(s, dtype=torch.uint8), np.float64, 1e-3)
    assert e.value.status == 5
    # a chunk-level defect (a bit width above 64) is found by the device decoder
    s = bytearray(O.encode(x, 1e-3))
    s[8 + 2 * 10] = 65
    with pytest.raises(api.SleekError) as e:
        api.decompress_from_host(torch.frombuffer(s, dtype=torch.uint8), np.float64, 1e-3, segment_bytes=3 * CS)
    assert e.value.status == 5
    good = torch.frombuffer(bytearray(O.encode(x, 1e-3)), dtype=torch.uint8)
    small = torch.empty(10, dtype=torch.float64, device="cuda")
    with pytest.raises(api.SleekError) as e:
        api.decompress_from_host(good, np.float64, 1e-3, out=small)
    assert e.value.status == 9
    with pytest.raises(api.SleekError) as e:
        api.compress_to_host(torch.from_numpy(x).cuda(), out=torch.empty(64, dtype=torch.uint8))
    assert e.value.status == 9
    # still exact afterwards
    assert api.compress_to_host(torch.from_numpy(x).cuda(), 1e-3).numpy().tobytes() == O.encode(x, 1e-3)
