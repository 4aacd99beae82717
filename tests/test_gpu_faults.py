"""Fault injection on the device decoder: random byte corruptions and
truncations of valid streams (planted on the host), decoded with the stream
length and output capacity given.  The device must agree with the host
validator on every stream -- accept exactly the streams the validator accepts,
decoding them bit-identically to the oracle, and report the others as a status
(corrupt stream, or capacity when the header asks for more than the output
holds) without a trap, a hang or a write outside the output."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sleek_b200 import api

pytestmark = pytest.mark.gpu

SLEEK_ERR_CORRUPT_STREAM = 5
SLEEK_ERR_CAPACITY = 9


def _corruptions(s, rng, count):
    for t in range(count):
        b = bytearray(s)
        if t % 5 == 4:
            b = b[: int(rng.integers(0, len(b)))]
        else:
            hi = (8, 8 + 8, len(b))[int(rng.integers(0, 3))]
            for _ in range(int(rng.integers(1, 4))):
                b[int(rng.integers(0, hi))] = int(rng.integers(0, 256))
        yield bytes(b)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("eb", [None, 1e-3])
def test_device_decoder_agrees_with_validator(cuda, dtype, eb):
    rng = np.random.default_rng(21 if eb is None else 22)
    n = 3 * 16384 // np.dtype(dtype).itemsize + 5
    x = (np.cumsum(rng.normal(0, 1, n)) * 0.3).astype(dtype)
    s = O.encode(x, eb)
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    guard = 64  # elements past the capacity that must stay untouched
    out = torch.empty(n + guard, dtype=tdt, device="cuda")
    size = torch.empty(1, dtype=torch.int64, device="cuda")
    info = api.sleek_error_bound(eb, dtype) if eb is not None else None
    seen = {"valid": 0, "corrupt": 0, "capacity": 0}
    for b in _corruptions(s, rng, 300):
        v = api.validate_stream(b, dtype)
        enc = torch.frombuffer(bytearray(b) or bytearray(1), dtype=torch.uint8).cuda()
        out.fill_(7.0)
        view = out[:n]
        args = (enc, view, size) if info is None else (info, enc, view, size)
        try:
            api.sleek_decompress_gpu(0, *args, encoded_bytes=len(b))
            got = int(size.item())
        except api.SleekError as e:  # rejected on the host (shorter than a header)
            assert len(b) < 8
            got = -e.status
        assert torch.all(out[n:] == 7.0)
        if v["valid"] and v["insize"] <= x.nbytes:
            assert got == v["insize"], (v, got)
            want = O.decode(b, dtype, eb)
            assert view[: got // x.itemsize].cpu().numpy().tobytes() == want.tobytes()
            seen["valid"] += 1
        elif v["valid"]:
            assert got == -SLEEK_ERR_CAPACITY, (v, got)
            seen["capacity"] += 1
        else:
            assert got in (-SLEEK_ERR_CORRUPT_STREAM, -SLEEK_ERR_CAPACITY), (v, got)
            if v["insize"] <= x.nbytes and v["reason"] != 1:
                assert got == -SLEEK_ERR_CORRUPT_STREAM, (v, got)
            seen["corrupt"] += 1
    assert seen["valid"] > 10 and seen["corrupt"] > 10, seen
    # the device is still usable and exact afterwards
    y = api.decompress(torch.frombuffer(bytearray(s), dtype=torch.uint8).cuda(), dtype, eb)
    assert y.cpu().numpy().tobytes() == O.decode(s, dtype, eb).tobytes()
