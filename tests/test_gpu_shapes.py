"""Launch shapes of the single-buffer kernels (threads per CTA, compute warps,
stages, CTAs per SM) and the autotuner that picks them: every shape writes the
same bytes as the oracle, and a tuned choice is applied per input-size bucket."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sleek_b200 import _capi, api, autotune

pytestmark = pytest.mark.gpu


@pytest.fixture
def default_shapes():
    yield
    L = _capi.lib()
    for dec in (0, 1):
        for w in (4, 8):
            for lossy in (0, 1):
                _capi.check(L.sleek_set_launch_shape(dec, w, lossy, -1, 0, 0))


def _field(n, dt, seed):
    rng = np.random.default_rng(seed)
    x = (np.cumsum(rng.normal(0, 1, n)) * 0.3).astype(dt)
    x[rng.choice(n, n // 500, replace=False)] = np.nan
    return x


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("eb", [None, 1e-3])
def test_every_shape_writes_the_oracle_bytes(cuda, default_shapes, dt, eb):
    L = _capi.lib()
    w = np.dtype(dt).itemsize
    x = _field(300 * 16384 // w + 77, dt, 11)
    t = torch.from_numpy(x).cuda()
    want = O.encode(x, eb)
    want_dec = O.decode(want, dt, eb).tobytes()
    for dec in (0, 1):
        for shape, ctas in autotune.single_candidates(bool(dec)):
            _capi.check(L.sleek_set_launch_shape(dec, w, int(eb is not None), -1, shape, ctas))
            s = api.compress(t, eb)
            assert s.cpu().numpy().tobytes() == want, (dec, shape, ctas)
            y = api.decompress(s, dt, eb)
            assert y.cpu().numpy().tobytes() == want_dec, (dec, shape, ctas)


def test_autotuner_applies_a_shape_per_size_bucket(cuda, default_shapes):
    x = torch.from_numpy(_field(2000 * 4096, np.float32, 12)).cuda()
    for dec in (False, True):
        r = autotune.tune_single(x, None, decompress=dec, use_cache=False)
        assert r["bucket_log2"] == (x.numel() * 4).bit_length() - 1
        assert len(r["ms"]) == len(autotune.single_candidates(dec))
        assert r["shape"]["shape"] == r["best"][0]
    # the tuned bucket still writes the oracle's stream
    assert api.compress(x, None).cpu().numpy().tobytes() == O.encode(x.cpu().numpy(), None)
