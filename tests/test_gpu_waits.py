"""Device-side time limits: a wait that nothing will ever satisfy (an mbarrier
without arrivals, a look-back whose predecessor never publishes) gives up after
its limit and reports it instead of hanging, and the device stays usable.  The
waits are the ones the encode and decode kernels use."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
from sleek_b200 import _capi, api

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("limit_ms", [20, 200])
def test_waits_give_up_after_their_limit(cuda, limit_ms):
    res = (C.c_longlong * 3)()
    _capi.check(_capi.lib().sleek_selftest_bounded_waits(limit_ms * 1_000_000, res))
    gave_up, lookback, ns = res[0], res[1], res[2]
    assert gave_up == 1 and lookback == -1
    assert 2 * limit_ms * 1e6 <= ns < 2 * limit_ms * 1e6 + 2e9
    # the context is intact: a compress right after is exact
    x = np.cumsum(np.random.default_rng(limit_ms).normal(0, 1, 50_000)).astype(np.float64)
    assert api.compress(torch.from_numpy(x).cuda(), 1e-3).cpu().numpy().tobytes() == O.encode(x, 1e-3)


def test_selftest_rejects_bad_limits(cuda):
    res = (C.c_longlong * 3)()
    assert _capi.lib().sleek_selftest_bounded_waits(0, res) == _capi.SLEEK_ERR_INVALID_ARG
    assert _capi.lib().sleek_selftest_bounded_waits(20_000_000_000, res) == _capi.SLEEK_ERR_INVALID_ARG
