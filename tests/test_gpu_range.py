"""Device value range (sleek_minmax_*), the input of the range-relative error
bound: equal to numpy's nanmin / nanmax on arrays with NaNs, infinities,
denormals, every start alignment and ragged lengths; NaN for an all-NaN or
empty array."""
import math

import numpy as np
import pytest
import torch

from sleek_b200 import api

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n", [1, 3, 5, 17, 1000, 4097, 1 << 20, (1 << 22) + 7])
@pytest.mark.parametrize("offset", [0, 1, 3])
def test_range_matches_numpy(cuda, dtype, n, offset):
    rng = np.random.default_rng(n * 7 + offset)
    x = (rng.normal(0, 1, n + offset) * 10 ** rng.uniform(-30, 30)).astype(dtype)
    if n > 10:
        k = rng.choice(n + offset, (n + offset) // 50 + 1, replace=False)
        x[k[: len(k) // 2]] = np.nan
        x[k[len(k) // 2:]] = 1e-40 if dtype == np.float32 else 1e-310
    t = torch.from_numpy(x).cuda()[offset:]  # element-aligned, not 16-byte aligned
    lo, hi = api.value_range(t)
    y = x[offset:]
    assert not np.all(np.isnan(y))
    assert (lo, hi) == (float(np.nanmin(y)), float(np.nanmax(y)))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_range_with_infinities_and_signed_zero(cuda, dtype):
    x = np.array([0.0, -0.0, 5.0, -np.inf, 3.0, np.inf, np.nan], dtype=dtype)
    assert api.value_range(torch.from_numpy(x).cuda()) == (-np.inf, np.inf)
    x = np.array([np.nan, 2.5, -7.25, np.nan], dtype=dtype)
    assert api.value_range(torch.from_numpy(x).cuda()) == (-7.25, 2.5)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_range_all_nan_and_empty(cuda, dtype):
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    for t in (torch.full((1000,), float("nan"), dtype=tdt, device="cuda"), torch.empty(0, dtype=tdt, device="cuda")):
        lo, hi = api.value_range(t)
        assert math.isnan(lo) and math.isnan(hi)


def test_range_relative_bound_in_the_data_precision(cuda):
    x = np.linspace(-3.3, 12.7, 100001).astype(np.float32)
    eb = api.range_relative_error_bound(torch.from_numpy(x).cuda(), 1e-3)
    want = (np.float32(x.max()) - np.float32(x.min())) * np.float32(1e-3)
    assert eb == float(np.float32(want))
