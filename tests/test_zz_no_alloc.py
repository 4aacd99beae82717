"""The allocation-free compress entry point (sleek_compress_f32_static).

It serves callers that cannot call cudaMalloc (device memory owned by a framework or
pool allocator, a fixed memory budget, paths that must not risk an allocation's device
synchronisation): its scratch is a device array inside the library, so its output must
equal the regular entry point's, bit for bit, call after call -- including when the
shared scratch still holds a previous call's contents.  This file is collected last so
that a failure here leaves every other test already run; it passes alone in a fresh
process as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from sleek_b200 import _capi, api

pytestmark = pytest.mark.gpu


def _field(n, seed):
    rng = np.random.default_rng(seed)
    x = (np.cumsum(rng.normal(0, 1, n)) * 0.25).astype(np.float32)
    x[rng.choice(n, max(1, n // 400), replace=False)] = np.nan
    return torch.from_numpy(x).cuda()


def _regular(x):
    enc = torch.zeros(api.sleek_upper_bound_size(x.numel() * 4), dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    _capi.check(_capi.lib().sleek_compress_f32(x.data_ptr(), x.numel(), enc.data_ptr(), size.data_ptr(),
                                               None, 0, torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return enc[: int(size.item())].cpu().numpy().tobytes()


def _static(x):
    enc = torch.zeros(api.sleek_upper_bound_size(x.numel() * 4), dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    _capi.check(_capi.lib().sleek_compress_f32_static(x.data_ptr(), x.numel(), enc.data_ptr(), size.data_ptr(),
                                                      torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    n = int(size.item())
    assert n > 0, f"device status {-n}"
    return enc[:n].cpu().numpy().tobytes()


def test_static_scratch_matches_regular_entry_on_consecutive_calls(cuda):
    # a larger call first, then a smaller one: the second starts with the first's
    # leftovers in the shared scratch
    for n, seed in ((40 * 4096 + 123, 1), (3 * 4096 + 7, 2), (1, 3)):
        x = _field(n, seed)
        assert _static(x) == _regular(x), n


def test_static_scratch_rejects_inputs_beyond_its_limit(cuda):
    x = torch.zeros(16, dtype=torch.float32, device="cuda")
    enc = torch.zeros(64, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    too_many = (1 << 30) // 4 + 1  # rejected before any device access
    rc = _capi.lib().sleek_compress_f32_static(x.data_ptr(), too_many, enc.data_ptr(), size.data_ptr(), None)
    assert rc == _capi.SLEEK_ERR_TOO_LARGE
