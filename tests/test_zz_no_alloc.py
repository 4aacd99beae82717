"""The allocation-free compress entry point (sleek_compress_f32_static).

It serves callers that cannot call cudaMalloc (device memory owned by a framework or
pool allocator, a fixed memory budget, paths that must not risk an allocation's device
synchronisation): its scratch is a device array inside the library, so its output must
equal the regular entry point's and the oracle's, bit for bit, call after call --
including when the shared scratch still holds a previous call's contents, and at the
documented size limit, where every look-back flag of the scratch is in use.  This file
is collected last so that a failure here leaves every other test already run; it passes
alone in a fresh process as well as after the other tests.
"""
import hashlib

import numpy as np
import pytest
import torch

from oracle import oracle as O
from sleek_b200 import _capi, api, workloads

pytestmark = pytest.mark.gpu

MAX_BYTES = 1 << 30  # SLEEK_STATIC_MAX_INPUT_BYTES in include/sleek_capi.h


def _field(n, seed):
    rng = np.random.default_rng(seed)
    x = (np.cumsum(rng.normal(0, 1, n)) * 0.25).astype(np.float32)
    if n:
        x[rng.choice(n, max(1, n // 400), replace=False)] = np.nan
    return torch.from_numpy(x).cuda()


def _regular(x):
    enc = torch.zeros(api.sleek_upper_bound_size(x.numel() * 4), dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    _capi.check(_capi.lib().sleek_compress_f32(x.data_ptr(), x.numel(), enc.data_ptr(), size.data_ptr(),
                                               None, 0, torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return enc[: int(size.item())].cpu().numpy().tobytes()


def _static(x, enc=None, size=None, stream=None):
    if enc is None:
        enc = torch.zeros(api.sleek_upper_bound_size(x.numel() * 4), dtype=torch.uint8, device="cuda")
    if size is None:
        size = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = stream if stream is not None else torch.cuda.current_stream()
    _capi.check(_capi.lib().sleek_compress_f32_static(x.data_ptr(), x.numel(), enc.data_ptr(), size.data_ptr(),
                                                      st.cuda_stream))
    st.synchronize()
    n = int(size.item())
    assert n > 0, f"device status {-n}"
    return enc[:n].cpu().numpy().tobytes()


def test_static_scratch_matches_regular_entry_and_oracle_on_consecutive_calls(cuda):
    # a larger call first, then smaller ones: each later call starts with the
    # previous call's leftovers in the shared scratch
    for n, seed in ((40 * 4096 + 123, 1), (3 * 4096 + 7, 2), (1, 3), (0, 4), (4096, 5)):
        x = _field(n, seed)
        got = _static(x)
        assert got == _regular(x), n
        assert got == O.encode(x.cpu().numpy(), None), n


def test_static_scratch_at_its_size_limit(cuda):
    # exactly SLEEK_STATIC_MAX_INPUT_BYTES: 65,536 chunks, every flag of the scratch
    # in use; the stream's digest equals the oracle's and the regular entry point's
    x = workloads.c2c_particles(MAX_BYTES // 4, device="cuda")
    assert x.numel() * 4 == MAX_BYTES
    got = hashlib.sha256(_static(x)).hexdigest()
    assert got == hashlib.sha256(O.encode(x.cpu().numpy(), None)).hexdigest()
    assert got == hashlib.sha256(_regular(x)).hexdigest()
    # a second call in a row, after a smaller one left its contents behind
    y = _field(5 * 4096 + 1, 6)
    assert _static(y) == O.encode(y.cpu().numpy(), None)
    assert hashlib.sha256(_static(x)).hexdigest() == got


def test_static_scratch_calls_allocate_no_device_memory(cuda):
    # A regular call on a stream the library has not seen allocates a workspace for
    # that stream (at least 1 MB).  The static entry point must not: after a first
    # call on this device (which may load the library's device code), free device
    # memory stays the same across calls on a new stream.
    x = _field(40 * 4096, 7)
    enc = torch.zeros(api.sleek_upper_bound_size(x.numel() * 4), dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    _static(x, enc, size)
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        out = _static(x, enc, size, stream=side)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert out == _regular(x)


def test_static_scratch_rejects_inputs_beyond_its_limit(cuda):
    x = torch.zeros(16, dtype=torch.float32, device="cuda")
    enc = torch.zeros(64, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    too_many = MAX_BYTES // 4 + 1  # rejected before any device access
    rc = _capi.lib().sleek_compress_f32_static(x.data_ptr(), too_many, enc.data_ptr(), size.data_ptr(), None)
    assert rc == _capi.SLEEK_ERR_TOO_LARGE
