"""Host logic of the native serving loop (no GPU): its arena follows the same
next-fit, coalescing policy as the Python loop's DevicePool, offset for offset,
and creating a server without a device fails cleanly."""
import ctypes as C

import numpy as np
import pytest
import torch

from sleek_b200 import _capi
from sleek_b200.serve import DevicePool


def _replay_native(size, ops):
    arr = (C.c_longlong * len(ops))(*ops)
    out = (C.c_longlong * len(ops))()
    _capi.check(_capi.lib().sleek_server_arena_replay(size, arr, len(ops), out))
    return list(out)


def _replay_pool(size, ops):
    pool = DevicePool(size, device="cpu")
    live, out = [], []
    for v in ops:
        if v > 0:
            off = pool.alloc(v)
            live.append((off, v))
            out.append(-1 if off is None else off)
        else:
            off, n = live[-v]
            pool.free(off, n)
            live[-v] = (None, n)
            out.append(pool.free_bytes)
    return out


def _random_ops(rng, size, n):
    """Allocations of log-uniform sizes and releases of random live ones; an
    allocation that finds no room (checked on the native arena) is never released."""
    ops, live, nalloc = [], [], 0
    for _ in range(n):
        if live and rng.random() < 0.45:
            ops.append(-live.pop(int(rng.integers(0, len(live)))))
        else:
            ops.append(int(np.exp(rng.uniform(0, np.log(size / 8)))))
            if _replay_native(size, ops)[-1] >= 0:
                live.append(nalloc)
            nalloc += 1
    return ops


@pytest.mark.parametrize("seed", range(4))
def test_native_arena_matches_the_python_pool(seed):
    rng = np.random.default_rng(seed)
    size = int(rng.choice([1 << 16, 1 << 20, 3 << 20]))
    ops = _random_ops(rng, size, 600)
    assert _replay_native(size, ops) == _replay_pool(size, ops)


def test_native_arena_coalesces_back_to_one_range():
    size = 1 << 20
    ops = [4096] * 200 + [-j for j in range(0, 200, 2)] + [-j for j in range(1, 200, 2)]
    got = _replay_native(size, ops)
    assert got[:200] == [4096 * j for j in range(200)]  # next-fit from the start, back to back
    assert got[-1] == size                                # everything free again
    assert _replay_native(size, ops + [size])[-1] == 0    # as one range: the whole arena fits
    assert got == _replay_pool(size, ops)


def test_server_create_without_a_device_fails_cleanly():
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = _capi.lib().sleek_server_create(None, 1 << 20, 2, 8, 1024, C.byref(h))
    assert rc != _capi.SLEEK_OK and not h.value


def test_server_arguments_are_checked():
    L = _capi.lib()
    h = C.c_void_p()
    assert L.sleek_server_create(None, 1 << 20, 0, 8, 1024, C.byref(h)) == _capi.SLEEK_ERR_INVALID_ARG
    assert L.sleek_server_create(None, 1 << 20, 2, 2000, 1024, C.byref(h)) == _capi.SLEEK_ERR_INVALID_ARG
    assert L.sleek_server_create(C.c_void_p(16), 1 << 20, 2, 8, 1024, C.byref(h)) == _capi.SLEEK_ERR_ALIGNMENT
    assert L.sleek_server_submit(None, None, 0) == _capi.SLEEK_ERR_INVALID_ARG
    # a release of an allocation that was never made
    ops = (C.c_longlong * 1)(0)
    assert L.sleek_server_arena_replay(1 << 20, ops, 1, (C.c_longlong * 1)()) == _capi.SLEEK_ERR_INVALID_ARG


def test_request_array_layout_matches_the_c_struct():
    # NativeServer builds requests as a numpy array handed to sleek_server_submit
    from sleek_b200.serve import SERVER_REQUEST_DTYPE

    assert C.sizeof(_capi.ServerRequest) == SERVER_REQUEST_DTYPE.itemsize
    for name, _ in _capi.ServerRequest._fields_:
        assert getattr(_capi.ServerRequest, name).offset == SERVER_REQUEST_DTYPE.fields[name][1], name
