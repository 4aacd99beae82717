"""Parity of the sm_100a kernels (through the C ABI) with the oracle.

Bar: compressed streams and decoded outputs bit-identical to the reference's,
pinned three ways -- the committed golden fixtures made by the reference CPU
codec, the oracle restatement on seeded inputs, and (where oracle/_ref was
built) the reference's own GPU kernels on the same device.  Lossy outputs are
also checked point-wise with the reference's MAXABS rule: finite values within
|x - x'| <= eb, non-finite values bit-identical.  Full-size inputs are checked
through size-independent properties (round trip, stream digest).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
from sleek_b200 import api, workloads
from sleek_b200._capi import SleekError
from tests.golden_io import cases, load, sha

pytestmark = pytest.mark.gpu
CASES = cases()


def gpu_encode(x: np.ndarray, eb=None) -> bytes:
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    return api.compress(t, eb).cpu().numpy().tobytes()


def gpu_decode(stream: bytes, dtype, eb=None) -> np.ndarray:
    s = torch.frombuffer(bytearray(stream), dtype=torch.uint8).cuda()
    return api.decompress(s, dtype, eb).cpu().numpy()


def maxabs_ok(x: np.ndarray, y: np.ndarray, eb: float) -> bool:
    """The reference's point-wise check (lossy_compressors_gpu/MAXABS_f32.h:66-81)."""
    fin = np.isfinite(x) & np.isfinite(y)
    nf = ~fin
    ib = np.uint32 if x.dtype == np.float32 else np.uint64
    nonfinite_ok = np.all((x[nf].view(ib) == y[nf].view(ib)) | (np.isnan(x[nf]) & np.isnan(y[nf])))
    err = np.abs(x[fin].astype(np.float64) - y[fin].astype(np.float64))
    return bool(nonfinite_ok) and (err.size == 0 or err.max() <= abs(eb))


# ---- golden fixtures (made by the reference CPU codec) ---------------------------

@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_encode_matches_golden(cuda, case):
    x, stream = load(case)
    assert gpu_encode(x, case["eb"]) == stream


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_decode_matches_golden(cuda, case):
    x, stream = load(case)
    y = gpu_decode(stream, x.dtype, case["eb"])
    assert sha(y.tobytes()) == case["decoded_sha256"]


# ---- seeded edge cases against the oracle -------------------------------------------

def _mixed(n, dt, seed):
    rng = np.random.default_rng(seed)
    x = (np.cumsum(rng.normal(0, 1, n)) * 0.37).astype(dt)
    k = max(1, n // 300)
    idx = rng.choice(n, k, replace=False)
    tiny = np.float32(1e-40) if dt == np.float32 else 1e-310
    x[idx] = np.array([np.nan, np.inf, -np.inf, tiny, -tiny, 0.0, -0.0], dt)[np.arange(k) % 7]
    return x


SIZES = [1, 2, 3, 31, 32, 33, 1023, 2047, 2048, 2049, 4095, 4096, 4097, 8191, 8192, 8193, 3 * 4096 + 1]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("eb", [None, 1e-2, 1e-5])
def test_sizes_match_oracle(cuda, dt, n, eb):
    x = _mixed(n, dt, n)
    s = gpu_encode(x, eb)
    assert s == O.encode(x, eb)
    y = gpu_decode(s, dt, eb)
    assert y.tobytes() == O.decode(s, dt, eb).tobytes()
    if eb is None:
        assert y.tobytes() == x.tobytes()
    else:
        assert maxabs_ok(x, y, eb)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_empty_input(cuda, dt):
    # the reference leaves this undefined; here it is an 8-byte header-only stream
    s = gpu_encode(np.zeros(0, dt))
    assert s == np.array([0], np.int64).tobytes()
    assert gpu_decode(s, dt).size == 0


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("kind", ["random_bits", "zeros", "constant", "alternating_sign", "ramp"])
def test_value_patterns(cuda, dt, kind):
    n = 3 * (16384 // np.dtype(dt).itemsize) + 17
    rng = np.random.default_rng(7)
    ib = np.uint32 if dt == np.float32 else np.uint64
    if kind == "random_bits":
        x = rng.integers(0, np.iinfo(ib).max, n, dtype=ib, endpoint=True).view(dt)
    elif kind == "zeros":
        x = np.zeros(n, dt)
    elif kind == "constant":
        x = np.full(n, 3.25, dt)
    elif kind == "alternating_sign":
        x = (np.where(np.arange(n) % 2, -1.0, 1.0) * rng.uniform(1, 2, n)).astype(dt)
    else:
        x = np.arange(n, dtype=dt)
    for eb in (None, 1e-3, 0.5):
        s = gpu_encode(x, eb)
        assert s == O.encode(x, eb), eb
        assert gpu_decode(s, dt, eb).tobytes() == O.decode(s, dt, eb).tobytes()


def test_f64_lossy_width_32_boundary(cuda):
    """64-bit lossy chunks whose widths are all at most 32 decode through 32-bit
    extraction and dequantization: a full chunk whose widest subchunk has exactly
    32 bits (codes up to 2^32 - 2), a 33-bit chunk in the same stream, and a
    partial last chunk with zero-width subchunks.  With eb = 1e-3 a value's code
    is about 2^10 |x|, so |x| in [2^21, 2^22) gives 32-bit codes."""
    rng = np.random.default_rng(11)
    v = 16384 // 8

    def band(lo, hi, n):
        return (rng.uniform(lo, hi, n) * np.where(rng.random(n) < 0.5, -1, 1)).astype(np.float64)

    x = np.concatenate([band(2 ** 21, 2 ** 22, v), band(2 ** 22, 2 ** 23, v), band(2 ** 21, 2 ** 22, 100)])
    x[5] = 2.0 ** 22 - 2.0 ** -9  # the largest code that still has 32 bits
    s = gpu_encode(x, 1e-3)
    assert s == O.encode(x, 1e-3)
    chunks = 3
    sizes = np.frombuffer(s[8:8 + 2 * chunks], np.uint16)
    off, widest = 8 + 2 * chunks, []
    for c in range(chunks):
        ln = np.frombuffer(s[off:off + 32], np.uint8)
        widest.append((int(ln.min()), int(ln.max())))
        off += int(sizes[c])
    assert widest == [(32, 32), (33, 33), (0, 32)]  # the cases this test is about
    y = gpu_decode(s, np.float64, 1e-3)
    assert y.tobytes() == O.decode(s, np.float64, 1e-3).tobytes()
    assert maxabs_ok(x, y, 1e-3)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("eb", [0.0, 1e-40, -1e-3, 1e-30, 1e3])
def test_error_bound_corner_cases(cuda, dt, eb):
    # eb = 0 and denormal eb exercise the implicit-1 quirk of quantize
    # (sleek_common_gpu.h:790-795); a negative eb uses |eb| (sleek_lossy_gpu.h:65)
    x = _mixed(5000, dt, 3)
    s = gpu_encode(x, eb)
    assert s == O.encode(x, eb)
    assert gpu_decode(s, dt, eb).tobytes() == O.decode(s, dt, eb).tobytes()


def test_error_bound_too_large_raises(cuda):
    x = torch.ones(100, device="cuda")
    with pytest.raises(SleekError):
        api.compress(x, 1e38)


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_unaligned_input_and_stream(cuda, dt):
    n = 20000
    base = torch.from_numpy(_mixed(n + 3, np.float32 if dt == torch.float32 else np.float64, 9)).cuda()
    for off in (1, 2, 3):
        x = base[off:off + n]  # element-aligned, not 16-byte aligned
        s = api.compress(x)
        assert s.cpu().numpy().tobytes() == O.encode(x.cpu().numpy())
        buf = torch.zeros(s.numel() + 64, dtype=torch.uint8, device="cuda")
        sv = buf[8:8 + s.numel()]
        sv.copy_(s)
        y = api.decompress(sv, np.float32 if dt == torch.float32 else np.float64)
        assert torch.equal(y.view(torch.int32 if dt == torch.float32 else torch.int64),
                           x.view(torch.int32 if dt == torch.float32 else torch.int64))


def test_repeated_calls_reuse_workspace(cuda):
    outs = []
    for v in range(4):
        x = _mixed(40000 + 1000 * v, np.float32, 100 + v)
        s = gpu_encode(x, None if v % 2 else 1e-3)
        assert s == O.encode(x, None if v % 2 else 1e-3)
        outs.append(s)
    assert len(set(outs)) == 4


def test_caller_workspace(cuda):
    x = torch.from_numpy(_mixed(70000, np.float64, 4)).cuda()
    from sleek_b200 import _capi
    need = _capi.lib().sleek_compress_workspace_size(x.numel() * 8)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    enc = torch.empty(api.sleek_upper_bound_size(x.numel() * 8), dtype=torch.uint8, device="cuda")
    size = torch.empty(1, dtype=torch.int64, device="cuda")
    api.sleek_compress_gpu(0, x, x.numel(), enc, size, workspace=ws, check=True)
    n = int(size.item())
    assert enc[:n].cpu().numpy().tobytes() == O.encode(x.cpu().numpy())
    small = torch.empty(8, dtype=torch.uint8, device="cuda")
    with pytest.raises(SleekError):
        api.sleek_compress_gpu(0, x, x.numel(), enc, size, workspace=small)


def test_library_workspace_resets_itself_between_calls(cuda):
    # The library-owned workspace of a stream is cleared once, when it is allocated;
    # every launch then leaves the other half clean for the next one.  A run of calls
    # whose chunk counts shrink and grow (growth past the first allocation included),
    # with decompressions, range reductions and a failed call in between, must give
    # the oracle's streams throughout.
    from sleek_b200 import _capi
    side = torch.cuda.Stream()
    sh = side.cuda_stream
    status = C.c_int(-1)
    seq = [(700 * 4096 + 5, np.float32, None), (3 * 2048, np.float64, 1e-3), (1, np.float32, 1e-2),
           (0, np.float64, None), (5000 * 4096 + 17, np.float32, None), (2 * 2048 + 1, np.float64, None),
           (700 * 2048, np.float64, 1e-6), (9, np.float32, None)]
    with torch.cuda.stream(side):
        for k, (n, dt, eb) in enumerate(seq):
            x = _mixed(max(n, 1), dt, 500 + k)[:n]
            t = torch.from_numpy(x).cuda()
            s = api.compress(t, eb)
            want = O.encode(x, eb)
            assert s.cpu().numpy().tobytes() == want, (k, n)
            y = api.decompress(s, dt, eb)
            assert y.cpu().numpy().tobytes() == O.decode(want, dt, eb).tobytes(), (k, n)
            if n:
                api.value_range(t)
            if k == 3:  # a failed decode on the same workspace, then good calls again
                b = bytearray(want if n else O.encode(_mixed(5000, dt, 9), eb))
                b[8] = 0xFF
                b[9] = 0x7F
                with pytest.raises(SleekError):
                    api.decompress(torch.frombuffer(b, dtype=torch.uint8).cuda(), dt, eb)
                _capi.check(_capi.lib().sleek_workspace_status(None, sh, C.byref(status)))
                assert status.value == _capi.SLEEK_ERR_CORRUPT_STREAM
        _capi.check(_capi.lib().sleek_workspace_status(None, sh, C.byref(status)))
        assert status.value == _capi.SLEEK_OK


def test_concurrent_streams_keep_their_own_workspaces(cuda):
    # Three streams, each with its library-owned workspace, take turns enqueueing
    # compress and decompress calls of different sizes and kinds with no host wait
    # in between; every stream and decoded array equals the oracle's.
    from sleek_b200 import _capi
    L = _capi.lib()
    streams = [torch.cuda.Stream() for _ in range(3)]
    jobs = []
    for k in range(12):
        dt = np.float32 if k % 2 else np.float64
        eb = None if k % 3 == 0 else (1e-3 if k % 3 == 1 else 1e-5)
        x = _mixed(int(30000 + 45000 * (k % 5)) + k, dt, 900 + k)
        t = torch.from_numpy(x).cuda()
        n = x.size * x.itemsize
        enc = torch.zeros(api.sleek_upper_bound_size(n), dtype=torch.uint8, device="cuda")
        dec = torch.zeros_like(t)
        sizes = torch.zeros(2, dtype=torch.int64, device="cuda")
        jobs.append((x, eb, t, enc, dec, sizes))
    torch.cuda.synchronize()
    w = lambda dt: "f32" if dt == np.float32 else "f64"
    for k, (x, eb, t, enc, dec, sizes) in enumerate(jobs):
        sh = streams[k % 3].cuda_stream
        pre = (api.sleek_error_bound(eb, x.dtype).c_struct(),) if eb is not None else ()
        mid = "_lossy" if eb is not None else ""
        _capi.check(getattr(L, f"sleek_compress{mid}_{w(x.dtype)}")(
            *pre, t.data_ptr(), t.numel(), enc.data_ptr(), sizes.data_ptr(), None, 0, sh))
        _capi.check(getattr(L, f"sleek_decompress{mid}_{w(x.dtype)}")(
            *pre, enc.data_ptr(), enc.numel(), dec.data_ptr(), t.numel() * x.itemsize, sizes[1:].data_ptr(),
            None, 0, sh))
    torch.cuda.synchronize()
    for x, eb, t, enc, dec, sizes in jobs:
        want = O.encode(x, eb)
        assert int(sizes[0]) == len(want)
        assert enc[:len(want)].cpu().numpy().tobytes() == want
        assert int(sizes[1]) == x.size * x.itemsize
        assert dec.cpu().numpy().tobytes() == O.decode(want, x.dtype, eb).tobytes()


def test_graph_replays_with_the_library_workspace(cuda):
    # Captured calls keep their workspace pointer; the workspace's epoch lives on the
    # device, so replaying the graph many times (encodes and decodes of different
    # sizes alternating on one stream) keeps every output equal to the oracle's.
    from sleek_b200 import _capi
    L = _capi.lib()
    side = torch.cuda.Stream()
    sh = side.cuda_stream
    xs = [_mixed(n, np.float64, 900 + n) for n in (300 * 2048 + 3, 5 * 2048, 40 * 2048 + 1)]
    ts = [torch.from_numpy(x).cuda() for x in xs]
    encs = [torch.zeros(api.sleek_upper_bound_size(x.nbytes), dtype=torch.uint8, device="cuda") for x in xs]
    decs = [torch.zeros_like(t) for t in ts]
    sizes = torch.zeros(2 * len(xs), dtype=torch.int64, device="cuda")

    def calls():
        for k, (t, e, d) in enumerate(zip(ts, encs, decs)):
            _capi.check(L.sleek_compress_f64(t.data_ptr(), t.numel(), e.data_ptr(), sizes[2 * k:].data_ptr(),
                                             None, 0, sh))
            _capi.check(L.sleek_decompress_f64(e.data_ptr(), e.numel(), d.data_ptr(), t.numel() * 8,
                                               sizes[2 * k + 1:].data_ptr(), None, 0, sh))

    with torch.cuda.stream(side):
        calls()  # outside capture: the stream's workspace exists before the capture
    side.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        calls()
    want = [O.encode(x, None) for x in xs]
    for rep in range(25):
        for e, d in zip(encs, decs):
            e.zero_()
            d.zero_()
        torch.cuda.synchronize()
        with torch.cuda.stream(side):
            g.replay()
        side.synchronize()
        for k, x in enumerate(xs):
            n = int(sizes[2 * k].item())
            assert encs[k][:n].cpu().numpy().tobytes() == want[k], (rep, k)
            assert int(sizes[2 * k + 1].item()) == x.nbytes
            assert decs[k].cpu().numpy().tobytes() == x.tobytes(), (rep, k)
    del g


# ---- malformed streams: an error status, never a trap ----------------------------------

def test_corrupt_streams_report_status(cuda):
    case = next(c for c in CASES if c["name"] == "f32_smooth_lossless")
    x, s = load(case)
    chunks = (len(x) * 4 + 16383) // 16384
    bad = []
    b = bytearray(s); b[8] = 0xFF; b[9] = 0x7F; bad.append(bytes(b))  # size > 16384
    b = bytearray(s); b[8 + 2 * chunks + 5] = 200; bad.append(bytes(b))  # ln > 32 in chunk 0
    b = bytearray(s); cs0 = int.from_bytes(s[8:10], "little")
    p = 8 + 2 * chunks + cs0 - 2
    b[p] ^= 0x01; bad.append(bytes(b))  # trailer mismatch
    bad.append(s[: len(s) - 100])  # truncated payload
    b = bytearray(s); b[0:8] = (10**12).to_bytes(8, "little"); bad.append(bytes(b))  # header beyond capacity
    for blob in bad:
        t = torch.frombuffer(bytearray(blob), dtype=torch.uint8).cuda()
        out = torch.empty(len(x), dtype=torch.float32, device="cuda")
        with pytest.raises(SleekError):
            api.decompress(t, np.float32, out=out)
    # the device is still usable afterwards
    assert gpu_encode(x) == s


# ---- full-size configs: oracle digest + size-independent properties ----------------------

def _roundtrip_full(x: torch.Tensor, eb):
    dt = np.float32 if x.dtype == torch.float32 else np.float64
    s = api.compress(x, eb)
    xs = x.cpu().numpy()
    assert sha(s.cpu().numpy().tobytes()) == sha(O.encode(xs, eb))
    y = api.decompress(s, dt, eb)
    if eb is None:
        ib = torch.int32 if x.dtype == torch.float32 else torch.int64
        assert torch.equal(y.view(ib), x.view(ib))
    else:
        assert maxabs_ok(xs, y.cpu().numpy(), eb)
    return s.numel()


@pytest.mark.parametrize("eb", [None])
def test_c0_signal_full(cuda, eb):
    x = workloads.c0_signal(1 << 24, device="cuda")
    n = _roundtrip_full(x, eb)
    assert n < x.numel() * 4


@pytest.mark.parametrize("eb", [None, 1e-2, 1e-4, 1e-6])
def test_c1_turbulence_full(cuda, eb):
    x = workloads.c1_turbulence(device="cuda")
    _roundtrip_full(x, eb)


@pytest.mark.parametrize("eb", [None, 1e-3])
def test_c2a_latlon_full(cuda, eb):
    x = workloads.c2a_latlon(device="cuda")
    _roundtrip_full(x, eb)


@pytest.mark.parametrize("eb", [None, 1e-3])
def test_c2b_lognormal_full(cuda, eb):
    x = workloads.c2b_lognormal(device="cuda")
    _roundtrip_full(x, eb)


@pytest.mark.parametrize("eb", [None, 1e-3])
def test_c2c_particles_full(cuda, eb):
    x = workloads.c2c_particles(device="cuda")
    _roundtrip_full(x, eb)


# ---- the reference's own GPU kernels, same device -------------------------------------

ref_gpu = O.ref_gpu()


@pytest.mark.skipif(ref_gpu is None, reason="reference GPU build (oracle/_ref) not present")
@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("eb", [None, 1e-3])
def test_matches_reference_gpu_kernels(cuda, dt, eb):
    x = _mixed(3 * 16384 // np.dtype(dt).itemsize * 5 + 11, dt, 77)
    t = torch.from_numpy(x).cuda()
    enc = torch.zeros(api.sleek_upper_bound_size(x.nbytes), dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    tag = "f32" if dt == np.float32 else "f64"
    blocks = ref_gpu.ref_gpu_blocks()
    torch.cuda.synchronize()
    if eb is None:
        getattr(ref_gpu, f"ref_gpu_compress_{tag}")(blocks, t.data_ptr(), x.size, enc.data_ptr(), size.data_ptr())
    else:
        getattr(ref_gpu, f"ref_gpu_compress_lossy_{tag}")(blocks, eb, t.data_ptr(), x.size, enc.data_ptr(),
                                                         size.data_ptr())
    torch.cuda.synchronize()
    ref_stream = enc[: int(size.item())].cpu().numpy().tobytes()
    assert gpu_encode(x, eb) == ref_stream
    dec = torch.zeros(x.size, dtype=t.dtype, device="cuda")
    dsize = torch.zeros(1, dtype=torch.int64, device="cuda")
    if eb is None:
        getattr(ref_gpu, f"ref_gpu_decompress_{tag}")(blocks, enc.data_ptr(), dec.data_ptr(), dsize.data_ptr())
    else:
        getattr(ref_gpu, f"ref_gpu_decompress_lossy_{tag}")(blocks, eb, enc.data_ptr(), dec.data_ptr(),
                                                           dsize.data_ptr())
    torch.cuda.synchronize()
    assert gpu_decode(ref_stream, dt, eb).tobytes() == dec.cpu().numpy().tobytes()
