"""Batched compress / decompress (one persistent launch for many arrays of uneven
sizes, mixed float32 / float64 and mixed error bounds) against the oracle and the
single-buffer entry points: every array's stream must be bit-identical to the
oracle's, decoded arrays bit-identical to the oracle's decode, alone or in the mix,
eagerly and replayed from a CUDA graph."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sleek_b200 import api
from sleek_b200.batch import BatchPlan, compress_batch, decompress_batch
from sleek_b200._capi import SleekError

pytestmark = pytest.mark.gpu


def _mix(n, seed=0):
    rng = np.random.default_rng(seed)
    arrays, ebs = [], []
    for i in range(n):
        dt = np.float32 if rng.random() < 0.5 else np.float64
        nbytes = int(np.exp(rng.uniform(np.log(4), np.log(600_000))))
        cnt = max(0, nbytes // np.dtype(dt).itemsize) if i % 17 else 0  # a few empty arrays
        x = (np.cumsum(rng.normal(0, 1, cnt)) * rng.uniform(0.01, 10)).astype(dt)
        if cnt > 10:
            x[rng.integers(0, cnt, cnt // 200 + 1)] = np.nan
        arrays.append(x)
        ebs.append(None if i % 2 == 0 else float(10 ** rng.uniform(-6, -1)))
    return arrays, ebs


def test_batch_compress_matches_oracle(cuda):
    arrays, ebs = _mix(60, 1)
    streams = compress_batch([torch.from_numpy(a).cuda() for a in arrays], ebs)
    for a, eb, s in zip(arrays, ebs, streams):
        assert s.cpu().numpy().tobytes() == O.encode(a, eb)


def test_batch_decompress_matches_oracle(cuda):
    arrays, ebs = _mix(60, 2)
    ref = [O.encode(a, eb) for a, eb in zip(arrays, ebs)]
    streams = [torch.frombuffer(bytearray(r), dtype=torch.uint8).cuda() for r in ref]
    outs = decompress_batch(streams, [a.dtype for a in arrays], ebs)
    for a, eb, r, o in zip(arrays, ebs, ref, outs):
        assert o.cpu().numpy().tobytes() == O.decode(r, a.dtype, eb).tobytes()


def test_batch_alone_equals_in_the_mix(cuda):
    arrays, ebs = _mix(30, 3)
    tens = [torch.from_numpy(a).cuda() for a in arrays]
    mixed = compress_batch(tens, ebs)
    for t, eb, s in zip(tens, ebs, mixed):
        alone = api.compress(t, eb) if t.numel() else compress_batch([t], [eb])[0]
        assert torch.equal(alone.cpu(), s.cpu())


def test_batch_graph_replay(cuda):
    arrays, ebs = _mix(40, 4)
    tens = [torch.from_numpy(a).cuda() for a in arrays]
    plan = BatchPlan.compress(tens, ebs)
    g = plan.graph()
    for _ in range(2):
        plan.sizes.zero_()
        g.replay()
        torch.cuda.synchronize()
        for a, eb, s in zip(arrays, ebs, plan.streams()):
            assert s.cpu().numpy().tobytes() == O.encode(a, eb)
    dplan = BatchPlan.decompress(plan.streams(), [a.dtype for a in arrays], ebs)
    dg = dplan.graph()
    dg.replay()
    torch.cuda.synchronize()
    for a, eb, o in zip(arrays, ebs, dplan.arrays()):
        assert o.cpu().numpy().tobytes() == O.decode(O.encode(a, eb), a.dtype, eb).tobytes()


def test_batch_larger_than_one_launch_group(cuda):
    rng = np.random.default_rng(5)
    arrays = [rng.normal(0, 1, int(rng.integers(1, 3000))).astype(np.float32) for _ in range(1100)]
    streams = compress_batch([torch.from_numpy(a).cuda() for a in arrays], [None] * len(arrays))
    for a, s in zip(arrays[::37], streams[::37]):
        assert s.cpu().numpy().tobytes() == O.encode(a)


def test_batch_grid_settings_do_not_change_output(cuda):
    arrays, ebs = _mix(20, 6)
    tens = [torch.from_numpy(a).cuda() for a in arrays]
    outs = []
    for grid in (1, 2, 0):
        p = BatchPlan.compress(tens, ebs, grid=grid)
        p.run()
        outs.append([s.cpu() for s in p.streams()])
    for a, b in zip(outs[0], outs[1]):
        assert torch.equal(a, b)
    for a, b in zip(outs[0], outs[2]):
        assert torch.equal(a, b)


def test_batch_corrupt_stream_reports_status(cuda):
    arrays, ebs = _mix(10, 7)
    ref = [bytearray(O.encode(a, eb)) for a, eb in zip(arrays, ebs)]
    k = next(i for i, a in enumerate(arrays) if a.size * a.itemsize > 20000)
    ref[k][8] = 0xFF  # first chunk size beyond 16384
    ref[k][9] = 0x7F
    streams = [torch.frombuffer(r, dtype=torch.uint8).cuda() for r in ref]
    with pytest.raises(SleekError):
        decompress_batch(streams, [a.dtype for a in arrays], ebs)
    # the device stays usable
    assert compress_batch([torch.from_numpy(arrays[k]).cuda()], [ebs[k]])[0].cpu().numpy().tobytes() == \
        O.encode(arrays[k], ebs[k])
