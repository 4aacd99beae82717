"""Sharded single-buffer compression, host side: shard ranges, stitching the
shards' segment streams into one stream and splitting it back, and the
distributed exchange (all-gather of payload totals, point-to-point table and
payload transfers) on gloo process groups of 2 and 3 ranks.  The segment codec
here is the oracle (CPU); the result must be byte-identical to the oracle's
stream of the whole array, and every rank must decode its own shard."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import oracle as O
from sleek_b200 import shard

CS = 16384


def _array(dtype, nbytes, seed=0):
    rng = np.random.default_rng(seed)
    x = (np.cumsum(rng.normal(0, 1, nbytes // np.dtype(dtype).itemsize)) * 0.2).astype(dtype)
    if x.size > 50:
        x[rng.integers(0, x.size, x.size // 50)] = np.nan
    return x


def test_shard_ranges_cover_every_chunk_once():
    for total in (0, 5, CS, CS + 4, 100 * CS + 8):
        for world in (1, 2, 3, 8):
            r = shard.shard_chunks(total, world)
            assert r[0][0] == 0 and r[-1][1] == (total + CS - 1) // CS
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [c1 - c0 for c0, c1 in r]
            assert max(sizes) - min(sizes) <= 1
            spans = [shard.shard_bytes(total, world, k) for k in range(world)]
            assert sum(b - a for a, b in spans) == total


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("eb", [None, 1e-3])
@pytest.mark.parametrize("world", [1, 2, 3, 7])
def test_stitch_and_split_match_whole_stream(dtype, eb, world):
    x = _array(dtype, 23 * CS + 8 * 3, world)
    whole = O.encode(x, eb)
    segs = []
    for k in range(world):
        b0, b1 = shard.shard_bytes(x.nbytes, world, k)
        part = x.view(np.uint8)[b0:b1].view(dtype)
        segs.append(torch.frombuffer(bytearray(O.encode(part, eb)), dtype=torch.uint8))
    st = shard.stitch(segs, x.nbytes)
    assert st.numpy().tobytes() == whole
    back = shard.split(torch.frombuffer(bytearray(whole), dtype=torch.uint8), shard.shard_chunks(x.nbytes, world))
    for a, b in zip(back, segs):
        assert torch.equal(a, b)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _enc(x, eb):
    return torch.frombuffer(bytearray(O.encode(x.numpy(), eb)), dtype=torch.uint8)


def _dec(s, dtype, eb):
    return torch.from_numpy(O.decode(s.numpy().tobytes(), dtype, eb).copy())


def _worker(rank, world, port, dtype, eb, nbytes, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        x = _array(dtype, nbytes, 42)
        b0, b1 = shard.shard_bytes(x.nbytes, world, rank)
        local = torch.from_numpy(x.view(np.uint8)[b0:b1].view(dtype).copy())
        out = shard.sharded_compress(local, x.nbytes, eb, owner=world - 1, encode=_enc)
        ok_c = (out.numpy().tobytes() == O.encode(x, eb)) if rank == world - 1 else out is None
        mine = shard.sharded_decompress(out if rank == world - 1 else None, dtype, eb, owner=world - 1, decode=_dec)
        want = O.decode(O.encode(x, eb), dtype, eb).view(np.uint8)[b0:b1]
        ok_d = mine.numpy().view(np.uint8).tobytes() == want.tobytes()
        q.put((rank, bool(ok_c), bool(ok_d)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dtype,eb,nbytes", [(2, np.float32, None, 9 * CS + 12),
                                                    (2, np.float64, 1e-4, 16 * CS),
                                                    (3, np.float32, 1e-2, 4 * CS + 40),
                                                    (3, np.float64, None, CS + 8)])  # one rank holds no chunk
def test_distributed_exchange_on_gloo(world, dtype, eb, nbytes):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, dtype, eb, nbytes, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(c and d for _, c, d in res), res
