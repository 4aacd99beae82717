"""Sharded single-buffer compression on the device: shards of one array encoded
separately by the device codec and stitched give the device stream of the whole
array byte for byte, and split segment streams decode on the device to the
matching slices; the distributed entry points run on a one-rank NCCL group.
(More ranks need more GPUs; the exchange itself is covered on gloo.)"""
import datetime
import os
import socket

import numpy as np
import pytest
import torch

from oracle import oracle as O
from sleek_b200 import api, shard

pytestmark = pytest.mark.gpu
CS = 16384


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("eb", [None, 1e-3])
@pytest.mark.parametrize("world", [2, 5, 8])
def test_device_shards_stitch_to_the_whole_stream(cuda, dtype, eb, world):
    rng = np.random.default_rng(world)
    n = (300 * CS + 24) // np.dtype(dtype).itemsize
    x = (np.cumsum(rng.normal(0, 1, n)) * 0.1).astype(dtype)
    t = torch.from_numpy(x).cuda()
    whole = api.compress(t, eb)
    tb = t.view(torch.uint8)
    segs = [api.compress(tb[b0:b1].view(t.dtype), eb)
            for b0, b1 in (shard.shard_bytes(x.nbytes, world, k) for k in range(world))]
    assert torch.equal(shard.stitch(segs, x.nbytes), whole)
    assert whole.cpu().numpy().tobytes() == O.encode(x, eb)
    ref = O.decode(O.encode(x, eb), dtype, eb).view(np.uint8)
    for k, s in enumerate(shard.split(whole, shard.shard_chunks(x.nbytes, world))):
        b0, b1 = shard.shard_bytes(x.nbytes, world, k)
        assert api.decompress(s, dtype, eb).cpu().numpy().view(np.uint8).tobytes() == ref[b0:b1].tobytes()


def test_one_rank_nccl_group(cuda):
    import torch.distributed as dist
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        x = torch.randn(40 * CS // 8 + 3, dtype=torch.float64, device="cuda").cumsum(0)
        out = shard.sharded_compress(x, x.numel() * 8, 1e-6)
        assert torch.equal(out, api.compress(x, 1e-6))
        y = shard.sharded_decompress(out, np.float64, 1e-6)
        assert torch.equal(y, api.decompress(out, np.float64, 1e-6))
    finally:
        dist.destroy_process_group()
