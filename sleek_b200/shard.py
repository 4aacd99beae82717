"""One large array compressed across several GPUs into ONE stream.

Chunks are independent apart from the exclusive scan of their sizes, so the
array splits into contiguous, chunk-aligned shards, one per rank (one process
per GPU).  Each rank encodes its shard with the device codec into a *segment
stream* -- a valid stream of its own, whose size table is a slice of the global
size table and whose payload area is a contiguous run of the global payload
area.  The only exchange the scan needs is an all-gather of the G per-shard
payload totals (8 bytes each); every rank then knows where its table slice and
payload run go, and sends them point to point (NCCL over NVLink on GPUs) into
the owner rank's stream buffer.  The result is byte-identical to compressing
the whole array on one GPU.

Decompression reverses it: the owner broadcasts the header and size table, each
rank computes its shard's payload range from the table, the owner sends each
rank its run, and every rank decodes its segment stream into its shard.

``stitch`` / ``split`` are the same layout arithmetic for shard streams held by
one process.  The codec is the device one (``api.compress`` / ``api.decompress``)
unless a caller passes its own ``encode`` / ``decode`` (used to exercise the
exchange on CPU-only process groups).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
import torch

CS = 16384


def shard_chunks(total_bytes: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous chunk ranges [c0, c1) per rank, as even as whole chunks allow."""
    chunks = (total_bytes + CS - 1) // CS
    base, extra = divmod(chunks, world)
    out, c = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((c, c + n))
        c += n
    return out


def shard_bytes(total_bytes: int, world: int, rank: int) -> Tuple[int, int]:
    """Byte range [b0, b1) of the array that rank `rank` holds."""
    c0, c1 = shard_chunks(total_bytes, world)[rank]
    return min(c0 * CS, total_bytes), min(c1 * CS, total_bytes)


def _header(n: int, device) -> torch.Tensor:
    return torch.from_numpy(np.array([n], np.int64).view(np.uint8).copy()).to(device)


def _insize(stream: torch.Tensor) -> int:
    return int(stream[:8].cpu().numpy().view(np.int64)[0])


def _payload_len(stream: torch.Tensor) -> Tuple[int, int]:
    """(chunks, payload bytes) of a segment stream"""
    n = _insize(stream)
    chunks = (n + CS - 1) // CS
    return chunks, stream.numel() - 8 - 2 * chunks


def stitch(segments: Sequence[torch.Tensor], total_bytes: int) -> torch.Tensor:
    """The stream of the whole array from the segment streams of its shards (in
    order; every shard but the last a whole number of chunks)."""
    dev = segments[0].device if segments else torch.device("cpu")
    chunks = (total_bytes + CS - 1) // CS
    parts = [_header(total_bytes, dev)]
    tables, payloads = [], []
    for s in segments:
        ch, _ = _payload_len(s)
        tables.append(s[8:8 + 2 * ch])
        payloads.append(s[8 + 2 * ch:])
    out = torch.cat(parts + tables + payloads)
    assert out.numel() >= 8 + 2 * chunks
    return out


def split(stream: torch.Tensor, ranges: Sequence[Tuple[int, int]]) -> List[torch.Tensor]:
    """Segment streams of the chunk ranges `ranges` of a whole stream."""
    total = _insize(stream)
    chunks = (total + CS - 1) // CS
    cs = stream[8:8 + 2 * chunks].cpu().numpy().view(np.uint16).astype(np.int64)
    starts = np.concatenate([[0], np.cumsum(cs)]) + 8 + 2 * chunks
    out = []
    for c0, c1 in ranges:
        nbytes = max(0, min(c1 * CS, total) - c0 * CS)
        out.append(torch.cat([_header(nbytes, stream.device), stream[8 + 2 * c0:8 + 2 * c1],
                              stream[int(starts[c0]):int(starts[c1])]]))
    return out


def _default_encode(x: torch.Tensor, eb):
    from . import api
    return api.compress(x, eb)


def _default_decode(s: torch.Tensor, dtype, eb):
    from . import api
    return api.decompress(s, dtype, eb)


def sharded_compress(x_local: torch.Tensor, total_bytes: int, eb: Optional[float] = None, group=None, owner: int = 0,
                     encode: Optional[Callable] = None) -> Optional[torch.Tensor]:
    """Every rank passes its shard (``shard_bytes(total_bytes, world, rank)`` of
    the array, flattened); the owner rank returns the stream of the whole array,
    the other ranks None.  One all-gather of per-shard payload totals, then one
    point-to-point transfer of table slice + payload per non-owner rank."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    b0, b1 = shard_bytes(total_bytes, world, rank)
    if x_local.numel() * x_local.element_size() != b1 - b0:
        raise ValueError(f"rank {rank} holds {x_local.numel() * x_local.element_size()} bytes, its shard is {b1 - b0}")
    seg = (encode or _default_encode)(x_local, eb) if b1 > b0 else _header(0, x_local.device)
    ch, payload = _payload_len(seg)
    sizes = torch.tensor([payload], dtype=torch.int64, device=x_local.device)
    allsizes = [torch.zeros_like(sizes) for _ in range(world)]
    dist.all_gather(allsizes, sizes, group=group)  # the scan's only exchange: 8 bytes per shard
    payloads = [int(t.item()) for t in allsizes]
    ranges = shard_chunks(total_bytes, world)
    chunks = ranges[-1][1]
    base = 8 + 2 * chunks
    pay_off = [base + sum(payloads[:r]) for r in range(world)]
    if rank == owner:
        out = torch.empty(base + sum(payloads), dtype=torch.uint8, device=x_local.device)
        out[:8] = _header(total_bytes, out.device)
        for r in range(world):
            c0, c1 = ranges[r]
            t_dst = out[8 + 2 * c0:8 + 2 * c1]
            p_dst = out[pay_off[r]:pay_off[r] + payloads[r]]
            if r == rank:
                t_dst.copy_(seg[8:8 + 2 * ch])
                p_dst.copy_(seg[8 + 2 * ch:])
            else:
                if t_dst.numel():
                    dist.recv(t_dst, src=r, group=group)
                if p_dst.numel():
                    dist.recv(p_dst, src=r, group=group)
        return out
    if ch:
        dist.send(seg[8:8 + 2 * ch].contiguous(), dst=owner, group=group)
    if payload:
        dist.send(seg[8 + 2 * ch:].contiguous(), dst=owner, group=group)
    return None


def sharded_decompress(stream: Optional[torch.Tensor], dtype, eb: Optional[float] = None, group=None, owner: int = 0,
                       device=None, decode: Optional[Callable] = None) -> torch.Tensor:
    """The owner passes the whole stream (others None); every rank returns its
    decoded shard (``shard_bytes`` of the original array)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = stream.device if stream is not None else (device or torch.device("cpu"))
    hdr = stream[:8].clone() if rank == owner else torch.empty(8, dtype=torch.uint8, device=dev)
    dist.broadcast(hdr, src=owner, group=group)
    total = int(hdr.cpu().numpy().view(np.int64)[0])
    ranges = shard_chunks(total, world)
    chunks = ranges[-1][1]
    table = stream[8:8 + 2 * chunks].clone() if rank == owner else torch.empty(2 * chunks, dtype=torch.uint8,
                                                                               device=dev)
    if chunks:
        dist.broadcast(table, src=owner, group=group)
    cs = table.cpu().numpy().view(np.uint16).astype(np.int64)
    starts = np.concatenate([[0], np.cumsum(cs)]) + 8 + 2 * chunks
    c0, c1 = ranges[rank]
    nbytes = max(0, min(c1 * CS, total) - c0 * CS)
    plen = int(starts[c1] - starts[c0])
    if rank == owner:
        for r in range(world):
            if r != owner:
                a, b = ranges[r]
                if starts[b] > starts[a]:
                    dist.send(stream[int(starts[a]):int(starts[b])].contiguous(), dst=r, group=group)
        payload = stream[int(starts[c0]):int(starts[c1])]
    else:
        payload = torch.empty(plen, dtype=torch.uint8, device=dev)
        if plen:
            dist.recv(payload, src=owner, group=group)
    seg = torch.cat([_header(nbytes, dev), table[2 * c0:2 * c1], payload])
    tdt = torch.float32 if np.dtype(dtype) == np.float32 else torch.float64
    if nbytes == 0:
        return torch.empty(0, dtype=tdt, device=dev)
    return (decode or _default_decode)(seg, dtype, eb)
