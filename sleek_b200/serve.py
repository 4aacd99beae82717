"""Serving loop: compress / decompress requests of different sizes, taken as they
arrive and run with continuous batching.

- Outputs live in one device-resident arena (``DevicePool``, next-fit with
  coalescing): a request is admitted only when its output fits in free HBM, and
  its memory returns to the pool when it completes.  A request that can never
  run (its output larger than the arena, or more chunks than a launch holds)
  fails at once with ``SLEEK_ERR_CAPACITY``, and so do the waiting requests when
  nothing is on the GPU to free memory (outputs kept by the caller fill the
  arena): the loop always ends.
- ``slots`` CUDA streams each own a reusable compress plan and a reusable
  decompress plan (``sleek_batch_plan_set_items``: no allocation per batch).  Any
  idle slot takes every admitted request waiting at that moment (up to the plan
  capacity and workspace), so requests that arrive while others are on the GPU
  join the next launch, and launches on different slots overlap on the device.
- Latency is measured from a request's arrival to the host seeing its batch
  complete; ``stats`` reports p50 / p99 and aggregate GB/s of uncompressed bytes.

Every request's result is bit-identical to running it alone through the
single-buffer entry points (the batched kernels produce the same streams).

``NativeServer`` is the same loop run by a thread of the library
(``sleek_server_*`` in ``include/sleek_capi.h``): the whole arrival trace is
submitted ahead with its arrival times and replayed by that thread, so no
interpreter sits between a request's arrival, its launch and its completion;
``Server`` keeps the loop in Python, where each step is visible.
"""
from __future__ import annotations

import bisect
import threading
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from . import _capi
from ._capi import C
from .api import sleek_upper_bound_size

GRANULE = 256
ITEM_DTYPE = np.dtype([("input", np.uint64), ("output", np.uint64), ("size_out", np.uint64),
                       ("num_elements", np.int64), ("stream_bytes", np.int64), ("elem_bytes", np.int32),
                       ("lossy", np.int32), ("error_bound", np.float64)])
assert ITEM_DTYPE.itemsize == 56  # sleek_batch_item
SERVER_REQUEST_DTYPE = np.dtype([("input", np.uint64), ("num_elements", np.int64), ("stream_bytes", np.int64),
                                 ("arrival_s", np.float64), ("error_bound", np.float64), ("tag", np.int64),
                                 ("op", np.int32), ("elem_bytes", np.int32), ("lossy", np.int32),
                                 ("keep", np.int32)])
assert SERVER_REQUEST_DTYPE.itemsize == 64  # sleek_server_request


class DevicePool:
    """Next-fit allocator over one device arena; free ranges are coalesced.

    The search starts at the free range holding the end of the last allocation
    and wraps around, so with outputs freed roughly in arrival order it finds a
    fit at once instead of walking past the small holes near the arena's start
    (replayed served traffic: 1.2 us per allocation and at most 9 free ranges,
    against 3-5 us and 74 for first-fit)."""

    def __init__(self, nbytes: int, device="cuda"):
        nbytes = (nbytes // GRANULE) * GRANULE
        self.arena = torch.empty(nbytes, dtype=torch.uint8, device=device)
        self.base = self.arena.data_ptr()
        self.size = nbytes
        self._starts = [0]          # sorted free range starts
        self._ends = {0: nbytes}    # start -> end
        self._rover = 0             # end of the last allocation
        self.free_bytes = nbytes

    @staticmethod
    def rounded(n: int) -> int:
        return max(GRANULE, (n + GRANULE - 1) // GRANULE * GRANULE)

    def alloc(self, n: int) -> Optional[int]:
        n = self.rounded(n)
        starts = self._starts
        m = len(starts)
        k = max(0, bisect.bisect_right(starts, self._rover) - 1)
        for j in range(m):
            i = k + j if k + j < m else k + j - m
            s = starts[i]
            e = self._ends[s]
            if e - s >= n:
                del self._ends[s]
                starts.pop(i)
                if e - s > n:
                    bisect.insort(starts, s + n)
                    self._ends[s + n] = e
                self.free_bytes -= n
                self._rover = s + n
                return s
        return None

    def free(self, off: int, n: int) -> None:
        n = self.rounded(n)
        s, e = off, off + n
        i = bisect.bisect_left(self._starts, s)
        if i < len(self._starts) and self._starts[i] == e:  # merge with the next range
            e = self._ends.pop(e)
            self._starts.pop(i)
        if i > 0 and self._ends[self._starts[i - 1]] == s:  # merge with the previous range
            s = self._starts[i - 1]
            self._ends[s] = e
        else:
            self._starts.insert(i, s)
            self._ends[s] = e
        self.free_bytes += n

    def view(self, off: int, n: int) -> torch.Tensor:
        return self.arena[off:off + n]


@dataclass
class Request:
    op: str                     # "compress" or "decompress"
    src: torch.Tensor           # compress: device values; decompress: device stream (uint8)
    dtype: np.dtype
    eb: Optional[float] = None
    num_elements: int = 0       # decompress: elements the stream decodes to
    arrival: float = 0.0        # seconds, on the server's clock
    rid: int = 0
    # filled by the server
    out_off: int = -1
    out_bytes: int = 0
    done: float = -1.0
    result_bytes: int = -1

    @property
    def raw_bytes(self) -> int:
        if self.op == "compress":
            return self.src.numel() * self.src.element_size()
        return self.num_elements * np.dtype(self.dtype).itemsize


@dataclass
class _Slot:
    stream: torch.cuda.Stream
    plans: dict
    ws: dict
    sizes: torch.Tensor
    sizes_host: torch.Tensor  # pinned; filled by an async copy on the slot's stream
    busy: bool = False
    event: Optional[torch.cuda.Event] = None
    reqs: List[Request] = field(default_factory=list)


class Server:
    def __init__(self, hbm_budget: int, slots: int = 4, max_batch: int = 512, max_batch_chunks: int = 1 << 16,
                 device="cuda"):
        self.pool = DevicePool(hbm_budget, device)
        self.max_batch = max_batch
        self.max_batch_chunks = max_batch_chunks
        L = _capi.lib()
        self._L = L
        self.slots: List[_Slot] = []
        for _ in range(slots):
            plans = {}
            for op, dec in (("compress", 0), ("decompress", 1)):
                h = _capi.C.c_void_p()
                _capi.check(L.sleek_batch_plan_create_reusable(max_batch, dec, _capi.C.byref(h)))
                plans[op] = h
            ws = {op: torch.zeros(8 * (32 + max_batch_chunks + 2 * max_batch), dtype=torch.uint8, device=device)
                  for op in ("compress", "decompress")}
            self.slots.append(_Slot(torch.cuda.Stream(device=device), plans, ws,
                                    torch.zeros(2 * max_batch, dtype=torch.int64, device=device),
                                    torch.zeros(2 * max_batch, dtype=torch.int64, pin_memory=True)))
        self.queue: List[Request] = []
        self.completed: List[Request] = []
        self.t0 = time.perf_counter()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    # ---- admission and dispatch ----------------------------------------------------------
    def submit(self, r: Request) -> None:
        chunks = (r.raw_bytes + 16383) // 16384
        if DevicePool.rounded(self._out_bytes(r)) > self.pool.size or chunks > self.max_batch_chunks:
            self._fail(r)  # can never be admitted
        else:
            self.queue.append(r)

    def _fail(self, r: Request) -> None:
        r.result_bytes = -_capi.SLEEK_ERR_CAPACITY
        r.done = self.now()
        self.completed.append(r)

    def _out_bytes(self, r: Request) -> int:
        if r.op == "compress":
            return sleek_upper_bound_size(r.raw_bytes)
        return r.raw_bytes

    def _take(self) -> List[Request]:
        """Admitted requests for one launch: outputs allocated from the pool, in
        arrival order, skipping (for now) those that do not fit yet.  Once the
        launch is full the rest of the queue stays as it is, in one slice (a
        burst's long queue is not walked request by request)."""
        take, chunks, keep = [], 0, []
        queue = self.queue
        for i, r in enumerate(queue):
            if len(take) == self.max_batch:
                keep.extend(queue[i:])
                break
            ch = (r.raw_bytes + 16383) // 16384
            if chunks + ch <= self.max_batch_chunks:
                n = self._out_bytes(r)
                off = self.pool.alloc(n)
                if off is not None:
                    r.out_off, r.out_bytes = off, n
                    take.append(r)
                    chunks += ch
                    continue
            keep.append(r)
        self.queue = keep
        return take

    def _launch(self, slot: _Slot, reqs: List[Request]) -> None:
        slot.reqs = reqs
        slot.busy = True
        k = 0
        with torch.cuda.stream(slot.stream):
            for op in ("compress", "decompress"):
                part = [r for r in reqs if r.op == op]
                if not part:
                    continue
                items = np.zeros(len(part), ITEM_DTYPE)
                comp = op == "compress"
                items["input"] = [r.src.data_ptr() for r in part]
                items["output"] = [self.pool.base + r.out_off for r in part]
                items["size_out"] = slot.sizes.data_ptr() + 8 * (k + np.arange(len(part), dtype=np.uint64))
                items["num_elements"] = [r.src.numel() if comp else r.num_elements for r in part]
                items["stream_bytes"] = [-1 if comp else r.src.numel() for r in part]
                items["elem_bytes"] = [np.dtype(r.dtype).itemsize for r in part]
                items["lossy"] = [int(r.eb is not None) for r in part]
                items["error_bound"] = [float(r.eb) if r.eb is not None else 0.0 for r in part]
                h = slot.plans[op]
                sh = slot.stream.cuda_stream
                _capi.check(self._L.sleek_batch_plan_set_items(h, items.ctypes.data, len(part), sh))
                ws = slot.ws[op]
                _capi.check(self._L.sleek_batch_plan_run(h, ws.data_ptr(), ws.numel(), sh))
                for i, r in enumerate(part):
                    r._slot_index = k + i
                k += len(part)
            # sizes come back with the batch, without a host wait on the device
            slot.sizes_host[:k].copy_(slot.sizes[:k], non_blocking=True)
            slot.event = torch.cuda.Event()
            slot.event.record(slot.stream)

    def poll(self) -> int:
        """Completes finished launches; returns how many requests completed."""
        n = 0
        for slot in self.slots:
            if slot.busy and slot.event.query():
                sizes = slot.sizes_host[: len(slot.reqs)].tolist() if slot.reqs else []
                t = self.now()
                for r in slot.reqs:
                    r.done = t
                    r.result_bytes = int(sizes[r._slot_index])
                    self.completed.append(r)
                n += len(slot.reqs)
                slot.busy = False
                slot.reqs = []
        return n

    def dispatch(self) -> None:
        for slot in self.slots:
            if not self.queue:
                return
            if not slot.busy:
                reqs = self._take()
                if reqs:
                    self._launch(slot, reqs)

    def result(self, r: Request) -> torch.Tensor:
        """A completed request's output (a view into the pool until released)."""
        if r.result_bytes < 0:
            raise _capi.SleekError(-r.result_bytes, "serve")
        return self.pool.view(r.out_off, r.result_bytes)

    def release(self, r: Request) -> None:
        if r.out_off >= 0:
            self.pool.free(r.out_off, r.out_bytes)
            r.out_off = -1

    # ---- driving a workload --------------------------------------------------------------
    def serve(self, requests: List[Request], keep=None) -> dict:
        """Feeds requests at their arrival times (seconds from now) and runs until all
        complete.  Outputs are released on completion unless ``keep(r)`` is true."""
        pending = sorted(requests, key=lambda r: r.arrival)
        self.t0 = time.perf_counter()
        self.completed = []
        i = 0
        while i < len(pending) or self.queue or any(s.busy for s in self.slots):
            t = self.now()
            while i < len(pending) and pending[i].arrival <= t:
                self.submit(pending[i])
                i += 1
            done_before = len(self.completed)
            self.poll()
            for r in self.completed[done_before:]:
                if keep is None or not keep(r):
                    self.release(r)
            self.dispatch()
            if self.queue and not any(s.busy for s in self.slots):
                # nothing in flight will free memory: what waits cannot be admitted
                for r in self.queue:
                    self._fail(r)
                self.queue = []
        for s in self.slots:
            s.stream.synchronize()
        return self.stats()

    def stats(self) -> dict:
        return _stats(self.completed)

    def close(self) -> None:
        for s in self.slots:
            s.stream.synchronize()
            for h in s.plans.values():
                self._L.sleek_batch_plan_destroy(h)
            s.plans = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _stats(completed: List[Request]) -> dict:
    lat = np.array([r.done - r.arrival for r in completed]) * 1e3
    span = max(r.done for r in completed) - min(r.arrival for r in completed)
    nbytes = sum(r.raw_bytes for r in completed)
    return {"requests": len(completed), "bytes": nbytes, "span_s": round(span, 4),
            "gbs": round(nbytes / span / 1e9, 1) if span > 0 else None,
            "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
            "errors": sum(1 for r in completed if r.result_bytes < 0)}


class NativeServer:
    """The serving loop of ``Server`` run by a thread of the library: requests are
    admitted at their arrival times on the server's clock when their output fits in
    the arena (a device tensor owned here), launched with the batched kernels on
    ``slots`` streams, and completed when the library's thread sees their launch
    finish.  Same results, same admission rules, same statistics as ``Server``."""

    def __init__(self, hbm_budget: int, slots: int = 4, max_batch: int = 512, max_batch_chunks: int = 1 << 16,
                 device="cuda"):
        self.arena = torch.empty((hbm_budget // GRANULE) * GRANULE, dtype=torch.uint8, device=device)
        self.base = self.arena.data_ptr()
        self._L = _capi.lib()
        h = C.c_void_p()
        _capi.check(self._L.sleek_server_create(self.base, self.arena.numel(), slots, max_batch, max_batch_chunks,
                                                C.byref(h)), "sleek_server_create")
        self._h = h
        self.completed: List[Request] = []
        self._serving = threading.Lock()  # serve() tags requests by position: one call at a time

    def now(self) -> float:
        t = C.c_double()
        _capi.check(self._L.sleek_server_now(self._h, C.byref(t)))
        return t.value

    def arena_info(self):
        """(free bytes, size) of the arena."""
        f, n = C.c_longlong(), C.c_longlong()
        _capi.check(self._L.sleek_server_arena_info(self._h, C.byref(f), C.byref(n)))
        return f.value, n.value

    def serve(self, requests: List[Request], keep=None, lead_s: float = 0.02) -> dict:
        """Submits the requests with their arrival times (seconds from now, plus a
        lead for the submission itself) and waits for all of them.  Outputs
        are returned to the arena on completion unless ``keep(r)`` is true.  Calls
        from several threads run one after the other (the C ABI itself takes
        submissions from any thread)."""
        with self._serving:
            return self._serve(requests, keep, lead_s)

    def _serve(self, requests: List[Request], keep, lead_s: float) -> dict:
        n = len(requests)
        arr = np.zeros(max(n, 1), SERVER_REQUEST_DTYPE)
        comp = np.array([r.op == "compress" for r in requests], dtype=bool)
        arr["input"][:n] = [r.src.data_ptr() for r in requests]
        arr["num_elements"][:n] = [r.src.numel() if c else r.num_elements for r, c in zip(requests, comp)]
        arr["stream_bytes"][:n] = [0 if c else r.src.numel() for r, c in zip(requests, comp)]
        arr["error_bound"][:n] = [float(r.eb) if r.eb is not None else 0.0 for r in requests]
        arr["tag"][:n] = np.arange(n)
        arr["op"][:n] = np.where(comp, 0, 1)
        arr["elem_bytes"][:n] = [np.dtype(r.dtype).itemsize for r in requests]
        arr["lossy"][:n] = [int(r.eb is not None) for r in requests]
        arr["keep"][:n] = [int(keep is not None and bool(keep(r))) for r in requests]
        rel = np.array([r.arrival for r in requests], dtype=np.float64)
        # arrivals on the server's clock, set once the array is built; the lead
        # covers the submission and the loop taking the requests in (a few
        # hundred ns per request)
        t0 = self.now() + lead_s + 5e-7 * n
        arr["arrival_s"][:n] = t0 + rel
        _capi.check(self._L.sleek_server_submit(self._h, arr.ctypes.data, n), "sleek_server_submit")
        buf = (_capi.ServerCompletion * 4096)()
        got = C.c_longlong()
        completed = []
        while len(completed) < n:
            _capi.check(self._L.sleek_server_poll(self._h, buf, len(buf), C.byref(got), 100), "sleek_server_poll")
            for k in range(got.value):
                c = buf[k]
                r = requests[c.tag]
                r.done = c.done_s - t0
                r.result_bytes = c.result_bytes
                r.out_off = (c.output - self.base) if c.output else -1
                r.out_bytes = max(c.result_bytes, 0)
                completed.append(r)
        self.completed = completed
        return self.stats()

    def result(self, r: Request) -> torch.Tensor:
        """A completed, kept request's output (a view into the arena until released)."""
        if r.result_bytes < 0:
            raise _capi.SleekError(-r.result_bytes, "serve")
        if r.out_off < 0:
            raise ValueError("the request's output was not kept")
        return self.arena[r.out_off:r.out_off + r.result_bytes]

    def release(self, r: Request) -> None:
        if r.out_off >= 0:
            _capi.check(self._L.sleek_server_release(self._h, C.c_void_p(self.base + r.out_off)))
            r.out_off = -1

    def stats(self) -> dict:
        return _stats(self.completed)

    def close(self) -> None:
        if self._h is not None:
            _capi.check(self._L.sleek_server_destroy(self._h), "sleek_server_destroy")
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
