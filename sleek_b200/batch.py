"""Batched compress / decompress: many arrays of uneven sizes, mixed float32 /
float64 and mixed error bounds in one persistent launch (per group of up to 1024
arrays), optionally captured in a CUDA graph.

Each array's stream is bit-identical to what ``sleek_compress_gpu`` produces for
it alone; the batched look-back is segmented per array.

    plan = BatchPlan.compress(arrays, error_bounds)    # validates, uploads tables
    plan.run()                                          # or plan.graph().replay()
    streams = plan.streams()                            # exact-size views
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np
import torch

from . import _capi
from .api import CS, SleekError, sleek_upper_bound_size, stream_size


def _elem(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return 4
    if t.dtype == torch.float64:
        return 8
    raise TypeError("SLEEK compresses float32 and float64 data")


class BatchPlan:
    """A validated batch with its device job tables and workspace.

    ``run`` only clears the workspace and launches (no host work, no allocation),
    so it can be captured in a CUDA graph (``graph``)."""

    def __init__(self, items, keep, decompress: bool, outputs, sizes, grid: int = 0):
        self._items = items
        self._keep = keep  # tensors the items point into
        self.decompress = decompress
        self.outputs = outputs
        self.sizes = sizes
        self.n = len(outputs)
        L = _capi.lib()
        arr = (_capi.BatchItem * max(1, self.n))(*items)
        h = C.c_void_p()
        _capi.check(L.sleek_batch_plan_create(C.cast(arr, C.c_void_p), self.n, int(decompress), C.byref(h)),
                    "sleek_batch_plan_create")
        self._h = h
        if grid:
            _capi.check(L.sleek_batch_plan_set_grid(h, int(grid)))
        wsb = int(L.sleek_batch_plan_workspace_size(h))
        dev = outputs[0].device if self.n else torch.device("cuda")
        self.workspace = torch.zeros(max(wsb, 8), dtype=torch.uint8, device=dev)
        self._graph = None

    # ---- construction -----------------------------------------------------------------
    @classmethod
    def compress(cls, arrays: Sequence[torch.Tensor], error_bounds: Optional[Sequence[Optional[float]]] = None,
                 grid: int = 0) -> "BatchPlan":
        """Plan compressing every array (eb None = lossless) into its own stream buffer."""
        arrays = [a.contiguous().view(-1) for a in arrays]
        if error_bounds is None:
            error_bounds = [None] * len(arrays)
        outs, sizes, items = [], torch.zeros(len(arrays), dtype=torch.int64, device="cuda"), []
        for i, (a, eb) in enumerate(zip(arrays, error_bounds)):
            w = _elem(a)
            out = torch.empty(max(sleek_upper_bound_size(a.numel() * w), 16), dtype=torch.uint8, device=a.device)
            outs.append(out)
            items.append(_capi.BatchItem(a.data_ptr() if a.numel() else out.data_ptr(), out.data_ptr(),
                                         sizes[i:].data_ptr(), a.numel(), -1, w, int(eb is not None),
                                         float(eb) if eb is not None else 0.0))
        return cls(items, arrays, False, outs, sizes, grid)

    @classmethod
    def decompress(cls, streams: Sequence[torch.Tensor], dtypes, error_bounds=None, num_elements=None,
                   grid: int = 0) -> "BatchPlan":
        """Plan decompressing every stream; ``num_elements`` (output capacities) default
        to the sizes recorded in the streams' headers."""
        n = len(streams)
        if error_bounds is None:
            error_bounds = [None] * n
        if num_elements is None:
            num_elements = [stream_size(s) // np.dtype(d).itemsize for s, d in zip(streams, dtypes)]
        outs, sizes, items = [], torch.zeros(n, dtype=torch.int64, device="cuda"), []
        for i, (s, d, eb, ne) in enumerate(zip(streams, dtypes, error_bounds, num_elements)):
            d = np.dtype(d)
            tdt = torch.float32 if d == np.float32 else torch.float64
            out = torch.empty(max(int(ne), 1), dtype=tdt, device=s.device)
            outs.append(out)
            items.append(_capi.BatchItem(s.data_ptr(), out.data_ptr(), sizes[i:].data_ptr(), int(ne), s.numel(),
                                         d.itemsize, int(eb is not None), float(eb) if eb is not None else 0.0))
        return cls(items, list(streams), True, outs, sizes, grid)

    # ---- execution ----------------------------------------------------------------------
    def run(self, stream=None) -> None:
        st = torch.cuda.current_stream() if stream is None else stream
        L = _capi.lib()
        _capi.check(L.sleek_batch_plan_run(self._h, self.workspace.data_ptr(),
                                           self.workspace.numel(), int(st.cuda_stream)), "sleek_batch_plan_run")

    def graph(self) -> torch.cuda.CUDAGraph:
        """The run captured once in a CUDA graph (replay with ``.replay()``)."""
        if self._graph is None:
            self.run()  # first run outside capture (occupancy queries, attributes)
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    self.run(stream=s)
            torch.cuda.current_stream().wait_stream(s)
            self._graph = g
        return self._graph

    # ---- results --------------------------------------------------------------------------
    def byte_sizes(self) -> list:
        v = self.sizes.cpu().tolist()
        bad = [x for x in v if x < 0]
        if bad:
            raise SleekError(-bad[0], "batch")
        return v

    def streams(self) -> list:
        """Compressed streams at their exact sizes (compress plans)."""
        return [o[:n] for o, n in zip(self.outputs, self.byte_sizes())]

    def arrays(self) -> list:
        """Decoded arrays at their exact sizes (decompress plans)."""
        return [o[: n // o.element_size()] for o, n in zip(self.outputs, self.byte_sizes())]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._graph = None
                _capi.lib().sleek_batch_plan_destroy(h)
            except Exception:
                pass
            self._h = None


def compress_batch(arrays, error_bounds=None):
    """Compresses many arrays in one launch; returns their streams."""
    p = BatchPlan.compress(arrays, error_bounds)
    p.run()
    return p.streams()


def decompress_batch(streams, dtypes, error_bounds=None):
    """Decompresses many streams in one launch; returns the arrays."""
    p = BatchPlan.decompress(streams, dtypes, error_bounds)
    p.run()
    return p.arrays()
