#!/usr/bin/env python3
"""Benchmark of the sm_100a SLEEK compress / decompress path.

Metric (the reference's convention, sleek_single_compressor.cu:123 and
memcpy.cu:128): GB/s of UNCOMPRESSED bytes, 1e9 bytes per GB.

Workload (default): the float64 turbulence-like field of 256 x 384 x 384 values
(301,989,888 bytes; seeded synthetic stand-in for the Miranda field), lossless
and absolute error bounds 1e-2, 1e-4, 1e-6.  One step = compress + decompress
of the field in each of the four modes (8 kernel launches, each preceded by a
workspace clear).  Inputs (302 MB) are larger than the 126 MB L2, so no flush is
needed between iterations.

  value     whole-job GB/s: uncompressed bytes through all compress and
            decompress passes of all ranks / max-over-ranks device time
  e2e       same metric through the public C-ABI calls with host buffers:
            per mode H2D of the input, compress, D2H of the stream, H2D of the
            stream, decompress, D2H of the output, all inside the timed region
  roofline  the dominant kernel's algorithmic bytes (uncompressed + stream
            bytes per launch) / its mean CUDA-event duration, against the
            measured HBM copy bandwidth in MEASURED_PEAKS.json
  cpu_baseline  the reference's own OpenMP CPU codec (oracle/_ref), all host
            threads, on the same field

Run: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU (torchrun, one process per GPU): every rank runs an independent
replica of the workload (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "compress/decompress GB/s (uncompressed bytes) vs D2D memcpy on 1 B200"
MODES = [None, 1e-2, 1e-4, 1e-6]
SHAPE = (256, 384, 384)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    return world, rank, local


def dist_max(v: float, world: int) -> float:
    if world == 1:
        return v
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        torch.distributed.barrier()


# ---------------------------------------------------------------------------------
# reference arm: the reference's own CPU codec on the host cores
# ---------------------------------------------------------------------------------

def cpu_reference_run(x: np.ndarray, repeats: int):
    """Times the reference CPU codec (compress + decompress, every mode) on x."""
    from oracle import oracle as O

    if O.ref_cpu() is None:
        return None, "port"
    t_total = 0.0
    nbytes = 0
    for _ in range(repeats):
        for eb in MODES:
            t0 = time.perf_counter()
            s = O.ref_encode(x, eb)
            t1 = time.perf_counter()
            O.ref_decode(s, x.dtype, eb)
            t2 = time.perf_counter()
            t_total += t2 - t0
            nbytes += 2 * x.nbytes
    return nbytes / t_total / 1e9, "reference"


def cpu_port_run(x: np.ndarray, repeats: int):
    from oracle import oracle as O

    t_total = 0.0
    nbytes = 0
    for _ in range(repeats):
        for eb in MODES:
            t0 = time.perf_counter()
            s = O.encode(x, eb)
            O.decode(s, x.dtype, eb)
            t_total += time.perf_counter() - t0
            nbytes += 2 * x.nbytes
    return nbytes / t_total / 1e9


def reference_gpu_kernels(x: torch.Tensor, reps: int = 5):
    """The reference's own GPU codec (its headers compiled for sm_100a into
    oracle/_ref) on the same field and modes: GB/s of uncompressed bytes through
    its public API (which allocates and frees scratch per call) and with its kernels
    launched on preallocated scratch; CUDA events on the legacy default stream it
    uses.  Its streams must equal this project's.  None when it was not built."""
    from oracle import oracle as O
    from sleek_b200 import api

    R = O.ref_gpu()
    if R is None:
        return None
    blocks = R.ref_gpu_blocks()
    N = x.numel() * 8
    enc = torch.empty(api.sleek_upper_bound_size(N), dtype=torch.uint8, device=x.device)
    dec = torch.empty_like(x)
    size = torch.zeros(2, dtype=torch.int64, device=x.device)
    carry = torch.zeros((N + 16383) // 16384 + 1, dtype=torch.int64, device=x.device)
    dflt = torch.cuda.default_stream(x.device)

    def timed(fn):
        with torch.cuda.stream(dflt):
            fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(dflt)
            for _ in range(reps):
                fn()
            e1.record(dflt)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps * 1e-3

    out = {"kernels": "reference d_encode / d_decode built for sm_100a, grid %d x 512" % blocks, "modes": {}}
    same = True
    for eb in MODES:
        lossy = int(eb is not None)
        if eb is None:
            api_c = lambda: R.ref_gpu_compress_f64(blocks, x.data_ptr(), x.numel(), enc.data_ptr(), size.data_ptr())
            api_d = lambda: R.ref_gpu_decompress_f64(blocks, enc.data_ptr(), dec.data_ptr(), size[1:].data_ptr())
        else:
            api_c = lambda: R.ref_gpu_compress_lossy_f64(blocks, eb, x.data_ptr(), x.numel(), enc.data_ptr(),
                                                         size.data_ptr())
            api_d = lambda: R.ref_gpu_decompress_lossy_f64(blocks, eb, enc.data_ptr(), dec.data_ptr(),
                                                           size[1:].data_ptr())
        k_c = lambda: R.ref_gpu_encode_prealloc_f64(blocks, x.data_ptr(), x.numel(), enc.data_ptr(), size.data_ptr(),
                                                    carry.data_ptr(), lossy, eb or 0.0)
        k_d = lambda: R.ref_gpu_decode_prealloc_f64(blocks, enc.data_ptr(), dec.data_ptr(), size[1:].data_ptr(),
                                                    carry.data_ptr(), lossy, eb or 0.0)
        t_ac, t_kc = timed(api_c), timed(k_c)
        S = int(size[0].item())
        same &= enc[:S].cpu().numpy().tobytes() == api.compress(x, eb).cpu().numpy().tobytes()
        t_ad, t_kd = timed(api_d), timed(k_d)
        out["modes"][str(eb)] = {"compress_api_gbs": round(N / t_ac / 1e9, 1), "compress_kernel_gbs": round(N / t_kc / 1e9, 1),
                                 "decompress_api_gbs": round(N / t_ad / 1e9, 1),
                                 "decompress_kernel_gbs": round(N / t_kd / 1e9, 1)}
    out["streams_identical_to_ours"] = bool(same)
    return out


def cpu_baseline(x_host: np.ndarray, max_seconds: float = 20.0):
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    cores = int(os.environ["OMP_NUM_THREADS"])
    t0 = time.perf_counter()
    v, kind = cpu_reference_run(x_host, 1)
    if v is None:
        v = cpu_port_run(x_host, 1)
        kind, cores = "port", 1
    el = time.perf_counter() - t0
    reps = max(1, min(5, int(max_seconds / max(el, 1e-3))))
    if reps > 1:
        v2 = cpu_reference_run(x_host, reps)[0] if kind == "reference" else cpu_port_run(x_host, reps)
        v = v2
    return {"value": round(v, 3), "unit": "GB/s", "cores": cores, "kind": kind,
            "sample": f"full {x_host.nbytes} B field, compress+decompress x 4 modes, {reps + 1} passes"}


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    from sleek_b200 import workloads

    dev = "cuda" if torch.cuda.is_available() else "cpu"
    x = workloads.c1_turbulence(SHAPE, device=dev).cpu().numpy()
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    from oracle import oracle as O

    kind = "reference" if O.ref_cpu() is not None else "port"
    cores = int(os.environ["OMP_NUM_THREADS"]) if kind == "reference" else 1
    run = (lambda r: cpu_reference_run(x, r)[0]) if kind == "reference" else (lambda r: cpu_port_run(x, r))
    for _ in range(args.warmup):
        run(1)
    t0 = time.perf_counter()
    steps_v = [run(1) for _ in range(args.steps)]
    el = time.perf_counter() - t0
    v = statistics.mean(steps_v)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * el / max(args.steps, 1), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args),
        "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "cores": cores, "kind": kind,
                         "sample": f"full {x.nbytes} B field, compress+decompress x 4 modes per step"},
        "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def bench_batched(dev, world, args):
    """The batched workload (1000 arrays, 4 KB - 64 MB, mixed dtypes and bounds):
    one graph-captured persistent launch vs 1000 sequential plain launches (also
    graph-captured, so host launch overhead is not counted against the plain
    form), with every stream and decoded array compared bit for bit."""
    from sleek_b200 import _capi, api, autotune, workloads
    from sleek_b200.batch import BatchPlan

    L = _capi.lib()
    arrays, ebs = workloads.batched_arrays(1000, device=dev)
    total = sum(a.numel() * a.element_size() for a in arrays)
    st = torch.cuda.current_stream()

    # sequential plain launches through the C ABI, one buffer per call, with the
    # library-owned workspace (one kernel launch per call)
    outs = [torch.empty(api.sleek_upper_bound_size(a.numel() * a.element_size()) + 16, dtype=torch.uint8,
                        device=dev) for a in arrays]
    szs = torch.zeros(len(arrays), dtype=torch.int64, device=dev)
    ebi = [None if eb is None else api.sleek_error_bound(eb, np.float32 if a.dtype == torch.float32
                                                         else np.float64).c_struct() for a, eb in zip(arrays, ebs)]

    def seq_compress(stream):
        sh = stream.cuda_stream
        for i, a in enumerate(arrays):
            t = "f32" if a.dtype == torch.float32 else "f64"
            if ebi[i] is None:
                rc = getattr(L, f"sleek_compress_{t}")(a.data_ptr(), a.numel(), outs[i].data_ptr(),
                                                       szs[i:].data_ptr(), None, 0, sh)
            else:
                rc = getattr(L, f"sleek_compress_lossy_{t}")(ebi[i], a.data_ptr(), a.numel(), outs[i].data_ptr(),
                                                             szs[i:].data_ptr(), None, 0, sh)
            _capi.check(rc)

    decs = [torch.empty_like(a) for a in arrays]
    dszs = torch.zeros(len(arrays), dtype=torch.int64, device=dev)

    def seq_decompress(stream):
        sh = stream.cuda_stream
        for i, a in enumerate(arrays):
            t = "f32" if a.dtype == torch.float32 else "f64"
            cap = a.numel() * a.element_size()
            if ebi[i] is None:
                rc = getattr(L, f"sleek_decompress_{t}")(outs[i].data_ptr(), outs[i].numel(), decs[i].data_ptr(), cap,
                                                         dszs[i:].data_ptr(), None, 0, sh)
            else:
                rc = getattr(L, f"sleek_decompress_lossy_{t}")(ebi[i], outs[i].data_ptr(), outs[i].numel(),
                                                               decs[i].data_ptr(), cap, dszs[i:].data_ptr(),
                                                               None, 0, sh)
            _capi.check(rc)

    def graph_of(fn):
        fn(st)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s2 = torch.cuda.Stream()
        s2.wait_stream(st)
        with torch.cuda.stream(s2):
            fn(s2)  # outside capture: the library-owned workspace of s2 exists before it
            with torch.cuda.graph(g, stream=s2):
                fn(s2)
        st.wait_stream(s2)
        return g

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    g_seq_c = graph_of(seq_compress)
    t_seq_c = timed(g_seq_c.replay)
    g_seq_d = graph_of(seq_decompress)
    t_seq_d = timed(g_seq_d.replay)

    plan = BatchPlan.compress(arrays, ebs)
    tuned_c = autotune.tune_plan(plan, f"c3-compress-{len(arrays)}", use_cache=False)
    t_bat_c = timed(plan.graph().replay)
    seq_sizes = szs.cpu().tolist()
    bat_streams = plan.streams()
    exact = all(int(n) == s.numel() and torch.equal(o[:int(n)], s)
                for o, n, s in zip(outs, seq_sizes, bat_streams))
    dplan = BatchPlan.decompress(bat_streams, [np.float32 if a.dtype == torch.float32 else np.float64
                                               for a in arrays], ebs,
                                 num_elements=[a.numel() for a in arrays])
    tuned_d = autotune.tune_plan(dplan, f"c3-decompress-{len(arrays)}", use_cache=False)
    t_bat_d = timed(dplan.graph().replay)
    exact = exact and all(torch.equal(d.view(torch.int32 if d.dtype == torch.float32 else torch.int64),
                                      o.view(torch.int32 if o.dtype == torch.float32 else torch.int64))
                          for d, o in zip(decs, dplan.arrays()))
    gbs = lambda ms: round(total / (ms * 1e-3) / 1e9, 1)
    return {
        "workload": "1000 arrays, log-uniform 4 KB-64 MB, f32/f64, half lossless / half lossy eb in [1e-6,1e-1]",
        "total_bytes": total,
        "compress_gbs": {"batched_graph": gbs(t_bat_c), "sequential_plain_graph": gbs(t_seq_c),
                         "speedup": round(t_seq_c / t_bat_c, 2)},
        "decompress_gbs": {"batched_graph": gbs(t_bat_d), "sequential_plain_graph": gbs(t_seq_d),
                           "speedup": round(t_seq_d / t_bat_d, 2)},
        "autotuned_ctas_per_sm": {"compress": tuned_c["best"], "decompress": tuned_d["best"]},
        "bit_exact_vs_plain": bool(exact),
    }


def serve_plain(reqs, dev) -> dict:
    """The per-buffer form of the served workload: every request, at its arrival
    time, is one plain call of the reference-shaped entry points
    (sleek_compress_* / sleek_decompress_*, library-owned workspace) on one stream;
    a request completes when the event recorded after its call has passed.  Same
    clock, latency and throughput definitions as Server.serve."""
    import collections

    from sleek_b200 import _capi, api

    L = _capi.lib()
    st = torch.cuda.Stream(dev)
    sh = st.cuda_stream
    maxraw = max(r.raw_bytes for r in reqs)
    out = torch.empty(api.sleek_upper_bound_size(maxraw) + 16, dtype=torch.uint8, device=dev)
    size = torch.zeros(1, dtype=torch.int64, device=dev)
    ebc = {}

    def call(r):
        dt = np.dtype(r.dtype)
        t = "f32" if dt == np.float32 else "f64"
        lossy = r.eb is not None
        if lossy and (r.eb, t) not in ebc:
            ebc[(r.eb, t)] = api.sleek_error_bound(r.eb, dt).c_struct()
        pre = (ebc[(r.eb, t)],) if lossy else ()
        mid = "_lossy" if lossy else ""
        if r.op == "compress":
            rc = getattr(L, f"sleek_compress{mid}_{t}")(*pre, r.src.data_ptr(), r.src.numel(), out.data_ptr(),
                                                       size.data_ptr(), None, 0, sh)
        else:
            rc = getattr(L, f"sleek_decompress{mid}_{t}")(*pre, r.src.data_ptr(), r.src.numel(), out.data_ptr(),
                                                         r.num_elements * dt.itemsize, size.data_ptr(), None, 0, sh)
        _capi.check(rc)

    pending = sorted(reqs, key=lambda r: r.arrival)
    inflight = collections.deque()
    n = len(pending)
    i = 0
    t0 = time.perf_counter()
    while i < n or inflight:
        now = time.perf_counter() - t0
        while i < n and pending[i].arrival <= now:
            call(pending[i])
            ev = torch.cuda.Event()
            ev.record(st)
            inflight.append((ev, pending[i]))
            i += 1
            if inflight[0][0].query():
                break
        while inflight and inflight[0][0].query():
            inflight.popleft()[1].done = time.perf_counter() - t0
    st.synchronize()
    lat = np.array([r.done - r.arrival for r in reqs]) * 1e3
    span = max(r.done for r in reqs) - min(r.arrival for r in reqs)
    nbytes = sum(r.raw_bytes for r in reqs)
    return {"requests": n, "bytes": nbytes, "span_s": round(span, 4), "gbs": round(nbytes / span / 1e9, 1),
            "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3)}


def bench_serve(dev, n_requests: int, seed: int = 4):
    """The served workload: Poisson arrivals at 70 % of the loop's measured peak,
    sizes log-uniform 1 KB - 256 MB, 60 / 40 compress / decompress, half lossy with
    bounds log-uniform in [1e-6, 1e-2], outputs in a device pool of up to 150 GB.
    Decompress requests read one of 256 distinct streams made beforehand by the
    compressor (about 5 GB in all, many times the 126 MB L2).  The loop is the
    library's native one (serve.NativeServer); the same arrival trace also runs
    through the Python loop (serve.Server) and through one plain entry-point call
    per request (serve_plain), and every form's peak is measured with every request
    queued at once.  1 % of
    the served requests are re-run alone through the single-buffer entry points and
    compared bit for bit; up to 200 of them (those of at most 8 MB) are kept on the
    host for the oracle check of the CPU-baseline leg."""
    from sleek_b200 import api
    from sleek_b200.serve import NativeServer, Request, Server

    rng = np.random.default_rng(20261203 + 4000 + seed)
    n_src = 1 << 31  # 8 GB of f32 + 8 GB of f64 source values
    g = torch.Generator(device=dev).manual_seed(20261203 + 4000)
    src32 = (torch.cumsum(torch.randn(n_src // 4, generator=g, device=dev), 0) * 1e-3).contiguous()
    src64 = (torch.cumsum(torch.randn(n_src // 8, generator=g, device=dev, dtype=torch.float64), 0) * 1e-3)
    lo, hi = np.log(1024), np.log(256 << 20)

    def pick(dt):
        src = src32 if dt == np.float32 else src64
        cnt = max(1, int(np.exp(rng.uniform(lo, hi))) // np.dtype(dt).itemsize)
        per16 = 16 // np.dtype(dt).itemsize  # request buffers start 16-byte aligned
        off = int(rng.integers(0, (src.numel() - cnt) // per16)) * per16
        return src[off:off + cnt]

    bank = []
    for i in range(256):
        dt = np.float32 if i % 2 else np.float64
        eb = None if (i // 2) % 2 == 0 else float(10 ** rng.uniform(-6, -2))
        x = pick(dt)
        bank.append((api.compress(x, eb), np.dtype(dt), eb, x.numel()))
    bank_bytes = sum(b[0].numel() for b in bank)

    def make(n, rate):
        reqs, t = [], 0.0
        for k in range(n):
            t += rng.exponential(1.0 / rate) if rate else 0.0
            if rng.random() < 0.6:
                dt = np.float32 if rng.random() < 0.5 else np.float64
                x = pick(dt)
                eb = None if rng.random() < 0.5 else float(10 ** rng.uniform(-6, -2))
                reqs.append(Request("compress", x, np.dtype(dt), eb, arrival=t, rid=k))
            else:
                st_, dt, eb, cnt = bank[int(rng.integers(0, len(bank)))]
                reqs.append(Request("decompress", st_, dt, eb, num_elements=cnt, arrival=t, rid=k))
        return reqs

    def clone(rs):
        return [Request(r.op, r.src, r.dtype, r.eb, num_elements=r.num_elements, arrival=r.arrival, rid=r.rid)
                for r in rs]

    free, _ = torch.cuda.mem_get_info()
    budget = int(min(150 << 30, free - (8 << 30)))
    # launches of up to 131,072 chunks (2 GB): capping them at the largest request
    # (256 MB) shortens the native loop's tail at equal load (p99 1.1 -> 0.9 ms)
    # but lowers its peak by 12 % and starves the Python loop, whose cost per
    # launch then dominates

    def py_server():
        return Server(hbm_budget=budget, slots=4, max_batch=512, max_batch_chunks=1 << 17)

    # peaks: everything queued at once -- plain calls, the Python loop, the native loop
    warm = make(min(2000, n_requests), 0.0)
    plain_peak = serve_plain(clone(warm), dev)["gbs"]
    srv = py_server()
    py_peak = srv.serve(clone(warm))["gbs"]
    srv.close()
    srv = None  # the arena goes back to the device before the next one
    torch.cuda.empty_cache()
    nat = NativeServer(hbm_budget=budget, slots=4, max_batch=512, max_batch_chunks=1 << 17)
    peak = nat.serve(clone(warm))["gbs"]
    reqs = make(n_requests, 0.0)
    mean_bytes = np.mean([r.raw_bytes for r in reqs])
    rate = 0.7 * peak * 1e9 / mean_bytes
    t = 0.0
    for r in reqs:
        t += rng.exponential(1.0 / rate)
        r.arrival = t
    plain_reqs, py_reqs = clone(reqs), clone(reqs)
    sample = set(int(i) for i in rng.choice(len(reqs), max(1, len(reqs) // 100), replace=False))
    stats = nat.serve(reqs, keep=lambda r: r.rid in sample)
    exact = True
    kept = []
    for r in reqs:
        if r.rid in sample:
            got = nat.result(r)
            alone = api.compress(r.src, r.eb) if r.op == "compress" else api.decompress(r.src, r.dtype, r.eb).view(
                torch.uint8)
            exact = exact and torch.equal(got, alone)
            if r.raw_bytes <= (8 << 20) and len(kept) < 200:
                kept.append((r.op, r.src.cpu().numpy(), np.dtype(r.dtype), r.eb, got.cpu().numpy()))
            nat.release(r)
    got = alone = None  # views of the arena
    nat.close()
    nat = None
    torch.cuda.empty_cache()
    # the same trace through the Python loop and through plain calls
    srv = py_server()
    py_stats = srv.serve(py_reqs)
    srv.close()
    srv = None
    torch.cuda.empty_cache()
    plain = serve_plain(plain_reqs, dev)
    stats.update({"loop": "native: one thread of the library admits, launches and completes (sleek_server_*)",
                  "target_load": 0.7, "peak_gbs": peak, "arrival_rate_per_s": round(rate, 1),
                  "hbm_budget_bytes": budget, "sample_checked": len(sample), "sample_bit_exact": bool(exact),
                  "decompress_bank": {"streams": len(bank), "bytes": bank_bytes},
                  "python_loop": {**py_stats, "peak_gbs": py_peak,
                                  "form": "the same loop in Python (serve.Server), same trace"},
                  "plain": {**plain, "peak_gbs": plain_peak,
                            "form": "one sleek_compress_*/sleek_decompress_* call per request, one stream"},
                  "served_over_plain": {"peak": round(peak / plain_peak, 2),
                                        "at_load_gbs": round(stats["gbs"] / plain["gbs"], 2)},
                  "workload": f"{n_requests} requests, Poisson at 70% of peak, 1 KB-256 MB log-uniform, "
                              "60/40 compress/decompress, 50% lossy eb in [1e-6,1e-2]"})
    return stats, kept


def served_oracle_check(kept) -> dict:
    """Checker for the served leg (CPU-baseline leg only): the kept sample of served
    results against the oracle."""
    from oracle import oracle as O

    ok = True
    for op, src, dt, eb, got in kept:
        if op == "compress":
            ok = ok and got.tobytes() == O.encode(src.view(dt), eb)
        else:
            ok = ok and got.tobytes() == O.decode(src.tobytes(), dt, eb).tobytes()
    return {"checked": len(kept), "bit_exact": bool(ok)}


def _graph_gbs(fn, nbytes, reps, stream):
    """GB/s of `nbytes` per call: `reps` calls captured in one CUDA graph, one warm
    replay, then one replay between CUDA events on `stream`."""
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        for _ in range(reps):
            fn()
    with torch.cuda.stream(stream):  # replay() launches on the current stream
        g.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.replay()
        e1.record(stream)
    torch.cuda.synchronize()
    del g
    return nbytes * reps / (e0.elapsed_time(e1) * 1e-3) / 1e9


def _copy_gbs(dst, src, reps, stream):
    """GB/s of a device-to-device copy of src's bytes (memcpy.cu:121-129): `reps`
    eager copies between CUDA events after three warm-up copies.  (A copy captured
    in a CUDA graph becomes a memcpy node, which ran at about half the speed of the
    eager copy on the B200, so the copy is not graph-timed.)"""
    n = src.numel() * src.element_size()
    with torch.cuda.stream(stream):
        for _ in range(3):
            dst.copy_(src)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            dst.copy_(src)
        e1.record(stream)
    torch.cuda.synchronize()
    return n * reps / (e0.elapsed_time(e1) * 1e-3) / 1e9


def _geomean(v):
    v = [float(x) for x in v]
    return float(np.exp(np.mean(np.log(v)))) if v else None


def bench_configs(dev, peak, extra_rows=None, reps=10, tune=True):
    """Every single-buffer configuration of the measurement table on the same device
    path, each beside a D2D copy of the same bytes (the reference's own comparison,
    memcpy.cu:121-129, made per input by compress_decompress_inputs_single.py:228-240):
    compress / decompress GB/s of uncompressed bytes, the compression ratio, the
    fraction of the copy's GB/s and of the HBM roofline ((N + S) / t over the measured
    copy bandwidth), then geomeans over every (configuration, mode) row as the
    reference's harness takes them (:250-257).  The C-ABI calls use the library-owned
    workspace and are captured `reps` times in a CUDA graph, replayed between CUDA
    events, so small inputs measure the device, not the Python call overhead; each
    result is checked by a round trip (exact for lossless, within the bound for lossy).
    `extra_rows` adds rows measured elsewhere (the float64 field of the main leg)."""
    from sleek_b200 import _capi, api, workloads

    L = _capi.lib()
    cases = [("c0 f32 signal 2^24", lambda: workloads.c0_signal(device=dev), (None,)),
             ("c2a f32 1800x3600", lambda: workloads.c2a_latlon(device=dev), (None, 1e-3)),
             ("c2b f32 512^3", lambda: workloads.c2b_lognormal(device=dev), (None, 1e-3)),
             ("c2c f32 2^28", lambda: workloads.c2c_particles(device=dev), (None, 1e-3))]
    out = dict(extra_rows or {})
    side = torch.cuda.Stream(dev)
    sh = side.cuda_stream
    for name, make, ebs in cases:
        x = make().contiguous().view(-1)
        N = x.numel() * x.element_size()
        enc = torch.empty(api.sleek_upper_bound_size(N), dtype=torch.uint8, device=dev)
        dec = torch.empty_like(x)
        size = torch.zeros(2, dtype=torch.int64, device=dev)
        memcpy = _copy_gbs(dec, x, reps, side)
        row = {"bytes": N, "memcpy_d2d_gbs": round(memcpy, 1)}
        for eb in ebs:
            if eb is None:
                fc = lambda: L.sleek_compress_f32(x.data_ptr(), x.numel(), enc.data_ptr(), size.data_ptr(),
                                                  None, 0, sh)
                fd = lambda: L.sleek_decompress_f32(enc.data_ptr(), enc.numel(), dec.data_ptr(), N,
                                                    size[1:].data_ptr(), None, 0, sh)
            else:
                e = api.sleek_error_bound(eb, np.float32).c_struct()
                fc = lambda: L.sleek_compress_lossy_f32(e, x.data_ptr(), x.numel(), enc.data_ptr(),
                                                        size.data_ptr(), None, 0, sh)
                fd = lambda: L.sleek_decompress_lossy_f32(e, enc.data_ptr(), enc.numel(), dec.data_ptr(), N,
                                                          size[1:].data_ptr(), None, 0, sh)
            shapes = None
            if tune:
                from sleek_b200 import autotune

                shapes = {d: _tuned_row(autotune.tune_single(x, eb, decompress=(d == "decompress"), use_cache=False))
                          for d in ("compress", "decompress")}
            with torch.cuda.stream(side):
                for _ in range(3):  # warm-up outside capture (grid sizes, attributes, workspace)
                    _capi.check(fc())
                    _capi.check(fd())
            side.synchronize()
            S = int(size[0].item())
            assert int(size[1].item()) == N, name
            if eb is None:
                assert torch.equal(dec.view(torch.int32), x.view(torch.int32)), name
            else:
                fin = torch.isfinite(x)
                assert bool(((dec[fin] - x[fin]).abs() <= eb).all()), name
            cg = _graph_gbs(lambda: _capi.check(fc()), N, reps, side)
            dg = _graph_gbs(lambda: _capi.check(fd()), N, reps, side)
            row[str(eb)] = _mode_row(N, S, cg, dg, memcpy, peak)
            if shapes:
                row[str(eb)]["launch_shapes"] = shapes
        out[name] = row
        del x, enc, dec
        torch.cuda.empty_cache()
    rows = [r for cfg in out.values() for k, r in cfg.items() if isinstance(r, dict)]
    out["geomean"] = {k: round(_geomean([r[k] for r in rows]), 3)
                      for k in ("ratio", "compress_gbs", "decompress_gbs")}
    out["geomean"]["memcpy_d2d_gbs"] = round(_geomean([c["memcpy_d2d_gbs"] for c in out.values()
                                                      if "memcpy_d2d_gbs" in c]), 1)
    for k in ("compress", "decompress"):
        out["geomean"][f"frac_of_memcpy_{k}"] = round(_geomean([r["frac_of_memcpy"][k] for r in rows]), 3)
        out["geomean"][f"roofline_frac_{k}"] = round(_geomean([r["roofline_frac"][k] for r in rows]), 3)
    out["all_at_least_0.8_of_memcpy"] = {k: all(r["frac_of_memcpy"][k] >= 0.8 for r in rows)
                                         for k in ("compress", "decompress")}
    out["timing"] = (f"{reps} calls per CUDA graph replay, CUDA events; copy: {reps} eager D2D copies of the same "
                     "bytes between CUDA events")
    return out


def _tuned_row(r):
    """The autotuner's choice as recorded in the bench line."""
    sh = r["shape"]
    return {"shape": sh["shape"], "threads": sh["threads"], "warps": sh["warps"], "stages": sh["stages"],
            "ctas_per_sm": r["best"][1] or "all that fit", "size_bucket_log2": r["bucket_log2"]}


def _mode_row(N, S, cg, dg, memcpy, peak):
    """One (configuration, mode) row: GB/s of N, fraction of the D2D copy and of the
    HBM roofline ((N + S) bytes moved per call over the measured copy bandwidth)."""
    return {"ratio": round(N / S, 3), "compress_gbs": round(cg, 1), "decompress_gbs": round(dg, 1),
            "frac_of_memcpy": {"compress": round(cg / memcpy, 3), "decompress": round(dg / memcpy, 3)},
            "roofline_frac": {"compress": round(cg * (N + S) / N / peak, 3),
                              "decompress": round(dg * (N + S) / N / peak, 3)}}


def bench_transfer(x, modes=(None, 1e-2, 1e-4), repeats=3):
    """Compressed device->host and host->device copies of the field against plain
    pinned cudaMemcpy of its N bytes: GB/s of uncompressed bytes, wall clock around
    the synchronous calls (median of `repeats` after one warm-up); the assembled
    host stream must equal the device stream byte for byte."""
    from sleek_b200 import api

    N = x.numel() * x.element_size()
    hraw = torch.empty(N, dtype=torch.uint8, pin_memory=True)
    hstream = torch.empty(api.sleek_upper_bound_size(N), dtype=torch.uint8, pin_memory=True)
    back = torch.empty_like(x)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(repeats):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return sorted(ts)[len(ts) // 2]

    xr = x.view(-1).view(torch.uint8)
    out = {"workload": "c1 f64 field, 301,989,888 B, pinned host buffers, 32 MiB segments",
           "plain_d2h_gbs": round(N / timed(lambda: hraw.copy_(xr)) / 1e9, 2),
           "plain_h2d_gbs": round(N / timed(lambda: back.view(-1).view(torch.uint8).copy_(hraw)) / 1e9, 2)}
    exact = True
    for eb in modes:
        h = api.compress_to_host(x, eb, out=hstream)
        exact &= h.numpy().tobytes() == api.compress(x, eb).cpu().numpy().tobytes()
        t_c = timed(lambda: api.compress_to_host(x, eb, out=hstream))
        n = h.numel()
        t_d = timed(lambda: api.decompress_from_host(hstream[:n], np.float64, eb, out=back))
        if eb is None:
            exact &= torch.equal(back.view(-1).view(torch.int64), x.view(-1).view(torch.int64))
        out[str(eb)] = {"ratio": round(N / n, 3), "compress_to_host_gbs": round(N / t_c / 1e9, 2),
                        "decompress_from_host_gbs": round(N / t_d / 1e9, 2)}
    out["bit_exact"] = bool(exact)
    return out


def config_dict(args):
    return {"workload": "c1 f64 turbulence field 256x384x384 (301,989,888 B), lossless + eb 1e-2/1e-4/1e-6, "
                        "compress+decompress per mode",
            "global_batch": 8 * args.gpus, "seq_len": None, "parallelism": f"replicas{args.gpus}",
            "l2": "inputs larger than L2 (302 MB > 126 MB), no flush"}


# ---------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg (profiling runs)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched (1000-array) comparison")
    ap.add_argument("--no-transfer", action="store_true", help="skip the compressed host<->device copy leg")
    ap.add_argument("--no-configs", action="store_true", help="skip the f32 configurations leg")
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes, no autotuning")
    ap.add_argument("--serve-requests", type=int, default=100000,
                    help="requests of the served workload leg (0 = skip; 100000 = the full workload)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world, rank, local = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        if world > 1:
            torch.distributed.destroy_process_group()
        return

    from sleek_b200 import _capi, api, workloads

    peak, peak_kind = peaks()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    L = _capi.lib()
    x = workloads.c1_turbulence(SHAPE, device=dev)
    N = x.numel() * 8
    cap = api.sleek_upper_bound_size(N)
    st = torch.cuda.current_stream()
    sh = st.cuda_stream
    # persistent device buffers, one stream buffer per mode
    enc = [torch.empty(cap, dtype=torch.uint8, device=dev) for _ in MODES]
    esz = torch.zeros(len(MODES), dtype=torch.int64, device=dev)
    dsz = torch.zeros(len(MODES), dtype=torch.int64, device=dev)
    dec = torch.empty_like(x)
    ebi = [None if eb is None else api.sleek_error_bound(eb, np.float64).c_struct() for eb in MODES]

    # the reference-shaped entry points with the library-owned workspace (NULL): the
    # kernels keep it ready themselves, so a call is one kernel launch
    def launch_c(i):
        if ebi[i] is None:
            rc = L.sleek_compress_f64(x.data_ptr(), x.numel(), enc[i].data_ptr(), esz[i:].data_ptr(), None, 0, sh)
        else:
            rc = L.sleek_compress_lossy_f64(ebi[i], x.data_ptr(), x.numel(), enc[i].data_ptr(),
                                            esz[i:].data_ptr(), None, 0, sh)
        _capi.check(rc, "compress")

    def launch_d(i):
        if ebi[i] is None:
            rc = L.sleek_decompress_f64(enc[i].data_ptr(), cap, dec.data_ptr(), N, dsz[i:].data_ptr(), None, 0, sh)
        else:
            rc = L.sleek_decompress_lossy_f64(ebi[i], enc[i].data_ptr(), cap, dec.data_ptr(), N,
                                              dsz[i:].data_ptr(), None, 0, sh)
        _capi.check(rc, "decompress")

    # launch shapes: the autotuner times the kernel shapes on this field, per mode and
    # direction, and the timed calls below use its choice
    tuned = {}
    if not args.no_tune:
        from sleek_b200 import autotune

        for i, eb in enumerate(MODES):
            tuned[str(eb)] = {d: _tuned_row(autotune.tune_single(x, eb, decompress=(d == "decompress"),
                                                                 use_cache=False))
                              for d in ("compress", "decompress")}

    # correctness gate before timing: every mode round-trips and sizes are sane
    for i in range(len(MODES)):
        launch_c(i)
        launch_d(i)
    torch.cuda.synchronize()
    S = [int(v) for v in esz.cpu().tolist()]
    assert all(s > 0 for s in S) and all(int(v) == N for v in dsz.cpu().tolist()), (S, dsz)

    # ---- per-kernel CUDA-event timing (the roofline numbers) ------------------------
    reps = 10
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(len(MODES) * reps)]
    for i in range(len(MODES)):
        launch_c(i)
        launch_d(i)
    torch.cuda.synchronize()
    k = 0
    for r in range(reps):
        for i in range(len(MODES)):
            e = ev[k]; k += 1
            e[0].record(st); launch_c(i); e[1].record(st)
            e[2].record(st); launch_d(i); e[3].record(st)
    torch.cuda.synchronize()
    tc = [0.0] * len(MODES)
    td = [0.0] * len(MODES)
    k = 0
    for r in range(reps):
        for i in range(len(MODES)):
            e = ev[k]; k += 1
            tc[i] += e[0].elapsed_time(e[1]) / reps
            td[i] += e[2].elapsed_time(e[3]) / reps
    # memcpy D2D baseline on the same bytes (memcpy.cu:121-129 convention)
    mc = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(3):
        dec.copy_(x)
    mc[0].record(st)
    for _ in range(reps):
        dec.copy_(x)
    mc[1].record(st)
    torch.cuda.synchronize()
    t_memcpy = mc[0].elapsed_time(mc[1]) / reps
    memcpy_gbs = N / (t_memcpy * 1e-3) / 1e9

    # ---- whole-step timing ------------------------------------------------------------
    def step():
        for i in range(len(MODES)):
            launch_c(i)
            launch_d(i)

    for _ in range(args.warmup):
        step()
    barrier(world)
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    t0.record(st)
    for _ in range(args.steps):
        step()
    t1.record(st)
    torch.cuda.synchronize()
    barrier(world)
    clocks = clk.stop()
    ms = t0.elapsed_time(t1)
    ms_max = dist_max(ms, world)
    bytes_per_step = 2 * N * len(MODES)
    value = bytes_per_step * args.steps * world / (ms_max * 1e-3) / 1e9

    # ---- end to end through the public API with host buffers ---------------------------
    # Per mode: pinned host array -> device, compress_to_host (only the stream crosses
    # PCIe, its size read back properly), decompress_from_host, device -> pinned host
    # array.  The next mode's input copy runs on its own stream during this mode's
    # codec calls and this mode's output copy during the next mode's, so both PCIe
    # directions carry data at once; every byte is copied inside the timed region.
    hin = torch.empty(x.numel(), dtype=torch.float64, pin_memory=True)
    hin.copy_(x.cpu())
    hstream = [torch.empty(cap, dtype=torch.uint8, pin_memory=True) for _ in MODES]
    hout = [torch.empty(x.numel(), dtype=torch.float64, pin_memory=True) for _ in range(2)]
    d_in = [torch.empty_like(x) for _ in range(2)]
    d_out = [torch.empty_like(x) for _ in range(2)]
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    got = [0] * len(MODES)
    h2d = sum(N + s for s in S)
    d2h = sum(s + N for s in S)

    def e2e_step():
        with torch.cuda.stream(s_in):
            s_in.wait_event(ev_out[0])
            d_in[0].copy_(hin, non_blocking=True)
            ev_in[0].record(s_in)
        for i, eb in enumerate(MODES):
            b = i % 2
            if i + 1 < len(MODES):  # prefetch the next input
                with torch.cuda.stream(s_in):
                    d_in[1 - b].copy_(hin, non_blocking=True)
                    ev_in[1 - b].record(s_in)
            st.wait_event(ev_in[b])
            h = api.compress_to_host(d_in[b], eb, out=hstream[i], stream=st)
            got[i] = h.numel()
            st.wait_event(ev_out[b])  # the output copy of mode i - 2 has finished with d_out[b]
            api.decompress_from_host(h, np.float64, eb, out=d_out[b], stream=st)
            s_out.wait_stream(st)
            with torch.cuda.stream(s_out):
                hout[b].copy_(d_out[b], non_blocking=True)
                ev_out[b].record(s_out)
        st.wait_stream(s_out)

    e2e_value = None
    if not args.no_e2e:
        for _ in range(2):
            e2e_step()
        # the host round trip is exact (lossless mode, checked outside the timed region)
        h = api.compress_to_host(d_in[0], None, out=hstream[0], stream=st)
        api.decompress_from_host(h, np.float64, None, out=d_out[0], stream=st)
        hout[0].copy_(d_out[0])
        assert torch.equal(hout[0].view(torch.int64), hin.view(torch.int64))
        torch.cuda.synchronize()
        barrier(world)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.e2e_steps):
            e2e_step()
        e1.record(st)
        torch.cuda.synchronize()
        e2e_ms = dist_max(e0.elapsed_time(e1), world)
        e2e_value = round(bytes_per_step * args.e2e_steps * world / (e2e_ms * 1e-3) / 1e9, 2)
        assert got == list(S), (got, S)

    # ---- roofline of the dominant kernel ----------------------------------------------
    t_enc = sum(tc)
    t_dec = sum(td)
    dom = "encode" if t_enc >= t_dec else "decode"
    per = tc if dom == "encode" else td
    alg_bytes = sum(N + s for s in S) / len(MODES)
    t_launch = sum(per) / len(MODES)
    achieved = alg_bytes / (t_launch * 1e-3) / 1e9

    # DRAM traffic of the dominant kernel per launch, from the committed ncu summary
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"k_{dom}_c1_f64.md")
    if os.path.exists(prof):
        for ln_ in open(prof):
            if ln_.startswith("traffic_bytes_per_launch"):
                traffic = int(ln_.split(":")[1].split()[0])
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args),
        "compress_gbs": {str(m): round(N / (tc[i] * 1e-3) / 1e9, 1) for i, m in enumerate(MODES)},
        "decompress_gbs": {str(m): round(N / (td[i] * 1e-3) / 1e9, 1) for i, m in enumerate(MODES)},
        "ratio": {str(m): round(N / S[i], 4) for i, m in enumerate(MODES)},
        "memcpy_d2d_gbs": round(memcpy_gbs, 1),
        "frac_of_memcpy": {
            "compress": round(len(MODES) * N / (t_enc * 1e-3) / 1e9 / memcpy_gbs, 3),
            "decompress": round(len(MODES) * N / (t_dec * 1e-3) / 1e9 / memcpy_gbs, 3)},
        "roofline": {"bound": "hbm", "kernel": f"k_{dom}<u64> (mean over the 4 modes)",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 3), "peak_kind": f"of {peak_kind}", "traffic": traffic,
                     "traffic_note": "ncu DRAM read+write of one lossless launch (profiles/); the L2 still holds "
                                     "part of the written stream when the kernel ends"},
        "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": 2 * len(MODES) * args.steps,
        "clocks": clocks,
        "launch_shapes": tuned or "defaults (--no-tune)",
    }
    if not args.no_batched:
        # free the single-buffer leg's buffers first
        del enc, dec, d_in, d_out, hin, hout, hstream
        torch.cuda.empty_cache()
        line["batched"] = bench_batched(dev, world, args)
    kept = []
    if args.serve_requests > 0:
        torch.cuda.empty_cache()
        line["served"], kept = bench_serve(dev, args.serve_requests)
    if not args.no_transfer:
        line["transfer"] = bench_transfer(x)
    if not args.no_configs:
        c1_row = {"bytes": N, "memcpy_d2d_gbs": round(memcpy_gbs, 1)}
        for i, m in enumerate(MODES):
            c1_row[str(m)] = _mode_row(N, S[i], N / (tc[i] * 1e-3) / 1e9, N / (td[i] * 1e-3) / 1e9, memcpy_gbs, peak)
        for i, m in enumerate(MODES):
            if tuned:
                c1_row[str(m)]["launch_shapes"] = tuned[str(m)]
        line["configs"] = bench_configs(dev, peak, {"c1 f64 256x384x384 (main leg, per-call CUDA events)": c1_row},
                                        tune=not args.no_tune)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference's own implementations on this box: its CPU codec (the baseline)
        # and, beside it, its GPU kernels built for sm_100a; the oracle checks the
        # kept sample of served results
        line["cpu_baseline"] = cpu_baseline(x.cpu().numpy())
        line["reference_gpu"] = reference_gpu_kernels(x)
        if kept:
            line["served"]["sample_oracle"] = served_oracle_check(kept)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
