"""Benchmark of the B200 hot path (one JSON line on rank 0).

Headline workload: the equi-join SELECT SUM(b.payload * p.value), COUNT(*)
FROM probe p JOIN build b ON p.fk = b.key WHERE b.attr < 20, with a 2M-row
build table and a 120M-row probe table per GPU (weak scaling: every rank
joins its own probe shard against the same build table, then the partial
SUM/COUNT are all-reduced over NCCL).  A step is the whole query: build
append (fused filter) + table build + fused probe/aggregate + finish.

`value` times it with every input resident in HBM; `e2e` times the same
query through the C ABI from pinned host buffers (host->device copies in the
timed region).  `roofline` is the fused probe kernel's algorithmic bytes
(16 B per probe row) over its CUDA-event duration against the measured HBM
copy bandwidth.  `operators` adds the lineitem-shaped fused
filter->project->aggregate (6,001,215 rows) and the 200M-row Zipf GROUP BY.

--impl reference times the CPU restatement of the engine's threaded plan
(the reference engine itself cannot be built: its kernels are oz-lang for
an absent compiler) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

BUILD_ROWS = 2_000_000
PROBE_ROWS = 120_000_000
FK_DOMAIN = 2_500_000
LINEITEM_ROWS = 6_001_215
ZIPF_ROWS = 200_000_000
ZIPF_PARTS = 4096
SERVE_TABLES = 16
JOIN_PARTS = 256
SERVE_BUDGET = 150 * 10**9
SERVE_WORKERS = 3
SERVE_COALESCE_ROWS = 8 << 20   # rows up to which waiting Zipf aggregations coalesce (0: off)
ZIPF_DISTINCT = 20_000_000
SORT_ROWS = 300_000_000
METRIC = "rows/s & HBM GB/s vs peak per operator; mixed-stream queries/s and p50/p99"


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows: list[list[str]] = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def pinned(q, nbytes: int, dtype, count: int) -> tuple[int, np.ndarray]:
    ptr = q.lib().qdb_gpu_host_alloc(nbytes)
    if not ptr:
        raise MemoryError("pinned allocation failed")
    arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), shape=(nbytes,)).view(dtype)[:count]
    return ptr, arr


class JoinWorkload:
    def __init__(self, q, rank: int):
        from qumirdb_b200 import queries
        self.q = q
        self.build_host = []
        self.probe_host = []
        self.ptrs = []
        for dt, n in [(np.int64, BUILD_ROWS), (np.int64, BUILD_ROWS), (np.int32, BUILD_ROWS)]:
            p, a = pinned(q, n * np.dtype(dt).itemsize, dt, n)
            self.ptrs.append(p)
            self.build_host.append(a)
        for dt, n in [(np.int64, PROBE_ROWS), (np.int64, PROBE_ROWS)]:
            p, a = pinned(q, n * np.dtype(dt).itemsize, dt, n)
            self.ptrs.append(p)
            self.probe_host.append(a)
        # The build table is the same on every rank; the probe shard is the rank's own.
        q.lib().qdb_gen_join(1, BUILD_ROWS, 0, FK_DOMAIN, *[a.ctypes.data for a in self.build_host], None, None)
        tmp = [np.empty(1, np.int64), np.empty(1, np.int64), np.empty(1, np.int32)]
        q.lib().qdb_gen_join(1000 + rank, 1, PROBE_ROWS, FK_DOMAIN, *[t.ctypes.data for t in tmp],
                             *[a.ctypes.data for a in self.probe_host])
        self.dev_build = q.DeviceRowSet(self.build_host)
        self.dev_probe = q.DeviceRowSet(self.probe_host)
        self.host_build = q.HostRowSet(self.build_host)
        self.host_probe = q.HostRowSet(self.probe_host)
        self.jspec, self.aspec = queries.join_sum(20)
        self.prog = q.compile_join_aggregate(self.jspec, self.aspec)
        self.rows = BUILD_ROWS + PROBE_ROWS
        self.h2d = BUILD_ROWS * 20 + PROBE_ROWS * 16

    def step(self, resident: bool = True) -> tuple[int, int]:
        q = self.q
        from qumirdb_b200 import abi
        J = q.RowJoin(self.prog)
        J.append(self.dev_build if resident else self.host_build)
        J.build()
        agg = q.Aggregate(self.prog)
        J.probe_aggregate(agg, self.dev_probe if resident else self.host_probe)
        out = agg.finish()
        vals, _ = q.read_rowset(out, [abi.I64, abi.I64])
        res = (int(vals[0][0]), int(vals[1][0]))
        q.release(out)
        return res


def combine_partials(dist, s: int, c: int, device: str = "cuda") -> tuple[int, int]:
    """The join's partial SUM(payload*value) and COUNT(*) of every rank's probe
    shard, summed over ranks (the one data-path collective: the partials are
    two int64 words; SUM wraps like the engine's reducer)."""
    import torch
    t = torch.tensor([s, c], device=device, dtype=torch.int64)
    dist.all_reduce(t)
    return int(t[0]), int(t[1])


def max_over_ranks(dist, ms: float, device: str = "cuda") -> float:
    """The slowest rank's time: the whole job is done when the last rank is."""
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def timed(q, fn, steps: int, warmup: int, dist=None, profile: bool = False):
    """Device time of `steps` calls of fn on the library's stream (events)."""
    import torch
    for _ in range(warmup):
        fn()
    stream = torch.cuda.ExternalStream(q.lib().qdb_gpu_get_stream())
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    q.synchronize()
    q.profile(profile)
    q.profile_read()
    launches0 = q.launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    results = [fn() for _ in range(steps)]
    end.record(stream)
    end.synchronize()
    torch.cuda.synchronize()
    ms = start.elapsed_time(end) / steps
    launches = q.launch_count() - launches0
    kernels = q.profile_read() if profile else []
    q.profile(False)
    if dist is not None:
        ms = max_over_ranks(dist, ms)
    return ms, results, launches, kernels


def kernel_avg(kernels, name, steps: int = 1):
    """Per-step device time of every launch of `name` (summed over the step's
    launches) and the units they processed per step."""
    ks = [(ms, units) for n, ms, units in kernels if n == name]
    if not ks:
        return None, None
    return sum(k[0] for k in ks) / steps, sum(k[1] for k in ks) / steps


def load_traffic() -> dict:
    p = ROOT / "profiles" / "traffic.json"
    return json.loads(p.read_text()) if p.exists() else {}


def lineitem_operator(q, peak):
    from qumirdb_b200 import abi, queries
    n = LINEITEM_ROWS
    cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64),
            np.empty(n, np.uint8), np.empty(n, np.uint8), np.empty(n, np.int32)]
    q.lib().qdb_gen_lineitem(0, n, *[c.ctypes.data for c in cols])
    spec = queries.lineitem_agg(int(cols[6].max()) - 90, flags=abi.OUT_DEVICE)
    prog = q.compile_aggregate(spec)
    drs = q.DeviceRowSet(cols)
    flush = q.DeviceBuffer(256 << 20)

    import torch
    stream = torch.cuda.ExternalStream(q.lib().qdb_gpu_get_stream())

    def query():
        agg = q.Aggregate(prog)
        agg.add(drs)
        out = agg.finish()
        q.release(out)

    # Each query runs after an L2 flush; only the query is timed (events
    # around it on the library's stream), the flush is not.
    for _ in range(3):
        flush_l2(q, flush)
        query()
    q.synchronize()
    q.profile(True)
    q.profile_read()
    launches0 = q.launch_count()
    times = []
    for _ in range(10):
        flush_l2(q, flush)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        query()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    launches = q.launch_count() - launches0
    kernels = q.profile_read()
    q.profile(False)
    ms = statistics.median(times)
    kname = "agg_update_sig" if any(k[0] == "agg_update_sig" for k in kernels) else "agg_update"
    kms, _ = kernel_avg(kernels, kname, 10)
    alg = n * 38
    return {"workload": "lineitem scan-filter-aggregate, 6,001,215 rows, GROUP BY flag, status",
            "rows_per_s": n / (ms / 1e3), "ms_per_query": ms, "kernel": kname, "kernel_ms": kms,
            "algorithmic_bytes": alg, "kernel_gbs": alg / (kms / 1e3) / 1e9 if kms else None,
            "frac_of_measured_hbm": (alg / (kms / 1e3) / 1e9) / peak if kms else None,
            "l2": "flushed between queries (256 MiB write)", "gpu_launches": launches / 10}


def lineitem_batched_operator(q, peak):
    """The config-0 lineitem table split into 64 contiguous partitions, each
    its own aggregate of the Q1-shaped program, all in one
    qdb_gpu_agg_dispatch_batch (the low-cardinality batched kernel) and one
    batched finalize per query; L2 flushed between queries."""
    from qumirdb_b200 import abi, queries
    n = LINEITEM_ROWS
    parts = 64
    cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64),
            np.empty(n, np.uint8), np.empty(n, np.uint8), np.empty(n, np.int32)]
    q.lib().qdb_gen_lineitem(0, n, *[c.ctypes.data for c in cols])
    prog = q.compile_aggregate(queries.lineitem_agg(int(cols[6].max()) - 90, flags=abi.OUT_DEVICE))
    bounds = np.linspace(0, n, parts + 1).astype(np.int64)
    rowsets = [q.DeviceRowSet([c[lo:hi] for c in cols]) for lo, hi in zip(bounds[:-1], bounds[1:])]
    flush = q.DeviceBuffer(256 << 20)

    import torch
    stream = torch.cuda.ExternalStream(q.lib().qdb_gpu_get_stream())

    def query():
        b = q.AggregateBatch(prog, parts)
        b.add(rowsets)
        b.finish().release()

    for _ in range(3):
        flush_l2(q, flush)
        query()
    q.synchronize()
    q.profile(True)
    q.profile_read()
    times = []
    for _ in range(10):
        flush_l2(q, flush)
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        query()
        e.record(stream)
        e.synchronize()
        times.append(a.elapsed_time(e))
    kernels = q.profile_read()
    q.profile(False)
    ms = statistics.median(times)
    kms, _ = kernel_avg(kernels, "agg_batch_update_low", 10)
    alg = n * 38
    return {"workload": "lineitem scan-filter-aggregate, 6,001,215 rows as 64 partitions, one batched launch",
            "rows_per_s": n / (ms / 1e3), "ms_per_query": ms, "kernel": "agg_batch_update_low", "kernel_ms": kms,
            "algorithmic_bytes": alg, "kernel_gbs": alg / (kms / 1e3) / 1e9 if kms else None,
            "frac_of_measured_hbm": (alg / (kms / 1e3) / 1e9) / peak if kms else None,
            "l2": "flushed between queries (256 MiB write)"}


def flush_l2(q, buf):
    q.lib().qdb_gpu_memset(buf.ptr, 0, buf.nbytes)


def zipf_operator(q, peak):
    from qumirdb_b200 import abi, queries
    n = ZIPF_ROWS
    cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.float64)]
    q.lib().qdb_gen_zipf(2, n, ZIPF_DISTINCT, 1.1, *[c.ctypes.data for c in cols])
    spec = queries.zipf_agg(expected_groups=ZIPF_DISTINCT, flags=abi.OUT_DEVICE)
    prog = q.compile_aggregate(spec)
    drs = q.DeviceRowSet(cols)
    del cols
    groups = []

    def step():
        agg = q.Aggregate(prog)
        agg.add(drs)
        groups.append(agg.groups)
        out = agg.finish()
        q.release(out)

    ms, _, launches, kernels = timed(q, step, 3, 1, profile=True)
    kname = "agg_update_high" if any(k[0] == "agg_update_high" for k in kernels) else "agg_update"
    kms, _ = kernel_avg(kernels, kname, 3)
    alg = n * 24
    return {"workload": "GROUP BY key (Zipf 1.1 over 20M), 200M rows, COUNT/SUM/MIN/MAX/SUM(f64)",
            "rows_per_s": n / (ms / 1e3), "ms_per_query": ms, "groups": groups[-1], "kernel": kname,
            "kernel_ms": kms, "algorithmic_bytes": alg,
            "kernel_gbs": alg / (kms / 1e3) / 1e9 if kms else None,
            "frac_of_measured_hbm": (alg / (kms / 1e3) / 1e9) / peak if kms else None,
            "l2": "inputs larger than L2", "gpu_launches": launches / 3}


def zipf_partition_sizes(parts: int = ZIPF_PARTS) -> np.ndarray:
    """Log-uniform partition sizes in [1e3, 1e6] rows (seeded)."""
    rng = np.random.default_rng(5)
    return np.exp(rng.uniform(np.log(1e3), np.log(1e6), parts)).astype(np.int64)


def zipf_batched_operator(q, peak):
    """The high-cardinality GROUP BY run as 4096 independent partitions of
    log-uniform size, each its own aggregate, all in one persistent launch
    per step (plus the batched finalize).  The partitions are consecutive
    slices of one Zipf(1.1 over 20M) stream, resident in HBM."""
    from qumirdb_b200 import abi, queries
    sizes = zipf_partition_sizes()
    n = int(sizes.sum())
    cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.float64)]
    q.lib().qdb_gen_zipf(6, n, ZIPF_DISTINCT, 1.1, *[c.ctypes.data for c in cols])
    prog = q.compile_aggregate(queries.zipf_agg(flags=abi.OUT_DEVICE))
    drs = q.DeviceRowSet(cols)
    del cols
    bounds = np.concatenate([[0], np.cumsum(sizes)])
    parts = q.RowSetPointers([q.SliceRowSet(drs, int(lo), int(hi)) for lo, hi in zip(bounds[:-1], bounds[1:])])
    groups = []

    def step():
        b = q.AggregateBatch(prog, len(parts))
        b.add(parts)
        groups.append(sum(b.groups))
        b.finish().release()

    ms, _, launches, _ = timed(q, step, 3, 3)
    _, _, _, kernels = timed(q, step, 2, 0, profile=True)
    kms, _ = kernel_avg(kernels, "agg_batch_update", 2)
    fms, _ = kernel_avg(kernels, "agg_finalize_batch", 2)
    alg = n * 24
    return {"workload": f"GROUP BY key (Zipf 1.1 over 20M) as {len(sizes)} independent partitions of "
                        f"log-uniform 1K-1M rows ({n} rows), COUNT/SUM/MIN/MAX/SUM(f64), one persistent launch",
            "rows_per_s": n / (ms / 1e3), "ms_per_query": ms, "groups": groups[-1], "kernel": "agg_batch_update",
            "kernel_ms": kms, "finalize_ms": fms, "algorithmic_bytes": alg,
            "kernel_gbs": alg / (kms / 1e3) / 1e9 if kms else None,
            "frac_of_measured_hbm": (alg / (kms / 1e3) / 1e9) / peak if kms else None,
            "l2": "inputs larger than L2", "gpu_launches": launches / 3, "autotune": q.autotune_info()}


def join_batched_operator(q, peak, w, steps: int = 3):
    """Config 1's join as the engine's partitioned plan: both sides split by
    the join key's hash into JOIN_PARTS partitions with the device shuffle
    (input preparation, untimed), then per step the partitions' build rows
    are appended in one batched call, all tables built in one, all probes run
    in one persistent launch and all aggregates finished in one batched
    finalize; SUM/COUNT summed over the partitions equal the single join's."""
    from qumirdb_b200 import abi
    hprog_b = q.compile_hash([(abi.I64,), (abi.I64,), (abi.I32,)], [0])
    hprog_p = q.compile_hash([(abi.I64,), (abi.I64,)], [0])
    bparts = q.shuffle(hprog_b, w.dev_build, JOIN_PARTS)
    pparts = q.shuffle(hprog_p, w.dev_probe, JOIN_PARTS)

    class View:
        def __init__(self, rs):
            self.rs = rs
            self.ptr = C.byref(rs)

    bviews = [View(bparts[i]) for i in range(JOIN_PARTS)]
    pviews = [View(pparts[i]) for i in range(JOIN_PARTS)]
    res = []

    def step():
        jb = q.RowJoinBatch(w.prog, JOIN_PARTS)
        jb.append_all(bviews)
        jb.build()
        jb.probe_aggregate(pviews)
        s = c = 0
        outs = jb.finish()
        for out in outs:
            vals, _ = q.read_rowset(out, [abi.I64, abi.I64])
            s += int(vals[0][0])
            c += int(vals[1][0])
        outs.release()
        jb.release()
        res.append((s, c))

    ms, _, launches, _ = timed(q, step, steps, 2 if steps > 1 else 0)
    _, _, _, kernels = timed(q, step, 2, 0, profile=True)
    kms, _ = kernel_avg(kernels, "join_agg_probe_batch", 2)
    bms, _ = kernel_avg(kernels, "join_build_batch", 2)
    alg = PROBE_ROWS * 16
    bparts.release()
    pparts.release()
    return {"workload": f"the 2M x 120M join split by key hash into {JOIN_PARTS} partitions (device shuffle), "
                        "one batched append, one batched build, one batched probe launch, one batched finalize",
            "rows_per_s": w.rows / (ms / 1e3), "ms_per_query": ms, "result": list(res[-1]),
            "kernel": "join_agg_probe_batch", "kernel_ms": kms, "build_batch_ms": bms,
            "frac_of_measured_hbm": (alg / (kms / 1e3) / 1e9) / peak if kms else None,
            "gpu_launches": launches / 3}


def serving_cpu_arm(tables, sample_rows: int = 4 << 20) -> dict:
    """The CPU arm of the serving stream: each table's query through the CPU
    restatement's threaded plans on all host threads, timed on a prefix of
    at most `sample_rows` rows of the same seeded table (the generators are
    deterministic per row) and scaled to the table's rows (these plans are
    linear in rows); queries/s is the table count over the summed service
    times (one query at a time, the engine's executor shape), p50/p99 the
    service times'."""
    from oracle import oracle as O
    from qumirdb_b200 import HostRowSet, queries
    threads = os.cpu_count() or 1
    secs = []
    for t in tables:
        m = min(t.rows, sample_rows)
        if t.template == "lineitem":
            cols = [np.empty(m, np.int64), np.empty(m, np.int64), np.empty(m, np.int64), np.empty(m, np.int64),
                    np.empty(m, np.uint8), np.empty(m, np.uint8), np.empty(m, np.int32)]
            O.lib().qdb_gen_lineitem(t.seed, m, *[c.ctypes.data for c in cols])
            spec = queries.lineitem_agg(t.cutoff)
            sec = O.lib().oracle_bench_aggregate(C.byref(spec.struct), HostRowSet(cols).ptr, threads, None)
        elif t.template == "zipf":
            cols = [np.empty(m, np.int64), np.empty(m, np.int64), np.empty(m, np.float64)]
            O.lib().qdb_gen_zipf(t.seed, m, max(1, t.rows // 10), 1.1, *[c.ctypes.data for c in cols])
            spec = queries.zipf_agg(expected_groups=max(1, m // 10))
            sec = O.lib().oracle_bench_aggregate(C.byref(spec.struct), HostRowSet(cols).ptr, threads, None)
        elif t.template == "join":
            nb = max(1, t.rows // 60)
            b = [np.empty(nb, np.int64), np.empty(nb, np.int64), np.empty(nb, np.int32)]
            p = [np.empty(m, np.int64), np.empty(m, np.int64)]
            O.lib().qdb_gen_join(t.seed, nb, m, nb + nb // 4, *[x.ctypes.data for x in b + p])
            s_, c_ = C.c_int64(), C.c_int64()
            sec = O.lib().oracle_bench_join_sum(b[0].ctypes.data, b[1].ctypes.data, b[2].ctypes.data, nb, 20,
                                                p[0].ctypes.data, p[1].ctypes.data, m, threads, C.byref(s_),
                                                C.byref(c_))
        else:
            k1, k2 = np.empty(m, np.int64), np.empty(m, np.int32)
            O.lib().qdb_gen_sort(t.seed, m, k1.ctypes.data, k2.ctypes.data, None)
            spec = queries.sort_k1_desc_k2()
            rs = HostRowSet([k1, k2, np.arange(m, dtype=np.int64)])
            t0 = time.perf_counter()
            O.top_k(spec, [rs], np.arange(m, dtype=np.int64), min(1000, m))
            sec = time.perf_counter() - t0
        secs.append(sec * t.rows / m)
    arr = np.array(secs)
    return {"queries_per_s": len(arr) / arr.sum(), "p50_ms": float(np.percentile(arr, 50)) * 1e3,
            "p99_ms": float(np.percentile(arr, 99)) * 1e3, "cores": threads,
            "sample": f"each table's query on a prefix of at most {sample_rows:,} rows, scaled to its rows"}


def serving_operator(q):
    """The mixed serving stream: Poisson arrivals of queries drawn uniformly
    from the four templates, each over its own resident seeded tables of
    log-uniform size 1M-100M rows, through the plain one-query-at-a-time path
    and through the serving loop (HBM-budget admission, worker streams,
    coalesced small aggregations).  The arrival rate is swept upward in
    multiples of the plain path's capacity; a rate is sustained when the
    completed queries/s keep up with it (>= 95%) and p99 stays within 500 ms,
    and each mode reports its best sustained rate."""
    from qumirdb_b200 import serving
    sizes = serving.log_uniform_sizes(SERVE_TABLES, 1_000_000, 100_000_000, seed=7)
    tables = [serving.Table(serving.TEMPLATES[i % 4], int(n), seed=50 + i).build() for i, n in enumerate(sizes)]
    resident = sum(t.nbytes for t in tables)
    progs = serving.Programs()
    max_sort = max(t.rows for t in tables if t.template == "sort")
    plain = serving.PlainServer(progs, max_sort, keep_results=False)
    # Service time of each query alone (also warms programs, pools, tuner).
    warm = [serving.Query(i, t, 0.0) for i, t in enumerate(tables)]
    plain.run(warm)
    calib = [serving.Query(i, t, 0.0) for i, t in enumerate(tables)]
    st = plain.run(calib)
    service = st["wall_s"] / len(tables)
    budget = SERVE_BUDGET
    out = {"workload": f"{len(tables)} resident tables (log-uniform 1M-100M rows, "
                       f"{int(sizes.sum())} rows, {resident / 1e9:.1f} GB), templates lineitem/join/zipf/sort, "
                       "Poisson arrivals", "plain_service_ms": service * 1e3, "budget_bytes": budget,
           "resident_bytes": resident, "sweeps": {}}
    srv = serving.BatchingServer(progs, budget, resident, workers=SERVE_WORKERS, small_rows=SERVE_COALESCE_ROWS,
                                 max_sort_rows=max_sort, keep_results=False)
    # Warm-up: the autotuner's search for the coalesced aggregation shape,
    # then the workers.
    small = [t for t in tables if t.template == "zipf" and t.rows <= (8 << 20)]
    if small:
        serving.run_agg_batch(progs, small * max(1, (32 << 20) // sum(t.rows for t in small)), keep=False)
    srv.warm(tables)
    srv.run(serving.make_stream(tables, 1.0 / service, 48, seed=99))
    for mode in ("plain", "serving"):
        runs = []
        for mult in (0.3, 0.5, 0.7, 0.85, 1.0, 1.2, 1.5, 2.0, 2.5, 3.0, 4.0):
            rate = mult / service
            count = int(max(48, min(1500, rate * 2.5)))
            stream = serving.make_stream(tables, rate, count, seed=int(mult * 10))
            stats = plain.run(stream) if mode == "plain" else srv.run(stream)
            stats["rate"] = rate
            offered = len(stream) / stream[-1].arrival     # the stream's own arrival rate
            stats["sustained"] = stats["p99_ms"] <= 500 and stats["queries_per_s"] >= 0.95 * offered
            runs.append(stats)
            if not stats["sustained"]:
                break
        ok = [r for r in runs if r["sustained"]] or runs[:1]
        best = max(ok, key=lambda r: r["queries_per_s"])
        out["sweeps"][mode] = runs
        out[mode] = {k: best[k] for k in ("rate", "queries_per_s", "p50_ms", "p99_ms")}
    srv.close()
    out["serving_over_plain_qps"] = out["serving"]["queries_per_s"] / out["plain"]["queries_per_s"]
    best = max((r for r in out["sweeps"]["serving"] if r["sustained"]), key=lambda r: r["queries_per_s"],
               default=out["sweeps"]["serving"][0])
    out["coalesced_queries"] = best.get("coalesced_queries", 0)
    out["batched_launches"] = best.get("batched_launches", 0)
    out["cpu"] = serving_cpu_arm(tables)
    return out


def sort_pass_plan_bytes(n: int) -> tuple[int, int]:
    """Algorithmic bytes of the device sort of (k1 i64 DESC, k2 i32 ASC) over
    n row ids, by the plan it runs: the id scan (row id 8: batch count and
    dense-run marks), extraction (row id 8 + k1 8 + k2 4 read, u32 k2 key 4 +
    u64 k1 key 8 written), the k2 stage's 3 non-constant digit passes (first
    4 + 8 then 2 x 16), the k1 stage's 8 passes (first a gather 4 + 8 + 12,
    then 7 x 24), the final row-id write from the positions and the marks
    (4 + 8; the ids are consecutive rows, so no copy of them is kept and the
    marks stay in L2).  Returns (total per sort, per u64 pass)."""
    per_row = 8 + 32 + (12 + 16 + 16) + (24 + 7 * 24) + 12
    return n * per_row, n * 24


def sort_operator(q, peak):
    from qumirdb_b200 import abi, queries
    n = SORT_ROWS
    batch = 1 << 22
    k1 = np.empty(n, np.int64)
    k2 = np.empty(n, np.int32)
    rowid = np.empty(n, np.int64)
    q.lib().qdb_gen_sort(3, n, k1.ctypes.data, k2.ctypes.data, rowid.ctypes.data)
    sizes = [min(batch, n - b) for b in range(0, n, batch)]
    store, at = [], 0
    for m in sizes:
        store.append(q.DeviceRowSet([k1[at:at + m], k2[at:at + m], rowid[at:at + m]]))
        at += m
    ids = np.concatenate([(np.int64(b) << 32) | np.arange(m, dtype=np.int64) for b, m in enumerate(sizes)])
    pristine = q.DeviceBuffer(ids.nbytes).upload(ids)
    work = q.DeviceBuffer(ids.nbytes)
    del ids
    sorter = q.Sort(q.compile_sort(queries.sort_k1_desc_k2(flags=abi.OUT_DEVICE)), store)
    topper = q.Sort(q.compile_sort(queries.top_k1(flags=abi.OUT_DEVICE)), store)
    import torch
    stream = torch.cuda.ExternalStream(q.lib().qdb_gpu_get_stream())

    def run(fn, steps, warmup):
        times = []
        kern = []
        for i in range(warmup + steps):
            q.lib().qdb_gpu_memcpy(work.ptr, pristine.ptr, work.nbytes)   # in place: restore the input order
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            if i >= warmup:
                q.profile(True)
                q.profile_read()
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            if i >= warmup:
                times.append(a.elapsed_time(b))
                kern.append(q.profile_read())
                q.profile(False)
        return statistics.median(times), kern

    ms, kern = run(lambda: sorter.sort(work), 3, 1)
    passes = [ms_ for ks in kern for name, ms_, _ in ks if name == "sort_pass_u64"]
    alg, per_pass = sort_pass_plan_bytes(n)
    pass_ms = statistics.median(passes) if passes else None
    tk_ms, tk_kern = run(lambda: topper.top_k(work, 1000), 3, 1)
    tk_alg = n * 16   # each row id read once (id scan) and each k1 read once (collect)
    tk_parts = {}                 # per kernel name: the median over steps of its summed time in a step
    for ks in tk_kern:
        step = {}
        for name, ms_, _ in ks:
            step[name] = step.get(name, 0.0) + ms_
        for name, v in step.items():
            tk_parts.setdefault(name, []).append(v)
    tk_parts = {name: statistics.median(v) for name, v in tk_parts.items()}
    collect_ms = tk_parts.get("topk_collect")
    line = {"workload": "ORDER BY k1 DESC, k2 ASC (stable) over 300,000,000 row ids in 72 batches; "
                        "top-N: ORDER BY k1 LIMIT 1000",
            "rows_per_s": n / (ms / 1e3), "ms_per_sort": ms, "algorithmic_bytes": alg,
            "bytes_per_row": alg // n, "sort_gbs": alg / (ms / 1e3) / 1e9,
            "frac_of_measured_hbm": alg / (ms / 1e3) / 1e9 / peak,
            "kernel": "sort_pass_u64", "kernel_ms": pass_ms,
            "kernel_gbs": per_pass / (pass_ms / 1e3) / 1e9 if pass_ms else None,
            "kernel_frac_of_measured_hbm": per_pass / (pass_ms / 1e3) / 1e9 / peak if pass_ms else None,
            "topk_ms": tk_ms, "topk_rows_per_s": n / (tk_ms / 1e3), "topk_algorithmic_bytes": tk_alg,
            "topk_gbs": tk_alg / (tk_ms / 1e3) / 1e9, "topk_kernels_ms": tk_parts,
            # The collect pass reads k1 alone here (every id tile is a dense run: no id reads).
            "topk_collect_gbs": n * 8 / (collect_ms / 1e3) / 1e9 if collect_ms else None,
            "topk_collect_frac_of_measured_hbm": n * 8 / (collect_ms / 1e3) / 1e9 / peak if collect_ms else None,
            "l2": "inputs larger than L2"}
    del store, pristine, work
    return line


def cpu_baseline_sort(sample: int) -> dict:
    from oracle import oracle as O
    k1 = np.empty(sample, np.int64)
    k2 = np.empty(sample, np.int32)
    O.lib().qdb_gen_sort(3, sample, k1.ctypes.data, k2.ctypes.data, None)
    threads = os.cpu_count() or 1
    sec = O.lib().oracle_bench_sort(k1.ctypes.data, k2.ctypes.data, sample, threads, None)
    return {"value": sample / sec, "unit": "rows/s", "cores": threads, "kind": "port",
            "sample": f"{sample:,} rows (of 300M): per-lane LSD + heap k-way merge of the CPU restatement",
            "seconds": sec}


def cpu_baseline_agg(kind: str, sample: int) -> dict:
    """The CPU restatement's threaded aggregate plan (per-lane partial
    tables, then the hash-partitioned final) on all host threads, over the
    lineitem table or a sample of the Zipf stream."""
    from oracle import oracle as O
    from qumirdb_b200 import HostRowSet, queries
    if kind == "lineitem":
        cols = [np.empty(sample, np.int64), np.empty(sample, np.int64), np.empty(sample, np.int64),
                np.empty(sample, np.int64), np.empty(sample, np.uint8), np.empty(sample, np.uint8),
                np.empty(sample, np.int32)]
        O.lib().qdb_gen_lineitem(0, sample, *[c.ctypes.data for c in cols])
        spec = queries.lineitem_agg(int(cols[6].max()) - 90)
        what = f"{sample:,} rows (the whole table)"
    else:
        cols = [np.empty(sample, np.int64), np.empty(sample, np.int64), np.empty(sample, np.float64)]
        O.lib().qdb_gen_zipf(2, sample, ZIPF_DISTINCT, 1.1, *[c.ctypes.data for c in cols])
        spec = queries.zipf_agg(expected_groups=ZIPF_DISTINCT)
        what = f"{sample:,} rows (of 200M) of the same Zipf stream"
    threads = os.cpu_count() or 1
    rs = HostRowSet(cols)
    sec = O.lib().oracle_bench_aggregate(C.byref(spec.struct), rs.ptr, threads, None)
    return {"value": sample / sec, "unit": "rows/s", "cores": threads, "kind": "port",
            "sample": what + ": per-lane partial tables + hash-partitioned final of the CPU restatement",
            "seconds": sec}


def cpu_baseline_join(sample_probe: int, steps: int = 1) -> dict:
    """The CPU restatement's threaded join plan over the bench's own seeded
    inputs (the same generators, linked into the oracle library, so this
    leg loads no device code)."""
    from oracle import oracle as O
    b = [np.empty(BUILD_ROWS, np.int64), np.empty(BUILD_ROWS, np.int64), np.empty(BUILD_ROWS, np.int32)]
    p = [np.empty(sample_probe, np.int64), np.empty(sample_probe, np.int64)]
    O.lib().qdb_gen_join(1, BUILD_ROWS, 0, FK_DOMAIN, *[x.ctypes.data for x in b], None, None)
    tmp = [np.empty(1, np.int64), np.empty(1, np.int64), np.empty(1, np.int32)]
    O.lib().qdb_gen_join(1000, 1, sample_probe, FK_DOMAIN, *[t.ctypes.data for t in tmp], *[x.ctypes.data for x in p])
    threads = os.cpu_count() or 1
    times = []
    s = C.c_int64()
    c = C.c_int64()
    for _ in range(steps):
        t = O.lib().oracle_bench_join_sum(b[0].ctypes.data, b[1].ctypes.data, b[2].ctypes.data, BUILD_ROWS, 20,
                                          p[0].ctypes.data, p[1].ctypes.data, sample_probe, threads, C.byref(s),
                                          C.byref(c))
        times.append(t)
    sec = min(times)
    what = "the whole 120,000,000-row probe" if sample_probe == PROBE_ROWS else \
        f"a probe sample of {sample_probe:,} rows (of 120M)"
    return {"value": (BUILD_ROWS + sample_probe) / sec, "unit": "rows/s", "cores": threads, "kind": "port",
            "sample": f"build 2,000,000 rows + {what}, threaded partitioned row-table plan of the CPU "
                      f"restatement (fastest of {steps} runs)", "seconds": sec, "times": times,
            "result": [s.value, c.value]}


JOIN_CONFIG = {"workload": "equi-join: build 2,000,000 rows (unique keys, attr<20 filter fused), probe "
                           "120,000,000 rows per GPU (fk uniform over 1..2.5M), SUM(payload*value), COUNT(*)",
               "build_rows": BUILD_ROWS, "probe_rows_per_gpu": PROBE_ROWS,
               "l2": "inputs larger than L2 (1.92 GB probe stream per step)"}


def reference_arm(args) -> None:
    """The reference's CPU path for the headline workload: the oracle's
    threaded partitioned row-join plan (the reference engine cannot be built
    here), on all host threads, over the whole 2M x 120M workload with the
    same seeded inputs; one step is one whole query.  Only the oracle
    library is loaded."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    steps = max(1, args.steps)
    cb = cpu_baseline_join(PROBE_ROWS, steps=args.warmup + steps)
    timed_s = cb["times"][args.warmup:]
    sec = statistics.median(timed_s)
    rows = BUILD_ROWS + PROBE_ROWS
    value = rows / sec
    line = {"metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded generators with the workload's shapes and distributions)",
            "impl": "reference",
            "config": dict(JOIN_CONFIG, parallelism=f"shard{world}", result=cb["result"]),
            "cpu_baseline": {"value": value, "unit": "rows/s", "cores": cb["cores"], "kind": "port",
                             "sample": cb["sample"].replace(f"(fastest of {args.warmup + steps} runs)",
                                                            f"(median of {steps} timed runs)")},
            "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profile_case(name: str, rows: int) -> None:
    """One workload run twice (a warm-up, then the launch a profiler
    captures) at `rows` rows; prints "done <name>".  The workloads are the
    bench's own generators at a size that a detailed capture finishes on."""
    import qumirdb_b200 as q
    from qumirdb_b200 import queries
    q.init(0)
    if name == "lineitem":
        n = rows or LINEITEM_ROWS
        cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64),
                np.empty(n, np.uint8), np.empty(n, np.uint8), np.empty(n, np.int32)]
        q.lib().qdb_gen_lineitem(0, n, *[c.ctypes.data for c in cols])
        prog = q.compile_aggregate(queries.lineitem_agg(int(cols[6].max()) - 90))
        drs = q.DeviceRowSet(cols)
        for _ in range(2):
            a = q.Aggregate(prog)
            a.add(drs)
            q.release(a.finish())
    elif name == "lineitem_batched":
        n = rows or LINEITEM_ROWS
        cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64),
                np.empty(n, np.uint8), np.empty(n, np.uint8), np.empty(n, np.int32)]
        q.lib().qdb_gen_lineitem(0, n, *[c.ctypes.data for c in cols])
        prog = q.compile_aggregate(queries.lineitem_agg(int(cols[6].max()) - 90))
        bounds = np.linspace(0, n, 65).astype(np.int64)
        rowsets = [q.DeviceRowSet([c[lo:hi] for c in cols]) for lo, hi in zip(bounds[:-1], bounds[1:])]
        for _ in range(2):
            b = q.AggregateBatch(prog, 64)
            b.add(rowsets)
            b.finish().release()
    elif name == "join":
        n = rows or PROBE_ROWS
        b = [np.empty(BUILD_ROWS, np.int64), np.empty(BUILD_ROWS, np.int64), np.empty(BUILD_ROWS, np.int32)]
        p = [np.empty(n, np.int64), np.empty(n, np.int64)]
        q.lib().qdb_gen_join(1, BUILD_ROWS, n, FK_DOMAIN, *[x.ctypes.data for x in b + p])
        j, a = queries.join_sum(20)
        prog = q.compile_join_aggregate(j, a)
        db, dp = q.DeviceRowSet(b), q.DeviceRowSet(p)
        for _ in range(2):
            J = q.RowJoin(prog)
            J.append(db)
            J.build()
            agg = q.Aggregate(prog)
            J.probe_aggregate(agg, dp)
            q.release(agg.finish())
    elif name == "join_batched":
        w = JoinWorkload(q, 0)
        for _ in range(2):
            join_batched_operator(q, 1.0, w, steps=1)
    elif name == "zipf":
        n = rows or ZIPF_ROWS
        cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.float64)]
        q.lib().qdb_gen_zipf(2, n, max(1, n // 10), 1.1, *[c.ctypes.data for c in cols])
        prog = q.compile_aggregate(queries.zipf_agg(expected_groups=max(1, n // 10)))
        drs = q.DeviceRowSet(cols)
        for _ in range(2):
            a = q.Aggregate(prog)
            a.add(drs)
            q.release(a.finish())
    elif name == "zipf_batched":
        from qumirdb_b200 import abi
        sizes = zipf_partition_sizes()
        if rows:
            sizes = np.maximum(1, sizes * rows // int(sizes.sum()))
        n = int(sizes.sum())
        cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.float64)]
        q.lib().qdb_gen_zipf(6, n, ZIPF_DISTINCT, 1.1, *[c.ctypes.data for c in cols])
        prog = q.compile_aggregate(queries.zipf_agg(flags=abi.OUT_DEVICE))
        drs = q.DeviceRowSet(cols)
        bounds = np.concatenate([[0], np.cumsum(sizes)])
        parts = q.RowSetPointers([q.SliceRowSet(drs, int(lo), int(hi)) for lo, hi in zip(bounds[:-1], bounds[1:])])
        for _ in range(2):
            b = q.AggregateBatch(prog, len(parts))
            b.add(parts)
            b.finish().release()
    elif name == "sort":
        n = rows or SORT_ROWS
        k1 = np.empty(n, np.int64)
        k2 = np.empty(n, np.int32)
        rid = np.arange(n, dtype=np.int64)
        q.lib().qdb_gen_sort(3, n, k1.ctypes.data, k2.ctypes.data, None)
        s = q.Sort(q.compile_sort(queries.sort_k1_desc_k2()), [q.DeviceRowSet([k1, k2, rid])])
        d = q.DeviceBuffer(rid.nbytes)
        for _ in range(2):
            d.upload(rid)
            s.sort(d)
    elif name == "topk":
        n = rows or SORT_ROWS
        k1 = np.empty(n, np.int64)
        k2 = np.empty(n, np.int32)
        rid = np.arange(n, dtype=np.int64)
        q.lib().qdb_gen_sort(3, n, k1.ctypes.data, k2.ctypes.data, None)
        s = q.Sort(q.compile_sort(queries.top_k1()), [q.DeviceRowSet([k1, k2, rid])])
        d = q.DeviceBuffer(rid.nbytes)
        for _ in range(2):
            d.upload(rid)
            s.top_k(d, 1000)
    q.synchronize()
    print("done", name, flush=True)


def compact_operators(ops: dict) -> dict:
    """The per-operator figures that go on the one JSON line: rows/s, time,
    the dominant kernel's time and fraction of the measured HBM peak, its
    ncu traffic over the algorithmic bytes, and the CPU baseline; the
    serving stream's best sustained points (the sweeps stay in --detail)."""
    traffic = load_traffic()

    def r(x, nd=4):
        return None if x is None else float(f"{x:.{nd}g}")

    out = {}
    for name in ("lineitem", "lineitem_batched", "zipf", "zipf_batched", "join_batched", "sort"):
        o = ops.get(name)
        if not o:
            continue
        c = {"rows_per_s": r(o.get("rows_per_s")), "ms": r(o.get("ms_per_query", o.get("ms_per_sort"))),
             "kernel": o.get("kernel"), "kernel_ms": r(o.get("kernel_ms")),
             "frac_of_measured_hbm": r(o.get("kernel_frac_of_measured_hbm", o.get("frac_of_measured_hbm")), 3)}
        ratio = traffic.get(f"{o.get('kernel')}_traffic_over_algorithmic")
        if ratio is not None:
            c["traffic_over_algorithmic"] = ratio
        if name == "sort":
            c.update({"sort_frac_of_measured_hbm": r(o.get("frac_of_measured_hbm"), 3),
                      "bytes_per_row": o.get("bytes_per_row"), "topk_ms": r(o.get("topk_ms")),
                      "topk_rows_per_s": r(o.get("topk_rows_per_s"))})
        if name in ("zipf", "zipf_batched"):
            c["groups"] = o.get("groups")
        if "finalize_ms" in o:
            c["finalize_ms"] = r(o.get("finalize_ms"))
        if "build_batch_ms" in o:
            c["build_batch_ms"] = r(o.get("build_batch_ms"))
            c["result"] = o.get("result")
        cb = o.get("cpu_baseline")
        if cb:
            c["cpu_baseline"] = {"rows_per_s": r(cb["value"]), "cores": cb["cores"], "kind": cb["kind"]}
        out[name] = c
    sv = ops.get("serving")
    if sv:
        pick = lambda d: {k: r(d[k]) for k in ("queries_per_s", "p50_ms", "p99_ms")}  # noqa: E731
        out["serving"] = {"plain": pick(sv["plain"]), "serving": pick(sv["serving"]),
                          "serving_over_plain_qps": r(sv["serving_over_plain_qps"], 3)}
        for k in ("cpu", "coalesced_queries", "batched_launches"):
            if k in sv:
                out["serving"][k] = sv[k] if not isinstance(sv[k], dict) else pick(sv[k])
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--no-operators", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-case", choices=["join", "join_batched", "sort", "topk", "lineitem",
                                               "lineitem_batched", "zipf", "zipf_batched"],
                    help="run one workload twice at --rows rows (for profiler captures) and exit")
    ap.add_argument("--rows", type=int, default=0)
    ap.add_argument("--detail", help="write every operator's full figures (serving sweeps included) to this file")
    ap.add_argument("--only", choices=["lineitem", "lineitem_batched", "zipf", "zipf_batched", "sort", "serving"],
                    help="run one operator's measurement and print its JSON")
    args = ap.parse_args()
    if args.only:
        import qumirdb_b200 as q
        q.init(0)
        peak, _ = peaks()
        fn = {"lineitem": lambda: lineitem_operator(q, peak),
              "lineitem_batched": lambda: lineitem_batched_operator(q, peak), "zipf": lambda: zipf_operator(q, peak),
              "zipf_batched": lambda: zipf_batched_operator(q, peak), "sort": lambda: sort_operator(q, peak),
              "serving": lambda: serving_operator(q)}[args.only]
        print(json.dumps({args.only: fn()}), flush=True)
        return
    if args.profile_case:
        profile_case(args.profile_case, args.rows)
        return
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        reference_arm(args)
        return

    import torch
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    import qumirdb_b200 as q
    q.init(local)
    peak, peak_kind = peaks()

    w = JoinWorkload(q, rank)

    def query():
        s, c = w.step(resident=True)
        if dist is not None:
            return combine_partials(dist, s, c)
        return s, c

    sampler = ClockSampler(local)
    sampler.start()
    ms, results, launches, kernels = timed(q, query, args.steps, args.warmup, dist=dist, profile=True)
    clocks = sampler.stop()
    kms, kunits = kernel_avg(kernels, "join_agg_probe", args.steps)
    alg_bytes = PROBE_ROWS * 16
    achieved = alg_bytes / (kms / 1e3) / 1e9 if kms else None
    traffic = load_traffic().get("join_agg_probe_bytes_per_probe_row")

    # The same query with the fused probe kept on the hashed bucket table
    # (QDB_JOIN_DIRECT=0): the build keys here are unique over a dense range,
    # so the measured step above probes the direct-address index instead.
    hashed = None
    if rank == 0 and world == 1:
        os.environ["QDB_JOIN_DIRECT"] = "0"
        try:
            hms, hres, _, hk = timed(q, lambda: w.step(resident=True), 5, 3, profile=True)
            hkms, _ = kernel_avg(hk, "join_agg_probe", 5)
            hashed = {"ms_per_step": hms, "kernel_ms": hkms,
                      "frac_of_measured_hbm": alg_bytes / (hkms / 1e3) / 1e9 / peak if hkms else None,
                      "same_result": list(hres[-1]) == list(results[-1])}
        finally:
            del os.environ["QDB_JOIN_DIRECT"]

    # End to end through the C ABI from pinned host buffers.
    def query_e2e():
        s, c = w.step(resident=False)
        if dist is not None:
            return combine_partials(dist, s, c)
        return s, c

    ms_e2e, _, _, _ = timed(q, query_e2e, max(1, min(args.steps, 3)), 1, dist=dist)

    line = {
        "metric": METRIC,
        "value": world * w.rows / (ms / 1e3),
        "unit": "rows/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int64",
        "data": "synthetic (seeded generators with the workload's shapes and distributions)",
        "config": dict(JOIN_CONFIG, parallelism=f"shard{world}", result=list(results[-1])),
        "roofline": {"bound": "hbm", "kernel": "join_agg_probe", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak if achieved else None,
                     "traffic": traffic * PROBE_ROWS if traffic else None,
                     "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms": kms},
        "e2e": {"value": world * w.rows / (ms_e2e / 1e3), "unit": "rows/s", "h2d_bytes_per_step": w.h2d,
                "d2h_bytes_per_step": 16},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if hashed:
        line["join_hashed_probe"] = {k: (round(v, 4) if isinstance(v, float) else v) for k, v in hashed.items()}
    if rank == 0 and world == 1 and not args.no_operators:
        ops = {}
        try:
            ops = {"lineitem": lineitem_operator(q, peak), "lineitem_batched": lineitem_batched_operator(q, peak),
                   "zipf": zipf_operator(q, peak),
                   "zipf_batched": zipf_batched_operator(q, peak), "join_batched": join_batched_operator(q, peak, w),
                   "sort": sort_operator(q, peak),
                   "serving": serving_operator(q)}
            if not args.no_cpu_baseline:
                ops["sort"]["cpu_baseline"] = {
                    k: v for k, v in cpu_baseline_sort(20_000_000).items() if k != "seconds"}
                ops["lineitem"]["cpu_baseline"] = {
                    k: v for k, v in cpu_baseline_agg("lineitem", LINEITEM_ROWS).items() if k != "seconds"}
                ops["zipf"]["cpu_baseline"] = {
                    k: v for k, v in cpu_baseline_agg("zipf", 20_000_000).items() if k != "seconds"}
        except Exception as e:  # reported, never hidden
            line["operators_error"] = repr(e)
        if args.detail:
            Path(args.detail).parent.mkdir(parents=True, exist_ok=True)
            Path(args.detail).write_text(json.dumps(ops, indent=1))
        line["operators"] = compact_operators(ops)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline_join(PROBE_ROWS)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
