#!/usr/bin/env python
"""Benchmark of the B200 gzip compression path (one JSON line on rank 0).

Workload (default): the 64 MiB synthetic log stream (seed 1) as a one-file
ustar archive (512 + 64 MiB + 1,024 bytes), cut into 2 MiB chunks (32 full +
a 1,536-byte tail), each chunk compressed into 128 KiB gzip members -- the
reference's `--backend gpu` behaviour on its single-stream throughput config.

* ``value``: input GB/s with inputs resident in HBM (device ABI call
  gpz_compress_device per step; L2 flushed between steps, steps timed with
  CUDA events on the launching stream, max over ranks).
* ``e2e``: the same metric through the public host API gpz_compress_batch
  (host buffers in, host gzip streams out; copies inside the timed region).
* ``roofline``: the dominant kernel's algorithmic bytes per launch
  ((1 + ratio) x input bytes) over its CUDA-event duration, against the
  measured HBM copy bandwidth; ``traffic`` from the committed ncu capture.
* ``cpu_baseline``: the CPU port of the same path (oracle, all host threads)
  on a bounded sample; ``gpzip_cpu_equiv``: zlib 1.3 level 5 per 2 MiB chunk
  on all host threads (the reference's gpzip-cpu path).

``--impl reference`` times the CPU port instead (rank 0 only).
Multi-GPU (torchrun): every rank compresses its own copy of the workload
(members are independent; no collective on the data path): weak scaling.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from gpzip_b200 import workloads as W  # noqa: E402

METRIC = "input GB/s/B200 at bit-exact tokens"
MEMBER = 128 * 1024
CHUNK = 2 << 20
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="logs", choices=["logs", "text", "binary", "uneven"])
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="seconds per arrival rate of the serving measurement (0: skip)")
    ap.add_argument("--serve-rates", default="1000,10000,50000")
    ap.add_argument("--serve-only", action="store_true", help="run only the serving measurement")
    ap.add_argument("--cpu-sample-mib", type=int, default=0,
                    help="MiB of the workload the CPU port times per step (0: all of it)")
    ap.add_argument("--no-configs", action="store_true", help="skip the per-config (text, binary) lines")
    ap.add_argument("--codec", default="gzip", choices=["gzip", "zstd"],
                    help="codec of the device-resident measurement (zstd: for profiling its kernels)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baselines (quick runs)")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-file batched vs plain measurement")
    ap.add_argument("--device-only", action="store_true",
                    help="only the device-resident steps (no e2e, no CPU baselines): for profiling")
    return ap.parse_args()


def workload(name: str):
    if name == "logs":
        data = W.config_logs_tar()
        desc = "logs-64MiB-ustar (seed 1): 32x2MiB chunks + 1536 B tail"
    elif name == "text":
        data = W.config_text()
        desc = "text-8MiB (seed 0): 4x2MiB chunks"
    else:
        data = W.config_binary()
        desc = "binary-272MiB (seed 2): 136x2MiB chunks"
    return data, desc


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


class Clocks:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"gpz_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names[1:], parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def chunk_parity(outs, workload: str):
    """(chunks whose gzip stream equals the oracle's, chunks): the oracle's
    per-chunk SHA-256 digests are committed with the tests
    (tests/golden/config_digests.json)."""
    import hashlib
    want = json.load(open(os.path.join(ROOT, "tests", "golden", "config_digests.json")))["sets"][workload]
    got = [hashlib.sha256(bytes(x)).hexdigest() for x in outs]
    return sum(int(a == b) for a, b in zip(got, want["chunk_sha256"])), want["chunks"]


def inflate_all(gz: bytes) -> bytes:
    import zlib
    out, rest = b"", gz
    while rest:
        d = zlib.decompressobj(31)
        out += d.decompress(rest)
        rest = d.unused_data
    return out


def cpu_port_rate(data: np.ndarray, sample_mib: int, threads: int):
    """The CPU port of the reference GPU path (oracle) on the workload, or on
    its first sample_mib MiB when sample_mib > 0."""
    from oracle import oracle as O
    sample = data[: min(data.size, sample_mib << 20)] if sample_mib > 0 else data
    spans = W.chunk_spans(sample.size, CHUNK)
    t0 = time.perf_counter()
    outs = [O.gzip_chunk(sample[o:o + n], MEMBER, threads=threads) for o, n in spans]
    dt = time.perf_counter() - t0
    return sample.size / dt / 1e9, sum(len(x) for x in outs) / sample.size, sample.size


def cpu_zlib_rate(data: np.ndarray, threads: int):
    from oracle import oracle as O
    t0 = time.perf_counter()
    gz = O.cpu_gzip_chunks(data, CHUNK, 5, threads=threads)
    dt = time.perf_counter() - t0
    return data.size / dt / 1e9, len(gz) / data.size


def uneven_items(scale: float = 1.0):
    """The 1,000-file mix (seed 3) cut into 2 MiB chunks + short remainders."""
    files = W.uneven_files(1000, seed=3, scale=scale)
    items = []
    for _, _, data in files:
        for o, n in W.chunk_spans(data.size, CHUNK):
            items.append(np.ascontiguousarray(data[o:o + n]))
    return items


def run_uneven(ctx, args, stream):
    """Batched persistent path vs the plain one-launch-per-chunk path, host API."""
    import torch
    items = uneven_items()
    total = sum(x.size for x in items)
    # one caller-owned output buffer, reused by both paths
    buf = np.zeros(ctx.batch_bound(items), dtype=np.uint8)
    for _ in range(max(1, args.warmup)):
        ctx.compress_batch(items, out=buf)
    times = []
    ctx.host_times(reset=True)
    for _ in range(max(1, args.steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        outs = ctx.compress_batch(items, out=buf)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    batched = total / (min(times) / 1e3) / 1e9
    host = {k: round(v / max(1, args.steps), 3) for k, v in ctx.host_times(reset=True).items()}
    outs = [bytes(o) for o in outs]  # the buffer is reused below
    pbuf = np.zeros_like(buf)
    ctx.compress_batch_plain(items[:8], out=pbuf)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    plain_outs = ctx.compress_batch_plain(items, out=pbuf)
    e1.record(stream)
    e1.synchronize()
    plain = total / (e0.elapsed_time(e1) / 1e3) / 1e9
    same = all(a == b for a, b in zip(outs, plain_outs))
    eq, tot = chunk_parity(outs, "uneven")
    return {"files": 1000, "chunks": len(items), "bytes": int(total), "batched_gbs": round(batched, 4),
            "parity": f"ok ({eq}/{tot} chunks equal the oracle's)" if eq == tot else f"FAILED ({eq}/{tot} chunks)",
            "plain_gbs": round(plain, 4), "batched_over_plain": round(batched / plain, 3),
            "batched_ms": round(min(times), 3), "outputs_identical": same, "host_ms_per_step": host,
            "ratio": round(sum(len(o) for o in outs) / total, 5)}


def inflate_rates(ctx, gz: bytes, want_len: int, steps: int = 5):
    """Decompression of the workload's gzip stream (the `gpzip x` path):
    gpz_inflate from page-locked host buffers, copies included (e2e), the
    device time of its kernels, and the gpzip-cpu equivalent, zlib inflate of
    the members on all host threads as parallel_decompress does with flate2."""
    import time as _t
    from concurrent.futures import ThreadPoolExecutor
    import zlib as _z

    import torch
    src = torch.empty(len(gz), dtype=torch.uint8, pin_memory=True).numpy()
    src[:] = np.frombuffer(gz, dtype=np.uint8)
    dst = torch.empty(max(want_len, 1), dtype=torch.uint8, pin_memory=True).numpy()
    for _ in range(2):
        ctx.inflate(src, out=dst)
    ts, dev = [], []
    for _ in range(steps):
        t0 = _t.perf_counter()
        n = len(ctx.inflate(src, out=dst))
        ts.append(_t.perf_counter() - t0)
        dev.append(ctx.inflate_device_ms())
    assert n == want_len
    hdr = bytes([0x1F, 0x8B, 0x08, 0, 0, 0, 0, 0, 0, 0xFF])
    starts, p = [], 0
    while True:
        q = gz.find(hdr, p)
        if q < 0:
            break
        starts.append(q)
        p = q + 10
    members = [gz[a:b] for a, b in zip(starts, starts[1:] + [len(gz)])]
    threads = os.cpu_count() or 1
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda m: _z.decompress(m, 31), members))
        t0 = _t.perf_counter()
        out_n = sum(len(x) for x in ex.map(lambda m: _z.decompress(m, 31), members))
        tc = _t.perf_counter() - t0
    assert out_n == want_len
    dms = statistics.median(dev)
    return {"value": round(want_len / min(ts) / 1e9, 4), "unit": "GB/s of output",
            "members": len(members), "in_bytes": len(gz), "out_bytes": want_len,
            "device_ms": round(dms, 4), "device_gbs": round(want_len / (dms / 1e3) / 1e9, 4),
            "cpu_zlib": {"value": round(want_len / tc / 1e9, 4), "threads": threads,
                         "what": "zlib inflate per member on a thread pool (parallel_decompress equivalent)"},
            "what": "gpz_inflate: page-locked host buffers, copies inside the timed region, wall clock"}


def writer_rate(ctx, data, rounds: int = 3, warm: int = 3):
    """The streaming writer (gpz_writer_*, ParallelChunkedWriter) as pack_tar
    drives it: the workload written in 1 MiB pieces, cut into 2 MiB chunks,
    16 in flight; input GB/s, best of `rounds` after `warm` untimed rounds
    (the passes a stream forms vary in size, so the first streams still meet
    size buckets whose launch graphs are not captured yet)."""
    import time as _t
    from gpzip_b200 import native

    class Count:
        n = 0

        def write(self, b):
            Count.n += len(b)

    view = np.ascontiguousarray(data)
    best = None
    for r in range(rounds + warm):
        Count.n = 0
        t0 = _t.perf_counter()
        with native.Writer(Count(), ctx=ctx, chunk_size=2 << 20, max_in_flight=16, sink_view=True) as w:
            for i in range(0, len(view), 1 << 20):
                w.write(view[i:i + (1 << 20)])
        t = _t.perf_counter() - t0
        if r >= warm:
            best = t if best is None else min(best, t)
    return {"value": round(len(view) / best / 1e9, 4), "unit": "GB/s", "out_bytes": Count.n,
            "what": "gpz_writer: 1 MiB writes, 2 MiB chunks, 16 in flight, wall clock; the sink takes each "
                    "member run as a view of the library's buffer"}


def chunk_fn_rate(ctx, chunks, threads: int = 16, rounds: int = 3):
    """The ChunkFn drop-in as ParallelChunkedWriter drives it: `threads`
    workers (max_in_flight for the gpu backend, gpu.rs:160-166) each call
    gpz_compress_chunk on their share of the chunks, concurrently; input GB/s
    over the whole set, best of `rounds` after one warm-up round."""
    import threading
    import time as _t
    L = ctx.L
    outs = [np.empty(ctx.bound(len(x)), dtype=np.uint8) for x in chunks]
    lens = [ctypes.c_size_t() for _ in chunks]
    failed = []

    def one_round():
        go = threading.Barrier(threads + 1)

        def worker(k):
            go.wait()
            for i in range(k, len(chunks), threads):
                a = chunks[i]
                rc = L.gpz_compress_chunk(ctx._h, a.ctypes.data, a.size, 5, outs[i].ctypes.data, outs[i].size,
                                          ctypes.byref(lens[i]))
                if rc:
                    failed.append(rc)

        th = [threading.Thread(target=worker, args=(k,)) for k in range(threads)]
        for t in th:
            t.start()
        go.wait()
        t0 = _t.perf_counter()
        for t in th:
            t.join()
        return _t.perf_counter() - t0

    one_round()
    ctx.host_times(reset=True)
    best = min(one_round() for _ in range(rounds))
    passes = ctx.host_times()["passes"] / rounds
    nbytes = sum(int(x.size) for x in chunks)
    if failed:
        return {"failed": sorted(set(failed))}
    return {"value": round(nbytes / best / 1e9, 4), "unit": "GB/s", "threads": threads, "calls": len(chunks),
            "passes_per_round": round(passes, 2), "out_bytes": int(sum(x.value for x in lens)),
            "what": "gpz_compress_chunk from concurrent caller threads (the ChunkFn drop-in), wall clock"}


def run_serving(device: int, seconds: float, rates, warm_seconds: float = 0.3):
    """Open-loop Poisson arrivals (seed 4), sizes log-uniform 4 KiB-16 MiB,
    content sliced from the three generators; continuous batching engine.
    Each rate first runs warm_seconds of the same arrival process (seed 5:
    graphs captured, pipelines primed), then the statistics are reset and
    the measured run starts."""
    import ctypes
    import threading
    import time as _t

    from gpzip_b200 import native
    pools = [W.text(48 << 20, seed=40), W.logs(48 << 20, seed=41), W.binary(48 << 20, seed=42)]
    results = []

    def drive(ctx, rate, secs, seed):
        """Submits one arrival process open loop while a poller collects the
        results; returns (requests, sizes, rejected, offered seconds, wall)."""
        L = ctx.L
        t, sizes, kinds, offs = W.serving_arrivals(rate, secs, seed=seed)
        sizes = np.minimum(sizes, (48 << 20) - 1)
        tickets = []
        lock = threading.Lock()
        done = threading.Event()

        def poller():
            buf = np.empty(ctx.bound(16 << 20), dtype=np.uint8)
            i = 0
            while True:
                with lock:
                    have = len(tickets)
                if i >= have:
                    if done.is_set():
                        with lock:
                            if i >= len(tickets):
                                return
                    _t.sleep(0.0005)
                    continue
                o = native.Out(buf.ctypes.data, buf.size, 0, 0)
                while L.gpz_poll(ctx._h, tickets[i], ctypes.byref(o), 1000) == native.GPZ_E_PENDING:
                    pass
                i += 1

        th = threading.Thread(target=poller)
        th.start()
        rejected = 0
        d = native.Desc()
        tk = ctypes.c_uint64()
        t0 = _t.perf_counter()
        for i in range(t.size):
            while _t.perf_counter() - t0 < t[i]:
                pass
            pool = pools[int(kinds[i])]
            n = int(sizes[i])
            off = int(offs[i] * (pool.size - n))
            d.in_, d.n, d.level = pool.ctypes.data + off, n, 5
            if L.gpz_submit_ref(ctx._h, ctypes.byref(d), ctypes.byref(tk)) == native.GPZ_OK:
                with lock:
                    tickets.append(tk.value)
            else:
                rejected += 1
        offered = _t.perf_counter() - t0
        done.set()
        th.join()
        return t.size, sizes, rejected, offered, _t.perf_counter() - t0

    for rate in rates:
        ctx = native.Context(device=device, pool_bytes=40 << 30)
        drive(ctx, rate, warm_seconds, seed=5)
        ctx.serve_reset_stats()
        ctx.host_times(reset=True)
        nreq, sizes, rejected, offered_s, wall = drive(ctx, rate, seconds, seed=4)
        st = ctx.serve_stats()
        host = {k: round(v, 1) for k, v in ctx.host_times().items()}
        lanes = [{k: (round(v, 3) if isinstance(v, float) else v) for k, v in ctx.lane_stats(i).items()}
                 for i in range(2)]
        small = int(np.sum(sizes <= (1 << 20)))
        results.append({
            "rate_per_s": rate, "seconds": seconds, "requests": int(nreq), "requests_le_1MiB": small,
            "completed": st["completed"], "rejected": rejected,
            "rejected_frac": round(rejected / max(1, nreq), 4),
            "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3), "p999_ms": round(st["p999_ms"], 3),
            "p50_le_1MiB_ms": round(st["p50_small_ms"], 3), "p99_le_1MiB_ms": round(st["p99_small_ms"], 3),
            "p999_le_1MiB_ms": round(st["p999_small_ms"], 3),
            "offered_gbs": round(float(np.sum(sizes)) / seconds / 1e9, 3),
            "throughput_gbs": round(st["bytes_in"] / wall / 1e9, 3), "batches": st["batches"],
            "submit_lag_s": round(offered_s - seconds, 3), "host_ms_total": host, "lanes": lanes, "wall_s": round(wall, 3)})
        ctx.close()
    return results


def gzip_check(outs, data, workload_name):
    """Every member inflates back to its chunk; every chunk equals the
    oracle's committed digest."""
    gz_all = b"".join(bytes(x) for x in outs)
    ok = inflate_all(gz_all) == data.tobytes()
    same, total = chunk_parity(outs, workload_name)
    return (f"ok ({same}/{total} chunks equal the oracle's; every member inflates)" if ok and same == total
            else f"FAILED (inflate={ok}, chunks equal to the oracle's: {same}/{total})")


def zstd_check(outs, data, workload_name):
    """Every chunk's frame equals the oracle's restatement (oracle/zstd_frame.c,
    on all host threads), and libzstd decodes the stream back to the input."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O
    spans = W.chunk_spans(data.size, CHUNK)
    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        want = list(ex.map(lambda on: O.zstd_chunk(data[on[0]:on[0] + on[1]], MEMBER), spans))
    same = sum(int(bytes(a) == b) for a, b in zip(outs, want))
    try:
        ok = O.zstd_decompress(b"".join(bytes(x) for x in outs), data.size) == data.tobytes()
    except ValueError:
        ok = False
    return (f"ok ({same}/{len(spans)} frames equal the oracle's; libzstd decodes the stream)"
            if ok and same == len(spans) else f"FAILED (libzstd={ok}, frames equal: {same}/{len(spans)})")


def zstd_measure(data, workload_name, desc, stream, flush, local, barrier):
    """The chunk-parallel zstd codec (GPZ_CODEC_ZSTD) on the workload:
    device-resident rate with its stage times, end to end through
    gpz_compress_batch, ratio, parity; beside it the gpzip-cpu zstd path,
    libzstd level 3 (the reference's level 5 mapping, compress.rs:91-99) per
    2 MiB chunk on all host threads."""
    import time as _t
    from concurrent.futures import ThreadPoolExecutor

    from gpzip_b200 import native
    from oracle import oracle as O
    zc = native.Context(device=local, member_bytes=MEMBER, flags=native.GPZ_FLAG_STAGE_TIMING,
                        codec=native.GPZ_CODEC_ZSTD)
    d = device_measure(zc, data, workload_name, 5, 3, stream, flush, local, 0, barrier, check=zstd_check)
    zc.close()
    ze = native.Context(device=local, member_bytes=MEMBER, codec=native.GPZ_CODEC_ZSTD)
    e = e2e_measure(ze, data, workload_name, 3, 2, stream, local, 0, 1, barrier, None, check=zstd_check)
    e.pop("_gz", None)
    ze.close()
    spans = W.chunk_spans(data.size, CHUNK)
    threads = os.cpu_count() or 1
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda on: O.zstd_compress(data[on[0]:on[0] + min(on[1], 1 << 16)], 3), spans[:threads]))
        t0 = _t.perf_counter()
        cpu_out = sum(len(x) for x in ex.map(lambda on: O.zstd_compress(data[on[0]:on[0] + on[1]], 3), spans))
        tc = _t.perf_counter() - t0
    names = native.STAGE_NAMES_ZSTD
    return {"workload": desc, "value": round(data.size * 5 / (d["total_ms"] / 1e3) / 1e9, 4), "unit": "GB/s",
            "ms_per_step": round(d["total_ms"] / 5, 4), "ratio": round(d["ratio"], 5), "parity": d["parity"],
            "stage_ms": {n: round(float(x), 4) for n, x in zip(names, d["stage_ms"])}, "e2e": e,
            "cpu_zstd": {"value": round(data.size / tc / 1e9, 4), "unit": "GB/s", "threads": threads,
                         "ratio": round(cpu_out / data.size, 5),
                         "what": "libzstd level 3, one frame per 2 MiB chunk, all host threads"}}


def device_measure(ctx, data, workload_name, steps, warmup, stream, flush, local, rank, barrier, clocks=False,
                   check=gzip_check):
    """gpz_compress_device on the workload resident in HBM: one checked
    pass, `warmup` untimed passes, then `steps` passes timed with CUDA
    events on the launching stream, L2 flushed before each."""
    import torch
    from gpzip_b200 import native
    spans = W.chunk_spans(data.size, CHUNK)
    offs, lens, pos = [], [], 0
    for o, n in spans:
        offs.append(pos)
        lens.append(n)
        pos += (n + 15) // 16 * 16
    packed = np.zeros(pos + 64, dtype=np.uint8)
    for (o, n), po in zip(spans, offs):
        packed[po:po + n] = data[o:o + n]
    d_in = torch.from_numpy(packed).to(f"cuda:{local}")
    del packed
    out_cap = ctx.bound(data.size) + 64 * len(spans)
    d_out = torch.empty(out_cap, dtype=torch.uint8, device=f"cuda:{local}")

    def step():
        return ctx.compress_device(d_in.data_ptr(), offs, lens, d_out.data_ptr(), out_cap, stream.cuda_stream)

    oo = step()
    parity = "unchecked"
    if rank == 0:
        host = d_out[:oo[-1]].cpu().numpy().copy()
        ctx.frame_host(host)
        gz_all = host.tobytes()
        parity = check([gz_all[a:b] for a, b in zip(oo[:-1], oo[1:])], data, workload_name)
        del host, gz_all
    ratio = oo[-1] / data.size
    for _ in range(warmup):
        step()
    barrier()
    clk = None
    if clocks:
        sampler = Clocks(local)
        sampler.start()
    times, stages = [], np.zeros(len(native.STAGE_NAMES))
    for _ in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        stages += np.array(ctx.stage_times())
    barrier()
    if clocks:
        clk = sampler.stop()
    out = {"total_ms": float(sum(times)), "stage_ms": stages / steps, "ratio": ratio, "parity": parity,
           "launches": ctx.last_launches(), "clocks": clk}
    del d_in, d_out
    torch.cuda.empty_cache()
    return out


def e2e_measure(ectx, data, workload_name, steps, warmup, stream, local, rank, world, barrier, dist,
                check=None):
    """gpz_compress_batch with host buffers: the step's input in page-locked
    host memory (the library uploads it directly), the caller's output
    buffer reused across calls; copies inside the timed region."""
    import torch
    spans = W.chunk_spans(data.size, CHUNK)
    host_in = torch.empty(data.size, dtype=torch.uint8, pin_memory=True).numpy()
    host_in[:] = data
    host_chunks = [host_in[o:o + n] for o, n in spans]
    buf = np.zeros(ectx.batch_bound(host_chunks), dtype=np.uint8)
    for _ in range(warmup):
        ectx.compress_batch(host_chunks, out=buf)
    barrier()
    e_times = []
    out_bytes = 0
    outs = None
    ectx.host_times(reset=True)
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        outs = ectx.compress_batch(host_chunks, out=buf)
        e1.record(stream)
        e1.synchronize()
        e_times.append(e0.elapsed_time(e1))
        out_bytes = sum(len(x) for x in outs)
    et = torch.tensor([sum(e_times)], device=f"cuda:{local}", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    value = data.size * len(e_times) * world / (float(et.item()) / 1e3) / 1e9
    host = {k: round(v / max(1, len(e_times)), 3) for k, v in ectx.host_times().items()}
    par = None
    if rank == 0 and check is not None:
        par = check(outs, data, workload_name)
    elif rank == 0:
        same, total = chunk_parity(outs, workload_name)
        par = f"ok ({same}/{total} chunks)" if same == total else f"FAILED ({same}/{total} chunks)"
    gz = b"".join(bytes(x) for x in outs)
    return {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": int(data.size),
            "d2h_bytes_per_step": int(out_bytes), "api": "gpz_compress_batch (host buffers; inputs page-locked)",
            "host_ms_per_step": host, "parity": par, "_gz": gz}


def roofline_of(kernel: str, kernel_ms: float, in_bytes: int, ratio: float, clk) -> dict:
    """The dominant stage against the measured HBM peak: algorithmic bytes
    (1 + ratio per input byte) over its event-timed duration; its committed
    ncu DRAM traffic and warp instructions scaled to this input; and the
    share of the SMs' issue slots those instructions fill at the sampled
    clock (148 SMs x 4 schedulers, one warp instruction per cycle each)."""
    peak, peak_kind = measured_peaks()
    algo = in_bytes * (1.0 + ratio)
    achieved = algo / (kernel_ms / 1e3) / 1e9
    tr = committed_traffic().get(kernel)
    traffic = round(tr["dram_bytes_per_input_byte"] * in_bytes) if tr else None
    r = {"bound": "hbm", "kernel": kernel, "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
         "frac": round(achieved / peak, 5), "traffic": traffic, "peak_kind": peak_kind,
         "algorithmic_bytes_per_launch": int(algo)}
    if tr and tr.get("warp_inst_per_input_byte"):
        mhz = (clk or {}).get("sm_mhz") or 1965.0
        inst = tr["warp_inst_per_input_byte"] * in_bytes
        r["issue_frac"] = round(inst / (148 * 4 * mhz * 1e6 * kernel_ms / 1e3), 4)
        r["limiter"] = tr.get("limiter")
    return r


def hybrid_rate(ctx, data, rounds: int = 2, warmup_chunks: int = 4, warm: int = 3):
    """The `--backend auto` writer (gpz_hybrid in gpz_writer_open_fn): CPU
    workers = host threads, 16 GPU permits on the device context, 2 MiB
    chunks, 1 MiB writes; input GB/s, best of `rounds` after `warm` untimed
    rounds, and the chunks each device took.  The first `warmup_chunks` chunks go to zlib on the host
    (4, as the reference's scheduler does); the in-order write waits for
    them, so on a 64 MiB input they bound the rate."""
    import time as _t
    from gpzip_b200 import native

    class Count:
        n = 0

        def write(self, b):
            Count.n += len(b)

    view = np.ascontiguousarray(data)
    cpu_workers = os.cpu_count() or 1
    best, split = None, None
    for r in range(rounds + warm):
        Count.n = 0
        with native.Hybrid(ctx=ctx, gpu_permits=16, warmup_chunks=warmup_chunks) as h:
            t0 = _t.perf_counter()
            with native.Writer(Count(), hybrid=h, chunk_size=CHUNK, max_in_flight=cpu_workers + 16,
                               sink_view=True) as w:
                for i in range(0, len(view), 1 << 20):
                    w.write(view[i:i + (1 << 20)])
            t = _t.perf_counter() - t0
            if r >= warm and (best is None or t < best):
                best, split = t, h.stats()
    return {"value": round(len(view) / best / 1e9, 4), "unit": "GB/s", "out_bytes": Count.n,
            "cpu_workers": cpu_workers, "gpu_permits": 16, "warmup_chunks": warmup_chunks,
            "cpu_chunks": split[0], "gpu_chunks": split[1],
            "ratio": round(Count.n / len(view), 5),
            "what": "gpz_hybrid chunk function in the streaming writer: 1 MiB writes, 2 MiB chunks, wall clock"}


def config_of(data, desc: str, world: int) -> dict:
    """The bench line's config, the same for both arms."""
    spans = W.chunk_spans(data.size, CHUNK)
    return {"workload": desc, "bytes": int(data.size), "chunk_bytes": CHUNK, "member_bytes": MEMBER,
            "members": sum(max(1, -(-n // MEMBER)) for _, n in spans), "level": 5,
            "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}"}


def run_reference(args, rank: int):
    """--impl reference: the CPU port of the path on all host threads, on the
    whole workload every step (or its first --cpu-sample-mib MiB)."""
    if rank != 0:
        return
    data, desc = workload(args.workload)
    threads = os.cpu_count() or 1
    sample_mib = args.cpu_sample_mib
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_port_rate(data, 2, threads)
    rates = []
    ratio = None
    for _ in range(args.steps):
        r, ratio, nbytes = cpu_port_rate(data, sample_mib, threads)
        rates.append(r)
    value = statistics.median(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(nbytes / (value * 1e9) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generators standing in for the reference's corpora)",
        "config": config_of(data, desc, args.gpus),
        "cpu_baseline": {"value": round(value, 5), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": (f"first {sample_mib} MiB" if sample_mib > 0 else "the whole workload")
                         + " per step, members on all host threads"},
        "e2e": {"value": round(value, 5), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "ratio": round(ratio, 5),
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from gpzip_b200 import native

    torch.cuda.set_device(local)
    if args.serve_only:
        if rank == 0:
            rates = [int(x) for x in args.serve_rates.split(",") if x]
            print(json.dumps({"serving": run_serving(local, args.serve_seconds, rates)}), flush=True)
        return
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    if args.workload == "uneven":
        uctx = native.Context(device=local, member_bytes=MEMBER)
        res = run_uneven(uctx, args, torch.cuda.current_stream())
        uctx.close()
        if rank == 0:
            line = {"metric": METRIC, "value": res["batched_gbs"], "unit": "GB/s", "n_gpus": world,
                    "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["batched_ms"],
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
                    "data": "synthetic (seeded generators standing in for the reference's corpora)",
                    "config": {"workload": "uneven-1000-files (seed 3): 2 MiB chunks + remainders, host API",
                               "member_bytes": MEMBER},
                    "uneven": res}
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    data, desc = workload(args.workload)
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")
    zstd_main = args.codec == "zstd"
    ctx = native.Context(device=local, member_bytes=MEMBER, flags=native.GPZ_FLAG_STAGE_TIMING,
                         codec=native.GPZ_CODEC_ZSTD if zstd_main else native.GPZ_CODEC_GZIP)
    dev = device_measure(ctx, data, args.workload, args.steps, args.warmup, stream, flush, local, rank, barrier,
                         clocks=True, check=zstd_check if zstd_main else gzip_check)
    ratio, parity, clk = dev["ratio"], dev["parity"], dev["clocks"]
    launches = dev["launches"] * args.steps
    t = torch.tensor([dev["total_ms"]], device=f"cuda:{local}", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    value = data.size * args.steps * world / (max_ms / 1e3) / 1e9

    # end to end through the public host API (host buffers, copies inside),
    # on a context with the production settings (graphs, autotuned shapes)
    ectx = native.Context(device=local, member_bytes=MEMBER)
    e2e = None if args.device_only else e2e_measure(ectx, data, args.workload, max(2, args.steps // 2),
                                                    max(args.warmup, 2), stream, local, rank, world, barrier, dist)
    spans = W.chunk_spans(data.size, CHUNK)
    inflate = None
    writer = None if args.device_only else writer_rate(ectx, data)
    hybrid = None
    if not (args.device_only or world > 1):
        hybrid = hybrid_rate(ectx, data)
        hybrid["no_warmup"] = hybrid_rate(ectx, data, warmup_chunks=0)
    if not args.device_only:
        inflate = inflate_rates(ectx, e2e.pop("_gz"), data.size)
    # pageable chunks, as a writer hands them over
    chunk_fn = None if args.device_only else chunk_fn_rate(ectx, [np.ascontiguousarray(data[o:o + n]) for o, n in spans])

    stage_ms = dev["stage_ms"]
    names = native.STAGE_NAMES_ZSTD if zstd_main else native.STAGE_NAMES
    dom = int(np.argmax(stage_ms))
    roofline = roofline_of(names[dom], stage_ms[dom], data.size, ratio, clk)

    cpu = None
    zl = None
    # the CPU baselines, serving and the uneven-file comparison are
    # single-GPU measurements: taken at N=1 only
    if rank == 0 and world == 1 and not (args.no_cpu or args.device_only):
        threads = os.cpu_count() or 1
        r, cr, nb = cpu_port_rate(data, args.cpu_sample_mib, threads)
        cpu = {"value": round(r, 5), "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": (f"first {args.cpu_sample_mib} MiB of the workload" if args.cpu_sample_mib > 0
                          else "the whole workload") + f" (CPU port of the reference GPU path, members on "
                                                       f"{threads} host threads)", "ratio": round(cr, 5)}
        zr, zratio = cpu_zlib_rate(data, threads)
        zl = {"value": round(zr, 4), "unit": "GB/s", "cores": threads, "ratio": round(zratio, 5),
              "what": "gpzip-cpu equivalent: zlib 1.3 level 5, one gzip member per 2 MiB chunk"}

    zstd = None
    if rank == 0 and world == 1 and not (args.device_only or args.no_configs):
        zstd = zstd_measure(data, args.workload, desc, stream, flush, local, barrier)

    # the other single-stream configs: 8 MiB text (plain-path config) and
    # 272 MiB mixed binary, device-resident and end to end, every chunk
    # compared with the oracle's committed digests
    per_config = None
    if rank == 0 and world == 1 and not (args.device_only or args.no_configs):
        per_config = {}
        for name in ("text", "binary"):
            if name == args.workload:
                continue
            cdata, cdesc = workload(name)
            cd = device_measure(ctx, cdata, name, 5, 3, stream, flush, local, rank, barrier)
            ce = e2e_measure(ectx, cdata, name, 3, 2, stream, local, rank, 1, barrier, None)
            ce.pop("_gz", None)
            cst = cd["stage_ms"]
            cdom = int(np.argmax(cst))
            per_config[name] = {
                "workload": cdesc, "bytes": int(cdata.size),
                "value": round(cdata.size * 5 / (cd["total_ms"] / 1e3) / 1e9, 4),
                "unit": "GB/s", "ms_per_step": round(cd["total_ms"] / 5, 4), "ratio": round(cd["ratio"], 5),
                "parity": cd["parity"], "e2e": ce,
                "stage_ms": {n: round(float(x), 4) for n, x in zip(names, cst)},
                "roofline": roofline_of(names[cdom], cst[cdom], cdata.size, cd["ratio"], clk)}
            del cdata

    serving = None
    if rank == 0 and world == 1 and args.serve_seconds > 0 and not args.device_only:
        rates = [int(x) for x in args.serve_rates.split(",") if x]
        serving = run_serving(local, args.serve_seconds, rates)

    # the 1,000-file uneven mix: batched persistent path vs the plain
    # one-launch-per-chunk path through the host API
    uneven = None
    if rank == 0 and world == 1 and not (args.device_only or args.no_uneven):
        uctx = native.Context(device=local, member_bytes=MEMBER)
        uneven = run_uneven(uctx, argparse.Namespace(steps=2, warmup=1), torch.cuda.current_stream())
        uctx.close()

    if world > 1:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generators standing in for the reference's corpora)",
            "config": config_of(data, desc, world),
            "roofline": roofline,
            "stage_ms": {n: round(float(x), 4) for n, x in zip(names, stage_ms)},
            "cpu_baseline": cpu,
            "gpzip_cpu_equiv": zl,
            "e2e": e2e,
            "chunk_fn": chunk_fn,
            "writer": writer,
            "hybrid": hybrid,
            "inflate": inflate,
            "gpu_launches": int(launches),
            "clocks": clk,
            "ratio": round(ratio, 5),
            "parity": parity,
            "per_config": per_config,
            "zstd": zstd,
            "serving": serving,
            "uneven": uneven,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    ectx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
