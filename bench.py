#!/usr/bin/env python
"""SA+ISA+LCP build throughput on B200 (Gsym/s), one JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload plain3g|plain100m|plain4m|batched|served]

The default workload is the human-scale plain build: 3.1 Gbp, 25 contigs,
Low-memory profile (64-bit construction, split40 SA storage, byte-coded LCP,
no resident ISA).  The batched-over-one-at-a-time ratio of the uneven
collection is a second invocation: ``--workload batched --count 1024``.

A step is one complete build of the workload: seed sort, doubling rounds,
ISA, LCP and packing.  ``value`` uses a device-resident text and device
output planes and the device time of each build (CUDA events recorded by the
library on its own stream, first to last); L2 is flushed (256 MiB write)
between steps.  ``e2e`` is the same build through the C ABI with pinned host
buffers, host<->device copies included.  With N > 1 (torchrun) every rank
builds its own replica (no collective: the path does not shard) and the
slowest rank's time counts.
"""
from __future__ import annotations

import argparse
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

METRIC = "SA+LCP build Gsym/s on 1 B200 (batched vs plain, bit-exact); % of HBM peak"
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="plain3g",
                    choices=["plain100m", "plain4m", "plain3g", "batched", "served"])
    ap.add_argument("--count", type=int, default=256,
                    help="references in the batched workload (1,024 in the full collection)")
    ap.add_argument("--batch-symbols", type=float, default=1.2e9,
                    help="HBM admission budget per batch launch (symbols)")
    ap.add_argument("--rate", type=float, default=200.0,
                    help="served workload: Poisson arrival rate (requests/s)")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="shrink the workload (profiling captures only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-workers", type=int, default=2,
                    help="collections: contexts building sub-batches side by side (e2e)")
    ap.add_argument("--e2e-batch-symbols", type=float, default=3e8,
                    help="collections: symbols per sub-batch (e2e)")
    ap.add_argument("--tune", action="append", default=[],
                    help="library tuning knob key=value (sufgpu_set_tuning)")
    return ap.parse_args()


def peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# Workloads
# ---------------------------------------------------------------------------
def workload(name: str, scale: float = 1.0, count: int = 256):
    from sufkit_b200 import synth
    if name == "plain4m":
        ref = synth.plain_4mbp(scale)
        desc = ("plain 4 Mbp build: 4 contigs (1.5/1.2/0.8/0.5 Mbp), uniform ACGT, "
                "0.1% N runs; Fast profile SA+ISA+raw LCP32, 32-bit storage")
        return [ref.logical_text()], desc
    if name == "plain3g":
        # SUFGPU_SYNTH_CACHE=<dir> keeps the generated text between runs of
        # one session (the generator is seeded: the file is the same text).
        cache = os.environ.get("SUFGPU_SYNTH_CACHE")
        desc = ("human-scale 3.1 Gbp plain build: 25 contigs (50-250 Mbp), GC 41%, 50% "
                "interspersed repeats, 1% segmental duplications, 150 Mbp of N in runs of "
                "10 kbp-3 Mbp; Low-memory profile: 64-bit construction, split40 SA storage, "
                "byte-coded LCP (32-bit anchors), no resident ISA")
        if cache:
            path = Path(cache) / f"human_scale_3gbp_{scale}.npy"
            if path.exists():
                return [np.load(path)], desc
            text = synth.human_scale_3gbp(scale).logical_text()
            path.parent.mkdir(parents=True, exist_ok=True)
            np.save(path, text)
            return [text], desc
        ref = synth.human_scale_3gbp(scale)
        desc = ("human-scale 3.1 Gbp plain build: 25 contigs (50-250 Mbp), GC 41%, 50% "
                "interspersed repeats, 1% segmental duplications, 150 Mbp of N in runs of "
                "10 kbp-3 Mbp; Low-memory profile: 64-bit construction, split40 SA storage, "
                "byte-coded LCP (32-bit anchors), no resident ISA")
        return [ref.logical_text()], desc
    if name == "batched":
        # Per-reference random streams (synth.uneven_reference), generated in
        # parallel: the collection tests/test_gpu_fullsize.py checks against
        # divsufsort64 reference by reference.
        texts = synth.uneven_texts(1024 if count <= 1024 else count, scale,
                                   indices=range(count))
        desc = (f"batched uneven collection: first {count} of 1,024 bacterial-like references "
                "(log-normal sizes, median 4 Mbp, clipped 0.5-12 Mbp, GC 30-70%, 1-8 contigs); "
                "SA + raw LCP32 per reference, 32-bit, HBM-admitted batch launches, "
                "compared with the plain build one reference at a time")
        return texts, desc
    ref = synth.repeat_rich_100mbp(scale)
    desc = ("repeat-rich 100 Mbp plain build: 24 contigs, GC 41%, 25% interspersed "
            "repeats (500 families, 5-15% divergence), 3% tandem repeats, 0.5% N runs; "
            "Fast profile SA+ISA+raw LCP32, 32-bit construction and storage")
    return [ref.logical_text()], desc


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, sm_max, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                sm_max.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(sm_max) if sm_max else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# Algorithmic-byte model of one build
# ---------------------------------------------------------------------------
def model_bytes(n: int, a_k: list[int], lcp_nonzero: int, w_sa: int, w_isa: int,
                lcp_kind: str, w_lcp: int = 4, anchors: int = 0, w_anchor: int = 4) -> int:
    """Algorithmic bytes B of one build of n symbols:

        B = n(1 + 2(8+W) + W)            seed: text read, one (key, idx) sort pass, rank write
          + sum_k 8 W A_k                doubling rounds over still-unsorted suffixes
          + n(W + w_isa)                 ISA emit
          + 6nW + 2C                     PHI scatter, PLCP read/write, LCP gather; C compares
          + n(W + w_sa)                  SA pack to the stored width
          + n w_lcp | n + 2 w_anchor #anchors   raw or byte-coded LCP

    with W = 4 if n-1 fits 32 bits else 8, A_k = #{suffixes i : m(i) >= 21 *
    2^(k-1)}, m(i) = max(LCP[ISA[i]], LCP[ISA[i]+1]) (LCP[n] = 0) and C =
    sum_p (PLCP[p] - max(PLCP[p-1] - 1, 0) + 1).  The last sum telescopes: for a
    sentinel-terminated text (PLCP of the last position is 0) C = n + #{rows r
    : LCP[r] >= 1}.  A_k and C depend only on the text."""
    W = 4 if n - 1 <= 0xFFFFFFFF else 8
    b = n * (1 + 2 * (8 + W) + W)
    b += sum(8 * W * a for a in a_k)
    b += n * (W + w_isa)
    b += n * 6 * W + 2 * (n + lcp_nonzero)
    b += n * (W + w_sa)
    b += n * w_lcp if lcp_kind == "raw" else n + 2 * w_anchor * anchors
    return int(b)


def text_statistics(lcp: np.ndarray, seed: int = 21) -> tuple[list[int], int]:
    """A_k (k = 1..R) and #{r : LCP[r] >= 1} from a row-order LCP (host)."""
    l = np.asarray(lcp).astype(np.int64)
    m = np.maximum(l, np.append(l[1:], 0))
    a_k, k = [], 1
    while True:
        a = int(np.count_nonzero(m >= seed * (1 << (k - 1))))
        if a == 0:
            break
        a_k.append(a)
        k += 1
    return a_k, int(np.count_nonzero(l >= 1))


def text_statistics_device(d_lcp, torch, seed: int = 21, chunk: int = 1 << 28):
    """text_statistics over a device-resident uint32 LCP plane (an int32
    tensor holding the bits), in chunks, with the counts reduced on the
    device: a multi-Gsym build needs no host copy of its LCP."""
    n = int(d_lcp.numel())
    counts = {}
    nonzero = 0
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        cur = d_lcp[s:e].to(torch.int64) & 0xFFFFFFFF
        nxt = torch.zeros_like(cur)
        nxt[: e - s - 1] = cur[1:]
        if e < n:
            nxt[e - s - 1] = int(d_lcp[e].item()) & 0xFFFFFFFF
        m = torch.maximum(cur, nxt)
        nonzero += int((cur >= 1).sum().item())
        k = 1
        while True:
            a = int((m >= seed * (1 << (k - 1))).sum().item())
            if a == 0:
                break
            counts[k] = counts.get(k, 0) + a
            k += 1
        del cur, nxt, m
    a_k = [counts[k] for k in sorted(counts)]
    return a_k, nonzero


def load_traffic(kernel: str):
    """DRAM bytes per algorithmic byte of `kernel`, from the committed ncu
    summary (profiles/traffic.json, measured on a 31 Mbp capture and scaled
    to a full launch by its algorithmic bytes), or None."""
    path = ROOT / "profiles" / "traffic.json"
    if not path.exists():
        return None
    entry = json.loads(path.read_text()).get(kernel)
    return entry["dram_per_algorithmic_byte"] if entry else None


# ---------------------------------------------------------------------------
# Reference arm and CPU baseline (the reference's own CPU build path)
# ---------------------------------------------------------------------------
def host_info() -> dict:
    """CPU model, logical CPUs, host RAM and the compiler that built the
    reference's CPU code (recorded beside every CPU timing)."""
    info = {"cpu": None, "nproc": os.cpu_count(), "ram_gb": None, "compiler": None}
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                info["cpu"] = line.split(":", 1)[1].strip()
                break
        for line in Path("/proc/meminfo").read_text().splitlines():
            if line.startswith("MemTotal"):
                info["ram_gb"] = round(int(line.split()[1]) / 1048576, 1)
                break
    except OSError:
        pass
    try:
        out = subprocess.run([os.environ.get("CXX", "g++"), "--version"], capture_output=True,
                             text=True, timeout=10).stdout
        info["compiler"] = (out.splitlines() or [None])[0]
    except (OSError, subprocess.TimeoutExpired):
        pass
    return info


def cpu_reference_step(text: np.ndarray, threads: int) -> float:
    import oracle
    t0 = time.perf_counter()
    oracle.ref_adapter(text, 64, threads)
    return time.perf_counter() - t0


def cpu_sample(texts: list[np.ndarray], symbols: int) -> np.ndarray:
    """A bounded prefix of the workload, re-terminated with the sentinel."""
    body = texts[0][: max(1, symbols - 1)]
    return np.concatenate([body[body != 0], np.zeros(1, np.uint8)])


def run_reference(args, texts, desc):
    import oracle
    if oracle.ref() is None:
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libsufref.so was not built"}))
        return
    threads = os.cpu_count() or 1
    sample = cpu_sample(texts, 20_000_000)
    for _ in range(args.warmup):
        cpu_reference_step(sample, threads)
    times = [cpu_reference_step(sample, threads) for _ in range(args.steps)]
    sec = sum(times) / len(times)
    value = sample.size / sec / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gsym/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": desc, "symbols_per_step": int(sample.size)},
        "cpu_baseline": {"value": value, "unit": "Gsym/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"first {sample.size} symbols of the workload text; "
                                   "libdivsufsort64 + ISA + Kasai LCP through "
                                   "detail::BuildDivsufsort64 (threads=%d)" % threads,
                         "host": host_info()},
        "e2e": {"value": value, "unit": "Gsym/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def run_served(args):
    """Workload 5 shape: Poisson arrivals into the served engine; p50/p99
    latency and aggregate Gsym/s against sequential plain builds."""
    import threading as th
    import sufkit_b200 as sg
    from sufkit_b200 import synth
    count = args.count
    scale = args.scale
    reqs = list(synth.served_stream(requests=count, scale=scale, rate_hz=args.rate))
    texts = [r.reference.logical_text() for r in reqs]
    arrivals = [r.arrival_s for r in reqs]
    total = sum(int(t.size) for t in texts)
    enc = sg.LcpEncoding.BYTE32
    # Pinned host text and output planes for every request (both modes use
    # the same buffers; allocation is outside the timed regions).
    pinned = []
    for t in texts:
        pt = sg.pinned_array(int(t.size))
        pt[:] = t
        planes = {"sa_low": sg.pinned_array(int(t.size), np.uint32),
                  "lcp": sg.pinned_array(int(t.size), np.uint8)}
        pinned.append((pt, planes))
    ctx = sg.Context(0)

    def one(pt, planes):
        return ctx.build_device(pt.ctypes.data, int(pt.size),
                                {k: v.ctypes.data for k, v in planes.items()},
                                sa_bits=32, isa_bits=0, lcp=enc)

    for pt, planes in pinned[:4]:
        one(pt, planes)  # warm the library and the device
    # Sequential plain builds, one request at a time.
    t0 = time.perf_counter()
    for pt, planes in pinned:
        one(pt, planes)
    seq = time.perf_counter() - t0
    ctx.close()
    def serve(delays):
        """One pass of the stream through a fresh server; `delays` are the
        submission times (seconds from the start).  Returns the server stats
        and the host wall time."""
        server = sg.Server(0, capacity_symbols=int(args.batch_symbols), max_instances=1024)
        tickets = [None] * count

        def submitter():
            start = time.perf_counter()
            for i, (a, (pt, planes)) in enumerate(zip(delays, pinned)):
                delay = a - (time.perf_counter() - start)
                if delay > 0:
                    time.sleep(delay)
                tickets[i] = server.submit(pt, 32, 0, enc, planes=planes)

        th_sub = th.Thread(target=submitter)
        t0 = time.perf_counter()
        th_sub.start()
        th_sub.join()
        for k in tickets:
            server.wait(k)
        wall = time.perf_counter() - t0
        st = server.stats()
        server.close()
        return st, wall

    # Poisson arrivals at the requested rate: latency (p50/p99) and the
    # throughput the stream offers.  Then the same requests all queued at
    # once: the served engine's capacity, against the sequential builds.
    st, wall = serve(arrivals)
    sat, sat_wall = serve([0.0] * count)
    line = {
        "metric": METRIC, "value": total / sat["span_seconds"] / 1e9, "unit": "Gsym/s",
        "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": sat["span_seconds"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": f"served stream: {count} requests, sizes log-normal 10 kbp-50 Mbp "
                               f"and 20% strain collections (50 copies at 0.1% SNP + 0.01% "
                               f"indel), all scaled x{scale}; SA + byte-coded LCP, 32-bit; host "
                               "buffers.  value: all requests queued at once (capacity); "
                               f"latency: Poisson arrivals at {args.rate} req/s",
                   "symbols": total, "p50_s": st["p50_seconds"], "p99_s": st["p99_seconds"],
                   "poisson_Gsym_s": total / st["span_seconds"] / 1e9,
                   "offered_Gsym_s": total / max(arrivals[-1], 1e-9) / 1e9,
                   "saturated_p50_s": sat["p50_seconds"], "saturated_p99_s": sat["p99_seconds"],
                   "sequential_Gsym_s": total / seq / 1e9,
                   "served_over_sequential": seq / sat["span_seconds"],
                   "iterations": sat["iterations"], "max_inflight": sat["max_inflight"],
                   "poisson_max_inflight": st["max_inflight"], "wall_s": wall + sat_wall},
    }
    print(json.dumps(line))


def main():
    args = parse_args()
    if args.workload == "served":
        run_served(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    sharded = args.workload == "batched" and world > 1 and args.impl == "ours"
    all_symbols = None
    if sharded:
        # N GPUs build a collection of N x count references, each its
        # bin-packed share (no collective on the data path).
        from sufkit_b200 import shard
        _, texts = shard.collection_share(args.count * world, world, rank, args.scale)
        desc = (f"batched uneven collection sharded over {world} GPUs: {args.count * world} "
                "bacterial-like references (log-normal sizes, median 4 Mbp, clipped 0.5-12 Mbp, "
                "GC 30-70%, 1-8 contigs), each GPU its bin-packed share of about "
                f"{args.count}; SA + raw LCP32 per reference, 32-bit")
    else:
        texts, desc = workload(args.workload, args.scale, args.count)
    if args.scale != 1.0:
        desc += f" (scaled x{args.scale})"

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, texts, desc)
        return

    import torch
    import sufkit_b200 as sg

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = sg.Context(local)
    for item in args.tune:
        key, value = item.split("=", 1)
        ctx.set_tuning(key, int(value))
    lcp_enc = sg.LcpEncoding.BYTE32 if args.workload == "plain3g" else sg.LcpEncoding.RAW32
    isa_bits = 0 if args.workload in ("batched", "plain3g") else 32
    sa_bits = 40 if args.workload == "plain3g" else 32

    # Device-resident inputs and outputs.
    n_total = sum(int(t.size) for t in texts)
    if sharded:
        all_symbols = int(shard.sum_over_ranks(n_total, dist, dev))
    d_texts = [torch.from_numpy(t).to(dev) for t in texts]
    lcp_dtype = torch.uint8 if lcp_enc == sg.LcpEncoding.BYTE32 else torch.int32
    d_out = [{"sa_low": torch.empty(t.size, dtype=torch.int32, device=dev),
              "sa_high": torch.empty(t.size, dtype=torch.uint8, device=dev) if sa_bits == 40 else None,
              "isa_low": torch.empty(t.size, dtype=torch.int32, device=dev) if isa_bits else None,
              "lcp": torch.empty(t.size, dtype=lcp_dtype, device=dev)} for t in texts]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def ptrs(o):
        return {k: (v.data_ptr() if v is not None else None) for k, v in o.items()}

    # Batches admitted by their symbol footprint (each launch holds at most
    # --batch-symbols symbols on the device).
    batches, cur, cur_n = [], [], 0
    for j, t in enumerate(texts):
        if cur and cur_n + t.size > args.batch_symbols:
            batches.append(cur)
            cur, cur_n = [], 0
        cur.append(j)
        cur_n += int(t.size)
    if cur:
        batches.append(cur)

    def device_step():
        if len(texts) == 1:
            return ctx.build_device(d_texts[0].data_ptr(), int(texts[0].size), ptrs(d_out[0]),
                                    sa_bits=sa_bits, isa_bits=isa_bits, lcp=lcp_enc)
        total = {"device_seconds": 0.0, "kernel_launches": 0}
        for b in batches:
            st = ctx.build_batch_device([(d_texts[j].data_ptr(), int(texts[j].size)) for j in b],
                                        [ptrs(d_out[j]) for j in b],
                                        sa_bits=32, isa_bits=isa_bits, lcp=lcp_enc)
            total["device_seconds"] += st["device_seconds"]
            total["kernel_launches"] += st["kernel_launches"]
        return total

    def one_at_a_time():
        seconds = 0.0
        for j, t in enumerate(texts):
            st = ctx.build_device(d_texts[j].data_ptr(), int(t.size), ptrs(d_out[j]),
                                  sa_bits=32, isa_bits=isa_bits, lcp=lcp_enc)
            seconds += st["device_seconds"]
        return seconds

    for _ in range(args.warmup):
        flush.fill_(1)
        torch.cuda.synchronize()
        device_step()

    # Timed region: K builds, L2 flushed between them (the per-kernel
    # profile is taken in separate builds afterwards: with it on, the library
    # drives rounds from the host instead of replaying captured graphs).
    clocks = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    device_seconds = 0.0
    launches = 0
    last_anchors = None
    wall0 = time.perf_counter()
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        torch.cuda.synchronize()
        st = device_step()
        device_seconds += st["device_seconds"]
        launches += st["kernel_launches"]
        last_anchors = st.get("anchors")
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    clock_info = clocks.stop()
    if dist is not None:
        dist.barrier()
    # Per-kernel CUDA-event profile of the same builds (same L2 flushing).
    prof_steps = max(3, args.steps // 2)
    ctx.set_profiling(True)
    for k in range(prof_steps):
        flush.fill_(k & 0xff)
        torch.cuda.synchronize()
        device_step()
    torch.cuda.synchronize()
    profile = ctx.profile()
    ctx.set_profiling(False)
    single = None
    if len(texts) > 1:
        one_at_a_time()  # warm
        flush.fill_(3)
        torch.cuda.synchronize()
        sec = one_at_a_time()
        single = {"one_at_a_time_Gsym_s": n_total / sec / 1e9,
                  "batched_over_one_at_a_time": (sec / (device_seconds / args.steps)),
                  "batches": len(batches), "references": len(texts)}

    from sufkit_b200 import shard
    step_seconds = shard.max_over_ranks(device_seconds / args.steps, dist, dev)
    # Replicas: every rank builds the whole workload; sharded: the ranks
    # together build the collection once.
    job_symbols = all_symbols if sharded else world * n_total
    value = job_symbols / step_seconds / 1e9

    # End to end through the C ABI with pinned host buffers.
    e2e = None
    if not args.no_e2e:
        pinned_text = [sg.pinned_array(int(t.size)) for t in texts]
        for src, dst in zip(texts, pinned_text):
            dst[:] = src
        host_out = []
        keep = []
        d2h = 0
        for t in texts:
            planes = {}
            layout = (("sa_low", np.uint32, True), ("sa_high", np.uint8, sa_bits == 40),
                      ("isa_low", np.uint32, bool(isa_bits)),
                      ("lcp", np.uint8 if lcp_enc == sg.LcpEncoding.BYTE32 else np.uint32, True))
            for key, dtype, on in layout:
                if not on:
                    continue
                arr = sg.pinned_array(int(t.size), dtype)
                keep.append(arr)
                planes[key] = arr.ctypes.data
                # Below 2^32 symbols the high planes of split coordinates are
                # all zero: the library fills them on the host, no copy.
                if not (key.endswith("_high") and len(texts) == 1 and t.size <= 0xFFFFFFFF):
                    d2h += arr.nbytes
            host_out.append(planes)
        def step():
            return e2e_step(ctx, pinned_text, host_out, isa_bits, lcp_enc, sa_bits,
                            args.e2e_batch_symbols, args.e2e_workers)
        for _ in range(2):
            step()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
        e2e_sec = shard.max_over_ranks((time.perf_counter() - t0) / args.steps, dist, dev)
        e2e = {"value": job_symbols / e2e_sec / 1e9, "unit": "Gsym/s",
               "h2d_bytes_per_step": n_total, "d2h_bytes_per_step": d2h,
               "ms_per_step": e2e_sec * 1e3}
        if len(texts) > 1:
            # Where the last step's sub-batches spent their time (host clock):
            # waiting for the compute gate, holding it, and copying after it.
            trace = ctx.collection_trace()
            e2e["collection"] = {
                "workers": args.e2e_workers, "batch_symbols": args.e2e_batch_symbols,
                "sub_batches": len(trace),
                "gate_wait_s": sum(t["gate_in"] - t["start"] for t in trace),
                "gate_held_s": sum(t["gate_out"] - t["gate_in"] for t in trace),
                "after_gate_s": sum(t["end"] - t["gate_out"] for t in trace),
                "span_s": max((t["end"] for t in trace), default=0.0)}

    # Roofline of the dominant kernel and of the whole build.
    peak, peak_kind = peaks()
    top = max(profile, key=lambda k: k["seconds"])
    achieved = top["bytes"] / top["seconds"] / 1e9 if top["seconds"] > 0 else 0.0
    traffic_ratio = load_traffic(top["kernel"])
    roofline = {"bound": "hbm", "kernel": top["kernel"], "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "launches_per_step": top["launches"] / prof_steps,
                "share_of_kernel_time": top["seconds"] / sum(k["seconds"] for k in profile),
                "traffic": (traffic_ratio * top["bytes"] / top["launches"])
                if traffic_ratio else None}
    kernels = sorted(({"kernel": k["kernel"], "ms_per_step": k["seconds"] * 1e3 / prof_steps,
                       "launches_per_step": k["launches"] / prof_steps,
                       "GBps": (k["bytes"] / k["seconds"] / 1e9) if k["seconds"] else None}
                      for k in profile), key=lambda k: -k["ms_per_step"])

    # Whole-build roofline: the algorithmic bytes of every build in a step
    # (A_k and C from each text's exact row LCP, reduced on the device) over
    # the step's device time.  A byte-coded build has no raw LCP plane, so one
    # extra build of the same text with raw LCP32 supplies it (the values
    # depend only on the text); the timed buffers are freed first.
    whole = None
    w_sa = {32: 4, 40: 5, 48: 6, 64: 8}[sa_bits]
    kind = "raw" if lcp_enc == sg.LcpEncoding.RAW32 else "byte"
    anchors_total = int(last_anchors) if last_anchors is not None else 0
    total_bytes = 0
    if kind == "raw":
        for j, t in enumerate(texts):
            a_k, nz = text_statistics_device(d_out[j]["lcp"], torch)
            total_bytes += model_bytes(int(t.size), a_k, nz, w_sa, isa_bits // 8, "raw")
    else:
        n0 = int(texts[0].size)
        d_out.clear()
        flush = None
        torch.cuda.empty_cache()
        d_sa = torch.empty(n0, dtype=torch.int32, device=dev)
        d_lcp = torch.empty(n0, dtype=torch.int32, device=dev)
        ctx.build_device(d_texts[0].data_ptr(), n0, {"sa_low": d_sa.data_ptr(),
                                                     "lcp": d_lcp.data_ptr()},
                         sa_bits=32, isa_bits=0, lcp=sg.LcpEncoding.RAW32)
        del d_sa
        ctx.close()  # the build arena is not needed any more
        torch.cuda.empty_cache()
        a_k, nz = text_statistics_device(d_lcp, torch)
        del d_lcp
        total_bytes = model_bytes(n0, a_k, nz, w_sa, isa_bits // 8, "byte",
                                  anchors=anchors_total)
    whole = {"algorithmic_bytes": total_bytes,
             "achieved_GBps": total_bytes / step_seconds / 1e9,
             "peak_GBps": peak, "frac": total_bytes / step_seconds / 1e9 / peak,
             "peak_source": peak_kind,
             "A_k": a_k if len(texts) == 1 else None,
             "anchors": anchors_total if kind == "byte" else None}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref() is not None:
            sample = cpu_sample(texts, 50_000_000)
            sec = cpu_reference_step(sample, 1)
            cpu = {"value": sample.size / sec / 1e9, "unit": "Gsym/s", "cores": 1,
                   "kind": "reference",
                   "sample": f"first {sample.size} symbols of the workload text, "
                             "libdivsufsort64 + Kasai LCP via detail::BuildDivsufsort64, "
                             "1 thread (divsufsort is serial)",
                   "host": host_info()}
            # The second CPU baseline: CaPS-SA as sufkit vendors it, all host
            # threads, SA + its construction LCP, same sample.
            threads = os.cpu_count() or 1
            width = 32 if sample.size <= 0xFFFFFFFF else 64
            _, _, caps_sec = oracle.ref_caps(sample, threads=threads, width=width)
            cpu["caps_sa"] = {"value": sample.size / caps_sec / 1e9, "unit": "Gsym/s",
                              "cores": threads, "kind": "reference",
                              "sample": f"the same {sample.size} symbols, detail::BuildCaps"
                                        f"{width} with LCP, {threads} threads"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Gsym/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_seconds * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32", "data": "synthetic",
            "config": {"workload": desc, "symbols": n_total, "job_symbols": job_symbols,
                       "l2": "flushed between steps (256 MiB device write)",
                       "parallelism": (f"{world} GPUs, bin-packed shares" if sharded
                                       else f"{world} independent replica(s)"),
                       "timing": "device time per build (library CUDA events), "
                                 "max over ranks", "wall_s": wall,
                       "build_roofline": whole, "batched": single, "kernels": kernels},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clock_info, "gpu_launches": launches,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def e2e_step(ctx, pinned_text, host_out, isa_bits, lcp_enc, sa_bits=32, batch_symbols=3e8,
             workers=2):
    """One build through the public API from pinned host buffers: a single
    reference, or a collection in sub-batches on `workers` contexts
    (sufgpu_build_collection), whose host copies overlap each other's kernels."""
    if len(pinned_text) == 1:
        t = pinned_text[0]
        return ctx.build_device(t.ctypes.data, int(t.size), host_out[0], sa_bits=sa_bits,
                                isa_bits=isa_bits, lcp=lcp_enc)
    return ctx.build_collection_device([(t.ctypes.data, int(t.size)) for t in pinned_text],
                                       host_out, sa_bits=32, isa_bits=isa_bits, lcp=lcp_enc,
                                       batch_symbols=int(batch_symbols), workers=workers)


if __name__ == "__main__":
    main()
