"""Autotuner for the build knobs (seed length, radix tile and block shape,
ballot-ranking threshold, packed-seed threshold, two-bit seed, the seed rank
write by window slots, and the round-compaction threshold at which the graph
rounds drop to a smaller bound).  The radix digit width is not a knob: every
radix kernel is compiled for 8-bit digits (their shared-memory histograms and
look-back words are sized by it).

    python -m sufkit_b200.autotune [--out sufkit_b200/tuning.json] [--quick]

For each size class (by the longest instance of a build) it builds a seeded
synthetic workload of that class on the GPU, times builds with the library's
own CUDA events (device seconds, best of a few), and tunes one knob at a time
(coordinate descent, two sweeps) starting from the built-in defaults.  The
winning settings per class go to a JSON table that ``Context`` loads by
default; the library applies a class's settings to every build whose longest
instance falls in it.  Knobs only change speed: every setting produces the
same SA, ISA and LCP, which the tuner re-checks on each class.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import Context, LcpEncoding, TUNING_PATH
from . import synth

# Candidate values per knob (0 for seed_symbols = choose from size/entropy).
CANDIDATES = {
    "seed_symbols": [0, 15, 16, 18, 19, 21],
    "sort_tile": [4096, 2048],
    "sort_block": [256, 512],
    "ballot_min_elems": [1 << 23, 0, 1 << 62],
    "packed_max_bits": [24, 0],
    "two_bit_seed": [1, 0],
    "rank_slots": [1, 0, 2],
    "graph_shrink": [4, 2, 16],
    "keys_sort_block": [256, 512],
    "seg_rank": [0, 1],
    "rank_cluster": [2, 0, 4],
    "seg_blocks": [3, 2],
    "seed_count_run": [1, 0],
    "batch_cluster": [1, 0],
}
DEFAULTS = {"seed_symbols": 0, "sort_tile": 4096, "sort_block": 256,
            "ballot_min_elems": 1 << 23, "packed_max_bits": 24, "two_bit_seed": 1,
            "rank_slots": 1, "graph_shrink": 4, "keys_sort_block": 256, "seg_rank": 0,
            "rank_cluster": 2, "seg_blocks": 3,
            "seed_count_run": 1, "batch_cluster": 1}


def workloads(quick: bool):
    """(max_symbols, name, texts, lcp) per size class."""
    s = 0.25 if quick else 1.0
    coll = synth.uneven_texts(1024, indices=range(32 if quick else 256))
    yield (1 << 24, "bacterial collection (batched)", coll, LcpEncoding.RAW32)
    yield (1 << 28, "repeat-rich 100 Mbp", [synth.repeat_rich_100mbp(s).logical_text()],
           LcpEncoding.RAW32)
    yield ((1 << 32) - 1, "human-scale 3.1 Gbp" + (" (scaled x0.1)" if quick else ""),
           [synth.human_scale_3gbp(0.1 if quick else 1.0).logical_text()], LcpEncoding.BYTE32)


def timed_build(ctx: Context, texts, lcp, reps: int):
    import torch
    dev = torch.device("cuda", 0)
    d_texts = [torch.from_numpy(t).to(dev) for t in texts]
    outs = []
    for t in texts:
        outs.append({"sa_low": torch.empty(t.size, dtype=torch.int32, device=dev),
                     "lcp": torch.empty(t.size, dtype=torch.uint8 if lcp == LcpEncoding.BYTE32
                                        else torch.int32, device=dev)})

    def ptrs(o):
        return {k: v.data_ptr() for k, v in o.items()}

    def run():
        if len(texts) == 1:
            return ctx.build_device(d_texts[0].data_ptr(), int(texts[0].size), ptrs(outs[0]),
                                    sa_bits=32, isa_bits=0, lcp=lcp)["device_seconds"]
        return ctx.build_batch_device([(d.data_ptr(), int(t.size)) for d, t in zip(d_texts, texts)],
                                      [ptrs(o) for o in outs], sa_bits=32, isa_bits=0,
                                      lcp=lcp)["device_seconds"]

    run()
    best = min(run() for _ in range(reps))
    digest = [np.frombuffer(o["sa_low"].cpu().numpy().tobytes(), np.uint8)[::4097].sum()
              for o in outs[:4]]
    return best, digest


def tune_class(ctx: Context, texts, lcp, reps: int, log):
    current = dict(DEFAULTS)

    def measure(settings):
        for k, v in settings.items():
            ctx.set_tuning(k, v)
        try:
            return timed_build(ctx, texts, lcp, reps)
        finally:
            for k, v in DEFAULTS.items():
                ctx.set_tuning(k, v)

    base_time, base_digest = measure(current)
    log(f"  defaults: {base_time * 1e3:.2f} ms")
    best_time = base_time
    for sweep in range(2):
        changed = False
        for key, values in CANDIDATES.items():
            for v in values:
                if v == current[key]:
                    continue
                trial = dict(current, **{key: v})
                t, digest = measure(trial)
                if digest != base_digest:
                    raise RuntimeError(f"{key}={v} changed the suffix array")
                log(f"  {key}={v}: {t * 1e3:.2f} ms")
                if t < best_time * 0.985:
                    best_time, current, changed = t, trial, True
        if not changed:
            break
    return current, base_time, best_time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(TUNING_PATH))
    ap.add_argument("--quick", action="store_true", help="smaller workloads, fewer repeats")
    args = ap.parse_args()
    import torch
    reps = 2 if args.quick else 3
    ctx = Context(0, tuning=None)
    classes = []
    t0 = time.time()
    for max_symbols, name, texts, lcp in workloads(args.quick):
        print(f"class <= {max_symbols} symbols: {name}", flush=True)
        settings, base, best = tune_class(ctx, texts, lcp, reps, lambda m: print(m, flush=True))
        changed = {k: v for k, v in settings.items() if v != DEFAULTS[k]}
        classes.append({"max_symbols": max_symbols, "workload": name,
                        "symbols": int(sum(t.size for t in texts)), "settings": changed,
                        "default_ms": base * 1e3, "tuned_ms": best * 1e3})
    table = {"device": torch.cuda.get_device_name(0), "tuned_seconds": time.time() - t0,
             "classes": classes}
    Path(args.out).write_text(json.dumps(table, indent=1) + "\n")
    print(json.dumps(table, indent=1))


if __name__ == "__main__":
    main()
