"""GPU: suffixes inside long single-symbol runs (N gaps, poly-A tracts) are
placed directly after the seed instead of by many doubling rounds.  Every
build here equals the oracle word for word, with the split on and off."""
import numpy as np
import pytest

import oracle
import sufkit_b200 as sg
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu


def expected(text):
    if oracle.ref() is not None:
        sa, isa, lcp, _ = oracle.ref_adapter(text, 64)
        return sa, isa, lcp
    return oracle.full_build(text)


def runs_text(rng, n, run_count, max_len, symbols=(2, 3, 4, 5, 6), sentinel=True):
    """Random ACGT body with runs of every symbol: lengths around the seed
    length (21), long ones, equal lengths and copies of one run + context so
    that run ends tie and need more rounds."""
    body = rng.integers(2, 6, size=n).astype(np.uint8)
    lengths = np.concatenate([
        np.array([20, 21, 22, 23, 41, 42, 43, 84, 85], np.int64),
        rng.integers(21, max_len + 1, size=run_count)])
    for L in lengths:
        c = int(rng.choice(symbols))
        start = int(rng.integers(0, max(1, n - L)))
        body[start:start + L] = c
    # Copies of one run with the same continuation (ties on the run end).
    unit = np.concatenate([np.full(500, 6, np.uint8), rng.integers(2, 6, 60).astype(np.uint8)])
    for _ in range(6):
        start = int(rng.integers(0, max(1, n - unit.size)))
        body[start:start + unit.size] = unit
    if sentinel:
        return np.concatenate([body, np.array([1, 0], np.uint8)])
    return body


def check(ctx, text, lcp=sg.LcpEncoding.RAW32):
    sa, isa, lcp_ref = expected(text)
    r = ctx.build(text, sa_bits=32, isa_bits=32, lcp=lcp, validate=True)
    assert (r.sa_low == sa).all(), "SA differs"
    assert (r.isa_low == isa).all(), "ISA differs"
    if lcp == sg.LcpEncoding.RAW32:
        assert (r.lcp == lcp_ref).all(), "LCP differs"
    else:
        primary, pos, val = oracle.bytecode(text, sa, isa, 32)
        assert (r.lcp == primary).all()
        assert (r.anchor_positions.astype(np.uint64) == pos).all()
        assert (r.anchor_values.astype(np.uint64) == val).all()
    return r


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_runs_of_every_symbol(ctx, seed):
    rng = np.random.default_rng(seed)
    t = runs_text(rng, 200_000, 300, 3000)
    r = check(ctx, t)
    assert r.stats["long_runs"] > 0


def test_runs_touching_the_end_without_sentinel(ctx):
    rng = np.random.default_rng(5)
    body = runs_text(rng, 50_000, 40, 800, sentinel=False)
    # Runs that end at the instance end, of the largest and smallest symbol.
    for tail in (6, 2):
        t = np.concatenate([body, np.full(700, tail, np.uint8)])
        r = check(ctx, t)
        assert r.stats["long_runs"] > 0


def test_adjacent_runs_and_whole_text_run(ctx):
    t = np.concatenate([np.full(3000, 6, np.uint8), np.full(2000, 2, np.uint8),
                        np.full(3000, 6, np.uint8), np.full(100, 5, np.uint8),
                        np.full(3000, 6, np.uint8), np.array([1, 0], np.uint8)])
    check(ctx, t)
    check(ctx, np.full(20_000, 4, np.uint8))
    check(ctx, np.concatenate([np.full(20_000, 4, np.uint8), np.zeros(1, np.uint8)]))


def test_split_on_and_off_agree(ctx):
    t = synth.human_scale_3gbp(scale=0.004).logical_text()
    on = ctx.build(t, sa_bits=40, isa_bits=0, lcp=sg.LcpEncoding.BYTE32)
    assert on.stats["long_runs"] > 0
    ctx.set_tuning("run_split", 0)
    try:
        off = ctx.build(t, sa_bits=40, isa_bits=0, lcp=sg.LcpEncoding.BYTE32)
    finally:
        ctx.set_tuning("run_split", 1)
    assert off.stats["long_runs"] == 0
    assert off.stats["active_rows"] > on.stats["active_rows"]
    assert (on.sa_low == off.sa_low).all() and (on.sa_high == off.sa_high).all()
    assert (on.lcp == off.lcp).all()
    assert (on.anchor_positions == off.anchor_positions).all()
    assert (on.anchor_values == off.anchor_values).all()


def test_byte_coded_with_runs(ctx):
    rng = np.random.default_rng(9)
    check(ctx, runs_text(rng, 100_000, 100, 5000), lcp=sg.LcpEncoding.BYTE32)


def test_batch_with_runs(ctx):
    rng = np.random.default_rng(13)
    texts = [runs_text(rng, int(n), 30, 2000, sentinel=bool(i % 2))
             for i, n in enumerate(rng.integers(3000, 40_000, size=16))]
    texts.append(np.full(3000, 6, np.uint8))
    batch = ctx.build_batch(texts, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32,
                            validate=True)
    for t, b in zip(texts, batch):
        sa, isa, lcp = expected(t)
        assert (b.sa_low == sa).all() and (b.isa_low == isa).all() and (b.lcp == lcp).all()
