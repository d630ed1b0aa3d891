"""GPU: the two-bit seed.  A single text of A, C, G, T with few other symbols
sorts 2-bit seed keys; windows that hold a separator, the sentinel, N or the
text end are placed exactly from the rare list.  Every build equals the
oracle word for word, and the code-table seed on the same text."""
import numpy as np
import pytest

import oracle
import sufkit_b200 as sg
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tctx():
    c = sg.Context(0, tuning=None)
    c.set_tuning("two_bit_min", 0)  # small texts take the two-bit seed too
    yield c
    c.close()


def expected(text):
    if oracle.ref() is not None:
        sa, isa, lcp, _ = oracle.ref_adapter(text, 64)
        return sa, isa, lcp
    return oracle.full_build(text)


def dna(rng, n, n_runs=0, n_single=0, separators=0, sentinel=True, poly=0):
    body = rng.integers(2, 6, size=n).astype(np.uint8)
    for _ in range(n_runs):
        L = int(rng.integers(1, 400))
        s = int(rng.integers(0, n))
        body[s:s + L] = 6
    for _ in range(poly):
        L = int(rng.integers(10, 300))
        s = int(rng.integers(0, n))
        body[s:s + L] = int(rng.integers(2, 7))
    body[rng.integers(0, n, size=n_single)] = 6
    body[rng.integers(0, n, size=separators)] = 1
    return np.concatenate([body, np.zeros(1, np.uint8)]) if sentinel else body


def check(c, text, two_bit=True, lcp=sg.LcpEncoding.RAW32):
    sa, isa, lcp_ref = expected(text)
    r = c.build(text, sa_bits=32, isa_bits=32, lcp=lcp, validate=True)
    assert (r.sa_low == sa).all(), "SA differs"
    assert (r.isa_low == isa).all(), "ISA differs"
    if lcp == sg.LcpEncoding.RAW32:
        assert (r.lcp == lcp_ref).all(), "LCP differs"
    else:
        primary, pos, val = oracle.bytecode(text, sa, isa, 32)
        assert (r.lcp == primary).all()
        assert (r.anchor_positions.astype(np.uint64) == pos).all()
        assert (r.anchor_values.astype(np.uint64) == val).all()
    if two_bit:
        assert r.stats["seed_code_bits"] == 2
        assert r.stats["seed_rare_rows"] > 0
    return r


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_dna_with_rare_symbols(tctx, seed):
    rng = np.random.default_rng(seed)
    check(tctx, dna(rng, 120_000, n_runs=20, n_single=30, separators=12, poly=10))


def test_without_sentinel_and_repeats(tctx):
    rng = np.random.default_rng(7)
    unit = rng.integers(2, 6, size=5000).astype(np.uint8)
    unit[100:130] = 6
    unit[2000] = 1
    t = np.concatenate([unit] * 12 + [dna(rng, 3000, sentinel=False)])
    check(tctx, t)
    check(tctx, np.concatenate([t, np.zeros(1, np.uint8)]))


@pytest.mark.parametrize("s", [1, 2, 3, 5, 8, 15])
def test_short_seeds_collide_more(tctx, s):
    """Short seeds put many rare rows under one two-bit key."""
    rng = np.random.default_rng(20 + s)
    t = dna(rng, 60_000, n_runs=30, n_single=60, separators=20, poly=5)
    tctx.set_tuning("seed_symbols", s)
    try:
        check(tctx, t)
    finally:
        tctx.set_tuning("seed_symbols", 0)


def test_unpacked_and_packed_keys(tctx):
    rng = np.random.default_rng(31)
    t = dna(rng, 200_000, n_runs=40, n_single=50, separators=24, poly=20)
    a = check(tctx, t)
    tctx.set_tuning("packed_max_bits", 0)
    try:
        b = check(tctx, t)
    finally:
        tctx.set_tuning("packed_max_bits", 24)
    assert (a.sa_low == b.sa_low).all()


def test_long_runs_of_every_symbol(tctx):
    """Runs of N and of A/C/G/T are split directly; runs of the separator are
    left to the rounds (their windows are rare rows)."""
    rng = np.random.default_rng(41)
    t = dna(rng, 150_000, n_runs=10, poly=30)
    body = t[:-1].copy()
    body[5000:5400] = 1   # a separator run
    body[9000:12000] = 6  # a long N run
    body[20000:23000] = 2
    t = np.concatenate([body, np.zeros(1, np.uint8)])
    r = check(tctx, t)
    assert r.stats["long_runs"] > 0


def test_too_many_rare_rows_falls_back(tctx):
    """Isolated Ns in 1% of positions leave about s x 1% windows rare: past
    the list's n/16, the build redoes the seed with the code-table keys."""
    rng = np.random.default_rng(51)
    t = dna(rng, 100_000, n_single=2000)
    r = check(tctx, t, two_bit=False)
    assert r.stats["seed_code_bits"] == 3


def test_byte_coded_lcp(tctx):
    rng = np.random.default_rng(61)
    check(tctx, dna(rng, 80_000, n_runs=10, separators=5, poly=40), lcp=sg.LcpEncoding.BYTE32)


def test_non_dna_alphabet_keeps_code_table(tctx):
    rng = np.random.default_rng(71)
    t = np.concatenate([rng.integers(1, 30, size=50_000).astype(np.uint8), np.zeros(1, np.uint8)])
    r = check(tctx, t, two_bit=False)
    assert r.stats["seed_code_bits"] > 2


@pytest.mark.parametrize("make", [
    lambda: synth.repeat_rich_100mbp(scale=0.05).logical_text(),
    lambda: synth.human_scale_3gbp(scale=0.002).logical_text(),
    lambda: synth.plain_4mbp(scale=1.0).logical_text(),
])
def test_workload_shapes_match_code_table_seed(make):
    """The benchmark shapes (scaled): two-bit and code-table seeds give the
    same planes, and both equal the oracle."""
    t = make()
    c = sg.Context(0, tuning=None)
    try:
        c.set_tuning("two_bit_min", 0)
        two = c.build(t, sa_bits=40, isa_bits=32, lcp=sg.LcpEncoding.BYTE32, validate=True)
        assert two.stats["seed_code_bits"] == 2
        c.set_tuning("two_bit_seed", 0)
        code = c.build(t, sa_bits=40, isa_bits=32, lcp=sg.LcpEncoding.BYTE32, validate=True)
        assert code.stats["seed_code_bits"] == 3
    finally:
        c.close()
    for f in ("sa_low", "sa_high", "isa_low", "isa_high", "lcp", "anchor_positions",
              "anchor_values"):
        a, b = getattr(two, f), getattr(code, f)
        assert (a is None and b is None) or (a == b).all(), f
    sa, isa, _ = expected(t)
    assert (two.sa == sa).all() and (two.isa == isa).all()


@pytest.mark.parametrize("two_bit_batch", [0, 1])
def test_two_bit_seed_in_batches(ctx, two_bit_batch):
    """Batches with two-bit seed keys: each instance's rare rows (windows that
    reach a separator, the sentinel, an N or the instance end) sorted by
    (instance, exact key) and placed within the instance.  Every instance
    equals the oracle, with and without the batch two-bit seed; instances of
    different sizes, N runs, contigs, and exact-key ties across instances."""
    from conftest import assert_oracle
    rng = np.random.default_rng(77)
    texts = [r.logical_text() for r in synth.uneven_collection(count=6, scale=0.01)]
    same = synth.random_text(rng, 3000, 4)
    texts += [same.copy(), same.copy()]                       # identical instances
    texts.append(synth.human_scale_3gbp(scale=0.0005).logical_text())  # N runs
    texts.append(np.concatenate([np.full(50, 6, np.uint8), synth.random_text(rng, 2000, 4)]))
    ctx.set_tuning("two_bit_min", 0)
    ctx.set_tuning("two_bit_batch", two_bit_batch)
    try:
        for lcp in (sg.LcpEncoding.RAW32, sg.LcpEncoding.BYTE32):
            batch = ctx.build_batch(texts, sa_bits=32, isa_bits=32, lcp=lcp, validate=True)
            assert (ctx.last_stats["seed_code_bits"] == 2) == bool(two_bit_batch)
            for t, b in zip(texts, batch):
                assert_oracle(b, t, lcp)
    finally:
        ctx.set_tuning("two_bit_min", 1 << 22)
        ctx.set_tuning("two_bit_batch", 1)
