"""GPU: a batch of uneven references equals each reference built alone, and
every instance equals the oracle's build of it (the reference's divsufsort64
when it was compiled)."""
import numpy as np
import pytest

import oracle
import sufkit_b200 as sg
from conftest import assert_oracle, oracle_build
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu


def test_batch_equals_single(ctx):
    refs = synth.uneven_collection(count=12, scale=0.01)
    texts = [r.logical_text() for r in refs]
    texts.append(np.array([0], np.uint8))              # one-symbol instance
    texts.append(np.full(5000, 6, np.uint8))           # no sentinel, one run
    texts.append(np.tile(np.array([2, 3], np.uint8), 3000))
    expected = [oracle_build(t) for t in texts]
    for lcp in (sg.LcpEncoding.RAW32, sg.LcpEncoding.BYTE32):
        batch = ctx.build_batch(texts, sa_bits=32, isa_bits=32, lcp=lcp, validate=True)
        for t, b, e in zip(texts, batch, expected):
            assert_oracle(b, t, lcp, e)
            s = ctx.build(t, sa_bits=32, isa_bits=32, lcp=lcp)
            assert (b.sa_low == s.sa_low).all()
            assert (b.isa_low == s.isa_low).all()
            assert (b.lcp == s.lcp).all()
            if lcp == sg.LcpEncoding.BYTE32:
                assert (b.anchor_positions == s.anchor_positions).all()
                assert (b.anchor_values == s.anchor_values).all()


def test_batch_against_oracle(ctx):
    rng = np.random.default_rng(11)
    texts = [synth.random_text(rng, int(n), 4) for n in rng.integers(1, 20000, size=40)]
    batch = ctx.build_batch(texts, sa_bits=64, isa_bits=0, lcp=sg.LcpEncoding.RAW64)
    for t, b in zip(texts, batch):
        assert_oracle(b, t, sg.LcpEncoding.RAW64)
        # and the C restatement agrees with the compiled reference
        sa, isa, lcp = oracle.full_build(t)
        assert (b.sa_low == sa).all() and (b.lcp == lcp).all()


@pytest.mark.parametrize("fused", [0, 1])
def test_batch_seed_first_pass_fused_or_separate(ctx, fused):
    """Batches whose seed keys come from the fused first-pass kernel (tiles
    follow instance boundaries, instances start at any byte offset) equal the
    oracle, as do batches sorted by the separate passes; packed (instances up
    to 2^24 symbols) and unpacked."""
    rng = np.random.default_rng(41)
    texts = [synth.random_text(rng, int(n), 4) for n in (1, 7, 4095, 4097, 10_001, 65_536)]
    texts += [r.logical_text() for r in synth.uneven_collection(count=5, scale=0.02)]
    big = [synth.repeat_rich_100mbp(scale=0.18).logical_text(),   # > 2^24 symbols: unpacked
           synth.random_text(rng, 3_333, 2)]
    ctx.set_tuning("seed_fused", fused)
    try:
        for batch_texts in (texts, big):
            batch = ctx.build_batch(batch_texts, sa_bits=32, isa_bits=32,
                                    lcp=sg.LcpEncoding.RAW32, validate=True)
            for t, b in zip(batch_texts, batch):
                assert_oracle(b, t, sg.LcpEncoding.RAW32)
    finally:
        ctx.set_tuning("seed_fused", 1)


@pytest.mark.parametrize("slots", [0, 1])
def test_batch_rank_write_by_slots_or_passes(ctx, slots):
    """A batch's seed rank write by per-instance window slots or by grouping
    passes: the same (oracle-equal) instances, including instances shorter
    than a window and exactly one window long."""
    rng = np.random.default_rng(43)
    texts = [synth.random_text(rng, int(n), 4) for n in (1, 2, 8191, 8192, 8193, 20_000)]
    texts += [r.logical_text() for r in synth.uneven_collection(count=4, scale=0.01)]
    ctx.set_tuning("rank_slots", slots)
    try:
        batch = ctx.build_batch(texts, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32,
                                validate=True)
        for t, b in zip(texts, batch):
            assert_oracle(b, t, sg.LcpEncoding.RAW32)
    finally:
        ctx.set_tuning("rank_slots", 1)


@pytest.mark.parametrize("cluster", [0, 1])
def test_batch_rank_write_cluster_windows(ctx, cluster):
    """A batch's rank write through 65536-position windows per instance held
    by two-block clusters (no grouping pass for instances of at most 2^16
    symbols, one for 2^20 and more), or through window slots: every instance
    equals the oracle."""
    rng = np.random.default_rng(65)
    small = [synth.random_text(rng, int(m), 4) for m in rng.integers(3000, 65_536, size=10)]
    large = [synth.random_text(rng, int(m), 4) for m in rng.integers(600_000, 1_100_000, size=3)]
    ctx.set_tuning("batch_cluster", cluster)
    try:
        for texts in (small, large + small[:3]):
            batch = ctx.build_batch(texts, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32,
                                    validate=True)
            for t, b in zip(texts, batch):
                assert_oracle(b, t, sg.LcpEncoding.RAW32)
    finally:
        ctx.set_tuning("batch_cluster", 1)
