"""GPU: sampled builds (sampling rate K > 1, as BuildDivsufsort's
sampling_rate) equal the reference's sampled divsufsort64 build word for
word: SA of the suffixes at multiples of K, their ISA and the LCP of
consecutive sampled rows, raw or byte-coded (primary bytes per sampled row
and anchors at sampled text positions, as the reference's
LcpStorage::BuildByteCodedDirect writes them for rate K)."""
import numpy as np
import pytest

import oracle
import sufkit_b200 as sg
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu


def expected_sampled(text, rate):
    if oracle.ref() is not None:
        return oracle.ref_adapter_sampled(text, rate, 64)
    sa, isa, lcp = oracle.full_build(text)
    return oracle.sample(sa, lcp, rate)


def texts():
    rng = np.random.default_rng(17)
    yield synth.repeat_rich_100mbp(scale=0.005).logical_text()
    yield synth.human_scale_3gbp(scale=0.002).logical_text()
    for n in (1, 2, 3, 31, 4097):
        yield synth.random_text(rng, n, 4)
    yield np.full(3000, 6, np.uint8)


@pytest.mark.parametrize("rate", [2, 3, 7, 32])
def test_sampled_equals_reference(ctx, rate):
    for t in texts():
        sa_k, isa_k, lcp_k = expected_sampled(t, rate)
        for sa_bits, lcp in ((32, sg.LcpEncoding.RAW32), (64, sg.LcpEncoding.RAW64),
                             (40, sg.LcpEncoding.RAW32)):
            r = ctx.build(t, sa_bits=sa_bits, isa_bits=sa_bits, lcp=lcp, validate=True,
                          sampling_rate=rate)
            assert (r.sa.astype(np.uint64) == sa_k).all(), (t.size, rate, sa_bits)
            assert (r.isa.astype(np.uint64) == isa_k).all()
            assert (r.lcp.astype(np.uint64) == lcp_k).all()


def test_sampled_batch_equals_single(ctx):
    rng = np.random.default_rng(5)
    ts = [synth.random_text(rng, int(n), 4) for n in rng.integers(1, 30_000, size=25)]
    ts.append(synth.repeat_rich_100mbp(scale=0.002).logical_text())
    batch = ctx.build_batch(ts, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32,
                            validate=True, sampling_rate=5)
    for t, b in zip(ts, batch):
        sa_k, isa_k, lcp_k = expected_sampled(t, 5)
        assert (b.sa_low == sa_k).all() and (b.isa_low == isa_k).all() and (b.lcp == lcp_k).all()


def expected_bytecode(text, sa_k, isa_k, lcp_k, rate, width):
    if oracle.ref() is not None:
        return oracle.ref_bytecode_sampled(text, sa_k, isa_k, rate, width)
    return oracle.sample_bytecode(sa_k, isa_k, lcp_k, rate)


def long_lcp_texts():
    rng = np.random.default_rng(23)
    yield synth.strain_collection(5, 20_000, rng).logical_text()   # LCPs ~20 kbp
    yield np.concatenate([np.full(3000, 2, np.uint8), np.array([1], np.uint8),
                          np.full(2000, 2, np.uint8), np.zeros(1, np.uint8)])
    yield synth.human_scale_3gbp(scale=0.002).logical_text()
    yield synth.random_text(rng, 5000, 4)  # no anchors


@pytest.mark.parametrize("rate", [2, 3, 8, 255, 256, 300])
def test_sampled_byte_coded_lcp_equals_reference(ctx, rate):
    for t in long_lcp_texts():
        sa_k, isa_k, lcp_k = expected_sampled(t, rate)
        for sa_bits, enc, width in ((32, sg.LcpEncoding.BYTE32, 32),
                                    (40, sg.LcpEncoding.BYTE64, 64)):
            primary, pos, val = expected_bytecode(t, sa_k, isa_k, lcp_k, rate, width)
            r = ctx.build(t, sa_bits=sa_bits, isa_bits=0, lcp=enc, validate=True,
                          sampling_rate=rate)
            assert (r.sa.astype(np.uint64) == sa_k).all(), (t.size, rate)
            assert np.array_equal(r.lcp, primary), (t.size, rate)
            assert np.array_equal(r.anchor_positions.astype(np.uint64), pos), (t.size, rate)
            assert np.array_equal(r.anchor_values.astype(np.uint64), val), (t.size, rate)


def test_sampled_byte_coded_batch_equals_single(ctx):
    ts = list(long_lcp_texts())
    batch = ctx.build_batch(ts, sa_bits=32, isa_bits=0, lcp=sg.LcpEncoding.BYTE32,
                            validate=True, sampling_rate=4)
    for t, b in zip(ts, batch):
        sa_k, isa_k, lcp_k = expected_sampled(t, 4)
        primary, pos, val = expected_bytecode(t, sa_k, isa_k, lcp_k, 4, 32)
        assert (b.sa_low == sa_k).all() and np.array_equal(b.lcp, primary)
        assert np.array_equal(b.anchor_positions.astype(np.uint64), pos)
        assert np.array_equal(b.anchor_values.astype(np.uint64), val)
