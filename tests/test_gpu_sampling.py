"""GPU: sampled builds (sampling rate K > 1, as BuildDivsufsort's
sampling_rate) equal the reference's sampled divsufsort64 build word for
word: SA of the suffixes at multiples of K, their ISA and the LCP of
consecutive sampled rows."""
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


def test_sampled_rejects_byte_coded_lcp(ctx):
    t = synth.random_text(np.random.default_rng(1), 1000, 4)
    with pytest.raises(sg.SufkitError) as e:
        ctx.build(t, sa_bits=32, isa_bits=0, lcp=sg.LcpEncoding.BYTE32, sampling_rate=4)
    assert e.value.code == sg.ErrorCode.INVALID_INPUT
