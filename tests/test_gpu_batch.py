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
