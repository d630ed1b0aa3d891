"""GPU: collections built in sub-batches on several contexts side by side
(sufgpu_build_collection).  Every instance equals a single build of it and
the oracle's build of it."""
import numpy as np
import pytest

import sufkit_b200 as sg
from conftest import assert_oracle, oracle_build
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu


def texts(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(2_000, 60_000))
        body = rng.integers(2, 6, size=n).astype(np.uint8)
        if i % 3 == 0:
            body[n // 3:n // 3 + 500] = 6
        out.append(np.concatenate([body, np.array([1], np.uint8), body[: n // 4],
                                   np.zeros(1, np.uint8)]))
    return out


@pytest.mark.parametrize("workers,batch_symbols", [(1, 200_000), (2, 150_000), (3, 1), (2, 0)])
def test_collection_equals_single_builds(ctx, workers, batch_symbols):
    ts = texts(23, workers * 10 + 1)
    got = ctx.build_collection(ts, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32,
                               validate=True, batch_symbols=batch_symbols, workers=workers)
    assert ctx.last_stats["symbols"] == sum(t.size for t in ts)
    for t, r in zip(ts, got):
        assert_oracle(r, t, sg.LcpEncoding.RAW32)
        one = ctx.build(t, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32)
        assert (r.sa_low == one.sa_low).all()
        assert (r.isa_low == one.isa_low).all()
        assert (r.lcp == one.lcp).all()


@pytest.mark.parametrize("lcp", [sg.LcpEncoding.RAW32, sg.LcpEncoding.RAW64, sg.LcpEncoding.NONE])
@pytest.mark.parametrize("workers", [2, 3])
def test_collection_sa_and_lcp_only(ctx, lcp, workers):
    """Without ISA a worker computes all planes first and copies after it
    leaves the shared gate (the packed SA staged in the rank buffer)."""
    ts = texts(31, 7 + workers)
    got = ctx.build_collection(ts, sa_bits=32, isa_bits=0, lcp=lcp, validate=True,
                               batch_symbols=120_000, workers=workers)
    for t, r in zip(ts, got):
        assert_oracle(r, t, lcp)
        one = ctx.build(t, sa_bits=32, isa_bits=0, lcp=lcp)
        assert (r.sa_low == one.sa_low).all()
        if lcp != sg.LcpEncoding.NONE:
            assert (r.lcp == one.lcp).all()


def test_collection_trace(ctx):
    ts = texts(12, 99)
    ctx.build_collection(ts, isa_bits=0, batch_symbols=100_000, workers=2)
    trace = ctx.collection_trace()
    assert len(trace) >= 2
    for t in trace:
        assert t["worker"] in (0, 1)
        assert 0 <= t["start"] <= t["gate_in"] <= t["gate_out"] <= t["end"]
    # The gate admits one build at a time.
    held = sorted((t["gate_in"], t["gate_out"]) for t in trace)
    for (a0, a1), (b0, b1) in zip(held, held[1:]):
        assert a1 <= b0


def test_collection_byte_coded_anchors_survive(ctx):
    """Anchors of every sub-batch stay readable after the later sub-batches."""
    ts = [synth.uneven_reference(i, 40_000 + 5_000 * i).logical_text() for i in range(9)]
    for t in ts[::3]:
        t[1000:1300] = 2  # long LCPs: anchors
    got = ctx.build_collection(ts, sa_bits=40, lcp=sg.LcpEncoding.BYTE32, batch_symbols=100_000,
                               workers=2)
    for t, r in zip(ts, got):
        assert_oracle(r, t, sg.LcpEncoding.BYTE32)
        one = ctx.build(t, sa_bits=40, isa_bits=0, lcp=sg.LcpEncoding.BYTE32)
        assert (r.sa == one.sa).all() and (r.lcp == one.lcp).all()
        assert (r.anchor_positions == one.anchor_positions).all()
        assert (r.anchor_values == one.anchor_values).all()


def test_collection_rejects_bad_arguments(ctx):
    with pytest.raises(sg.SufkitError):
        ctx.build_collection(texts(2, 5), workers=0)
    with pytest.raises(sg.SufkitError):
        ctx.build_collection(texts(2, 5), workers=9)
    assert ctx.build_collection([], workers=2) == []
