"""GPU: continuously batched (served) builds equal standalone builds.

Requests of mixed size and encoding are submitted while earlier ones are on
the GPU; each result must equal Context.build of the same text (and hence the
reference's divsufsort64 build)."""
import numpy as np
import pytest

import oracle
import sufkit_b200 as sg
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu

ENCODINGS = [(32, 32, sg.LcpEncoding.RAW32), (32, 0, sg.LcpEncoding.BYTE32),
             (40, 0, sg.LcpEncoding.BYTE32), (64, 64, sg.LcpEncoding.RAW64)]


def _texts():
    rng = np.random.default_rng(99)
    texts = [synth.random_text(rng, int(n), 4) for n in (1, 2, 100, 5000, 200_000, 1_500_000)]
    texts.append(synth.strain_collection(copies=8, genome_bp=150_000, rng=rng).logical_text())
    texts.append(synth.repeat_rich_100mbp(scale=0.01).logical_text())
    texts.append(np.concatenate([np.full(20_000, 6, np.uint8), np.array([1, 0], np.uint8)]))
    texts.append(rng.integers(0, 256, size=30_000).astype(np.uint8))
    return texts


def _same(a: sg.BuildResult, b: sg.BuildResult):
    for key in ("sa_low", "sa_high", "isa_low", "isa_high", "lcp", "anchor_positions",
                "anchor_values"):
        x, y = getattr(a, key), getattr(b, key)
        assert (x is None) == (y is None), key
        if x is not None:
            assert x.dtype == y.dtype and (x == y).all(), key


def test_served_results_equal_standalone(ctx):
    texts = _texts()
    with sg.Server(0, capacity_symbols=1 << 25, max_instances=64) as server:
        tickets = []
        # First wave, then a second wave submitted while the first runs.
        for i, t in enumerate(texts[:5]):
            sa_bits, isa_bits, lcp = ENCODINGS[i % len(ENCODINGS)]
            tickets.append((i, server.submit(t, sa_bits, isa_bits, lcp)))
        first = server.wait(tickets[0][1])
        for i, t in enumerate(texts[5:], start=5):
            sa_bits, isa_bits, lcp = ENCODINGS[i % len(ENCODINGS)]
            tickets.append((i, server.submit(t, sa_bits, isa_bits, lcp)))
        results = {tickets[0][0]: first}
        for i, ticket in tickets[1:]:
            results[i] = server.wait(ticket)
        stats = server.stats()
    assert stats["completed"] == len(texts)
    assert stats["p99_seconds"] >= stats["p50_seconds"] > 0
    for i, t in enumerate(texts):
        sa_bits, isa_bits, lcp = ENCODINGS[i % len(ENCODINGS)]
        alone = ctx.build(t, sa_bits, isa_bits, lcp)
        _same(results[i], alone)
    # And against the reference for one mixed-in request.
    t = texts[7]
    sa, isa, lcp_ref = oracle.full_build(t) if oracle.ref() is None else oracle.ref_adapter(t)[:3]
    assert (results[7].sa == sa).all()


def test_served_admission_under_small_arena(ctx):
    rng = np.random.default_rng(5)
    texts = [synth.random_text(rng, int(n), 4) for n in rng.integers(50_000, 400_000, size=24)]
    with sg.Server(0, capacity_symbols=1_000_000, max_instances=8) as server:
        tickets = [server.submit(t, 32, 32, sg.LcpEncoding.RAW32) for t in texts]
        results = [server.wait(k) for k in tickets]
        stats = server.stats()
    assert stats["completed"] == len(texts) and stats["max_inflight"] <= 8
    for t, r in zip(texts, results):
        alone = ctx.build(t, 32, 32, sg.LcpEncoding.RAW32)
        _same(r, alone)


def test_served_rejects_oversize():
    with sg.Server(0, capacity_symbols=100_000, max_instances=4) as server:
        ticket = server.submit(np.zeros(200_000, np.uint8) + 2, 32, 0, sg.LcpEncoding.NONE)
        with pytest.raises(sg.SufkitError) as err:
            server.wait(ticket)
        assert err.value.code == sg.ErrorCode.INVALID_INPUT
