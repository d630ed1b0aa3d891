"""GPU: continuously batched (served) builds equal standalone builds.

Requests of mixed size and encoding are submitted while earlier ones are on
the GPU; each result must equal Context.build of the same text and the
oracle's build (the reference's divsufsort64 when it was compiled), and the
server's per-request iteration counts must show that requests were merged
into a batch whose earlier members were still mid-rounds."""
import numpy as np
import pytest

import sufkit_b200 as sg
from conftest import assert_oracle, oracle_build
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
        assert_oracle(results[i], t, lcp)
        alone = ctx.build(t, sa_bits, isa_bits, lcp)
        _same(results[i], alone)


def test_served_requests_overlap_in_the_running_batch(ctx):
    """Continuous batching, not a queue: a request admitted while others are
    mid-rounds shares their doubling rounds.  The long-LCP strain collection
    (about 14 rounds) is submitted first; small requests follow while it runs.
    Some request must be admitted at an iteration > 0 with requests in flight,
    and finish before a request admitted earlier does; every result is the
    same in the mix as alone and as the oracle's."""
    rng = np.random.default_rng(17)
    long_lcp = synth.strain_collection(copies=12, genome_bp=200_000, rng=rng).logical_text()
    small = [synth.random_text(rng, int(n), 4) for n in (3_000, 40_000, 120_000, 7_000, 60_000)]
    texts = [long_lcp] + small
    expected = [oracle_build(t) for t in texts]
    with sg.Server(0, capacity_symbols=1 << 24, max_instances=16) as server:
        tickets = [server.submit(long_lcp, 32, 0, sg.LcpEncoding.BYTE32)]
        import time
        deadline = time.monotonic() + 30
        while server.stats()["iterations"] < 1 and time.monotonic() < deadline:
            time.sleep(0.0005)  # the long request is on the GPU, mid-rounds
        for t in small:
            tickets.append(server.submit(t, 32, 32, sg.LcpEncoding.RAW32))
        results = [server.wait(k) for k in tickets]
        stats = server.stats()
    assert stats["max_inflight"] > 1
    infos = [r.stats for r in results]
    merged = [i for i, st in enumerate(infos) if st["inflight_at_admit"] > 0
              and st["admit_iteration"] > 0]
    assert merged, f"no request joined a running batch: {infos}"
    # Overlap: a request admitted later finished no later than one admitted earlier.
    assert any(infos[j]["admit_iteration"] > infos[i]["admit_iteration"]
               and infos[j]["finish_iteration"] <= infos[i]["finish_iteration"]
               for i in range(len(infos)) for j in range(len(infos)) if i != j)
    for t, r, e, lcp in zip(texts, results, expected,
                            [sg.LcpEncoding.BYTE32] + [sg.LcpEncoding.RAW32] * len(small)):
        assert_oracle(r, t, lcp, e)
        alone = ctx.build(t, 32, 0 if lcp == sg.LcpEncoding.BYTE32 else 32, lcp)
        _same(r, alone)


def test_served_admission_under_small_arena(ctx):
    rng = np.random.default_rng(5)
    texts = [synth.random_text(rng, int(n), 4) for n in rng.integers(50_000, 400_000, size=24)]
    with sg.Server(0, capacity_symbols=1_000_000, max_instances=8) as server:
        tickets = [server.submit(t, 32, 32, sg.LcpEncoding.RAW32) for t in texts]
        results = [server.wait(k) for k in tickets]
        stats = server.stats()
    assert stats["completed"] == len(texts) and stats["max_inflight"] <= 8
    for t, r in zip(texts, results):
        assert_oracle(r, t, sg.LcpEncoding.RAW32)
        alone = ctx.build(t, 32, 32, sg.LcpEncoding.RAW32)
        _same(r, alone)


def test_served_rejects_oversize():
    with sg.Server(0, capacity_symbols=100_000, max_instances=4) as server:
        ticket = server.submit(np.zeros(200_000, np.uint8) + 2, 32, 0, sg.LcpEncoding.NONE)
        with pytest.raises(sg.SufkitError) as err:
            server.wait(ticket)
        assert err.value.code == sg.ErrorCode.INVALID_INPUT
