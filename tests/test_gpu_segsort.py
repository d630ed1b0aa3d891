"""GPU: doubling rounds sort their groups in shared memory; rounds with a group
too large for one block take the global passes.  Both give the oracle's
output word for word, and the two strategies agree with each other.  Every
test runs with the round's second step fused into the shared-memory sort
(seg_rank) and as the separate round_rank pass over sorted keys."""
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


@pytest.fixture(autouse=True, params=[1, 0], ids=["seg_rank", "seg_sort+round_rank"])
def round_step2(request, ctx):
    ctx.set_tuning("seg_rank", request.param)
    yield request.param
    ctx.set_tuning("seg_rank", 1)


def build(ctx, text, seg_sort=1):
    ctx.set_tuning("seg_sort", seg_sort)
    try:
        return ctx.build(text, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32, validate=True)
    finally:
        ctx.set_tuning("seg_sort", 1)


def test_small_groups_stay_in_shared_memory(ctx):
    t = synth.repeat_rich_100mbp(scale=0.01).logical_text()
    r = build(ctx, t)
    sa, isa, lcp = expected(t)
    assert r.stats["rounds"] > 0 and r.stats["seg_sort_fallbacks"] == 0
    assert (r.sa_low == sa).all() and (r.isa_low == isa).all() and (r.lcp == lcp).all()
    g = build(ctx, t, seg_sort=0)
    assert (g.sa_low == r.sa_low).all() and (g.lcp == r.lcp).all()


@pytest.mark.parametrize("period", [2, 5, 33])
def test_large_groups_fall_back(ctx, period):
    rng = np.random.default_rng(period)
    unit = rng.integers(2, 6, size=period).astype(np.uint8)
    tandem = np.tile(unit, 150_000 // period)
    flank = rng.integers(2, 6, size=5000).astype(np.uint8)
    t = np.concatenate([flank, tandem, flank[::-1], tandem, np.array([1, 0], np.uint8)])
    r = build(ctx, t)
    sa, isa, lcp = expected(t)
    assert r.stats["seg_sort_fallbacks"] > 0
    assert (r.sa_low == sa).all() and (r.isa_low == isa).all() and (r.lcp == lcp).all()


def test_groups_of_every_size_up_to_a_block(ctx):
    # Repeat families with 2..3000 copies of one 40-symbol unit and random
    # context: groups straddle windows and fill blocks to the limit.
    rng = np.random.default_rng(21)
    parts = []
    for copies in (2, 3, 17, 255, 1024, 2047, 2048, 2049, 3000):
        unit = rng.integers(2, 6, size=40).astype(np.uint8)
        for _ in range(copies):
            parts.append(unit)
            parts.append(rng.integers(2, 6, size=int(rng.integers(1, 9))).astype(np.uint8))
    t = np.concatenate(parts + [np.array([1, 0], np.uint8)])
    r = build(ctx, t)
    sa, isa, lcp = expected(t)
    assert (r.sa_low == sa).all() and (r.isa_low == isa).all() and (r.lcp == lcp).all()


@pytest.mark.parametrize("kind", ["repeats", "tandem"])
def test_graph_rounds_equal_host_rounds(ctx, kind):
    """Repeated builds of one layout replay captured round graphs (from the
    second build on); a round with a group beyond a block stops the graph and
    is finished by the host.  Every build equals the host-driven one."""
    if kind == "repeats":
        t = synth.repeat_rich_100mbp(scale=0.01).logical_text()
    else:
        rng = np.random.default_rng(3)
        unit = rng.integers(2, 6, size=3).astype(np.uint8)
        t = np.concatenate([rng.integers(2, 6, size=3000).astype(np.uint8),
                            np.tile(unit, 40_000), np.array([1, 0], np.uint8)])
    ctx.set_tuning("graph_rounds", 0)
    try:
        host = ctx.build(t, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32, validate=True)
    finally:
        ctx.set_tuning("graph_rounds", 1)
    for _ in range(3):
        r = ctx.build(t, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32, validate=True)
        assert (r.sa_low == host.sa_low).all() and (r.isa_low == host.isa_low).all()
        assert (r.lcp == host.lcp).all()
        assert r.stats["rounds"] == host.stats["rounds"]
        assert r.stats["active_rows"] == host.stats["active_rows"]
        assert r.stats["seg_sort_fallbacks"] == host.stats["seg_sort_fallbacks"]
    if kind == "tandem":
        assert host.stats["seg_sort_fallbacks"] > 0


@pytest.mark.parametrize("small", [0, 2, 96, 4096])
def test_rank_by_counting_or_passes(ctx, small):
    """Round tiles ranked by counting inside their groups (groups of at most
    `small` rows) or by the shared-memory radix passes (0: always passes;
    4096: counting for every tile that fits a block): the same oracle-equal
    build on repeat-rich text, tandem repeats and a long run."""
    rng = np.random.default_rng(5)
    texts = [synth.repeat_rich_100mbp(scale=0.01).logical_text(),
             np.concatenate([np.tile(synth.random_text(rng, 7, 4)[:6], 3000),
                             synth.random_text(rng, 20000, 4)]),
             np.concatenate([np.full(30000, 2, np.uint8), synth.random_text(rng, 5000, 4)])]
    ctx.set_tuning("seg_small_group", small)
    ctx.set_tuning("graph_rounds", 0)  # cached round graphs hold the knob of their capture
    try:
        for t in texts:
            r = ctx.build(t, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32, validate=True)
            sa, isa, lcp = expected(t)
            assert (r.sa_low == sa).all() and (r.isa_low == isa).all() and (r.lcp == lcp).all()
    finally:
        ctx.set_tuning("seg_small_group", 96)
        ctx.set_tuning("graph_rounds", 1)


@pytest.mark.parametrize("blocks", [2, 3])
def test_round_sort_register_caps(ctx, blocks):
    """The round sort compiled for two or three blocks per SM (register cap):
    the same oracle-equal build on repeat-rich text and tandem repeats."""
    rng = np.random.default_rng(8)
    texts = [synth.repeat_rich_100mbp(scale=0.01).logical_text(),
             np.concatenate([np.tile(synth.random_text(rng, 9, 4)[:8], 2000),
                             synth.random_text(rng, 30000, 4)])]
    ctx.set_tuning("seg_blocks", blocks)
    try:
        for t in texts:
            r = build(ctx, t)
            sa, isa, lcp = expected(t)
            assert (r.sa_low == sa).all() and (r.isa_low == isa).all() and (r.lcp == lcp).all()
    finally:
        ctx.set_tuning("seg_blocks", 3)
