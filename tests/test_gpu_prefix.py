"""GPU: the Fast index's exact k-mer prefix directory built from the device
SA equals the reference's FastPrefixIndex (and its k selection) entry for
entry."""
import numpy as np
import pytest

import oracle
import sufkit_b200 as sg
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["plain4m", "repeat_rich", "runs"])
def test_directory_equals_reference(ctx, name):
    if name == "plain4m":
        t = synth.plain_4mbp().logical_text()          # k = 10
    elif name == "repeat_rich":
        t = synth.repeat_rich_100mbp(scale=0.01).logical_text()
    else:
        t = synth.human_scale_3gbp(scale=0.0005).logical_text()  # N runs, contigs
    resident = t.size * 12
    k = sg.prefix_select_k(t.size, resident)
    assert k >= 8
    r = ctx.build(t, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32, prefix_k=k)
    if oracle.ref() is not None:
        rk, table, kmers, entries = oracle.ref_prefix_directory(t, resident)
        assert rk == k
        assert r.stats["prefix_kmers"] == kmers and r.stats["prefix_entries"] == entries
    else:
        table = oracle.prefix_directory(t, r.sa_low, k)
    assert (r.prefix_intervals == table).all()


@pytest.mark.parametrize("k", [1, 3, 6])
def test_directory_any_k(ctx, k):
    rng = np.random.default_rng(k)
    t = np.concatenate([rng.integers(2, 7, size=20_000).astype(np.uint8), [1],
                        rng.integers(2, 6, size=5_000).astype(np.uint8), [1, 0]]).astype(np.uint8)
    r = ctx.build(t, sa_bits=32, isa_bits=0, lcp=sg.LcpEncoding.NONE, prefix_k=k)
    sa, _, _ = oracle.full_build(t)
    assert (r.prefix_intervals == oracle.prefix_directory(t, sa, k)).all()


def test_directory_rejections(ctx):
    t = synth.random_text(np.random.default_rng(0), 5000, 4)
    for kwargs in ({"prefix_k": 11}, {"prefix_k": 4, "sampling_rate": 2}):
        with pytest.raises(sg.SufkitError) as e:
            ctx.build(t, sa_bits=32, isa_bits=0, lcp=sg.LcpEncoding.NONE, **kwargs)
        assert e.value.code == sg.ErrorCode.INVALID_INPUT
