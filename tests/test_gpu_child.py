"""GPU: the compact CHILD table against the reference.

The expected table is the CHILD section of a .sufidx that the reference's own
SuffixArray::Build (acceleration kLcpChild) saved for the same FASTA, read
back from the file; texts without a FASTA form use the C restatement of
BuildChildFor (pinned against those files by tests/test_oracle.py)."""
import numpy as np
import pytest

import oracle
import sufkit_b200 as sg
from conftest import oracle_build
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu

LCP_CHILD = 2  # sufkit::SaAcceleration::kLcpChild


@pytest.mark.parametrize("make", [lambda: synth.repeat_rich_100mbp(scale=0.01),
                                  lambda: synth.human_scale_3gbp(scale=0.001),
                                  lambda: synth.strain_collection(6, 40_000,
                                                                  np.random.default_rng(3))],
                         ids=["repeat-rich", "human-scale", "strains"])
def test_child_equals_reference_sufidx(ctx, tmp_path, make):
    if oracle.ref() is None:
        pytest.skip("the reference library was not built")
    ref = make()
    fasta = tmp_path / "r.fa"
    ref.write_fasta(fasta)
    out = oracle.sufkit_index(fasta, tmp_path / "r.sufidx", 0, 32, 32, acceleration=LCP_CHILD)
    assert out["rc"] == 0, out.get("error")
    expected = oracle.sufidx_coordinates(tmp_path / "r.sufidx", oracle.SECTION_CHILD)
    text = ref.logical_text()
    for enc in (sg.LcpEncoding.RAW32, sg.LcpEncoding.BYTE32):
        r = ctx.build(text, sa_bits=32, isa_bits=0, lcp=enc, child=True)
        assert np.array_equal(r.child.astype(np.uint64), expected), "CHILD differs"


def test_child_edge_cases(ctx):
    rng = np.random.default_rng(8)
    texts = [np.array([0], np.uint8), np.array([3, 0], np.uint8),
             np.concatenate([np.full(70_000, 2, np.uint8), np.zeros(1, np.uint8)]),  # rising LCP
             np.tile(np.array([2, 3, 4], np.uint8), 20_000),
             synth.random_text(rng, 100_000, 2), synth.random_text(rng, 40_000, 4, sentinel=False),
             rng.integers(0, 256, size=50_000).astype(np.uint8)]
    for t in texts:
        _, _, lcp = oracle_build(t)
        r = ctx.build(t, sa_bits=32, isa_bits=0, lcp=sg.LcpEncoding.RAW32, child=True)
        assert np.array_equal(r.child.astype(np.uint64), oracle.child(lcp)), t.size


def test_child_rejects_what_it_cannot_build(ctx):
    t = synth.random_text(np.random.default_rng(1), 1000, 4)
    with pytest.raises(sg.SufkitError):
        ctx.build(t, lcp=sg.LcpEncoding.NONE, child=True)
    with pytest.raises(sg.SufkitError):
        ctx.build(t, lcp=sg.LcpEncoding.RAW32, sampling_rate=4, child=True)
