"""CPU: the oracle restatement against the reference's golden vectors and,
where the reference library was built here, against the reference itself."""
import numpy as np
import pytest

import oracle
from sufkit_b200 import synth


def test_port_matches_golden(golden):
    for name, case in golden.items():
        t = case["text"]
        sa, isa, lcp = oracle.full_build(t)
        assert (sa == case["sa"]).all(), name
        assert (isa == case["isa"]).all(), name
        assert (lcp == case["lcp"]).all(), name
        primary, pos, val = oracle.bytecode(t, sa, isa, 32)
        assert (primary == case["primary"]).all(), name
        assert (pos == case["anchor_pos"]).all(), name
        assert (val == case["anchor_val"]).all(), name


def test_golden_logical_text_pins_encoding(golden):
    # tests/test_sufkit.cpp:219-221 (2-contig... 3-record reference.fa)
    expected = [2, 3, 4, 5, 6, 2, 3, 4, 5, 1, 5, 5, 5, 2, 3, 4, 5, 2, 2, 2, 1, 2, 2, 2, 1, 0]
    assert golden["reference_fa"]["text"].tolist() == expected


@pytest.mark.parametrize("n", [1, 2, 3, 7, 64, 1000, 20000])
def test_port_matches_reference_random(n):
    if oracle.ref() is None:
        pytest.skip("reference library not built")
    rng = np.random.default_rng(n)
    for alphabet in (1, 2, 4):
        t = synth.random_text(rng, n, alphabet)
        sa, isa, lcp, _ = oracle.ref_adapter(t)
        psa, pisa, plcp = oracle.full_build(t)
        assert (psa == sa).all() and (pisa == isa).all() and (plcp == lcp).all()
        for width in (32, 64):
            a = oracle.bytecode(t, sa, isa, width)
            b = oracle.ref_bytecode(t, sa, isa, width)
            for x, y in zip(a, b):
                assert (x == y).all()


def test_port_matches_reference_synthetic():
    if oracle.ref() is None:
        pytest.skip("reference library not built")
    t = synth.plain_4mbp(scale=0.05).logical_text()
    sa, isa, lcp, _ = oracle.ref_adapter(t)
    psa, pisa, plcp = oracle.full_build(t)
    assert (psa == sa).all() and (plcp == lcp).all()


def test_bytecode_separate_overflow_runs():
    # tests/test_lcp_storage.cpp:225-245: LCP {0,300,299,10,400,399} with the
    # identity ISA opens anchors at 1 and 4 only.  Text order = row order here.
    lcp = np.array([0, 300, 299, 10, 400, 399], np.uint64)
    opens = [p for p in range(lcp.size)
             if lcp[p] >= 255 and not (p > 0 and lcp[p - 1] == lcp[p] + 1)]
    assert opens == [1, 4]
    if oracle.ref() is not None:
        isa = np.arange(6, dtype=np.uint64)
        _, pos, val = oracle.ref_bytecode_from_raw(lcp, isa, 32)
        assert pos.tolist() == [1, 4] and val.tolist() == [300, 400]


def test_guide_block_boundaries():
    # tests/test_lcp_storage.cpp:247-272: anchors at 4095, 4096, 8193.
    pos = np.array([4095, 4096, 8193], np.uint64)
    g = oracle.guide(pos, 9000)
    # guide[b] = first anchor at or after b * 4096, b = 0..ceil(9000/4096).
    assert g.tolist() == [0, 1, 2, 3]


@pytest.mark.parametrize("bits", [0, 32, 40, 48, 64])
def test_pack_matches_reference(bits):
    if oracle.ref() is None:
        pytest.skip("reference library not built")
    rng = np.random.default_rng(bits)
    symbol_count = {0: 1 << 33, 32: 1 << 32, 40: 1 << 40, 48: 1 << 48, 64: 1 << 50}[bits]
    v = rng.integers(0, symbol_count, size=5000, dtype=np.uint64)
    v[:3] = [0, symbol_count - 1, min(symbol_count - 1, 0xFFFFFFFF)]
    a = oracle.pack(v, symbol_count, bits)
    b = oracle.ref_pack(v, symbol_count, bits)
    assert a[0] == b[0]
    assert (a[1] == b[1]).all()
    if a[2] is not None:
        assert (a[2] == b[2]).all()


def test_pack_rejects_out_of_range():
    with pytest.raises(ValueError):
        oracle.pack(np.array([5], np.uint64), 5, 32)  # value >= symbol count
    with pytest.raises(ValueError):
        oracle.pack(np.array([1], np.uint64), (1 << 32) + 2, 32)  # text too big for 32


@pytest.mark.parametrize("rate", [2, 3, 7, 32])
def test_sampling_restatement_matches_reference(golden, rate):
    """The sampling of a complete build (oracle.sample) equals the reference's
    BuildDivsufsort64 with sampling_rate K (SA, ISA, LCP of sampled rows)."""
    if oracle.ref() is None:
        pytest.skip("reference library not built")
    rng = np.random.default_rng(rate)
    texts = [case["text"] for case in list(golden.values())[:20]]
    texts += [np.concatenate([rng.integers(2, 6, size=n).astype(np.uint8), [0]]).astype(np.uint8)
              for n in (1, 2, 5, 100, 5000)]
    for t in texts:
        sa, isa, lcp, _ = oracle.ref_adapter(t, 64)
        sa_k, isa_k, lcp_k = oracle.sample(sa, lcp, rate)
        r_sa, r_isa, r_lcp = oracle.ref_adapter_sampled(t, rate, 64)
        assert (sa_k == r_sa.astype(np.int64)).all()
        assert (isa_k == r_isa.astype(np.int64)).all()
        assert (lcp_k == r_lcp.astype(np.int64)).all()


def test_prefix_directory_restatement_matches_reference():
    """oracle.prefix_directory (from the SA) equals the reference's
    FastPrefixIndex (built from its own SA/ISA, read back with Lookup)."""
    if oracle.ref() is None:
        pytest.skip("reference library not built")
    texts = [synth.plain_4mbp(scale=0.2).logical_text(),
             synth.repeat_rich_100mbp(scale=0.003).logical_text()]
    for t, want_k in zip(texts, (9, 8)):
        resident = t.size * 12  # SA + ISA + LCP, 32-bit
        k, table, kmers, entries = oracle.ref_prefix_directory(t, resident)
        assert k == want_k
        import sufkit_b200 as sg
        assert sg.prefix_select_k(t.size, resident) == k
        sa = oracle.ref_divsufsort64(t)
        mine = oracle.prefix_directory(t, sa, k)
        assert (mine == table).all()
        assert int((mine != (t.size | (t.size << 32))).sum()) == entries


def test_child_restatement_matches_reference_sufidx(tmp_path):
    """The C restatement of BuildChildFor equals the CHILD section the
    reference's SuffixArray::Build saves (acceleration kLcpChild)."""
    from sufkit_b200 import synth
    if oracle.ref() is None:
        pytest.skip("the reference library was not built")
    refs = [synth.repeat_rich_100mbp(scale=0.001), synth.human_scale_3gbp(scale=0.0002),
            synth.plain_4mbp(scale=0.005),
            synth.strain_collection(4, 5_000, np.random.default_rng(2))]
    for i, ref in enumerate(refs):
        fasta = tmp_path / f"{i}.fa"
        ref.write_fasta(fasta)
        out = oracle.sufkit_index(fasta, tmp_path / f"{i}.sufidx", 0, 32, 32, acceleration=2)
        assert out["rc"] == 0, out.get("error")
        child = oracle.sufidx_coordinates(tmp_path / f"{i}.sufidx", oracle.SECTION_CHILD)
        sa_file = oracle.sufidx_coordinates(tmp_path / f"{i}.sufidx", oracle.SECTION_SUFFIX_ARRAY)
        sa, isa, lcp = oracle.full_build(ref.logical_text())
        assert np.array_equal(sa_file, sa)
        assert np.array_equal(oracle.child(lcp), child)


def test_child_restatement_edge_cases():
    # Decreasing, increasing, constant and single-row LCP arrays.
    for lcp in ([0], [0, 5, 4, 3, 2, 1], [0, 1, 2, 3, 4], [0, 2, 2, 2, 2], [3, 1, 3, 1, 3]):
        out = oracle.child(np.array(lcp, np.uint64))
        assert out.size == len(lcp) and (out <= len(lcp)).all()


def test_sampled_bytecode_restatement_matches_reference():
    """oracle.sample_bytecode (the sampled byte coding restated from a sampled
    build's SA, ISA and LCP) equals LcpStorage::BuildByteCodedDirect with
    sampling rate K."""
    from sufkit_b200 import synth
    if oracle.ref() is None:
        pytest.skip("the reference library was not built")
    rng = np.random.default_rng(4)
    texts = [synth.strain_collection(3, 3000, rng).logical_text(),
             np.concatenate([np.full(1500, 2, np.uint8), np.zeros(1, np.uint8)]),
             synth.human_scale_3gbp(scale=0.0002).logical_text()]
    for t in texts:
        for rate in (2, 5, 255, 256, 400):
            sa, isa, lcp = oracle.ref_adapter_sampled(t, rate)
            for width in (32, 64):
                a = oracle.ref_bytecode_sampled(t, sa, isa, rate, width)
                b = oracle.sample_bytecode(sa, isa, lcp, rate)
                assert all(np.array_equal(x, y) for x, y in zip(a, b)), (t.size, rate, width)


def test_caps_sa_baseline_matches_divsufsort():
    """The CaPS-SA constructor sufkit vendors (compiled into the oracle as the
    second CPU baseline) gives divsufsort's SA and LCP."""
    from sufkit_b200 import synth
    if oracle.ref() is None:
        pytest.skip("the reference library was not built")
    rng = np.random.default_rng(12)
    for t in (synth.repeat_rich_100mbp(scale=0.002).logical_text(),
              synth.human_scale_3gbp(scale=0.0001).logical_text(),
              synth.random_text(rng, 5000, 2)):
        sa, lcp, sec = oracle.ref_caps(t, threads=4)
        ref_sa, _, ref_lcp, _ = oracle.ref_adapter(t, 64)
        assert np.array_equal(sa, ref_sa) and np.array_equal(lcp, ref_lcp) and sec >= 0
