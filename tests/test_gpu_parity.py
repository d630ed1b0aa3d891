"""GPU parity: every build through the C ABI equals the reference's
divsufsort64 build (SA, ISA, Kasai LCP, byte-coded LCP, packed planes) word
for word."""
import numpy as np
import pytest

import oracle
import sufkit_b200 as sg
from sufkit_b200 import synth, verify

pytestmark = pytest.mark.gpu


def expected(text):
    """(sa, isa, lcp) from the reference when built here, else the port."""
    if oracle.ref() is not None:
        sa, isa, lcp, _ = oracle.ref_adapter(text, 64)
        return sa, isa, lcp
    return oracle.full_build(text)


def check_full(ctx, text, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32):
    text = np.ascontiguousarray(text, np.uint8)
    sa, isa, lcp_ref = expected(text)
    r = ctx.build(text, sa_bits=sa_bits, isa_bits=isa_bits, lcp=lcp, validate=True)
    assert (r.sa == sa).all(), "SA differs"
    if isa_bits:
        assert (r.isa == isa).all(), "ISA differs"
    if lcp in (sg.LcpEncoding.RAW32, sg.LcpEncoding.RAW64):
        assert (r.lcp.astype(np.uint64) == lcp_ref).all(), "LCP differs"
    elif lcp in (sg.LcpEncoding.BYTE32, sg.LcpEncoding.BYTE64):
        width = 32 if lcp == sg.LcpEncoding.BYTE32 else 64
        primary, pos, val = oracle.bytecode(text, sa, isa, width)
        assert (r.lcp == primary).all(), "primary bytes differ"
        assert (r.anchor_positions.astype(np.uint64) == pos).all(), "anchor positions differ"
        assert (r.anchor_values.astype(np.uint64) == val).all(), "anchor values differ"
    return r


def test_golden_cases(ctx, golden):
    for name, case in golden.items():
        t = case["text"]
        r = ctx.build(t, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32, validate=True)
        assert (r.sa_low == case["sa"]).all(), name
        assert (r.isa_low == case["isa"]).all(), name
        assert (r.lcp == case["lcp"]).all(), name
        b = ctx.build(t, sa_bits=32, isa_bits=0, lcp=sg.LcpEncoding.BYTE32)
        assert (b.lcp == case["primary"]).all(), name
        assert (b.anchor_positions == case["anchor_pos"]).all(), name
        assert (b.anchor_values == case["anchor_val"]).all(), name


@pytest.mark.parametrize("n", [1, 2, 3, 4, 15, 16, 17, 255, 4095, 4096, 4097, 65537])
def test_small_sizes(ctx, n):
    rng = np.random.default_rng(n)
    for alphabet in (1, 2, 4):
        check_full(ctx, synth.random_text(rng, n, alphabet))


def test_no_sentinel_arbitrary_bytes(ctx):
    rng = np.random.default_rng(7)
    for n in (1, 2, 10, 1000, 50000):
        check_full(ctx, rng.integers(0, 256, size=n).astype(np.uint8))
        check_full(ctx, np.full(n, 65, np.uint8))
        check_full(ctx, np.tile(np.array([1, 2, 1], np.uint8), n)[:n])


def test_periodic_and_runs(ctx):
    # Long runs and short periods force the most doubling rounds.
    for period in (1, 2, 3, 7, 50):
        unit = (np.arange(period) % 4 + 2).astype(np.uint8)
        body = np.tile(unit, 200_000 // period + 1)[:200_000]
        check_full(ctx, np.concatenate([body, np.array([1, 0], np.uint8)]))


@pytest.mark.parametrize("sa_bits", [32, 40, 48, 64])
def test_storage_widths(ctx, sa_bits):
    t = synth.plain_4mbp(scale=0.01).logical_text()
    check_full(ctx, t, sa_bits=sa_bits, isa_bits=sa_bits, lcp=sg.LcpEncoding.RAW64)
    r = ctx.build(t, sa_bits=sa_bits, isa_bits=sa_bits)
    if sa_bits in (40, 48):
        assert r.sa_high is not None and not r.sa_high.any()
        _, low, high = oracle.pack(r.sa, t.size, sa_bits)
        assert (low == r.sa_low).all() and (high == r.sa_high).all()


@pytest.mark.parametrize("width", [32, 64])
def test_byte_coded(ctx, width):
    enc = sg.LcpEncoding.BYTE32 if width == 32 else sg.LcpEncoding.BYTE64
    t = synth.repeat_rich_100mbp(scale=0.005).logical_text()
    check_full(ctx, t, isa_bits=0, lcp=enc)
    # Overflow anchors from long runs and tandem repeats.
    runs = np.concatenate([np.full(3000, 6, np.uint8), np.array([2, 3], np.uint8),
                           np.full(1000, 6, np.uint8), np.array([1, 0], np.uint8)])
    check_full(ctx, runs, isa_bits=0, lcp=enc)


def test_workload1_full_size(ctx):
    """Workload 1 (4,000,005 symbols): word for word against the reference."""
    t = synth.plain_4mbp().logical_text()
    r = check_full(ctx, t)
    assert r.stats["symbols"] == 4_000_005


def test_workload2_scaled_word_for_word(ctx):
    t = synth.repeat_rich_100mbp(scale=0.05).logical_text()
    check_full(ctx, t)


def test_workload2_full_size_properties(ctx):
    """Workload 2 at 100,000,025 symbols: size-independent exactness checks
    (permutation, equal prefixes by hash, ordered first mismatch, ISA inverse)."""
    t = synth.repeat_rich_100mbp().logical_text()
    r = ctx.build(t, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32, validate=True)
    verify.check_suffix_array(t, r.sa_low, r.lcp)
    isa = r.isa_low.astype(np.int64)
    assert (r.sa_low[isa] == np.arange(t.size)).all()


def test_strain_collection_long_lcp(ctx):
    ref = synth.strain_collection(copies=8, genome_bp=200_000)
    check_full(ctx, ref.logical_text(), isa_bits=0, lcp=sg.LcpEncoding.BYTE32)


def test_divsufsort_dropins(ctx):
    t = synth.plain_4mbp(scale=0.01).logical_text()
    sa, _, _ = expected(t)
    assert (ctx.divsufsort64(t) == sa.astype(np.int64)).all()
    assert (ctx.divsufsort(t) == sa.astype(np.int32)).all()
    if oracle.ref() is not None:
        assert (ctx.divsufsort64(t) == oracle.ref_divsufsort64(t)).all()


def test_build_cuda_mirror(ctx):
    t = synth.plain_4mbp(scale=0.01).logical_text()
    sa, isa, lcp = expected(t)
    r64 = sg.build_cuda64(t, 1, True, True, 1)
    assert r64.suffix_array.dtype == np.int64 and (r64.suffix_array == sa.astype(np.int64)).all()
    assert (r64.isa == isa).all() and (r64.lcp == lcp).all()
    r32 = sg.build_cuda32(t, 1, True, False, 1)
    assert r32.suffix_array.dtype == np.int32 and (r32.lcp == lcp).all()
    assert r32.isa.size == 0
    sa_k, isa_k, lcp_k = oracle.sample(sa, lcp, 2)
    r2 = sg.build_cuda32(t, 2, True, True, 1)
    assert (r2.suffix_array == sa_k).all() and (r2.isa == isa_k).all() and (r2.lcp == lcp_k).all()
    with pytest.raises(sg.SufkitError) as e:
        sg.build_cuda32(t, 0, True, False, 1)
    assert e.value.code == sg.ErrorCode.INVALID_INPUT


def test_invalid_inputs(ctx):
    t = np.zeros(4, np.uint8)
    with pytest.raises(sg.SufkitError) as e:
        ctx.build(t, sa_bits=33)
    assert e.value.code == sg.ErrorCode.INVALID_INPUT
    r = ctx.build(np.zeros(0, np.uint8))
    assert r.sa_low.size == 0


def test_workload3_scaled_low_memory(ctx):
    """Workload 3 shape at 1% (31 Mbp, long N runs and segmental duplications):
    split40 SA and byte-coded LCP word for word against the reference."""
    t = synth.human_scale_3gbp(scale=0.01).logical_text()
    r = check_full(ctx, t, sa_bits=40, isa_bits=0, lcp=sg.LcpEncoding.BYTE32)
    # The N runs are split directly after the seed instead of by ~17 rounds.
    assert r.stats["long_runs"] > 0 and r.stats["rounds"] < 10


def test_libdivsufsort_abi_library(ctx):
    """sufkit_b200/libdivsufsort_cuda.so: divsufsort / divsufsort64 with
    libdivsufsort's exact C ABI equal the reference's divsufsort64."""
    import ctypes
    from pathlib import Path
    lib = ctypes.CDLL(str(Path(sg.__file__).resolve().parent / "libdivsufsort_cuda.so"))
    lib.divsufsort64.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
    lib.divsufsort.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32]
    rng = np.random.default_rng(31)
    for t in (synth.plain_4mbp(scale=0.02).logical_text(), synth.random_text(rng, 1, 4),
              rng.integers(0, 256, size=5000).astype(np.uint8)):
        sa, _, _ = expected(t)
        sa64 = np.empty(t.size, np.int64)
        sa32 = np.empty(t.size, np.int32)
        assert lib.divsufsort64(t.ctypes.data, sa64.ctypes.data, t.size) == 0
        assert lib.divsufsort(t.ctypes.data, sa32.ctypes.data, t.size) == 0
        assert (sa64 == sa.astype(np.int64)).all() and (sa32 == sa.astype(np.int32)).all()
        if oracle.ref() is not None:
            assert (sa64 == oracle.ref_divsufsort64(t)).all()


@pytest.mark.parametrize("slots", [0, 2])
def test_rank_write_by_slots_or_passes(ctx, slots):
    """The seed rank write of a single text by window slots (rank_slots=2)
    and by radix passes (0) give the same (oracle-equal) build."""
    t = synth.repeat_rich_100mbp(scale=0.03).logical_text()
    ctx.set_tuning("rank_slots", slots)
    try:
        check_full(ctx, t, isa_bits=32, lcp=sg.LcpEncoding.RAW32)
    finally:
        ctx.set_tuning("rank_slots", 1)


@pytest.mark.parametrize("shape", [("sort_block", 256, 512), ("keys_sort_block", 256, 512),
                                   ("sort_tile", 4096, 2048)])
def test_onesweep_tile_shapes(ctx, shape):
    """Onesweep passes of 256 x 16, 512 x 8 and 256 x 8 keys per block, for
    key-value sorts (unpacked seed) and keys-only sorts (packed seed, rank
    grouping): the same (oracle-equal) build."""
    knob, default, other = shape
    ctx.set_tuning(knob, other)
    try:
        for t in (synth.repeat_rich_100mbp(scale=0.03).logical_text(),   # unpacked seed
                  synth.plain_4mbp(scale=0.5).logical_text()):          # packed seed
            check_full(ctx, t, isa_bits=32, lcp=sg.LcpEncoding.RAW32)
    finally:
        ctx.set_tuning(knob, default)


@pytest.mark.parametrize("cluster", [0, 2, 4])
def test_rank_write_cluster_windows(ctx, cluster):
    """The single-text rank write through 65536-position windows held by a
    cluster of two or four blocks (one grouping pass for 22 position bits,
    none for 16) or through 2048-position windows (two passes, one): the same
    (oracle-equal) build."""
    rng = np.random.default_rng(16)
    ctx.set_tuning("rank_cluster", cluster)
    try:
        for t in (synth.repeat_rich_100mbp(scale=0.03).logical_text(),   # 3 Mbp: 22 bits
                  synth.random_text(rng, 60_000, 4),                     # 16 bits
                  synth.random_text(rng, 65_536, 4)):                    # one full window
            check_full(ctx, t, isa_bits=32, lcp=sg.LcpEncoding.RAW32)
    finally:
        ctx.set_tuning("rank_cluster", 2)


@pytest.mark.parametrize("fused", [0, 1])
@pytest.mark.parametrize("two_bit", [0, 1])
def test_seed_first_pass_fused_or_separate(ctx, fused, two_bit):
    """Seed keys generated by the kernel that also does the first radix pass,
    or written in position order and sorted by the separate passes: the same
    (oracle-equal) build, for code-table and two-bit seeds, packed and not."""
    for t in (synth.repeat_rich_100mbp(scale=0.02).logical_text(),     # > 2^24: unpacked
              synth.human_scale_3gbp(scale=0.002).logical_text(),      # N runs
              synth.plain_4mbp(scale=0.5).logical_text()):             # packed
        ctx.set_tuning("seed_fused", fused)
        ctx.set_tuning("two_bit_min", 0 if two_bit else 1 << 62)
        try:
            check_full(ctx, t, isa_bits=32, lcp=sg.LcpEncoding.RAW32)
            check_full(ctx, t, sa_bits=40, isa_bits=0, lcp=sg.LcpEncoding.BYTE32)
        finally:
            ctx.set_tuning("seed_fused", 1)
            ctx.set_tuning("two_bit_min", 1 << 22)


@pytest.mark.parametrize("tma", [0, 1])
def test_onesweep_bulk_tile_load(ctx, tma):
    """Single-segment radix passes with the tile's keys loaded by one bulk
    (TMA) copy or by per-thread loads: the same (oracle-equal) build."""
    t = synth.repeat_rich_100mbp(scale=0.03).logical_text()
    ctx.set_tuning("tma_tile", tma)
    try:
        check_full(ctx, t, isa_bits=32, lcp=sg.LcpEncoding.RAW32)
        check_full(ctx, synth.random_text(np.random.default_rng(3), 9_999, 2))
    finally:
        ctx.set_tuning("tma_tile", 0)


@pytest.mark.parametrize("long_run", [0, 1])
def test_seed_histograms_short_or_long_runs(ctx, long_run):
    """Seed digit histograms counted with 16 or 64 keys per thread (the
    counting kernel of the fused first pass): the same (oracle-equal) build
    for two-bit and code-table seeds, packed or not, and for a batch whose
    tiles cross instance boundaries."""
    rng = np.random.default_rng(64)
    ctx.set_tuning("seed_count_run", long_run)
    try:
        for t in (synth.repeat_rich_100mbp(scale=0.02).logical_text(),
                  synth.human_scale_3gbp(scale=0.002).logical_text(),
                  synth.plain_4mbp(scale=0.5).logical_text(),
                  synth.random_text(rng, 70_000, 20)):
            check_full(ctx, t, isa_bits=32, lcp=sg.LcpEncoding.RAW32)
        texts = [synth.random_text(rng, int(m), 4) for m in rng.integers(1, 30_000, size=12)]
        rs = ctx.build_batch(texts, sa_bits=32, isa_bits=0, lcp=sg.LcpEncoding.RAW32)
        for t, r in zip(texts, rs):
            sa, _, lcp = expected(t)
            assert (r.sa == sa).all() and (r.lcp.astype(np.uint64) == lcp).all()
    finally:
        ctx.set_tuning("seed_count_run", 1)
