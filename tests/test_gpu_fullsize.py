"""GPU: parity at the workloads' full sizes.

* repeat-rich 100 Mbp (Fast profile: SA + ISA + raw LCP32): word for word
  against the reference's divsufsort64 + Kasai (detail::BuildDivsufsort64,
  compiled from its sources);
* bacterial collection, all 1,024 references (~4.5 Gsym, SA + raw LCP32,
  built as a collection in sub-batches): every reference word for word
  against divsufsort64, compared by blake2b digests of the rows; the
  reference builds run in spawned worker processes on the host's cores while
  the GPU builds;
* human-scale 3.1 Gbp (Low-memory profile: split40 SA, byte-coded LCP with
  32-bit anchors): a word-for-word CPU build does not fit the test's time and
  host memory, so the full build is checked through size-independent
  properties on the device (verify.check_suffix_array_device: permutation,
  order at the first mismatch, equal prefixes by two polynomial hashes) on the
  exact SA and LCP of a raw build of the same text, and the Low-memory planes
  (split40 SA, byte primaries, anchors) are compared word for word with that
  build and with the byte coding restated from it on the device;
* one served strain collection at full size (50 copies of a 2 Mbp genome at
  0.1% SNP + 0.01% indel, so most suffixes share kbp prefixes with 49 others):
  SA and byte-coded LCP against divsufsort64.
"""
import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor

import numpy as np
import pytest

import oracle
import sufkit_b200 as sg
from sufkit_b200 import synth, verify

pytestmark = pytest.mark.gpu


def _need_reference():
    if oracle.ref() is None:
        pytest.skip("the reference library was not built")


def test_repeat_rich_100mbp_full_size_word_for_word():
    _need_reference()
    text = synth.repeat_rich_100mbp().logical_text()
    assert text.size == 100_000_025
    with sg.Context(0) as ctx:
        r = ctx.build(text, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32, validate=True)
    sa, isa, lcp, _ = oracle.ref_adapter(text, 64)
    assert np.array_equal(r.sa_low, sa.astype(np.uint32)), "SA differs"
    assert np.array_equal(r.isa_low, isa.astype(np.uint32)), "ISA differs"
    assert np.array_equal(r.lcp, lcp.astype(np.uint32)), "LCP differs"


def test_bacterial_collection_all_1024_references_word_for_word():
    _need_reference()
    count = 1024
    sizes = synth.uneven_sizes(count)
    workers = max(1, min(32, (os.cpu_count() or 2) - 1))
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        # Reference builds first (they take longest), GPU builds meanwhile.
        futures = [ex.submit(oracle.uneven_reference_digests, (i, sizes[i])) for i in range(count)]
        ours = {}
        with sg.Context(0) as ctx:
            step = 128
            for s in range(0, count, step):
                idx = list(range(s, min(count, s + step)))
                texts = synth.uneven_texts(count, indices=idx, workers=workers)
                results = ctx.build_collection(texts, sa_bits=32, isa_bits=0,
                                               lcp=sg.LcpEncoding.RAW32, batch_symbols=300_000_000)
                for i, t, r in zip(idx, texts, results):
                    ours[i] = (int(t.size),) + oracle.digest_planes(r.sa_low, r.lcp)
        total = 0
        for f in futures:
            i, n, d_sa, d_lcp = f.result()
            assert ours[i][0] == n
            assert ours[i][1] == d_sa, f"reference {i}: SA differs"
            assert ours[i][2] == d_lcp, f"reference {i}: LCP differs"
            total += n
    assert total > 4_000_000_000


def test_human_scale_3gbp_full_size_device_checked():
    torch = pytest.importorskip("torch")
    text = synth.human_scale_3gbp().logical_text()
    n = int(text.size)
    assert n > 3_000_000_000
    dev = torch.device("cuda", 0)
    d_text = torch.from_numpy(text).to(dev)
    i32 = torch.int32
    with sg.Context(0) as ctx:
        # The Low-memory build as the profile stores it.
        low = torch.empty(n, dtype=i32, device=dev)
        high = torch.empty(n, dtype=torch.uint8, device=dev)
        prim = torch.empty(n, dtype=torch.uint8, device=dev)
        ctx.build_device(d_text.data_ptr(), n, {"sa_low": low.data_ptr(), "sa_high": high.data_ptr(),
                                                "lcp": prim.data_ptr()},
                         sa_bits=40, isa_bits=0, lcp=sg.LcpEncoding.BYTE32, validate=True)
        anchor_pos, anchor_val = ctx.last_anchors
        # The same text with raw LCP32: the exact rows the properties check.
        sa = torch.empty(n, dtype=i32, device=dev)
        lcp = torch.empty(n, dtype=i32, device=dev)
        ctx.build_device(d_text.data_ptr(), n, {"sa_low": sa.data_ptr(), "lcp": lcp.data_ptr()},
                         sa_bits=32, isa_bits=0, lcp=sg.LcpEncoding.RAW32)
    assert bool((low == sa).all().item()), "split40 low plane differs from the SA"
    assert int(high.max().item()) == 0, "split40 high plane must be 0 below 2^32"
    del low, high
    torch.cuda.empty_cache()
    verify.check_suffix_array_device(d_text, sa, lcp, torch)
    primary, pos, val = verify.bytecode_device(sa, lcp, torch)
    assert bool((primary == prim).all().item()), "byte-coded primaries differ"
    assert pos.numel() == anchor_pos.size > 0
    assert np.array_equal(pos.cpu().numpy(), anchor_pos.astype(np.int64)), "anchor positions differ"
    assert np.array_equal(val.cpu().numpy(), anchor_val.astype(np.int64)), "anchor values differ"


def test_served_strain_collection_full_size_against_divsufsort():
    _need_reference()
    ref = synth.strain_collection(50, 2_000_000, np.random.default_rng(20260826))
    text = ref.logical_text()
    assert text.size > 99_000_000
    with sg.Server(0, capacity_symbols=1 << 28, max_instances=8) as server:
        ticket = server.submit(text, 32, 0, sg.LcpEncoding.BYTE32)
        r = server.wait(ticket)
    sa, isa, lcp, _ = oracle.ref_adapter(text, 64)
    assert int(lcp.max()) > 1_000  # copies agree over kbp stretches between their SNPs
    assert np.array_equal(r.sa_low, sa.astype(np.uint32)), "SA differs"
    primary, pos, val = oracle.bytecode(text, sa, isa, 32)
    assert np.array_equal(r.lcp, primary), "byte-coded primaries differ"
    assert np.array_equal(r.anchor_positions.astype(np.uint64), pos), "anchor positions differ"
    assert np.array_equal(r.anchor_values.astype(np.uint64), val), "anchor values differ"


def _mem_available_gb() -> float:
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable"):
                return int(line.split()[1]) / 1048576
    except OSError:
        pass
    return 0.0


@pytest.mark.skipif(os.environ.get("SUFGPU_FULL_REFERENCE_3G") != "1",
                    reason="opt-in (SUFGPU_FULL_REFERENCE_3G=1): divsufsort64 at 3.1 Gsym takes "
                           "about 10 minutes and 80 GB of host memory")
def test_human_scale_3gbp_word_for_word_against_divsufsort64():
    """The full 3.1 Gbp build word for word against the reference's
    BuildDivsufsort64 (SA and LCP compared by blake2b digests of their rows).
    Needs about 110 GB of free host memory; skipped below that."""
    torch = pytest.importorskip("torch")
    _need_reference()
    if _mem_available_gb() < 110:
        pytest.skip("not run: host RAM")
    text = synth.human_scale_3gbp().logical_text()
    n = int(text.size)
    dev = torch.device("cuda", 0)
    d_text = torch.from_numpy(text).to(dev)
    sa = torch.empty(n, dtype=torch.int32, device=dev)
    lcp = torch.empty(n, dtype=torch.int32, device=dev)
    with sg.Context(0) as ctx:
        ctx.build_device(d_text.data_ptr(), n, {"sa_low": sa.data_ptr(), "lcp": lcp.data_ptr()},
                         sa_bits=32, isa_bits=0, lcp=sg.LcpEncoding.RAW32, validate=True)
    ours = oracle.digest_planes(sa.cpu().numpy().view(np.uint32), lcp.cpu().numpy().view(np.uint32))
    del sa, lcp, d_text
    torch.cuda.empty_cache()
    ref_sa, _, ref_lcp, _ = oracle.ref_adapter(text, 64)
    assert ours == oracle.digest_planes(ref_sa, ref_lcp)
