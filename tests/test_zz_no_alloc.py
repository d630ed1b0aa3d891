"""GPU: the allocation-free LCP entry point.

sufgpu_lcp_noalloc serves callers that can't call cudaMalloc (code running
under another framework's allocator, inside allocation-locked callbacks, or in
loops that must not block on an allocation): all of its scratch is one fixed
array inside the library.  These tests call it through the C ABI on
device-resident inputs and compare it with the LCP that the regular entry
point (sufgpu_build) produces and with the oracle's Kasai LCP (the
reference's divsufsort64 build when it was compiled, else the C
restatement), on consecutive calls, so stale scratch contents from the
previous call cannot leak into the next result.  The file is named to be
collected last.
"""
import numpy as np
import pytest

import oracle
import sufkit_b200 as sg
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu

MAX = 1 << 18  # SUFGPU_NOALLOC_MAX_SYMBOLS


def _inputs():
    rng = np.random.default_rng(2024)
    repeat_rich = synth.repeat_rich_100mbp(scale=0.0025).logical_text()  # long rows
    runs = np.concatenate([np.tile(np.array([2, 3, 4], np.uint8), 20_000),
                           np.full(9_000, 6, np.uint8), synth.random_text(rng, 50_000, 4)])
    at_limit = synth.random_text(rng, MAX, 2)
    return [repeat_rich, runs, at_limit, repeat_rich]


def _noalloc(lib, torch, text, sa):
    dev = torch.device("cuda", 0)
    d_text = torch.from_numpy(text).to(dev)
    d_sa = torch.from_numpy(sa.view(np.int32)).to(dev)
    d_lcp = torch.full((text.size,), -1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    status = lib.sufgpu_lcp_noalloc(d_text.data_ptr(), d_sa.data_ptr(), text.size,
                                    d_lcp.data_ptr(), None)
    torch.cuda.synchronize()
    return status, d_lcp.cpu().numpy().view(np.uint32)


def _oracle_lcp(text):
    if oracle.ref() is not None:
        return oracle.ref_adapter(text, 64)[2]
    return oracle.full_build(text)[2]


def test_noalloc_lcp_matches_build_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    lib = sg.library()
    with sg.Context(0) as ctx:
        for text in _inputs():
            assert text.size <= MAX
            built = ctx.build(text, sa_bits=32, isa_bits=0, lcp=sg.LcpEncoding.RAW32)
            status, lcp = _noalloc(lib, torch, text, built.sa_low)
            assert status == 0
            assert (lcp == built.lcp).all()
            assert (lcp.astype(np.uint64) == _oracle_lcp(text).astype(np.uint64)).all()


def test_noalloc_flags_suffix_array_entries_out_of_range():
    """An SA entry >= n is caught by the row kernel's range check (the row's
    text compare is skipped, so nothing is read past the text) and the call
    reports a build failure; the next call with a valid SA is exact again."""
    torch = pytest.importorskip("torch")
    lib = sg.library()
    text = synth.random_text(np.random.default_rng(7), 5000, 4)
    sa = oracle.suffix_array(text).astype(np.uint32)
    bad = sa.copy()
    bad[1234] = text.size + 100_000
    status, _ = _noalloc(lib, torch, text, bad)
    assert status == sg.ErrorCode.BUILD_FAILURE + 1
    status, lcp = _noalloc(lib, torch, text, sa)
    assert status == 0
    assert (lcp.astype(np.uint64) == _oracle_lcp(text).astype(np.uint64)).all()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = sg.library()
    # Rejected before any device access, so null pointers are fine here.
    assert lib.sufgpu_lcp_noalloc(None, None, MAX + 1, None, None) == sg.ErrorCode.INVALID_INPUT + 1
