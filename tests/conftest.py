import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "reference_cases.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


def golden_cases():
    data = np.load(GOLDEN)
    names = sorted({k.split("/")[0] for k in data.files})
    return {name: {f: data[f"{name}/{f}"] for f in
                   ("text", "sa", "isa", "lcp", "primary", "anchor_pos", "anchor_val")}
            for name in names}


@pytest.fixture(scope="session")
def golden():
    return golden_cases()


@pytest.fixture(scope="session")
def ctx():
    import sufkit_b200
    c = sufkit_b200.Context(0)
    yield c
    c.close()


# ---------------------------------------------------------------------------
# Direct comparison of a build result with the oracle
# ---------------------------------------------------------------------------
def oracle_build(text):
    """(sa, isa, lcp) as uint64 from the reference's divsufsort64 + Kasai when
    it was compiled, else from the C restatement."""
    import oracle
    if oracle.ref() is not None:
        sa, isa, lcp, _ = oracle.ref_adapter(text, 64)
    else:
        sa, isa, lcp = oracle.full_build(text)
    return sa.astype(np.uint64), isa.astype(np.uint64), lcp.astype(np.uint64)


def _joined(low, high):
    v = np.asarray(low).astype(np.uint64)
    if high is not None:
        v |= np.asarray(high).astype(np.uint64) << np.uint64(32)
    return v


def assert_oracle(result, text, lcp_encoding, expected=None):
    """Every plane of a BuildResult equals the oracle's build of `text`:
    SA (low/high planes joined), ISA when present, raw LCP or the byte-coded
    primaries and anchors (restated from the oracle's SA and ISA)."""
    import oracle
    import sufkit_b200 as sg
    sa, isa, lcp = expected if expected is not None else oracle_build(text)
    assert np.array_equal(_joined(result.sa_low, result.sa_high), sa), "SA differs from the oracle"
    if result.isa_low is not None:
        assert np.array_equal(_joined(result.isa_low, result.isa_high), isa), "ISA differs"
    enc = sg.LcpEncoding(lcp_encoding)
    if enc in (sg.LcpEncoding.RAW32, sg.LcpEncoding.RAW64):
        assert np.array_equal(np.asarray(result.lcp).astype(np.uint64), lcp), "LCP differs"
    elif enc in (sg.LcpEncoding.BYTE32, sg.LcpEncoding.BYTE64):
        width = 32 if enc == sg.LcpEncoding.BYTE32 else 64
        primary, pos, val = oracle.bytecode(text, sa, isa, width)
        assert np.array_equal(result.lcp, primary), "byte-coded primaries differ"
        assert np.array_equal(result.anchor_positions.astype(np.uint64), pos), "anchors differ"
        assert np.array_equal(result.anchor_values.astype(np.uint64), val), "anchor values differ"
