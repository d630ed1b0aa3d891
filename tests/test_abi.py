"""CPU: the C-ABI library loads, exports every declared entry point, and its
FASTA normalizer equals GenomeReference::FromFasta (no GPU needed)."""
import gzip
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
import sufkit_b200 as sg

HEADER = Path(__file__).resolve().parents[1] / "include" / "sufgpu" / "sufgpu.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"SUFGPU_API[^;(]*?\b(sufgpu_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = sg.library()
    declared = declared_symbols()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(sg.exported_symbols()) == sorted(declared)


def test_max_symbols_and_device_bytes():
    lib = sg.library()
    assert lib.sufgpu_max_symbols() == 2**32 - 1
    b = lib.sufgpu_device_bytes(100_000_025, None)
    assert 30 * 100_000_025 < b < 45 * 100_000_025


FASTA_CASES = {
    "plain": b">chr1 first\nACGTNACGT\n>chr2 second\nTTTACGTAAA\n>chr3 third\nAAA\n",
    "crlf": b">a desc\r\nACGT\r\nacgt\r\n>b\r\nNNNN\r\n",
    "blank_lines": b"\n\n>x\n\nAC\n\nGT\n>y\nRYKM acgt\n",
    "iupac_lower": b">q\nacgtnRYSWKMBDHVN-.*\n",
    "no_trailing_newline": b">z\nACGTACGT",
    "fastq": b"@r1\nACGT\n+\nIIII\n@r2\nGGCC\n+r2\nIIII\n",
    "tabs_spaces": b">t\tcomment here\nAC GT\tAC\n",
    "header_at_eof": b">a\nACGT\n>",
}
BAD_CASES = {
    "empty_name": b">\nACGT\n",
    "duplicate": b">a\nAC\n>a\nGT\n",
    "empty_sequence": b">a\n>b\nAC\n",
    "no_records": b"ACGT\n",
}


@pytest.mark.parametrize("name", sorted(FASTA_CASES))
def test_encode_fasta_matches_reference(tmp_path, name):
    path = tmp_path / f"{name}.fa"
    path.write_bytes(FASTA_CASES[name])
    ours, fp, _ = sg.encode_fasta(path)
    if oracle.ref() is None:
        pytest.skip("reference library not built")
    ref, ref_fp = oracle.ref_encode_fasta(path)
    assert ours.tolist() == ref.tolist()
    assert fp == ref_fp
    gz = tmp_path / f"{name}.fa.gz"
    gz.write_bytes(gzip.compress(FASTA_CASES[name]))
    ours_gz, fp_gz, _ = sg.encode_fasta(gz)
    assert ours_gz.tolist() == ref.tolist() and fp_gz == ref_fp


@pytest.mark.parametrize("name", sorted(BAD_CASES))
def test_encode_fasta_rejects_like_reference(tmp_path, name):
    path = tmp_path / f"{name}.fa"
    path.write_bytes(BAD_CASES[name])
    with pytest.raises(sg.SufkitError) as err:
        sg.encode_fasta(path)
    assert err.value.code == sg.ErrorCode.INVALID_INPUT
    if oracle.ref() is not None:
        with pytest.raises(ValueError):
            oracle.ref_encode_fasta(path)


def test_encode_fasta_missing_file(tmp_path):
    with pytest.raises(sg.SufkitError) as err:
        sg.encode_fasta(tmp_path / "missing.fa")
    assert err.value.code == sg.ErrorCode.IO_ERROR


def test_synthetic_fasta_round_trip(tmp_path):
    from sufkit_b200 import synth
    ref = synth.plain_4mbp(scale=0.002)
    path = tmp_path / "w1.fa"
    ref.write_fasta(path)
    ours, _, records = sg.encode_fasta(path)
    assert records == 4
    assert ours.tolist() == ref.encoded().tolist()
    if oracle.ref() is not None:
        theirs, _ = oracle.ref_encode_fasta(path)
        assert (theirs == ours).all()


def test_context_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(sg.SufkitError) as err:
        sg.Context(0)
    assert err.value.code == sg.ErrorCode.BUILD_FAILURE


def test_sufkit_dropin_library_fails_loudly_without_a_device(tmp_path):
    """sufkit's own Build through the drop-in constructor raises
    sufkit::Error(kBuildFailure) when no CUDA device is usable: there is no
    CPU fallback behind it."""
    import oracle
    import torch
    from sufkit_b200 import synth
    if not oracle.REF_CUDA_PATH.exists():
        pytest.skip("libsufref_cuda.so was not built")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    fasta = tmp_path / "a.fa"
    synth.plain_4mbp(scale=0.01).write_fasta(fasta)
    out = oracle.sufkit_index(fasta, tmp_path / "g.sufidx", 0, 32, 32, cuda=True)
    assert out["rc"] == 6  # 1 + ErrorCode::kBuildFailure
    assert "CUDA" in out["error"]
    assert not (tmp_path / "g.sufidx").exists()


def test_divsufsort_abi_library_exports_exactly_libdivsufsorts_entry_points():
    """libdivsufsort_cuda.so exports divsufsort and divsufsort64, as
    include/sufgpu/divsufsort_cuda.h declares them, and nothing else; without
    a device both return -2 (divsufsort's allocation-failure code) and reject
    bad arguments with -1."""
    import ctypes
    import subprocess
    import torch
    root = Path(__file__).resolve().parents[1]
    lib_path = root / "sufkit_b200" / "libdivsufsort_cuda.so"
    header = (root / "include" / "sufgpu" / "divsufsort_cuda.h").read_text()
    declared = sorted(re.findall(r"saint_t\s+(divsufsort\w*)\s*\(", header))
    assert declared == ["divsufsort", "divsufsort64"]
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True,
                         text=True, check=True).stdout
    exported = sorted(line.split()[-1] for line in out.splitlines() if " T " in line)
    assert exported == declared
    lib = ctypes.CDLL(str(lib_path))
    lib.divsufsort64.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
    lib.divsufsort.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32]
    t = np.array([3, 2, 0], np.uint8)
    sa = np.zeros(3, np.int64)
    assert lib.divsufsort64(None, sa.ctypes.data, 3) == -1
    assert lib.divsufsort64(t.ctypes.data, sa.ctypes.data, -1) == -1
    if not torch.cuda.is_available():
        assert lib.divsufsort64(t.ctypes.data, sa.ctypes.data, 3) == -2
