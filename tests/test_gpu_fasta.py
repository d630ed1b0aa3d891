"""GPU: FASTA normalisation and fingerprint on the device against the
reference's GenomeReference::FromFasta (compiled from its sources): the
logical bytes and the FNV-1a 64 fingerprint must be identical, for the FASTA
shapes kseq accepts (line widths, CRLF, lowercase and IUPAC codes, blank lines,
descriptions, bytes before the first header, '>' inside a sequence line)."""
import numpy as np
import pytest

import oracle
import sufkit_b200 as sg
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu


def _need_reference():
    if oracle.ref() is None:
        pytest.skip("the reference library was not built")


def _records(rng, count, lo, hi):
    out = []
    for i in range(count):
        n = int(rng.integers(lo, hi))
        seq = synth._ASCII[rng.integers(2, 7, size=n)].tobytes()
        out.append((f"chr{i}".encode(), seq))
    return out


def _fasta(records, width=80, eol=b"\n", desc=b"", blank=False, final_eol=True):
    parts = []
    for name, seq in records:
        parts.append(b">" + name + (b" " + desc if desc else b"") + eol)
        for s in range(0, len(seq), width):
            parts.append(seq[s:s + width] + eol)
        if blank:
            parts.append(eol)
    data = b"".join(parts)
    if not final_eol and data.endswith(eol):
        data = data[: -len(eol)]
    return data


def _shapes():
    rng = np.random.default_rng(20260901)
    recs = _records(rng, 5, 1, 5000)
    lower = [(n, s.lower()) for n, s in recs]
    iupac = [(n, bytes(rng.choice(list(b"ACGTNRYKMSWacgtnrykmsw"), size=len(s)).astype(np.uint8)))
             for n, s in recs]
    yield "80 columns", _fasta(recs)
    yield "60 columns, descriptions", _fasta(recs, 60, desc=b"synthetic contig len=1")
    yield "one base per line", _fasta(recs[:2], 1)
    yield "no final newline", _fasta(recs, 70, final_eol=False)
    yield "CRLF", _fasta(recs, 61, eol=b"\r\n")
    yield "CRLF with blank lines", _fasta(recs, 50, eol=b"\r\n", blank=True)
    yield "lowercase", _fasta(lower, 77)
    yield "IUPAC codes", _fasta(iupac, 80)
    yield "blank lines", _fasta(recs, 33, blank=True)
    yield "junk before the first header", b"junk line\n\n" + _fasta(recs)
    yield "'>' inside a sequence line", b">a\nAC>GT\nTT\n>b\nGG\n"
    yield "single base records", b">x\nA\n>y\nC\n>z\nN"
    yield "long human-scale", _fasta([(b"c%d" % i, synth._ASCII[c].tobytes())
                                      for i, c in enumerate(synth.human_scale_3gbp(0.003).contigs)])


@pytest.mark.parametrize("name,data", list(_shapes()), ids=[s[0] for s in _shapes()])
def test_device_fasta_equals_reference(ctx, tmp_path, name, data):
    _need_reference()
    path = tmp_path / "in.fa"
    path.write_bytes(data)
    expected, fp = oracle.ref_encode_fasta(path)
    got, got_fp, records = ctx.encode_fasta_bytes(data)
    assert np.array_equal(got, expected), name
    assert got_fp == fp, name
    assert records == int(np.count_nonzero(expected == 1))


def test_device_fasta_matches_host_reader_on_synthetic_references(ctx, tmp_path):
    for i, ref in enumerate([synth.repeat_rich_100mbp(0.02), synth.plain_4mbp(0.3)]):
        path = tmp_path / f"{i}.fa"
        ref.write_fasta(path)
        host, host_fp, host_records = sg.encode_fasta(path)
        got, fp, records = ctx.encode_fasta_bytes(path.read_bytes())
        assert np.array_equal(got, host) and fp == host_fp and records == host_records
        assert np.array_equal(np.append(got, 0), ref.logical_text())


@pytest.mark.parametrize("data,code", [
    (b"", sg.ErrorCode.INVALID_INPUT),                          # no record
    (b"ACGT\n", sg.ErrorCode.INVALID_INPUT),                    # no header
    (b">a\nAC\n>a\nGT\n", sg.ErrorCode.INVALID_INPUT),          # duplicate name
    (b">a\n>b\nGT\n", sg.ErrorCode.INVALID_INPUT),              # empty record
    (b">\nAC\n", sg.ErrorCode.INVALID_INPUT),                   # empty name
    (b">a\nACGT", None),                                       # valid, no final newline
    (b"@r1\nACGT\n+\nIIII\n", sg.ErrorCode.UNSUPPORTED_BACKEND),  # FASTQ
    (b">a\nAC\n+\nII\n", sg.ErrorCode.UNSUPPORTED_BACKEND),     # '+' line
    (b">a\r\n\r\nACGT\r\n", sg.ErrorCode.UNSUPPORTED_BACKEND),  # lone CR kept by kseq
])
def test_device_fasta_errors_follow_the_reader(ctx, data, code):
    if code is None:
        got, _, records = ctx.encode_fasta_bytes(data)
        assert records == 1 and list(got) == [2, 3, 4, 5, 1]
        return
    with pytest.raises(sg.SufkitError) as err:
        ctx.encode_fasta_bytes(data)
    assert err.value.code == code


def test_device_fasta_full_size_repeat_rich(ctx, tmp_path):
    """The 100 Mbp workload's FASTA (larger than 64 MiB: 16 KiB fingerprint
    chunks) against the reference's reader."""
    _need_reference()
    ref = synth.repeat_rich_100mbp()
    path = tmp_path / "w2.fa"
    ref.write_fasta(path)
    expected, fp = oracle.ref_encode_fasta(path)
    got, got_fp, records = ctx.encode_fasta_bytes(path.read_bytes())
    assert got.size == expected.size == 100_000_024
    assert np.array_equal(got, expected) and got_fp == fp and records == 24
