"""GPU: the drop-in inside sufkit's own code path.

oracle/_ref/libsufref_cuda.so is sufkit's sources with src/divsufsort_backend.cpp
replaced by sufkit_b200/integration/divsufsort_backend_cuda.cpp, which defines
BuildDivsufsort32/64 on the sufgpu C ABI.  Each case builds one FASTA through
sufkit's public SuffixArray::Build + Save twice -- stock divsufsort
(libsufref.so) and the GPU drop-in -- and requires:

  * the two .sufidx files to be byte-identical (every section: coordinates,
    LCP planes, metadata, CRCs);
  * SuffixArray::Load of the GPU-built file by the stock library to succeed
    (Load validates the container, CRCs and semantics) and answer Count and
    SuffixAt exactly as the stock file does.
"""
import filecmp

import pytest

import oracle
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu

FAST, LOW_MEMORY = 0, 1


def _need_libraries():
    if not oracle.REF_PATH.exists() or not oracle.REF_CUDA_PATH.exists():
        pytest.skip("the reference libraries were not built (make -C oracle ref cuda_seam)")


CASES = [
    # (name, reference, profile, coordinate width, storage width)
    ("plain 4 Mbp, Fast, 32-bit", lambda: synth.plain_4mbp(), FAST, 32, 32),
    ("plain 4 Mbp, Fast, 64-bit construction", lambda: synth.plain_4mbp(scale=0.25), FAST, 64, 0),
    ("human-scale x0.002, Low-memory split40 byte-coded",
     lambda: synth.human_scale_3gbp(scale=0.002), LOW_MEMORY, 64, 40),
    ("repeat-rich x0.02, Low-memory split48",
     lambda: synth.repeat_rich_100mbp(scale=0.02), LOW_MEMORY, 64, 48),
]


@pytest.mark.parametrize("name,make,profile,width,storage", CASES, ids=[c[0] for c in CASES])
def test_sufidx_from_gpu_dropin_equals_divsufsort(tmp_path, name, make, profile, width, storage):
    _need_libraries()
    fasta = tmp_path / "ref.fa"
    make().write_fasta(fasta)
    cpu_file, gpu_file = tmp_path / "cpu.sufidx", tmp_path / "gpu.sufidx"
    cpu = oracle.sufkit_index(fasta, cpu_file, profile, width, storage)
    gpu = oracle.sufkit_index(fasta, gpu_file, profile, width, storage, cuda=True)
    assert cpu["rc"] == 0, cpu.get("error")
    assert gpu["rc"] == 0, gpu.get("error")
    assert gpu["info"] == cpu["info"]
    assert filecmp.cmp(cpu_file, gpu_file, shallow=False), f"{name}: .sufidx files differ"
    rows = 5000
    a = oracle.sufkit_load(cpu_file, "ACGTA", rows)
    b = oracle.sufkit_load(gpu_file, "ACGTA", rows)
    assert b["rc"] == 0, b.get("error")
    assert (a["count"], a["rows"], a["info"]) == (b["count"], b["rows"], b["info"])
    assert b["count"] > 0


def test_gpu_dropin_rejects_what_divsufsort_rejects(tmp_path):
    """An empty FASTA fails in both builds with the same error category path
    (the drop-in raises sufkit::Error like the stock constructor)."""
    _need_libraries()
    fasta = tmp_path / "empty.fa"
    fasta.write_bytes(b"")
    cpu = oracle.sufkit_index(fasta, tmp_path / "c.sufidx", FAST, 32, 32)
    gpu = oracle.sufkit_index(fasta, tmp_path / "g.sufidx", FAST, 32, 32, cuda=True)
    assert cpu["rc"] != 0 and gpu["rc"] != 0
    assert cpu["rc"] == gpu["rc"]
