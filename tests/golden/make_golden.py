"""Regenerates tests/golden/*.npz from the reference's own compiled code.

Run where the sufkit sources are at $SUFKIT_REFERENCE (default: the build
container's checkout):  make -C oracle ref && python tests/golden/make_golden.py

Inputs are the reference's own test texts, rebuilt from the generators its C++
tests use (paths inside the sufkit project):
  * reference_fa: tests/data/reference.fa read by GenomeReference::FromFasta
    (the logical text pinned at tests/test_sufkit.cpp:219-221);
  * caps_runs_*: tests/test_caps_backend.cpp:47-54 (N runs of 16..4096 with a
    separator, a hard-boundary symbol and a trailing run of A);
  * caps_random_*: tests/test_caps_backend.cpp:55-64 (xorshift texts over
    {1..6} with 777-long N insertions);
  * lcp_all_a / lcp_random_bytes: tests/test_lcp_storage.cpp:331-338 (no
    sentinel; arbitrary bytes);
  * differential_*: tests/test_sufkit.cpp:1180-1196 (3 records x 40 bases over
    ACGTN from the LCG with seed 0x20260822).
Outputs per case come from libdivsufsort64 and detail::BuildDivsufsort64 (SA,
ISA, Kasai LCP) and LcpStorage::BuildByteCodedDirect (32- and 64-bit anchors).
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import oracle  # noqa: E402

REF = Path(os.environ.get("SUFKIT_REFERENCE", "/root/reference"))
OUT = Path(__file__).resolve().parent


def caps_runs():
    cases = {}
    for length in (16, 255, 256, 257, 1024, 4096):
        text = [6] * length + [1, 0]
        cases[f"caps_runs_{length}_a"] = list(text)
        text.insert(0, 2)
        text[length // 2] = 3
        cases[f"caps_runs_{length}_b"] = list(text)
        text[len(text) - 1:len(text) - 1] = [2] * (length + 1)
        cases[f"caps_runs_{length}_c"] = list(text)
    return cases


def caps_random():
    cases = {}
    mask = (1 << 64) - 1
    state = 947123
    for trial in range(96):
        text = []
        for _ in range(16 + trial * 13):
            state ^= (state << 13) & mask
            state ^= state >> 7
            state ^= (state << 17) & mask
            text.append(1 + state % 6)
        if trial % 3 == 0:
            text[7:7] = [6] * 777
        text.append(0)
        cases[f"caps_random_{trial:02d}"] = text
    return cases


def lcp_storage_texts():
    state = 0xC0FFEE
    rnd = []
    for _ in range(1537):
        state = (state * 1664525 + 1013904223) & 0xFFFFFFFF
        rnd.append(state >> 24)
    return {"lcp_all_a": [ord("A")] * 1025, "lcp_random_bytes": rnd}


def differential():
    cases = {}
    mask = (1 << 64) - 1
    state = 0x20260822

    def nxt():
        nonlocal state
        state = (state * 6364136223846793005 + 1442695040888963407) & mask
        return state

    alphabet = [2, 3, 4, 5, 6]  # A C G T N after normalization
    for trial in range(25):
        text = []
        for _ in range(3):
            for _ in range(40):
                text.append(alphabet[nxt() % 5])
            text.append(1)
        text.append(0)
        cases[f"differential_{trial:02d}"] = text
        # The C++ test then draws 12 query patterns from the same generator.
        for _ in range(12):
            for _ in range(1 + nxt() % 8):
                nxt()
    return cases


def main():
    if oracle.ref() is None:
        sys.exit("oracle/_ref/libsufref.so is missing: make -C oracle ref")
    cases = {}
    encoded, _ = oracle.ref_encode_fasta(REF / "tests" / "data" / "reference.fa")
    cases["reference_fa"] = list(encoded) + [0]
    cases.update(caps_runs())
    cases.update(caps_random())
    cases.update(lcp_storage_texts())
    cases.update(differential())
    arrays = {}
    for name, text in cases.items():
        t = np.asarray(text, np.uint8)
        sa64 = oracle.ref_divsufsort64(t).astype(np.uint32)
        sa, isa, lcp, _ = oracle.ref_adapter(t, 64)
        assert (sa.astype(np.uint32) == sa64).all()
        p32, a32, v32 = oracle.ref_bytecode(t, sa, isa, 32)
        arrays[f"{name}/text"] = t
        arrays[f"{name}/sa"] = sa64
        arrays[f"{name}/isa"] = isa.astype(np.uint32)
        arrays[f"{name}/lcp"] = lcp.astype(np.uint32)
        arrays[f"{name}/primary"] = p32
        arrays[f"{name}/anchor_pos"] = a32.astype(np.uint32)
        arrays[f"{name}/anchor_val"] = v32.astype(np.uint32)
    np.savez_compressed(OUT / "reference_cases.npz", **arrays)
    print(f"{len(cases)} cases -> {OUT / 'reference_cases.npz'}")


if __name__ == "__main__":
    main()
