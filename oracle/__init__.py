"""Test infrastructure only: ctypes loaders for the CPU oracle.

* ``port()``  -> liboracle.so, our C restatement (oracle/sa_oracle.c).
* ``ref()``   -> _ref/libsufref.so, the reference's own sources compiled by
  oracle/Makefile (None when it has not been built).
* ``sufkit_index(...)`` / ``sufkit_load(...)`` run sufkit's public
  SuffixArray::Build + Save and Load in a child process, through libsufref.so
  or through _ref/libsufref_cuda.so (the same sources with the constructor
  translation unit replaced by the sufgpu drop-in), so that both builds of
  one FASTA can be compared as saved files.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, and only as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_PATH = HERE / "liboracle.so"
REF_PATH = HERE / "_ref" / "libsufref.so"
REF_CUDA_PATH = HERE / "_ref" / "libsufref_cuda.so"

P = ctypes.c_void_p
U64 = ctypes.c_uint64


def build(reference: Optional[str] = None, cuda_seam: bool = False) -> None:
    """Compiles liboracle.so, and _ref/libsufref.so when the reference tree is
    available (make -C oracle); with cuda_seam also _ref/libsufref_cuda.so
    (needs sufkit_b200/libsufgpu.so)."""
    cmd = ["make", "-C", str(HERE), "-j8", "-s"]
    if reference:
        cmd.append(f"REF={reference}")
    subprocess.run(cmd, check=True)
    if cuda_seam and REF_PATH.exists():
        subprocess.run(cmd + ["cuda_seam"], check=True)


_port = None
_ref = None


def port() -> ctypes.CDLL:
    global _port
    if _port is None:
        if not PORT_PATH.exists():
            build()
        lib = ctypes.CDLL(str(PORT_PATH))
        lib.oracle_suffix_sort.argtypes = [P, U64, P]
        lib.oracle_isa.argtypes = [P, U64, P]
        lib.oracle_kasai_lcp.argtypes = [P, U64, P, P, P]
        lib.oracle_kasai_lcp.restype = None
        lib.oracle_bytecode_lcp.argtypes = [P, U64, P, P, ctypes.c_int, P, P, P, U64]
        lib.oracle_bytecode_lcp.restype = ctypes.c_int64
        lib.oracle_bytecode_guide.argtypes = [P, U64, U64, P]
        lib.oracle_bytecode_guide.restype = U64
        lib.oracle_bytecode_exact.argtypes = [P, P, P, U64, U64, U64]
        lib.oracle_bytecode_exact.restype = U64
        lib.oracle_pack.argtypes = [P, U64, U64, ctypes.c_int, P, P, P]
        lib.oracle_is_permutation.argtypes = [P, U64]
        lib.oracle_child.argtypes = [P, U64, P]
        lib.oracle_child.restype = None
        _port = lib
    return _port


def ref() -> Optional[ctypes.CDLL]:
    global _ref
    if _ref is None:
        if not REF_PATH.exists():
            return None
        lib = ctypes.CDLL(str(REF_PATH))
        lib.sufref_last_error.restype = ctypes.c_char_p
        lib.sufref_divsufsort64.argtypes = [P, P, ctypes.c_int64]
        lib.sufref_divsufsort32.argtypes = [P, P, ctypes.c_int32]
        lib.sufref_prefix_directory.argtypes = [P, U64, U64, P, P, P, P]
        lib.sufref_adapter_build_sampled.argtypes = [ctypes.c_int, P, U64, ctypes.c_uint32,
                                                     ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
                                                     P, P, P, P]
        lib.sufref_adapter_build.argtypes = [ctypes.c_int, P, U64, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_uint32, P, P, P, P]
        lib.sufref_pack.argtypes = [P, U64, U64, ctypes.c_int, P, P, P, P]
        lib.sufref_bytecoded_direct.argtypes = [P, U64, P, P, ctypes.c_int, P, P, P, U64, P]
        lib.sufref_bytecoded_from_raw.argtypes = [P, P, U64, ctypes.c_int, P, P, P, U64, P]
        lib.sufref_caps_build.argtypes = [ctypes.c_int, P, U64, ctypes.c_uint32, P, P, P]
        lib.sufref_bytecoded_direct_sampled.argtypes = [P, U64, P, P, U64, ctypes.c_uint32,
                                                        ctypes.c_int, P, P, P, U64, P]
        lib.sufref_bytecoded_exact.argtypes = [P, U64, P, P, U64, P, P, U64, P]
        lib.sufref_encode_fasta.argtypes = [ctypes.c_char_p, P, U64, P, P]
        lib.sufref_encode_fasta.restype = ctypes.c_int64
        lib.sufref_suffix_array_build.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
                                                  ctypes.c_char_p, P, P]
        lib.sufref_suffix_array_rows.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, P, U64]
        _ref = lib
    return _ref


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


# --------------------------------------------------------------------------
# Port (C restatement)
# --------------------------------------------------------------------------
def suffix_array(text: np.ndarray) -> np.ndarray:
    t = np.ascontiguousarray(text, np.uint8)
    sa = np.empty(t.size, np.uint64)
    if port().oracle_suffix_sort(_p(t), t.size, _p(sa)) != 0:
        raise MemoryError("oracle suffix sort failed")
    return sa


def inverse(sa: np.ndarray) -> np.ndarray:
    sa = np.ascontiguousarray(sa, np.uint64)
    isa = np.empty(sa.size, np.uint64)
    if port().oracle_isa(_p(sa), sa.size, _p(isa)) != 0:
        raise ValueError("not a permutation")
    return isa


def kasai(text: np.ndarray, sa: np.ndarray, isa: np.ndarray) -> np.ndarray:
    t = np.ascontiguousarray(text, np.uint8)
    sa = np.ascontiguousarray(sa, np.uint64)
    isa = np.ascontiguousarray(isa, np.uint64)
    lcp = np.empty(t.size, np.uint64)
    port().oracle_kasai_lcp(_p(t), t.size, _p(sa), _p(isa), _p(lcp))
    return lcp


def bytecode(text: np.ndarray, sa: np.ndarray, isa: np.ndarray, width: int = 32):
    """(primary, anchor_positions, anchor_values) as uint8 / uint64 arrays."""
    t = np.ascontiguousarray(text, np.uint8)
    sa = np.ascontiguousarray(sa, np.uint64)
    isa = np.ascontiguousarray(isa, np.uint64)
    primary = np.empty(t.size, np.uint8)
    cap = max(16, t.size)
    pos = np.empty(cap, np.uint64)
    val = np.empty(cap, np.uint64)
    k = port().oracle_bytecode_lcp(_p(t), t.size, _p(sa), _p(isa), width, _p(primary),
                                   _p(pos), _p(val), cap)
    if k < 0:
        raise ValueError("byte coding failed")
    return primary, pos[:k].copy(), val[:k].copy()


def guide(anchor_positions: np.ndarray, n: int) -> np.ndarray:
    a = np.ascontiguousarray(anchor_positions, np.uint64)
    out = np.empty(2 + max(n, 1) // 4096 + 1, np.uint64)
    k = port().oracle_bytecode_guide(_p(a), a.size, n, _p(out))
    return out[:k].copy()


def pack(values: np.ndarray, symbol_count: int, bits: int):
    """(width, low32 or native64, high or None)."""
    v = np.ascontiguousarray(values, np.uint64)
    low = np.empty(v.size, np.uint32)
    high8 = np.empty(v.size, np.uint8)
    high16 = np.empty(v.size, np.uint16)
    native = np.empty(v.size, np.uint64)
    width = bits
    resolved = port().oracle_pack(_p(v), v.size, symbol_count, bits, _p(low),
                                  _p(high16 if bits == 48 else high8), _p(native))
    if resolved < 0:
        raise ValueError("coordinate out of range for the storage width")
    width = resolved
    if width == 64:
        return width, native, None
    if width == 40:
        return width, low, high8
    if width == 48:
        return width, low, high16
    return width, low, None


def child(lcp: np.ndarray) -> np.ndarray:
    """Compact CHILD table of a row-order LCP array (uint64; n = no link)."""
    l = np.ascontiguousarray(lcp, np.uint64)
    out = np.empty(l.size, np.uint64)
    port().oracle_child(_p(l), l.size, _p(out))
    return out


def full_build(text: np.ndarray):
    """(sa, isa, lcp) from the port."""
    sa = suffix_array(text)
    isa = inverse(sa)
    return sa, isa, kasai(text, sa, isa)


# --------------------------------------------------------------------------
# Reference (compiled sufkit sources)
# --------------------------------------------------------------------------
def _check(lib, rc):
    if rc != 0:
        raise RuntimeError(f"reference call failed ({rc}): {lib.sufref_last_error().decode()}")


def ref_adapter(text: np.ndarray, width: int = 64, threads: int = 1):
    """detail::BuildDivsufsort{width}: (sa, isa, lcp, seconds[3])."""
    lib = ref()
    t = np.ascontiguousarray(text, np.uint8)
    sa = np.empty(t.size, np.uint64)
    isa = np.empty(t.size, np.uint64)
    lcp = np.empty(t.size, np.uint64)
    sec = (ctypes.c_double * 3)()
    _check(lib, lib.sufref_adapter_build(width, _p(t), t.size, 1, 1, threads, _p(sa), _p(isa),
                                         _p(lcp), sec))
    return sa, isa, lcp, list(sec)


def ref_caps(text: np.ndarray, threads: int = 1, width: int = 32, lcp: bool = True):
    """detail::BuildCaps32/64 (CaPS-SA as vendored by sufkit): (sa, lcp or
    None, seconds) with `threads` workers."""
    lib = ref()
    t = np.ascontiguousarray(text, np.uint8)
    sa = np.empty(max(t.size, 1), np.uint64)
    l = np.empty(max(t.size, 1), np.uint64) if lcp else None
    sec = (ctypes.c_double * 1)()
    _check(lib, lib.sufref_caps_build(width, _p(t), t.size, threads, _p(sa),
                                      _p(l) if lcp else None, sec))
    return sa[: t.size], (l[: t.size] if lcp else None), sec[0]


def ref_adapter_sampled(text: np.ndarray, rate: int, width: int = 64, threads: int = 1):
    """detail::BuildDivsufsort{width} with sampling rate K: (sa, isa, lcp) of
    the ceil(n / K) sampled rows."""
    lib = ref()
    t = np.ascontiguousarray(text, np.uint8)
    cap = max(1, (t.size + rate - 1) // rate)
    sa = np.empty(cap, np.uint64)
    isa = np.empty(cap, np.uint64)
    lcp = np.empty(cap, np.uint64)
    rows = ctypes.c_uint64()
    _check(lib, lib.sufref_adapter_build_sampled(width, _p(t), t.size, rate, 1, 1, threads,
                                                 _p(sa), _p(isa), _p(lcp), ctypes.byref(rows)))
    k = rows.value
    return sa[:k].copy(), isa[:k].copy(), lcp[:k].copy()


def sample(sa: np.ndarray, lcp: np.ndarray, rate: int):
    """Restatement of the sampling of src/divsufsort_backend.cpp:62-150 from a
    complete (sa, lcp): keep rows with sa % K == 0; ISA[p / K] = sampled row;
    LCP of consecutive sampled rows = min of the complete LCP over the rows
    after the previous sampled row up to this one (0 for the first)."""
    sa = np.asarray(sa, np.int64)
    lcp = np.asarray(lcp, np.int64)
    rows = np.flatnonzero(sa % rate == 0)
    sa_k = sa[rows]
    isa_k = np.empty(sa_k.size, np.int64)
    isa_k[sa_k // rate] = np.arange(sa_k.size)
    lcp_k = np.zeros(sa_k.size, np.int64)
    if rows.size > 1:
        # Segment j >= 1 is rows[j-1]+1 .. rows[j]: [starts[j-1], starts[j]).
        starts = rows + 1
        lcp_k[1:] = np.minimum.reduceat(np.append(lcp, 0), starts)[: rows.size - 1]
    return sa_k, isa_k, lcp_k


def ref_prefix_directory(text: np.ndarray, resident_core_bytes: int):
    """FastPrefixIndex::Build with default options over the reference's SA:
    (k, intervals[4^k] as begin | end << 32 with (n, n) for absent k-mers,
    indexed k-mers, nonempty entries)."""
    lib = ref()
    t = np.ascontiguousarray(text, np.uint8)
    out = np.empty(1 << 20, np.uint64)
    k = ctypes.c_uint32()
    kmers = ctypes.c_uint64()
    entries = ctypes.c_uint64()
    _check(lib, lib.sufref_prefix_directory(_p(t), t.size, int(resident_core_bytes),
                                            ctypes.byref(k), _p(out), ctypes.byref(kmers),
                                            ctypes.byref(entries)))
    return k.value, out[: (1 << (2 * k.value)) if k.value else 0].copy(), kmers.value, entries.value


def prefix_directory(text: np.ndarray, sa: np.ndarray, k: int) -> np.ndarray:
    """Restatement of the Fast index's k-mer directory
    (src/fast_prefix_index.cpp:131-205): for each k-mer of bytes 2..5 the SA
    rows [begin, end) of the suffixes starting with it, packed
    begin | end << 32, (n, n) where absent."""
    t = np.ascontiguousarray(text, np.uint8)
    n = t.size
    sa = np.asarray(sa, np.int64)
    table = np.full(1 << (2 * k), n | (n << 32), np.uint64)
    if n < k:
        return table
    windows = np.lib.stride_tricks.sliding_window_view(t, k)  # position p: t[p:p+k]
    canonical = ((windows >= 2) & (windows <= 5)).all(axis=1)
    weights = (1 << (2 * np.arange(k - 1, -1, -1))).astype(np.int64)
    keys = ((windows.astype(np.int64) - 2) & 3) @ weights
    rows_pos = sa  # row r -> position sa[r]
    valid_rows = np.flatnonzero((rows_pos <= n - k) & canonical[np.minimum(rows_pos, n - k)])
    if valid_rows.size == 0:
        return table
    row_keys = keys[rows_pos[valid_rows]]
    first = np.ones(valid_rows.size, bool)
    first[1:] = (row_keys[1:] != row_keys[:-1]) | (valid_rows[1:] != valid_rows[:-1] + 1)
    last = np.ones(valid_rows.size, bool)
    last[:-1] = first[1:]
    begins = valid_rows[first].astype(np.uint64)
    ends = (valid_rows[last] + 1).astype(np.uint64)
    table[row_keys[first]] = begins | (ends << np.uint64(32))
    return table


def ref_divsufsort64(text: np.ndarray) -> np.ndarray:
    lib = ref()
    t = np.ascontiguousarray(text, np.uint8)
    sa = np.empty(t.size, np.int64)
    _check(lib, lib.sufref_divsufsort64(_p(t), _p(sa), t.size))
    return sa


def ref_bytecode(text: np.ndarray, sa: np.ndarray, isa: np.ndarray, width: int = 32):
    lib = ref()
    t = np.ascontiguousarray(text, np.uint8)
    sa = np.ascontiguousarray(sa, np.uint64)
    isa = np.ascontiguousarray(isa, np.uint64)
    primary = np.empty(t.size, np.uint8)
    cap = max(16, t.size)
    pos = np.empty(cap, np.uint64)
    val = np.empty(cap, np.uint64)
    count = U64()
    _check(lib, lib.sufref_bytecoded_direct(_p(t), t.size, _p(sa), _p(isa), width, _p(primary),
                                            _p(pos), _p(val), cap, ctypes.addressof(count)))
    k = count.value
    return primary, pos[:k].copy(), val[:k].copy()


def ref_bytecode_sampled(text: np.ndarray, sa_k: np.ndarray, isa_k: np.ndarray, rate: int,
                         width: int = 32):
    """LcpStorage::BuildByteCodedDirect of a sampled build (rate K): primary
    bytes per sampled row, anchor positions and values (uint64)."""
    lib = ref()
    t = np.ascontiguousarray(text, np.uint8)
    sa = np.ascontiguousarray(sa_k, np.uint64)
    isa = np.ascontiguousarray(isa_k, np.uint64)
    rows = sa.size
    primary = np.empty(max(rows, 1), np.uint8)
    cap = rows + 1
    pos = np.empty(cap, np.uint64)
    val = np.empty(cap, np.uint64)
    count = ctypes.c_uint64()
    _check(lib, lib.sufref_bytecoded_direct_sampled(_p(t), t.size, _p(sa), _p(isa), rows, rate,
                                                    width, _p(primary), _p(pos), _p(val), cap,
                                                    ctypes.byref(count)))
    k = count.value
    return primary[:rows].copy(), pos[:k].copy(), val[:k].copy()


def sample_bytecode(sa_k: np.ndarray, isa_k: np.ndarray, lcp_k: np.ndarray, rate: int):
    """Restatement of the sampled byte coding (src/lcp_storage.cpp:304-420,
    K > 1) from a sampled build's SA, dense ISA and row LCP: primary =
    min(LCP, 255) per sampled row; an anchor opens at sample position s*K
    when PLCP_K[s] >= 255 unless sample s-1 overflowed too with PLCP_K[s-1]
    >= K and PLCP_K[s-1] - K == PLCP_K[s]."""
    lcp = np.asarray(lcp_k, np.int64)
    primary = np.minimum(lcp, 255).astype(np.uint8)
    plcp = lcp[np.asarray(isa_k, np.int64)]
    over = plcp >= 255
    prev = np.concatenate([[-1], plcp[:-1]])
    prev_over = np.concatenate([[False], over[:-1]])
    cont = prev_over & (prev >= rate) & (prev - rate == plcp)
    opens = np.flatnonzero(over & ~cont)
    return primary, (opens * rate).astype(np.uint64), plcp[opens].astype(np.uint64)


def ref_bytecode_from_raw(lcp: np.ndarray, isa: np.ndarray, width: int = 32):
    lib = ref()
    lcp = np.ascontiguousarray(lcp, np.uint64)
    isa = np.ascontiguousarray(isa, np.uint64)
    primary = np.empty(lcp.size, np.uint8)
    cap = max(16, lcp.size)
    pos = np.empty(cap, np.uint64)
    val = np.empty(cap, np.uint64)
    count = U64()
    _check(lib, lib.sufref_bytecoded_from_raw(_p(lcp), _p(isa), lcp.size, width, _p(primary),
                                              _p(pos), _p(val), cap, ctypes.addressof(count)))
    k = count.value
    return primary, pos[:k].copy(), val[:k].copy()


def ref_pack(values: np.ndarray, symbol_count: int, bits: int):
    lib = ref()
    v = np.ascontiguousarray(values, np.uint64)
    low = np.empty(v.size, np.uint32)
    high = np.empty(v.size, np.uint16 if bits == 48 else np.uint8)
    native = np.empty(v.size, np.uint64)
    width = ctypes.c_int()
    _check(lib, lib.sufref_pack(_p(v), v.size, symbol_count, bits, _p(low), _p(high),
                                _p(native), ctypes.addressof(width)))
    w = width.value
    if w == 64:
        return w, native, None
    return w, low, (high if w in (40, 48) else None)


def ref_encode_fasta(path) -> tuple[np.ndarray, int]:
    lib = ref()
    need = U64()
    fp = U64()
    raw = str(path).encode()
    rc = lib.sufref_encode_fasta(raw, None, 0, ctypes.addressof(need), ctypes.addressof(fp))
    if rc == -1:
        raise ValueError(lib.sufref_last_error().decode())
    out = np.empty(need.value, np.uint8)
    rc = lib.sufref_encode_fasta(raw, _p(out), need.value, ctypes.addressof(need),
                                 ctypes.addressof(fp))
    if rc < 0:
        raise ValueError(lib.sufref_last_error().decode())
    return out, fp.value


# --------------------------------------------------------------------------
# sufkit's public build/save/load, in a child process (two libraries export
# the same sufkit symbols, so each run gets a process of its own)
# --------------------------------------------------------------------------
_CHILD = r"""
import ctypes, json, sys
args = json.loads(sys.argv[1])
lib = ctypes.CDLL(args["lib"])
lib.sufref_last_error.restype = ctypes.c_char_p
out = {}
if args["op"] == "build":
    f = lib.sufref_suffix_array_build
    f.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_uint32, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p]
    stats = (ctypes.c_double * 12)()
    info = (ctypes.c_uint64 * 6)()
    rc = f(args["fasta"].encode(), args["profile"], args["width"], args["storage"],
           args["acceleration"], args["threads"], args["save"].encode(), stats, info)
    out = {"rc": rc, "stats": list(stats), "info": list(info)}
else:
    f = lib.sufref_load_query
    f.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_uint64, ctypes.c_void_p]
    occ = ctypes.c_uint64()
    rows = (ctypes.c_uint64 * args["rows"])()
    info = (ctypes.c_uint64 * 3)()
    rc = f(args["path"].encode(), args["pattern"].encode(), ctypes.byref(occ), rows,
           args["rows"], info)
    out = {"rc": rc, "count": occ.value, "rows": list(rows), "info": list(info)}
if out["rc"] != 0:
    out["error"] = lib.sufref_last_error().decode()
print(json.dumps(out))
"""


def _child(args: dict) -> dict:
    import json
    import sys
    proc = subprocess.run([sys.executable, "-c", _CHILD, json.dumps(args)], capture_output=True,
                          text=True, timeout=3600)
    if proc.returncode != 0:
        raise RuntimeError(f"child failed ({proc.returncode}): {proc.stderr[-2000:]}")
    return json.loads(proc.stdout.strip().splitlines()[-1])


def sufkit_index(fasta, save_path, profile: int = 0, coordinate_width: int = 64,
                 storage_width: int = 0, acceleration: int = -1, threads: int = 1,
                 cuda: bool = False) -> dict:
    """SuffixArray::Build of a FASTA with sufkit's own code, then Save.
    profile 0 = Fast, 1 = Low-memory; cuda selects libsufref_cuda.so."""
    lib = REF_CUDA_PATH if cuda else REF_PATH
    return _child({"op": "build", "lib": str(lib), "fasta": str(fasta), "profile": profile,
                   "width": coordinate_width, "storage": storage_width,
                   "acceleration": acceleration, "threads": threads, "save": str(save_path)})


def sufkit_load(path, pattern: str, rows: int) -> dict:
    """SuffixArray::Load (full validation) with the reference's own library,
    then Count(pattern) and SuffixAt(0..rows)."""
    return _child({"op": "load", "lib": str(REF_PATH), "path": str(path), "pattern": pattern,
                   "rows": rows})


# --------------------------------------------------------------------------
# Digests for full-size collection checks (run in spawned worker processes)
# --------------------------------------------------------------------------
def digest_planes(sa: np.ndarray, lcp: np.ndarray) -> tuple[str, str]:
    """blake2b of the SA and LCP rows as little-endian uint32 words (equal
    digests <=> equal rows, word for word)."""
    import hashlib
    sa32 = np.ascontiguousarray(np.asarray(sa).astype(np.uint32))
    lcp32 = np.ascontiguousarray(np.asarray(lcp).astype(np.uint32))
    return (hashlib.blake2b(sa32.tobytes(), digest_size=20).hexdigest(),
            hashlib.blake2b(lcp32.tobytes(), digest_size=20).hexdigest())


def uneven_reference_digests(task) -> tuple[int, int, str, str]:
    """Reference `index` of the bacterial collection (its own random stream,
    sufkit_b200.synth.uneven_reference), built by the reference's
    divsufsort64 + Kasai: (index, n, SA digest, LCP digest)."""
    from sufkit_b200 import synth
    index, total = task
    text = synth.uneven_reference(index, total).logical_text()
    sa, _, lcp, _ = ref_adapter(text, 64)
    d_sa, d_lcp = digest_planes(sa, lcp)
    return index, int(text.size), d_sa, d_lcp


# --------------------------------------------------------------------------
# Reading coordinate sections of a saved .sufidx (container layout of
# src/serialization.cpp:305-360: an 80-byte header, then 32-byte section
# entries {type u32, flags u32, offset u64, size u64, crc u32, 0 u32};
# coordinate sections of src/sa_codec.cpp:466-512: a 56-byte codec header
# {magic, version, codec, 0 (u32 each); symbols, count, low bytes, high bytes,
# 0 (u64 each)}, then the low plane and the high plane)
# --------------------------------------------------------------------------
SECTION_SUFFIX_ARRAY, SECTION_ISA, SECTION_LCP, SECTION_CHILD = 3, 5, 6, 7


def sufidx_sections(path) -> dict:
    import struct
    data = Path(path).read_bytes()
    count = struct.unpack_from("<I", data, 24)[0]
    out = {}
    for k in range(count):
        typ, _flags, off, size, _crc, _pad = struct.unpack_from("<IIQQII", data, 80 + 32 * k)
        out[typ] = (off, size)
    return out


def sufidx_coordinates(path, section: int) -> np.ndarray:
    """The values of one coordinate section (SA, ISA or CHILD) as uint64."""
    import struct
    off, size = sufidx_sections(path)[section]
    with open(path, "rb") as f:
        f.seek(off)
        blob = f.read(size)
    _magic, _version, _codec, _zero, _symbols, count, low_bytes, high_bytes, _res = \
        struct.unpack_from("<IIIIQQQQQ", blob, 0)
    body = blob[56:]
    if low_bytes == count * 8:
        return np.frombuffer(body, np.uint64, count).copy()
    low = np.frombuffer(body, np.uint32, count).astype(np.uint64)
    if high_bytes == count:
        low |= np.frombuffer(body, np.uint8, count, low_bytes).astype(np.uint64) << np.uint64(32)
    elif high_bytes == 2 * count:
        low |= np.frombuffer(body, np.uint16, count, low_bytes).astype(np.uint64) << np.uint64(32)
    return low
