"""sufkit_b200: Python host side of the sufgpu B200 construction engine.

Every call goes through the C ABI of ``libsufgpu.so`` (include/sufgpu/sufgpu.h)
with ctypes; the arrays live in numpy (host) or in any object exposing a device
pointer.  The names mirror the reference's constructor interface
(``detail::BuildDivsufsort32/64``, src/divsufsort_backend.hpp:13-33 in sufkit):
``build_cuda32`` / ``build_cuda64`` return the same fields (suffix_array, isa,
lcp and per-phase seconds) and raise :class:`SufkitError` with the reference's
``ErrorCode`` categories.

There is no CPU fallback: importing works anywhere, but every build needs the
compiled library and a CUDA device, and fails loudly without them.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

_HERE = Path(__file__).resolve().parent
LIBRARY_PATH = _HERE / "libsufgpu.so"
# Per-size knob table written by the autotuner (python -m sufkit_b200.autotune).
TUNING_PATH = _HERE / "tuning.json"


class ErrorCode(enum.IntEnum):
    """sufkit::ErrorCode (include/sufkit/types.hpp:708-721)."""

    INVALID_INPUT = 0
    IO_ERROR = 1
    UNSUPPORTED_BACKEND = 2
    CORRUPT_INDEX = 3
    VERSION_MISMATCH = 4
    BUILD_FAILURE = 5


class SufkitError(RuntimeError):
    """Mirror of sufkit::Error: a stable category plus a message."""

    def __init__(self, code: ErrorCode, message: str):
        super().__init__(message)
        self.code = ErrorCode(code)


class LcpEncoding(enum.IntEnum):
    """detail::LcpEncoding (src/lcp_storage.hpp:53-59)."""

    NONE = 0
    RAW32 = 1
    RAW64 = 2
    BYTE32 = 3
    BYTE64 = 4


FLAG_VALIDATE = 1
FLAG_PLANE_CRC = 2
FLAG_CHILD = 4


class _Desc(ctypes.Structure):
    _fields_ = [("sa_storage_bits", ctypes.c_uint32),
                ("isa_storage_bits", ctypes.c_uint32),
                ("lcp_encoding", ctypes.c_uint32),
                ("flags", ctypes.c_uint32),
                ("sampling_rate", ctypes.c_uint32),
                ("prefix_k", ctypes.c_uint32)]


class _Outputs(ctypes.Structure):
    _fields_ = [("sa_low", ctypes.c_void_p), ("sa_high", ctypes.c_void_p),
                ("isa_low", ctypes.c_void_p), ("isa_high", ctypes.c_void_p),
                ("lcp", ctypes.c_void_p), ("prefix_intervals", ctypes.c_void_p),
                ("child", ctypes.c_void_p)]


class _Anchors(ctypes.Structure):
    _fields_ = [("positions", ctypes.c_void_p), ("values", ctypes.c_void_p),
                ("count", ctypes.c_uint64), ("coordinate_bits", ctypes.c_uint32)]


class _Stats(ctypes.Structure):
    _fields_ = [("h2d_seconds", ctypes.c_double), ("sa_seconds", ctypes.c_double),
                ("isa_seconds", ctypes.c_double), ("lcp_seconds", ctypes.c_double),
                ("storage_seconds", ctypes.c_double), ("d2h_seconds", ctypes.c_double),
                ("total_seconds", ctypes.c_double), ("device_seconds", ctypes.c_double),
                ("symbols", ctypes.c_uint64),
                ("rounds", ctypes.c_uint32), ("seed_symbols", ctypes.c_uint32),
                ("active_rows", ctypes.c_uint64), ("active_first", ctypes.c_uint64),
                ("irreducible_long", ctypes.c_uint64),
                ("anchors", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint32),
                ("long_runs", ctypes.c_uint32), ("seg_sort_fallbacks", ctypes.c_uint32),
                ("seed_rare_rows", ctypes.c_uint32), ("prefix_kmers", ctypes.c_uint64),
                ("prefix_entries", ctypes.c_uint64), ("plane_crc", ctypes.c_uint32 * 5),
                ("seed_code_bits", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_
             if name != "plane_crc"}
        d["plane_crc"] = dict(zip(("sa_low", "sa_high", "isa_low", "isa_high", "lcp"),
                                  list(self.plane_crc)))
        return d


class _ServerConfig(ctypes.Structure):
    _fields_ = [("capacity_symbols", ctypes.c_uint64), ("max_instances", ctypes.c_uint32),
                ("flags", ctypes.c_uint32)]


class _RequestInfo(ctypes.Structure):
    _fields_ = [("queue_seconds", ctypes.c_double), ("latency_seconds", ctypes.c_double),
                ("rounds", ctypes.c_uint32), ("seed_symbols", ctypes.c_uint32),
                ("anchors", _Anchors), ("admit_iteration", ctypes.c_uint64),
                ("finish_iteration", ctypes.c_uint64), ("inflight_at_admit", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("symbols", ctypes.c_uint64),
                ("iterations", ctypes.c_uint64), ("max_inflight", ctypes.c_uint64),
                ("queued", ctypes.c_uint64), ("inflight", ctypes.c_uint64),
                ("p50_seconds", ctypes.c_double), ("p99_seconds", ctypes.c_double),
                ("span_seconds", ctypes.c_double), ("symbols_per_second", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class _Instance(ctypes.Structure):
    _fields_ = [("text", ctypes.c_void_p), ("n", ctypes.c_uint64),
                ("out", _Outputs), ("anchors", _Anchors)]


_lib: Optional[ctypes.CDLL] = None

# Exported symbols of the C ABI with their ctypes signatures.
_SIGNATURES = {
    "sufgpu_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]),
    "sufgpu_destroy": (None, [ctypes.c_void_p]),
    "sufgpu_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "sufgpu_max_symbols": (ctypes.c_uint64, []),
    "sufgpu_device_bytes": (ctypes.c_uint64, [ctypes.c_uint64, ctypes.c_void_p]),
    "sufgpu_build": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                    ctypes.POINTER(_Desc), ctypes.POINTER(_Outputs),
                                    ctypes.POINTER(_Anchors), ctypes.POINTER(_Stats)]),
    "sufgpu_divsufsort64": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_int64]),
    "sufgpu_divsufsort": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_int32]),
    "sufgpu_build_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(_Instance),
                                          ctypes.c_uint32, ctypes.POINTER(_Desc),
                                          ctypes.POINTER(_Stats)]),
    "sufgpu_build_collection": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(_Instance),
                                               ctypes.c_uint64, ctypes.POINTER(_Desc),
                                               ctypes.c_uint64, ctypes.c_uint32,
                                               ctypes.POINTER(_Stats)]),
    "sufgpu_collection_parts": (ctypes.c_uint64, [ctypes.c_void_p]),
    "sufgpu_collection_trace": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64,
                                               ctypes.POINTER(ctypes.c_uint32),
                                               ctypes.POINTER(ctypes.c_double)]),
    "sufgpu_set_profiling": (None, [ctypes.c_void_p, ctypes.c_int]),
    "sufgpu_profile_count": (ctypes.c_uint32, [ctypes.c_void_p]),
    "sufgpu_profile_entry": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32,
                                            ctypes.POINTER(ctypes.c_char_p),
                                            ctypes.POINTER(ctypes.c_uint64),
                                            ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_uint64)]),
    "sufgpu_set_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int64]),
    "sufgpu_prefix_select_k": (ctypes.c_uint32, [ctypes.c_uint64, ctypes.c_uint64]),
    "sufgpu_encode_fasta_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_uint64, ctypes.c_void_p,
                                                  ctypes.c_uint64, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_void_p]),
    "sufgpu_crc32_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                           ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]),
    "sufgpu_set_tuning_class": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p,
                                               ctypes.c_int64]),
    "sufgpu_clear_tuning_classes": (None, [ctypes.c_void_p]),
    "sufgpu_lcp_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    "sufgpu_server_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                            ctypes.POINTER(_ServerConfig)]),
    "sufgpu_server_destroy": (None, [ctypes.c_void_p]),
    "sufgpu_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                            ctypes.POINTER(_Desc), ctypes.POINTER(_Outputs),
                                            ctypes.POINTER(ctypes.c_uint64)]),
    "sufgpu_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.POINTER(_RequestInfo)]),
    "sufgpu_server_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.POINTER(ctypes.c_int)]),
    "sufgpu_server_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "sufgpu_server_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(_ServerStats)]),
    "sufgpu_host_alloc": (ctypes.c_void_p, [ctypes.c_uint64]),
    "sufgpu_host_free": (None, [ctypes.c_void_p]),
    "sufgpu_encode_fasta": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_uint64,
                                           ctypes.POINTER(ctypes.c_uint64),
                                           ctypes.POINTER(ctypes.c_uint64),
                                           ctypes.POINTER(ctypes.c_uint64)]),
}


def library() -> ctypes.CDLL:
    """Loads libsufgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIBRARY_PATH.exists():
            raise SufkitError(ErrorCode.UNSUPPORTED_BACKEND,
                              f"{LIBRARY_PATH} is missing: run python -m sufkit_b200.build")
        lib = ctypes.CDLL(str(LIBRARY_PATH))
        for name, (restype, argtypes) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def _ptr(a: Optional[np.ndarray]) -> Optional[int]:
    if a is None:
        return None
    return a.ctypes.data


def _raise(status: int, message: str):
    raise SufkitError(ErrorCode(status - 1), message)


def _as_text(text) -> np.ndarray:
    if isinstance(text, (bytes, bytearray, memoryview)):
        return np.frombuffer(bytes(text), dtype=np.uint8)
    arr = np.ascontiguousarray(text)
    if arr.dtype != np.uint8:
        raise SufkitError(ErrorCode.INVALID_INPUT, "text must be uint8")
    return arr


def _plane_dtype(bits: int):
    return np.uint64 if bits == 64 else np.uint32


def _high_dtype(bits: int):
    return {40: np.uint8, 48: np.uint16}.get(bits)


def compose(low: np.ndarray, high: Optional[np.ndarray]) -> np.ndarray:
    """Decodes a (low, high) coordinate plane pair to uint64 values."""
    out = low.astype(np.uint64)
    if high is not None:
        out |= high.astype(np.uint64) << np.uint64(32)
    return out


@dataclass
class BuildResult:
    """Planes of one build (host numpy arrays)."""

    sa_low: np.ndarray
    sa_high: Optional[np.ndarray] = None
    isa_low: Optional[np.ndarray] = None
    isa_high: Optional[np.ndarray] = None
    lcp: Optional[np.ndarray] = None
    anchor_positions: Optional[np.ndarray] = None
    anchor_values: Optional[np.ndarray] = None
    prefix_intervals: Optional[np.ndarray] = None
    child: Optional[np.ndarray] = None
    stats: dict = field(default_factory=dict)

    @property
    def sa(self) -> np.ndarray:
        return compose(self.sa_low, self.sa_high)

    @property
    def isa(self) -> Optional[np.ndarray]:
        return None if self.isa_low is None else compose(self.isa_low, self.isa_high)


class Context:
    """One CUDA device with its stream and grown device buffers.

    ``tuning`` names a knob table from the autotuner (default: the packaged
    sufkit_b200/tuning.json when it exists); ``None`` keeps the library's
    built-in defaults.  Knobs change speed only, never results."""

    def __init__(self, device: int = 0, tuning="default"):
        lib = library()
        handle = ctypes.c_void_p()
        status = lib.sufgpu_create(ctypes.byref(handle), device)
        if status != 0:
            _raise(status, lib.sufgpu_last_error(None).decode())
        self._lib = lib
        self._h = handle
        self.last_stats: dict = {}
        if tuning == "default":
            tuning = TUNING_PATH if TUNING_PATH.exists() else None
        if tuning is not None:
            self.load_tuning(tuning)

    def load_tuning(self, path) -> None:
        """Applies an autotuner table: {"classes": [{"max_symbols": m,
        "settings": {key: value}}, ...]} (replaces earlier classes)."""
        import json
        table = json.loads(Path(path).read_text())
        self._lib.sufgpu_clear_tuning_classes(self._h)
        for cls in table.get("classes", []):
            for key, value in cls.get("settings", {}).items():
                self.set_tuning_class(int(cls["max_symbols"]), key, int(value))

    def set_tuning_class(self, max_symbols: int, key: str, value: int) -> None:
        status = self._lib.sufgpu_set_tuning_class(self._h, int(max_symbols), key.encode(),
                                                   int(value))
        if status != 0:
            _raise(status, self._error())

    def clear_tuning_classes(self) -> None:
        self._lib.sufgpu_clear_tuning_classes(self._h)

    def close(self):
        if self._h:
            self._lib.sufgpu_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _error(self) -> str:
        return self._lib.sufgpu_last_error(self._h).decode()

    def _alloc_outputs(self, n: int, sa_bits: int, isa_bits: int, lcp: LcpEncoding):
        planes = {"sa_low": np.empty(n, _plane_dtype(sa_bits))}
        if _high_dtype(sa_bits):
            planes["sa_high"] = np.empty(n, _high_dtype(sa_bits))
        if isa_bits:
            planes["isa_low"] = np.empty(n, _plane_dtype(isa_bits))
            if _high_dtype(isa_bits):
                planes["isa_high"] = np.empty(n, _high_dtype(isa_bits))
        if lcp in (LcpEncoding.RAW32, LcpEncoding.RAW64):
            planes["lcp"] = np.empty(n, np.uint32 if lcp == LcpEncoding.RAW32 else np.uint64)
        elif lcp in (LcpEncoding.BYTE32, LcpEncoding.BYTE64):
            planes["lcp"] = np.empty(n, np.uint8)
        return planes

    @staticmethod
    def _outputs(planes: dict) -> _Outputs:
        return _Outputs(*(_ptr(planes.get(k)) for k in
                          ("sa_low", "sa_high", "isa_low", "isa_high", "lcp",
                           "prefix_intervals", "child")))

    @staticmethod
    def _anchors(a: _Anchors, lcp: LcpEncoding):
        if lcp not in (LcpEncoding.BYTE32, LcpEncoding.BYTE64):
            return None, None
        dtype = np.uint32 if a.coordinate_bits == 32 else np.uint64
        if a.count == 0 or not a.positions:
            return np.empty(0, dtype), np.empty(0, dtype)
        size = int(a.count) * np.dtype(dtype).itemsize
        pos = np.frombuffer(ctypes.string_at(a.positions, size), dtype=dtype).copy()
        val = np.frombuffer(ctypes.string_at(a.values, size), dtype=dtype).copy()
        return pos, val

    def build(self, text, sa_bits: int = 32, isa_bits: int = 32,
              lcp: LcpEncoding = LcpEncoding.RAW32, validate: bool = False,
              sampling_rate: int = 1, prefix_k: int = 0,
              plane_crc: bool = False, child: bool = False) -> BuildResult:
        """One complete build of ``text`` (the logical text including its
        sentinel).  Returns host planes; see include/sufgpu/sufgpu.h.  With
        sampling_rate K > 1 the planes hold the ceil(n / K) suffixes at
        positions that are multiples of K.  prefix_k > 0 also returns the Fast
        index's k-mer directory (4^k entries begin | end << 32).  child also
        returns the compact CHILD table (uint32 rows, n = no link)."""
        t = _as_text(text)
        n = int(t.size)
        lcp = LcpEncoding(lcp)
        planes = self._alloc_outputs(_rows(n, sampling_rate), sa_bits, isa_bits, lcp)
        if prefix_k:
            planes["prefix_intervals"] = np.empty(1 << (2 * prefix_k), np.uint64)
        if child:
            planes["child"] = np.empty(n, np.uint32)
        flags = ((FLAG_VALIDATE if validate else 0) | (FLAG_PLANE_CRC if plane_crc else 0)
                 | (FLAG_CHILD if child else 0))
        desc = _Desc(sa_bits, isa_bits, int(lcp), flags, int(sampling_rate), int(prefix_k))
        out = self._outputs(planes)
        anchors = _Anchors()
        stats = _Stats()
        status = self._lib.sufgpu_build(self._h, _ptr(t), n, ctypes.byref(desc),
                                        ctypes.byref(out), ctypes.byref(anchors),
                                        ctypes.byref(stats))
        if status != 0:
            _raise(status, self._error())
        pos, val = self._anchors(anchors, lcp)
        self.last_stats = stats.as_dict()
        return BuildResult(anchor_positions=pos, anchor_values=val,
                           stats=self.last_stats, **planes)

    def build_batch(self, texts: Sequence, sa_bits: int = 32, isa_bits: int = 0,
                    lcp: LcpEncoding = LcpEncoding.RAW32,
                    validate: bool = False, sampling_rate: int = 1) -> list[BuildResult]:
        """Builds many independent references with the same launches."""
        ts = [_as_text(t) for t in texts]
        lcp = LcpEncoding(lcp)
        all_planes = [self._alloc_outputs(_rows(int(t.size), sampling_rate), sa_bits, isa_bits,
                                          lcp) for t in ts]
        arr = (_Instance * len(ts))()
        for j, (t, planes) in enumerate(zip(ts, all_planes)):
            arr[j].text = _ptr(t)
            arr[j].n = int(t.size)
            arr[j].out = self._outputs(planes)
        desc = _Desc(sa_bits, isa_bits, int(lcp), FLAG_VALIDATE if validate else 0,
                     int(sampling_rate))
        stats = _Stats()
        status = self._lib.sufgpu_build_batch(self._h, arr, len(ts), ctypes.byref(desc),
                                              ctypes.byref(stats))
        if status != 0:
            _raise(status, self._error())
        self.last_stats = stats.as_dict()
        results = []
        for j, planes in enumerate(all_planes):
            pos, val = self._anchors(arr[j].anchors, lcp)
            results.append(BuildResult(anchor_positions=pos, anchor_values=val,
                                       stats=self.last_stats, **planes))
        return results

    def build_collection(self, texts: Sequence, sa_bits: int = 32, isa_bits: int = 0,
                         lcp: LcpEncoding = LcpEncoding.RAW32, validate: bool = False,
                         sampling_rate: int = 1, batch_symbols: int = 0,
                         workers: int = 2) -> list[BuildResult]:
        """Builds a collection in sub-batches of at most ``batch_symbols``
        symbols on ``workers`` contexts side by side (sufgpu_build_collection);
        each result equals a single build of that text."""
        ts = [_as_text(t) for t in texts]
        lcp = LcpEncoding(lcp)
        all_planes = [self._alloc_outputs(_rows(int(t.size), sampling_rate), sa_bits, isa_bits,
                                          lcp) for t in ts]
        arr = (_Instance * max(1, len(ts)))()
        for j, (t, planes) in enumerate(zip(ts, all_planes)):
            arr[j].text = _ptr(t)
            arr[j].n = int(t.size)
            arr[j].out = self._outputs(planes)
        desc = _Desc(sa_bits, isa_bits, int(lcp), FLAG_VALIDATE if validate else 0,
                     int(sampling_rate))
        stats = _Stats()
        status = self._lib.sufgpu_build_collection(self._h, arr, len(ts), ctypes.byref(desc),
                                                   int(batch_symbols), int(workers),
                                                   ctypes.byref(stats))
        if status != 0:
            _raise(status, self._error())
        self.last_stats = stats.as_dict()
        results = []
        for j, planes in enumerate(all_planes):
            pos, val = self._anchors(arr[j].anchors, lcp)
            results.append(BuildResult(anchor_positions=pos, anchor_values=val,
                                       stats=self.last_stats, **planes))
        return results

    def build_collection_device(self, texts: Sequence[tuple[int, int]], outs: Sequence[dict],
                                sa_bits: int = 32, isa_bits: int = 0,
                                lcp: LcpEncoding = LcpEncoding.RAW32, batch_symbols: int = 0,
                                workers: int = 2) -> dict:
        """sufgpu_build_collection from (pointer, length) texts into raw
        output pointers (host or device)."""
        arr = (_Instance * max(1, len(texts)))()
        for j, ((ptr, n), o) in enumerate(zip(texts, outs)):
            arr[j].text = ptr
            arr[j].n = n
            arr[j].out = _Outputs(*(o.get(k) for k in ("sa_low", "sa_high", "isa_low",
                                                       "isa_high", "lcp")))
        desc = _Desc(sa_bits, isa_bits, int(LcpEncoding(lcp)), 0)
        stats = _Stats()
        status = self._lib.sufgpu_build_collection(self._h, arr, len(texts), ctypes.byref(desc),
                                                   int(batch_symbols), int(workers),
                                                   ctypes.byref(stats))
        if status != 0:
            _raise(status, self._error())
        self.last_stats = stats.as_dict()
        return self.last_stats

    def collection_trace(self) -> list[dict]:
        """Per sub-batch of the last collection build: its worker and the host
        seconds (since the call began) at which it started, took the compute
        gate, left it, and finished."""
        out = []
        worker = ctypes.c_uint32()
        times = (ctypes.c_double * 4)()
        for i in range(int(self._lib.sufgpu_collection_parts(self._h))):
            if self._lib.sufgpu_collection_trace(self._h, i, ctypes.byref(worker), times) != 0:
                break
            out.append({"worker": int(worker.value), "start": times[0], "gate_in": times[1],
                        "gate_out": times[2], "end": times[3]})
        return out

    def encode_fasta_bytes(self, raw) -> tuple[np.ndarray, int, int]:
        """FASTA bytes (plain, in host memory) normalised on the device
        (sufgpu_encode_fasta_device): (logical bytes without the sentinel,
        FNV-1a 64 fingerprint, record count).  Raises SufkitError with
        UNSUPPORTED_BACKEND for FASTQ and other input only the host reader
        (encode_fasta) parses."""
        buf = np.frombuffer(raw, np.uint8) if isinstance(raw, (bytes, bytearray)) else \
            np.ascontiguousarray(raw, np.uint8)
        out = np.empty(buf.size + 1, np.uint8)
        size = ctypes.c_uint64()
        fp = ctypes.c_uint64()
        count = ctypes.c_uint64()
        status = self._lib.sufgpu_encode_fasta_device(self._h, _ptr(buf), buf.size, _ptr(out),
                                                      out.size, ctypes.byref(size),
                                                      ctypes.byref(fp), ctypes.byref(count))
        if status != 0:
            _raise(status, self._error())
        return out[: size.value].copy(), int(fp.value), int(count.value)

    def crc32_device(self, ptr: int, nbytes: int, crc_in: int = 0) -> int:
        """zlib's crc32(crc_in, data, nbytes) of device memory at ptr."""
        out = ctypes.c_uint32()
        status = self._lib.sufgpu_crc32_device(self._h, ptr, int(nbytes), int(crc_in),
                                               ctypes.byref(out))
        if status != 0:
            _raise(status, self._error())
        return int(out.value)

    def set_tuning(self, key: str, value: int) -> None:
        status = self._lib.sufgpu_set_tuning(self._h, key.encode(), int(value))
        if status != 0:
            _raise(status, self._error())

    def set_profiling(self, enable: bool = True) -> None:
        self._lib.sufgpu_set_profiling(self._h, int(enable))

    def profile(self) -> list[dict]:
        """Per-kernel totals since profiling was enabled."""
        out = []
        for i in range(self._lib.sufgpu_profile_count(self._h)):
            name = ctypes.c_char_p()
            launches = ctypes.c_uint64()
            seconds = ctypes.c_double()
            nbytes = ctypes.c_uint64()
            self._lib.sufgpu_profile_entry(self._h, i, ctypes.byref(name), ctypes.byref(launches),
                                           ctypes.byref(seconds), ctypes.byref(nbytes))
            out.append({"kernel": name.value.decode(), "launches": launches.value,
                        "seconds": seconds.value, "bytes": nbytes.value})
        return out

    def build_device(self, text_ptr: int, n: int, out_ptrs: dict, sa_bits: int = 32,
                     isa_bits: int = 32, lcp: LcpEncoding = LcpEncoding.RAW32,
                     validate: bool = False) -> dict:
        """Build from a device-resident text into device-resident planes
        (raw pointers, e.g. from torch tensors).  Returns the stats."""
        desc = _Desc(sa_bits, isa_bits, int(LcpEncoding(lcp)), FLAG_VALIDATE if validate else 0)
        out = _Outputs(*(out_ptrs.get(k) for k in ("sa_low", "sa_high", "isa_low", "isa_high", "lcp",
                                                   "prefix_intervals", "child")))
        anchors = _Anchors()
        stats = _Stats()
        status = self._lib.sufgpu_build(self._h, text_ptr, n, ctypes.byref(desc), ctypes.byref(out),
                                        ctypes.byref(anchors), ctypes.byref(stats))
        if status != 0:
            _raise(status, self._error())
        self.last_stats = stats.as_dict()
        # Byte-coded builds: the overflow anchors (host copies), else (None, None).
        self.last_anchors = self._anchors(anchors, LcpEncoding(lcp))
        return self.last_stats

    def build_batch_device(self, texts: Sequence[tuple[int, int]], outs: Sequence[dict],
                           sa_bits: int = 32, isa_bits: int = 0,
                           lcp: LcpEncoding = LcpEncoding.RAW32, validate: bool = False) -> dict:
        """Batched build from (pointer, length) texts into raw output pointers."""
        arr = (_Instance * len(texts))()
        for j, ((ptr, n), o) in enumerate(zip(texts, outs)):
            arr[j].text = ptr
            arr[j].n = n
            arr[j].out = _Outputs(*(o.get(k) for k in ("sa_low", "sa_high", "isa_low",
                                                       "isa_high", "lcp")))
        desc = _Desc(sa_bits, isa_bits, int(LcpEncoding(lcp)), FLAG_VALIDATE if validate else 0)
        stats = _Stats()
        status = self._lib.sufgpu_build_batch(self._h, arr, len(texts), ctypes.byref(desc),
                                              ctypes.byref(stats))
        if status != 0:
            _raise(status, self._error())
        self.last_stats = stats.as_dict()
        return self.last_stats

    def divsufsort64(self, text) -> np.ndarray:
        """Drop-in for libdivsufsort's divsufsort64 (returns the int64 SA)."""
        t = _as_text(text)
        sa = np.empty(t.size, np.int64)
        rc = self._lib.sufgpu_divsufsort64(self._h, _ptr(t), _ptr(sa), int(t.size))
        if rc != 0:
            raise SufkitError(ErrorCode.BUILD_FAILURE, f"divsufsort64 returned {rc}: {self._error()}")
        return sa

    def divsufsort(self, text) -> np.ndarray:
        t = _as_text(text)
        sa = np.empty(t.size, np.int32)
        rc = self._lib.sufgpu_divsufsort(self._h, _ptr(t), _ptr(sa), int(t.size))
        if rc != 0:
            raise SufkitError(ErrorCode.BUILD_FAILURE, f"divsufsort returned {rc}: {self._error()}")
        return sa


class Server:
    """Continuously batched builds (sufgpu_server_*): submit references while
    others are on the GPU; each result equals Context.build of the same text."""

    def __init__(self, device: int = 0, capacity_symbols: int = 0, max_instances: int = 0):
        lib = library()
        handle = ctypes.c_void_p()
        cfg = _ServerConfig(capacity_symbols, max_instances, 0)
        status = lib.sufgpu_server_create(ctypes.byref(handle), device, ctypes.byref(cfg))
        if status != 0:
            _raise(status, "cannot create the build server: " + lib.sufgpu_last_error(None).decode())
        self._lib = lib
        self._h = handle
        self._pending: dict[int, tuple] = {}

    def submit(self, text, sa_bits: int = 32, isa_bits: int = 0,
               lcp: LcpEncoding = LcpEncoding.RAW32, validate: bool = False,
               planes: Optional[dict] = None) -> int:
        """Queues one build.  ``planes`` may supply the output arrays (for
        example pinned ones from pinned_array); otherwise they are allocated."""
        t = np.ascontiguousarray(_as_text(text))
        lcp = LcpEncoding(lcp)
        if planes is None:
            planes = Context._alloc_outputs(None, int(t.size), sa_bits, isa_bits, lcp)
        desc = _Desc(sa_bits, isa_bits, int(lcp), FLAG_VALIDATE if validate else 0)
        out = Context._outputs(planes)
        ticket = ctypes.c_uint64()
        status = self._lib.sufgpu_server_submit(self._h, _ptr(t), int(t.size), ctypes.byref(desc),
                                                ctypes.byref(out), ctypes.byref(ticket))
        if status != 0:
            _raise(status, "submit rejected")
        # Keep the text and the planes alive until the request completes.
        self._pending[ticket.value] = (t, planes, lcp)
        return ticket.value

    def wait(self, ticket: int) -> BuildResult:
        info = _RequestInfo()
        status = self._lib.sufgpu_server_wait(self._h, ticket, ctypes.byref(info))
        t, planes, lcp = self._pending.pop(ticket)
        if status != 0:
            self._lib.sufgpu_server_release(self._h, ticket)
            _raise(status, f"served build {ticket} failed")
        pos, val = Context._anchors(info.anchors, lcp)
        self._lib.sufgpu_server_release(self._h, ticket)
        stats = {"queue_seconds": info.queue_seconds, "latency_seconds": info.latency_seconds,
                 "rounds": info.rounds, "seed_symbols": info.seed_symbols,
                 "admit_iteration": info.admit_iteration,
                 "finish_iteration": info.finish_iteration,
                 "inflight_at_admit": info.inflight_at_admit}
        return BuildResult(anchor_positions=pos, anchor_values=val, stats=stats, **planes)

    def stats(self) -> dict:
        st = _ServerStats()
        self._lib.sufgpu_server_get_stats(self._h, ctypes.byref(st))
        return st.as_dict()

    def close(self):
        if self._h:
            self._lib.sufgpu_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class CudaBuildResult:
    """Field-for-field mirror of detail::DivSufsortBuildResult<Index>
    (src/divsufsort_backend.hpp:13-25)."""

    suffix_array: np.ndarray
    isa: np.ndarray
    lcp: np.ndarray
    sa_seconds: float = 0.0
    isa_seconds: float = 0.0
    lcp_seconds: float = 0.0


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def prefix_select_k(suffix_count: int, resident_core_bytes: int) -> int:
    """FastPrefixIndex::SelectK with its default options: the directory's k
    (8..10) for an index of this size, 0 for none."""
    return int(library().sufgpu_prefix_select_k(int(suffix_count), int(resident_core_bytes)))


def _rows(n: int, sampling_rate: int) -> int:
    """Rows of a plane: n, or ceil(n / K) for sampling rate K > 1."""
    return n if sampling_rate <= 1 else (n + sampling_rate - 1) // sampling_rate


def _build_cuda(width: int, text, sampling_rate: int, retain_lcp: bool, retain_isa: bool,
                threads: int) -> CudaBuildResult:
    """Same contract as BuildDivsufsort<Index> (src/divsufsort_backend.cpp:24-157):
    SA in Index (the suffixes at multiples of sampling_rate), ISA/LCP as uint64
    when retained."""
    t = _as_text(text)
    if sampling_rate < 1:
        raise SufkitError(ErrorCode.INVALID_INPUT, "sampling rate must be at least 1")
    if threads == 0:
        raise SufkitError(ErrorCode.INVALID_INPUT, "thread count must be greater than zero")
    limit = np.iinfo(np.int32).max if width == 32 else np.iinfo(np.int64).max
    if t.size > limit:
        raise SufkitError(ErrorCode.INVALID_INPUT,
                          f"reference is too large for divsufsort{width}")
    ctx = default_context()
    r = ctx.build(t, sa_bits=64 if width == 64 else 32,
                  isa_bits=64 if (retain_isa or retain_lcp) else 0,
                  lcp=LcpEncoding.RAW64 if retain_lcp else LcpEncoding.NONE,
                  sampling_rate=sampling_rate)
    sa = r.sa_low.astype(np.int32 if width == 32 else np.int64, copy=False)
    st = r.stats
    return CudaBuildResult(
        suffix_array=sa,
        isa=r.isa_low if retain_isa else np.empty(0, np.uint64),
        lcp=r.lcp if retain_lcp else np.empty(0, np.uint64),
        sa_seconds=st["sa_seconds"], isa_seconds=st["isa_seconds"],
        lcp_seconds=st["lcp_seconds"])


def build_cuda32(text, sampling_rate: int = 1, retain_lcp: bool = False,
                 retain_isa: bool = False, threads: int = 1) -> CudaBuildResult:
    return _build_cuda(32, text, sampling_rate, retain_lcp, retain_isa, threads)


def build_cuda64(text, sampling_rate: int = 1, retain_lcp: bool = False,
                 retain_isa: bool = False, threads: int = 1) -> CudaBuildResult:
    return _build_cuda(64, text, sampling_rate, retain_lcp, retain_isa, threads)


class _Pinned:
    def __init__(self, nbytes: int):
        self.addr = library().sufgpu_host_alloc(max(1, nbytes))
        if not self.addr:
            raise SufkitError(ErrorCode.BUILD_FAILURE, "cannot allocate pinned host memory")

    def __del__(self):
        try:
            library().sufgpu_host_free(self.addr)
        except Exception:
            pass


def pinned_array(count: int, dtype=np.uint8) -> np.ndarray:
    """A numpy array in page-locked host memory (freed with the array)."""
    dtype = np.dtype(dtype)
    holder = _Pinned(count * dtype.itemsize)
    buf = (ctypes.c_uint8 * max(1, count * dtype.itemsize)).from_address(holder.addr)
    arr = np.frombuffer(buf, dtype=np.uint8)[: count * dtype.itemsize].view(dtype)
    arr.flags.writeable = True
    _PINNED_OWNERS[id(arr)] = holder
    import weakref
    weakref.finalize(arr, _PINNED_OWNERS.pop, id(arr), None)
    return arr


_PINNED_OWNERS: dict = {}


def encode_fasta(path) -> tuple[np.ndarray, int, int]:
    """GenomeReference::FromFasta normalization: (encoded bytes without the
    sentinel, FNV-1a fingerprint, record count)."""
    lib = library()
    size = ctypes.c_uint64()
    fp = ctypes.c_uint64()
    recs = ctypes.c_uint64()
    raw = str(path).encode()
    status = lib.sufgpu_encode_fasta(raw, None, 0, ctypes.byref(size), ctypes.byref(fp),
                                     ctypes.byref(recs))
    if status not in (0,):
        _raise(status, f"cannot normalize FASTA {path}")
    out = np.empty(size.value, np.uint8)
    status = lib.sufgpu_encode_fasta(raw, _ptr(out), size.value, ctypes.byref(size),
                                     ctypes.byref(fp), ctypes.byref(recs))
    if status != 0:
        _raise(status, f"cannot normalize FASTA {path}")
    return out, fp.value, recs.value


def logical_text(encoded: np.ndarray) -> np.ndarray:
    """Appends the unique 0 sentinel (src/suffix_array.cpp:4113-4117)."""
    return np.concatenate([np.asarray(encoded, np.uint8), np.zeros(1, np.uint8)])
