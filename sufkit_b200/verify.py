"""Size-independent checks of a built SA/LCP pair (vectorized numpy).

A suffix array with its LCP array is exact iff
  (1) SA is a permutation of [0, n),
  (2) for every adjacent pair (a, b) = (SA[r-1], SA[r]) with l = LCP[r]:
      the first l symbols of a and b are equal, and
  (3) either a + l == n (a is a proper prefix of b) or b + l < n and
      text[a + l] < text[b + l].
(2) is checked with a polynomial hash of text prefixes modulo two 31-bit
primes, (1) and (3) exactly.  Used by tests at sizes where the CPU oracle is
too slow; the kernels under test never call it.
"""
from __future__ import annotations

import numpy as np

_PRIMES = (2147483629, 2147483587)
_BASE = 1_000_003


def _prefix_hash(text: np.ndarray, p: int):
    n = text.size
    block = 1 << 12
    small = np.empty(block, np.uint64)
    small[0] = 1
    for i in range(1, block):
        small[i] = small[i - 1] * _BASE % p
    big_count = n // block + 2
    big = np.empty(big_count, np.uint64)
    big[0] = 1
    step = int(small[block - 1]) * _BASE % p
    for i in range(1, big_count):
        big[i] = big[i - 1] * step % p

    def power(k):
        k = np.asarray(k, np.uint64)
        return small[k % block] * big[k // block] % p

    inv_base = pow(_BASE, p - 2, p)
    small_inv = np.empty(block, np.uint64)
    small_inv[0] = 1
    for i in range(1, block):
        small_inv[i] = small_inv[i - 1] * inv_base % p
    big_inv = np.empty(big_count, np.uint64)
    big_inv[0] = 1
    step_inv = int(small_inv[block - 1]) * inv_base % p
    for i in range(1, big_count):
        big_inv[i] = big_inv[i - 1] * step_inv % p
    idx = np.arange(n, dtype=np.uint64)
    terms = (text.astype(np.uint64) + 1) * (small_inv[idx % block] * big_inv[idx // block] % p) % p
    h = np.zeros(n + 1, np.uint64)
    # Cumulative sums stay below 2^63 in chunks of 2^31 terms.
    chunk = 1 << 30
    acc = 0
    for s in range(0, n, chunk):
        c = np.cumsum(terms[s:s + chunk]) % p
        h[s + 1:s + 1 + c.size] = (c + acc) % p
        acc = int(h[s + c.size])
    return h, power


def _substring_hashes(h, power, p, starts, length):
    # sum_{k<l} t[s+k] B^{-(s+k)} * B^{s} = sum t[s+k] B^{-k}
    v = (h[starts + length] + p - h[starts]) % p
    return v * power(starts) % p


def check_suffix_array(text: np.ndarray, sa: np.ndarray, lcp: np.ndarray | None = None) -> None:
    """Raises AssertionError when SA (and LCP, if given) are not exact."""
    text = np.ascontiguousarray(text, np.uint8)
    n = text.size
    sa = np.asarray(sa).astype(np.uint64)
    assert sa.size == n
    seen = np.bincount(sa.astype(np.int64), minlength=n) if n else np.zeros(0)
    assert n == 0 or (seen.max() == 1 and seen.min() == 1), "SA is not a permutation"
    if n < 2:
        if lcp is not None and n == 1:
            assert int(lcp[0]) == 0
        return
    a = sa[:-1]
    b = sa[1:]
    if lcp is None:
        raise ValueError("LCP required for the order check")
    l = np.asarray(lcp).astype(np.uint64)
    assert int(l[0]) == 0, "LCP[0] must be 0"
    l = l[1:]
    assert (a + l <= n).all() and (b + l <= n).all(), "LCP exceeds suffix length"
    # (3) ordering at the first mismatch
    a_end = a + l == n
    ok = a_end.copy()
    inside = ~a_end & (b + l < n)
    ok[inside] = text[(a + l)[inside]] < text[(b + l)[inside]]
    assert ok.all(), f"order/LCP mismatch at rows {np.flatnonzero(~ok)[:5] + 1}"
    # (2) equal prefixes of length l
    for p in _PRIMES:
        h, power = _prefix_hash(text, p)
        ha = _substring_hashes(h, power, p, a, l)
        hb = _substring_hashes(h, power, p, b, l)
        bad = np.flatnonzero(ha != hb)
        assert bad.size == 0, f"prefix mismatch at rows {bad[:5] + 1}"


def plcp_from(sa: np.ndarray, lcp: np.ndarray) -> np.ndarray:
    out = np.empty(sa.size, np.uint64)
    out[np.asarray(sa, np.int64)] = np.asarray(lcp, np.uint64)
    return out
