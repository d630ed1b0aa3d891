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


# ---------------------------------------------------------------------------
# The same checks on device tensors (torch), for builds whose host copies
# would not fit: a 3.1 Gsym text needs ~80 GB of device memory here.
# ---------------------------------------------------------------------------
def _u32(t, torch):
    """int32 tensor holding uint32 bits -> int64 values."""
    return t.to(torch.int64) & 0xFFFFFFFF


def _device_powers(p: int, count: int, torch, dev):
    """B^k mod p for k < count as small[k & 0xffff] * big[k >> 16] mod p."""
    small = [1] * 65536
    for i in range(1, 65536):
        small[i] = small[i - 1] * _BASE % p
    step = small[65535] * _BASE % p
    big_n = count // 65536 + 2
    big = [1] * big_n
    for i in range(1, big_n):
        big[i] = big[i - 1] * step % p
    return (torch.tensor(small, dtype=torch.int64, device=dev),
            torch.tensor(big, dtype=torch.int64, device=dev))


def _pow_of(k, tables, p):
    small, big = tables
    return small[k & 0xFFFF] * big[k >> 16] % p


def check_suffix_array_device(d_text, d_sa, d_lcp, torch, chunk: int = 1 << 26) -> None:
    """check_suffix_array for device tensors: d_text uint8 (n), d_sa and d_lcp
    int32 holding uint32 values (n rows).  (1) and (3) exactly, (2) by the
    polynomial hash H[i] = sum_{j<i} (t[j]+1) B^j mod p (two 31-bit primes),
    comparing (H[a+l]-H[a]) B^b with (H[b+l]-H[b]) B^a."""
    dev = d_text.device
    n = int(d_text.numel())
    assert int(d_sa.numel()) == n and int(d_lcp.numel()) == n
    if n == 0:
        return
    # (1) permutation: every entry in [0, n) and every position hit.
    seen = torch.zeros(n, dtype=torch.uint8, device=dev)
    for s in range(0, n, chunk):
        v = _u32(d_sa[s:s + chunk], torch)
        assert int(v.max().item()) < n, "SA entry out of range"
        seen[v] = 1
    assert bool((seen == 1).all().item()), "SA is not a permutation"
    del seen
    assert int(_u32(d_lcp[:1], torch).item()) == 0, "LCP[0] must be 0"
    # (3) order at the first mismatch, and the LCP range.
    for s in range(1, n, chunk):
        e = min(n, s + chunk)
        a = _u32(d_sa[s - 1:e - 1], torch)
        b = _u32(d_sa[s:e], torch)
        l = _u32(d_lcp[s:e], torch)
        assert bool(((a + l <= n) & (b + l <= n)).all().item()), "LCP exceeds suffix length"
        a_end = a + l == n
        inside = ~a_end & (b + l < n)
        ta = d_text[torch.where(inside, a + l, torch.zeros_like(a))].to(torch.int16)
        tb = d_text[torch.where(inside, b + l, torch.zeros_like(b))].to(torch.int16)
        ok = a_end | (inside & (ta < tb))
        if not bool(ok.all().item()):
            bad = torch.nonzero(~ok).flatten()[:5] + s
            raise AssertionError(f"order/LCP mismatch at rows {bad.tolist()}")
    # (2) equal prefixes of length l, one prime at a time.
    for p in _PRIMES:
        tables = _device_powers(p, n + 1, torch, dev)
        h = torch.zeros(n + 1, dtype=torch.int64, device=dev)
        carry = 0
        for s in range(0, n, chunk):
            e = min(n, s + chunk)
            k = torch.arange(s, e, dtype=torch.int64, device=dev)
            terms = (d_text[s:e].to(torch.int64) + 1) * _pow_of(k, tables, p) % p
            c = torch.cumsum(terms, 0)  # < 2^26 * 2^31: no overflow
            h[s + 1:e + 1] = (c + carry) % p
            carry = int(h[e].item())
            del k, terms, c
        for s in range(1, n, chunk):
            e = min(n, s + chunk)
            a = _u32(d_sa[s - 1:e - 1], torch)
            b = _u32(d_sa[s:e], torch)
            l = _u32(d_lcp[s:e], torch)
            ha = (h[a + l] - h[a]) % p
            hb = (h[b + l] - h[b]) % p
            lhs = ha * _pow_of(b, tables, p) % p
            rhs = hb * _pow_of(a, tables, p) % p
            if not bool((lhs == rhs).all().item()):
                bad = torch.nonzero(lhs != rhs).flatten()[:5] + s
                raise AssertionError(f"prefix mismatch at rows {bad.tolist()}")
        del h


def bytecode_device(d_sa, d_lcp, torch, chunk: int = 1 << 26):
    """Byte-coded LCP of a single text from its exact SA and row LCP on the
    device: primary[r] = min(LCP[r], 255) and the text-ordered anchors, the
    positions p with PLCP[p] >= 255 that do not continue the run of p-1
    (PLCP[p-1] >= 255 and PLCP[p-1] - 1 == PLCP[p]); the restated rule of
    LcpStorage::BuildByteDataDirect (src/lcp_storage.cpp:394-412).  Returns
    (primary uint8, anchor positions int64, anchor values int64) tensors."""
    dev = d_sa.device
    n = int(d_sa.numel())
    primary = torch.empty(n, dtype=torch.uint8, device=dev)
    plcp = torch.empty(n, dtype=torch.int32, device=dev)
    for s in range(0, n, chunk):
        l = _u32(d_lcp[s:s + chunk], torch)
        primary[s:s + chunk] = torch.clamp(l, max=255).to(torch.uint8)
        plcp[_u32(d_sa[s:s + chunk], torch)] = d_lcp[s:s + chunk]
    pos, val = [], []
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        cur = _u32(plcp[s:e], torch)
        prev = torch.empty_like(cur)
        prev[1:] = cur[:-1]
        prev[0] = _u32(plcp[s - 1:s], torch)[0] if s > 0 else 0
        over = cur >= 255
        cont = over & (prev >= 255) & (prev - 1 == cur)
        if s == 0:
            cont[0] = False
        opens = torch.nonzero(over & ~cont).flatten()
        pos.append(opens + s)
        val.append(cur[opens])
    del plcp
    return primary, torch.cat(pos), torch.cat(val)
