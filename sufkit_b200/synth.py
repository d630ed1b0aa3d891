"""Seeded synthetic references with the shapes of the five build workloads.

Every generator returns encoded contigs in sufkit's logical-text alphabet
(A/C/G/T = 2..5, N = 6; src/reference_data.hpp:20-26) so that
``logical_text(contigs)`` equals what GenomeReference::FromFasta +
SuffixArray::Build would hand the constructor for the same FASTA
(src/genome_reference.cpp:131-156, src/suffix_array.cpp:4113-4117).
``write_fasta`` writes that FASTA for the reference's own reader.

Seeds are 20260822 + workload index.  ``scale`` shrinks a workload
proportionally (tests use small scales; benchmarks use 1.0).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Iterator, Optional

import numpy as np

BASE_SEED = 20260822
A, C, G, T, N = 2, 3, 4, 5, 6
_ASCII = np.frombuffer(b"??ACGTN", dtype=np.uint8)


def _bases(rng: np.random.Generator, n: int, gc: float) -> np.ndarray:
    """i.i.d. bases with the given GC fraction (resolution 1/65536), via a
    16-bit uniform draw and three thresholds (fast for multi-Gbp inputs)."""
    u = rng.integers(0, 1 << 16, size=n, dtype=np.uint16)
    at = int(round((1.0 - gc) / 2 * 65536))
    cg = int(round(gc / 2 * 65536))
    out = np.full(n, T, np.uint8)
    out[u < at + 2 * cg] = G
    out[u < at + cg] = C
    out[u < at] = A
    return out


def _mutate(rng: np.random.Generator, seq: np.ndarray, rate: float, gc: float) -> np.ndarray:
    out = seq.copy()
    hits = rng.random(out.size) < rate
    k = int(hits.sum())
    if k:
        # A substitution always changes the base.
        shift = rng.integers(1, 4, size=k).astype(np.uint8)
        out[hits] = ((out[hits] - A + shift) % 4) + A
    return out


def _n_runs(rng, genome: np.ndarray, total: int, lo: int, hi: int, log: bool) -> None:
    placed = 0
    while placed < total:
        if log:
            length = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        else:
            length = int(rng.integers(lo, hi + 1))
        length = min(length, total - placed, genome.size)
        if length <= 0:
            break
        start = int(rng.integers(0, genome.size - length + 1))
        genome[start:start + length] = N
        placed += length


def _interspersed(rng, genome: np.ndarray, fraction: float, families: int, gc: float,
                  lo: int = 300, hi: int = 6000, div=(0.05, 0.15), consensus=None) -> None:
    if consensus is None:
        lengths = np.exp(rng.uniform(np.log(lo), np.log(hi), size=families)).astype(np.int64)
        consensus = [_bases(rng, int(L), gc) for L in lengths]
    target = int(fraction * genome.size)
    placed = 0
    while placed < target:
        f = int(rng.integers(0, families))
        cons = consensus[f]
        L = min(cons.size, genome.size)
        start = int(rng.integers(0, genome.size - L + 1))
        genome[start:start + L] = _mutate(rng, cons[:L], rng.uniform(*div), gc)
        placed += L


def _tandem(rng, genome: np.ndarray, fraction: float, gc: float) -> None:
    target = int(fraction * genome.size)
    placed = 0
    while placed < target:
        period = int(rng.integers(1, 51))
        copies = int(rng.integers(5, 201))
        unit = _bases(rng, period, gc)
        arr = np.tile(unit, copies)[: genome.size]
        start = int(rng.integers(0, genome.size - arr.size + 1))
        genome[start:start + arr.size] = arr
        placed += arr.size


def _segdups(rng, genome: np.ndarray, fraction: float, gc: float) -> None:
    target = int(fraction * genome.size)
    placed = 0
    while placed < target:
        L = min(int(rng.integers(10_000, 200_001)), genome.size // 2)
        src = int(rng.integers(0, genome.size - L + 1))
        dst = int(rng.integers(0, genome.size - L + 1))
        genome[dst:dst + L] = _mutate(rng, genome[src:src + L], rng.uniform(0.01, 0.03), gc)
        placed += L


def _split(genome: np.ndarray, lengths: np.ndarray) -> list[np.ndarray]:
    cuts = np.cumsum(lengths)[:-1]
    return np.split(genome, cuts)


def _scaled_lengths(raw: np.ndarray, total: int) -> np.ndarray:
    lengths = np.maximum(1, np.floor(raw / raw.sum() * total)).astype(np.int64)
    lengths[-1] += total - lengths.sum()
    return lengths


@dataclass
class Reference:
    """One reference: its contigs in logical-text bytes (no separators)."""

    contigs: list[np.ndarray]

    @property
    def total_bases(self) -> int:
        return int(sum(c.size for c in self.contigs))

    def encoded(self) -> np.ndarray:
        """GenomeReference bytes: every contig followed by a 1 separator."""
        parts = []
        for c in self.contigs:
            parts.append(c)
            parts.append(np.ones(1, np.uint8))
        return np.concatenate(parts) if parts else np.zeros(0, np.uint8)

    def logical_text(self) -> np.ndarray:
        """Encoded bytes plus the 0 sentinel SuffixArray::Build appends."""
        return np.concatenate([self.encoded(), np.zeros(1, np.uint8)])

    def write_fasta(self, path, width: int = 80) -> None:
        with open(path, "wb") as f:
            for i, c in enumerate(self.contigs):
                f.write(b">contig%d synthetic\n" % i)
                ascii_ = _ASCII[c]
                for s in range(0, ascii_.size, width):
                    f.write(ascii_[s:s + width].tobytes() + b"\n")


def plain_4mbp(scale: float = 1.0, seed: Optional[int] = None) -> Reference:
    """Workload 1: 4 contigs (1.5/1.2/0.8/0.5 Mbp), uniform ACGT, 0.1% of
    positions in N runs of geometric length 1-100 (mean ~10)."""
    rng = np.random.default_rng(BASE_SEED + 0 if seed is None else seed)
    lengths = (np.array([1.5e6, 1.2e6, 0.8e6, 0.5e6]) * scale).astype(np.int64)
    lengths = np.maximum(lengths, 1)
    genome = _bases(rng, int(lengths.sum()), 0.5)
    target = int(0.001 * genome.size)
    placed = 0
    while placed < target:
        L = min(int(min(100, rng.geometric(0.1))), target - placed)
        s = int(rng.integers(0, genome.size - L + 1))
        genome[s:s + L] = N
        placed += L
    return Reference(_split(genome, lengths))


def repeat_rich_100mbp(scale: float = 1.0, seed: Optional[int] = None) -> Reference:
    """Workload 2: 24 contigs (U(1,8) Mbp scaled to 100 Mbp), GC 41%; 25% from
    500 repeat families (consensus log-uniform 300 bp-6 kbp, copies at 5-15%
    substitution divergence), 3% tandem repeats (period 1-50, 5-200 copies),
    0.5% N in runs."""
    rng = np.random.default_rng(BASE_SEED + 1 if seed is None else seed)
    total = max(1000, int(100e6 * scale))
    lengths = _scaled_lengths(rng.uniform(1e6, 8e6, size=24), total)
    genome = _bases(rng, total, 0.41)
    _interspersed(rng, genome, 0.25, 500, 0.41)
    _tandem(rng, genome, 0.03, 0.41)
    _n_runs(rng, genome, int(0.005 * total), 10, 5000, log=True)
    return Reference(_split(genome, lengths))


def _human_contig(task) -> np.ndarray:
    """One contig of the human-scale reference from its own random stream:
    bases at GC 41%, interspersed copies of the shared repeat families up to
    50% of the contig, segmental duplications (10-200 kbp at 1-3% divergence)
    up to 1%, and the contig's share of the N runs (log-uniform lengths)."""
    seed, index, length, consensus, n_budget, lo, hi = task
    rng = np.random.default_rng([seed, index])
    genome = np.empty(length, np.uint8)
    step = 1 << 25  # bounded temporaries for 250 Mbp contigs
    for s in range(0, length, step):
        genome[s:s + step] = _bases(rng, min(step, length - s), 0.41)
    _interspersed(rng, genome, 0.50, len(consensus), 0.41, consensus=consensus)
    _segdups(rng, genome, 0.01, 0.41)
    _n_runs(rng, genome, n_budget, lo, hi, log=True)
    return genome


def human_scale_3gbp(scale: float = 1.0, seed: Optional[int] = None,
                     workers: Optional[int] = None) -> Reference:
    """Workload 3: 25 contigs (50-250 Mbp scaled to 3.1 Gbp), GC 41%; 50%
    interspersed repeats from 500 families as in workload 2, 1% segmental
    duplications (10-200 kbp at 1-3% divergence), 150 Mbp of N in runs of
    10 kbp-3 Mbp (scaled), spread over the contigs by length.

    Each contig comes from its own random stream (seed, contig index), so the
    contigs are generated in parallel (spawned worker processes, safe after
    CUDA initialisation) for large scales; the result does not depend on the
    number of workers."""
    base = BASE_SEED + 2 if seed is None else seed
    rng = np.random.default_rng(base)
    total = max(10_000, int(3.1e9 * scale))
    lengths = _scaled_lengths(rng.uniform(50e6, 250e6, size=25), total)
    fam_len = np.exp(rng.uniform(np.log(300), np.log(6000), size=500)).astype(np.int64)
    consensus = [_bases(rng, int(L), 0.41) for L in fam_len]
    n_total = int(150e6 * scale)
    hi = max(20, int(3e6 * min(1.0, scale * 10)))
    lo = min(10_000, hi // 2)
    n_share = _scaled_lengths(lengths.astype(np.float64), n_total) if n_total >= 25 else \
        np.zeros(25, np.int64)
    tasks = [(base, i, int(lengths[i]), consensus, int(n_share[i]), lo, hi) for i in range(25)]
    if workers is None:
        import os
        workers = min(25, os.cpu_count() or 1) if total >= 64_000_000 else 1
    if workers > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            contigs = list(ex.map(_human_contig, tasks))
    else:
        contigs = [_human_contig(t) for t in tasks]
    return Reference(contigs)


def uneven_collection(count: int = 1024, scale: float = 1.0,
                      seed: Optional[int] = None) -> list[Reference]:
    """Workload 4: bacterial-like genomes, lengths log-normal (median 4 Mbp,
    clipped to 0.5-12 Mbp; sigma 0.5 gives ~4.5 Gbp for 1,024), GC U(30%,70%),
    1-8 contigs each."""
    rng = np.random.default_rng(BASE_SEED + 3 if seed is None else seed)
    sizes = np.clip(rng.lognormal(np.log(4e6), 0.5, size=count), 0.5e6, 12e6) * scale
    refs = []
    for size in sizes:
        gc = rng.uniform(0.30, 0.70)
        total = max(64, int(size))
        k = int(rng.integers(1, 9))
        lengths = _scaled_lengths(rng.uniform(0.2, 1.0, size=k), total)
        refs.append(Reference(_split(_bases(rng, total, gc), lengths)))
    return refs


def uneven_sizes(count: int, scale: float = 1.0, seed: Optional[int] = None) -> list[int]:
    """Lengths of a bacterial collection of `count` references (log-normal,
    median 4 Mbp, clipped to 0.5-12 Mbp), without generating the sequences."""
    rng = np.random.default_rng(BASE_SEED + 13 if seed is None else seed)
    sizes = np.clip(rng.lognormal(np.log(4e6), 0.5, size=count), 0.5e6, 12e6) * scale
    return [max(64, int(x)) for x in sizes]


def uneven_reference(index: int, total: int, seed: Optional[int] = None) -> Reference:
    """Reference `index` of such a collection with its own random stream, so
    that any subset (one GPU's share) is generated without the rest: GC
    U(30%,70%), 1-8 contigs."""
    rng = np.random.default_rng([BASE_SEED + 13 if seed is None else seed, index])
    gc = rng.uniform(0.30, 0.70)
    k = int(rng.integers(1, 9))
    lengths = _scaled_lengths(rng.uniform(0.2, 1.0, size=k), total)
    return Reference(_split(_bases(rng, total, gc), lengths))


def _uneven_text(task) -> np.ndarray:
    index, total, seed = task
    return uneven_reference(index, total, seed).logical_text()


def uneven_texts(count: int = 1024, scale: float = 1.0, indices=None,
                 seed: Optional[int] = None, workers: Optional[int] = None) -> list[np.ndarray]:
    """Logical texts of references `indices` (default: all) of a bacterial
    collection of `count` (uneven_sizes lengths, uneven_reference streams),
    generated in spawned worker processes when the total is large; the result
    does not depend on the number of workers."""
    sizes = uneven_sizes(count, scale, None if seed is None else seed)
    idx = list(range(count)) if indices is None else list(indices)
    tasks = [(i, sizes[i], seed) for i in idx]
    if workers is None:
        import os
        total = sum(sizes[i] for i in idx)
        workers = min(32, os.cpu_count() or 1) if total >= 64_000_000 else 1
    if workers > 1 and len(tasks) > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(_uneven_text, tasks, chunksize=4))
    return [_uneven_text(t) for t in tasks]


def strain_collection(copies: int = 50, genome_bp: int = 2_000_000,
                      rng: Optional[np.random.Generator] = None) -> Reference:
    """50 copies of one random genome at 0.1% SNP + 0.01% indel divergence."""
    rng = rng or np.random.default_rng(BASE_SEED + 4)
    base = _bases(rng, genome_bp, 0.5)
    contigs = []
    for _ in range(copies):
        c = _mutate(rng, base, 0.001, 0.5)
        indel = np.flatnonzero(rng.random(c.size) < 0.0001)
        if indel.size:
            keep = np.ones(c.size, bool)
            keep[indel[::2]] = False  # deletions
            c = c[keep]
            ins = indel[1::2]
            ins = ins[ins < c.size]
            c = np.insert(c, ins, _bases(rng, ins.size, 0.5))
        contigs.append(c.astype(np.uint8))
    return Reference(contigs)


@dataclass
class Request:
    arrival_s: float
    reference: Reference


def served_stream(requests: int = 20_000, scale: float = 1.0, rate_hz: float = 50.0,
                  seed: Optional[int] = None) -> Iterator[Request]:
    """Workload 5: Poisson arrivals; sizes log-normal clipped to 10 kbp-50 Mbp;
    20% of requests are strain collections (50 x 2 Mbp at 0.1% SNP + 0.01%
    indel; sizes scaled by ``scale``)."""
    rng = np.random.default_rng(BASE_SEED + 4 if seed is None else seed)
    t = 0.0
    for _ in range(requests):
        t += rng.exponential(1.0 / rate_hz)
        if rng.random() < 0.2:
            ref = strain_collection(50, max(1000, int(2e6 * scale)), rng)
        else:
            size = int(np.clip(rng.lognormal(np.log(1e6), 1.2), 1e4, 5e7) * scale)
            ref = Reference([_bases(rng, max(16, size), rng.uniform(0.3, 0.7))])
        yield Request(t, ref)


def random_text(rng: np.random.Generator, n: int, alphabet: int = 4,
                sentinel: bool = True) -> np.ndarray:
    """Small random logical texts for parity tests."""
    body = rng.integers(2, 2 + alphabet, size=max(0, n - (1 if sentinel else 0))).astype(np.uint8)
    return np.concatenate([body, np.zeros(1, np.uint8)]) if sentinel else body
