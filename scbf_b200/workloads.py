"""Seeded synthetic sequencing workloads with the shapes of the benchmark configurations.

No public dataset is used by the reference's benchmarks; these generators produce uniform
random genomes (optionally with planted repeat families) and reads with the stated coverage,
strand mix, substitution / indel rates and runs of N.  Every function returns
``(data, offsets)``: the reads concatenated as ASCII bytes (uint8) and ``n + 1`` uint64
offsets, the layout the C ABI takes.  The heavy lifting is in csrc/scb_workloads.cpp
(libscb_workloads.so), multi-threaded with one random stream per read.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libscb_workloads.so")
LETTERS = np.frombuffer(b"ACGT", dtype=np.uint8)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build

            build.build_workloads()
        L = C.CDLL(LIB_PATH)
        vp, u64 = C.c_void_p, C.c_uint64
        L.scbw_random_genome.argtypes = [vp, u64, u64]
        L.scbw_short_reads.argtypes = [vp, u64, u64, u64, u64, C.c_double, C.c_double, C.c_int, vp, vp]
        L.scbw_lognormal_lengths.argtypes = [u64, C.c_double, C.c_double, u64, u64, u64, vp]
        L.scbw_noisy_reads.argtypes = [vp, u64, u64, vp, u64, C.c_double, C.c_double, C.c_double, vp, vp, vp]
        L.scbw_plant_repeats.argtypes = [vp, u64, u64, u64, u64, C.c_double, C.c_double, C.c_double, C.c_double, u64]
        L.scbw_to_ascii.argtypes = [vp, u64, vp]
        L.scbw_gather_reads.argtypes = [vp, vp, vp, u64, vp, vp]
        _lib = L
    return _lib


def random_genome(length: int, seed: int = 1) -> np.ndarray:
    """Uniform i.i.d. genome as letter indices 0..3 (A, C, G, T)."""
    g = np.empty(int(length), dtype=np.uint8)
    lib().scbw_random_genome(g.ctypes.data, g.size, seed)
    return g


def repeat_genome(genome_len: int, seed: int = 1, repeat_frac: float = 0.05, n_families: int = 500,
                  fam_min: int = 1_000, fam_max: int = 5_000, copy_lo: float = 10.0, copy_hi: float = 1e4,
                  divergence: float = 0.02) -> np.ndarray:
    """Random genome where about ``repeat_frac`` of the bases are copies of repeat families
    (lengths U{fam_min..fam_max}, copy numbers log-uniform in [copy_lo, copy_hi] scaled to the
    repeat budget, ``divergence`` substitutions between copies)."""
    g = random_genome(genome_len, seed)
    lib().scbw_plant_repeats(g.ctypes.data, g.size, n_families, fam_min, fam_max, copy_lo, copy_hi,
                             repeat_frac, divergence, seed)
    return g


def short_reads(genome_len: int = 0, n_reads: int | None = None, read_len: int = 150, seed: int = 1,
                sub_rate: float = 0.0, n_rate: float = 0.0, n_max_run: int = 10,
                coverage: float | None = None, genome: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Fixed-length reads sampled uniformly from a genome, 50/50 strands, with substitutions
    (per-base rate) and runs of N (about ``n_rate`` of the bases, runs of U{1..n_max_run})."""
    g = random_genome(genome_len, seed) if genome is None else np.ascontiguousarray(genome, dtype=np.uint8)
    if n_reads is None:
        n_reads = int(round((coverage or 1.0) * g.size / read_len))
    out = np.empty(max(n_reads * read_len, 1), dtype=np.uint8)
    offsets = np.zeros(n_reads + 1, dtype=np.uint64)
    lib().scbw_short_reads(g.ctypes.data, g.size, n_reads, read_len, seed + 1, sub_rate, n_rate, n_max_run,
                           out.ctypes.data, offsets.ctypes.data)
    return out[: n_reads * read_len], offsets


def noisy_reads(genome: np.ndarray, template_lens: np.ndarray, seed: int, sub: float, ins: float,
                dele: float) -> tuple[np.ndarray, np.ndarray]:
    """Reads copied from random positions / strands of ``genome`` with the given error rates."""
    g = np.ascontiguousarray(genome, dtype=np.uint8)
    t = np.ascontiguousarray(template_lens, dtype=np.uint64)
    n = t.size
    lens = np.zeros(n, dtype=np.uint64)
    L = lib()
    L.scbw_noisy_reads(g.ctypes.data, g.size, n, t.ctypes.data, seed, sub, ins, dele, lens.ctypes.data, None, None)
    offsets = np.zeros(n + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    out = np.empty(max(int(offsets[-1]), 1), dtype=np.uint8)
    L.scbw_noisy_reads(g.ctypes.data, g.size, n, t.ctypes.data, seed, sub, ins, dele, None, offsets.ctypes.data,
                       out.ctypes.data)
    return out[: int(offsets[-1])], offsets


def interleave(parts: list[tuple[np.ndarray, np.ndarray]], seed: int) -> tuple[np.ndarray, np.ndarray]:
    """Concatenate several batches and shuffle their reads (seeded)."""
    data = np.concatenate([d[: int(o[-1])] for d, o in parts])
    base = 0
    offs = []
    for _, o in parts:
        offs.append(o[:-1].astype(np.uint64) + np.uint64(base))
        base += int(o[-1])
    src_off = np.concatenate(offs + [np.array([base], dtype=np.uint64)])
    lens = np.diff(src_off.astype(np.int64))
    order = np.random.default_rng(seed).permutation(lens.size).astype(np.uint64)
    new_off = np.zeros(lens.size + 1, dtype=np.uint64)
    new_off[1:] = np.cumsum(lens[order.astype(np.int64)])
    out = np.empty(max(base, 1), dtype=np.uint8)
    lib().scbw_gather_reads(data.ctypes.data, src_off.ctypes.data, order.ctypes.data, lens.size, out.ctypes.data,
                            new_off.ctypes.data)
    return out[:base], new_off


def mixed_reads(genome_len: int, coverage: float, seed: int = 1, short_frac: float = 0.7, short_len: int = 150,
                short_err: float = 0.01, long_median: float = 10_000, long_sigma: float = 0.8,
                long_min: int = 1_000, long_max: int = 100_000, long_err: float = 0.05,
                genome: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Uneven-length batch: ``short_frac`` of the bases from short reads (substitutions), the rest
    from log-normal long reads (median ``long_median``, clipped) with sub:ins:del = 2:1:1 errors;
    short and long reads interleave."""
    g = random_genome(genome_len, seed) if genome is None else genome
    total = int(coverage * g.size)
    n_short = int(total * short_frac) // short_len
    s_data, s_off = short_reads(n_reads=n_short, read_len=short_len, seed=seed + 11, sub_rate=short_err, genome=g)
    long_budget = total - n_short * short_len
    est_n = max(1, int(long_budget / long_median) * 2 + 16)
    lens = np.zeros(est_n, dtype=np.uint64)
    lib().scbw_lognormal_lengths(est_n, float(long_median), float(long_sigma), long_min, long_max, seed + 13,
                                 lens.ctypes.data)
    cum = np.cumsum(lens)
    n_long = int(np.searchsorted(cum, long_budget)) + 1
    l_data, l_off = noisy_reads(g, lens[:n_long], seed + 17, long_err * 0.5, long_err * 0.25, long_err * 0.25)
    return interleave([(s_data, s_off), (l_data, l_off)], seed + 19)


def random_sequences(n: int, len_lo: int, len_hi: int, seed: int = 1, genome: np.ndarray | None = None,
                     from_genome_frac: float = 0.5, err: float = 0.01) -> tuple[np.ndarray, np.ndarray]:
    """Sequences with log-uniform lengths in [len_lo, len_hi]; ``from_genome_frac`` of them come
    from ``genome`` with substitutions, the rest are uniform random ACGT."""
    rng = np.random.default_rng(seed)
    lens = np.exp(rng.uniform(np.log(len_lo), np.log(len_hi), n)).astype(np.uint64)
    from_g = rng.random(n) < from_genome_frac if genome is not None else np.zeros(n, bool)
    parts = []
    if from_g.any():
        parts.append(noisy_reads(genome, lens[from_g], seed + 1, err, 0.0, 0.0))
    if (~from_g).any():
        rnd = random_genome(int(lens[~from_g].sum()), seed + 2)
        off = np.zeros(int((~from_g).sum()) + 1, dtype=np.uint64)
        off[1:] = np.cumsum(lens[~from_g])
        parts.append((LETTERS[rnd], off))
    return interleave(parts, seed + 3)


def config1(seed: int = 1):
    """1 Mbp uniform genome, 30x of 150 bp reads, both strands, 0.5% substitutions, no N."""
    return short_reads(genome_len=1_000_000, coverage=30, read_len=150, seed=seed, sub_rate=0.005)


def config2(seed: int = 1, scale: float = 1.0):
    """100 Mbp uniform genome, 20x of 150 bp reads (~13.3M reads), 1% substitutions, 1% N in runs
    of 1-10.  ``scale`` shrinks the genome (same coverage) for quick runs."""
    return short_reads(genome_len=int(100_000_000 * scale), coverage=20, read_len=150, seed=seed, sub_rate=0.01,
                       n_rate=0.01, n_max_run=10)


def config3(seed: int = 1, scale: float = 1.0):
    """50 Mbp genome with 5% from 500 repeat families (1-5 kbp, copy number log-uniform 10..10^4,
    2% divergence), 30x of 150 bp reads with 1% substitutions."""
    g = repeat_genome(int(50_000_000 * scale), seed=seed)
    return short_reads(coverage=30, read_len=150, seed=seed, sub_rate=0.01, genome=g)


def config4(seed: int = 1, scale: float = 1.0):
    """200 Mbp genome at 15x: 70% of bases from 150 bp reads (1% errors), 30% from log-normal long
    reads (median 10 kbp, 1-100 kbp) with 5% errors (sub:ins:del = 2:1:1)."""
    return mixed_reads(int(200_000_000 * scale), coverage=15, seed=seed)


def split(data: np.ndarray, offsets: np.ndarray) -> list[bytes]:
    """Back to a list of byte strings (small batches only)."""
    return [data[int(offsets[i]):int(offsets[i + 1])].tobytes() for i in range(len(offsets) - 1)]
