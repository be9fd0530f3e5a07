"""Seeded synthetic sequencing workloads with the shapes of the benchmark configurations.

No public dataset is used by the reference's benchmarks; these generators produce uniform
random genomes and reads with the stated coverage, strand mix, substitution / indel rates and
runs of N.  Every function returns ``(data, offsets)``: the reads concatenated as ASCII bytes
(uint8) and ``n + 1`` uint64 offsets, the layout the C ABI takes.
"""
from __future__ import annotations

import numpy as np

LETTERS = np.frombuffer(b"ACGT", dtype=np.uint8)
N_BYTE = ord("N")


def random_genome(length: int, rng: np.random.Generator) -> np.ndarray:
    """Uniform i.i.d. genome as letter indices 0..3 (A, C, G, T)."""
    return rng.integers(0, 4, length, dtype=np.uint8)


def _apply_substitutions(reads: np.ndarray, rate: float, rng: np.random.Generator) -> None:
    if rate <= 0:
        return
    mask = rng.random(reads.shape, dtype=np.float32) < rate
    shift = rng.integers(1, 4, int(mask.sum()), dtype=np.uint8)
    reads[mask] = (reads[mask] + shift) % 4


def _apply_n_runs(flat: np.ndarray, offsets: np.ndarray, rate: float, max_run: int,
                  rng: np.random.Generator) -> None:
    """Replace about ``rate`` of all bases by N, in runs of U{1..max_run}, clipped at read ends."""
    total = flat.size
    if rate <= 0 or total == 0:
        return
    mean_run = (1 + max_run) / 2.0
    n_runs = int(round(rate * total / mean_run))
    if n_runs == 0:
        return
    starts = rng.integers(0, total, n_runs, dtype=np.int64)
    lens = rng.integers(1, max_run + 1, n_runs, dtype=np.int64)
    read_idx = np.searchsorted(offsets, starts, side="right") - 1
    ends = offsets[read_idx + 1].astype(np.int64)
    for step in range(max_run):
        pos = starts + step
        ok = (step < lens) & (pos < ends)
        flat[pos[ok]] = N_BYTE


def short_reads(genome_len: int, n_reads: int | None = None, read_len: int = 150, seed: int = 1,
                sub_rate: float = 0.0, n_rate: float = 0.0, n_max_run: int = 10,
                coverage: float | None = None, genome: np.ndarray | None = None,
                chunk: int = 1 << 20) -> tuple[np.ndarray, np.ndarray]:
    """Fixed-length reads sampled uniformly from a random genome, 50/50 strands."""
    rng = np.random.default_rng(seed)
    g = random_genome(genome_len, rng) if genome is None else genome
    if n_reads is None:
        n_reads = int(round((coverage or 1.0) * g.size / read_len))
    out = np.empty(n_reads * read_len, dtype=np.uint8)
    cols = np.arange(read_len, dtype=np.int64)
    for r0 in range(0, n_reads, chunk):
        r1 = min(n_reads, r0 + chunk)
        starts = rng.integers(0, g.size - read_len + 1, r1 - r0, dtype=np.int64)
        reads = g[starts[:, None] + cols[None, :]]
        rev = rng.random(r1 - r0) < 0.5
        reads[rev] = 3 - reads[rev][:, ::-1]
        _apply_substitutions(reads, sub_rate, rng)
        out[r0 * read_len:r1 * read_len] = LETTERS[reads].reshape(-1)
    offsets = np.arange(0, (n_reads + 1) * read_len, read_len, dtype=np.uint64)
    _apply_n_runs(out, offsets.astype(np.int64), n_rate, n_max_run, rng)
    return out, offsets


def _noisy_copy(template: np.ndarray, sub: float, ins: float, dele: float,
                rng: np.random.Generator) -> np.ndarray:
    """Copy of a letter-index template with substitutions, insertions and deletions."""
    u = rng.random(template.size)
    counts = np.ones(template.size, dtype=np.int64)
    counts[u < dele] = 0
    is_ins = (u >= dele) & (u < dele + ins)
    counts[is_ins] = 2
    out = np.repeat(template, counts)
    # the second copy of each inserted base becomes a random base
    ins_pos = np.cumsum(counts)[is_ins] - 1
    out[ins_pos] = rng.integers(0, 4, ins_pos.size, dtype=np.uint8)
    is_sub = (u >= dele + ins) & (u < dele + ins + sub)
    sub_pos = np.cumsum(counts)[is_sub] - 1
    out[sub_pos] = (out[sub_pos] + rng.integers(1, 4, sub_pos.size, dtype=np.uint8)) % 4
    return out


def mixed_reads(genome_len: int, coverage: float, seed: int = 1, short_frac: float = 0.7,
                short_len: int = 150, short_err: float = 0.01, long_median: int = 10_000,
                long_sigma: float = 0.8, long_min: int = 1_000, long_max: int = 100_000,
                long_err: float = 0.05, max_bases: int | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Uneven-length batch: ``short_frac`` of bases from short reads, the rest from log-normal
    long reads (median ``long_median``, clipped) with sub:ins:del = 2:1:1 errors.  Reads are
    shuffled so short and long reads interleave."""
    rng = np.random.default_rng(seed)
    g = random_genome(genome_len, rng)
    total = int(coverage * genome_len) if max_bases is None else int(max_bases)
    n_short = int(total * short_frac) // short_len
    s_data, _ = short_reads(genome_len, n_short, short_len, seed=seed + 1, sub_rate=short_err, genome=g)
    s_reads = s_data.reshape(n_short, short_len)
    long_budget = total - n_short * short_len
    longs = []
    used = 0
    while used < long_budget:
        L = int(np.clip(rng.lognormal(np.log(long_median), long_sigma), long_min, long_max))
        L = min(L, g.size)
        st = int(rng.integers(0, g.size - L + 1))
        tpl = g[st:st + L]
        if rng.random() < 0.5:
            tpl = 3 - tpl[::-1]
        r = _noisy_copy(tpl, long_err * 0.5, long_err * 0.25, long_err * 0.25, rng)
        longs.append(LETTERS[r])
        used += r.size
    pieces = [s_reads[i] for i in range(n_short)] + longs
    order = rng.permutation(len(pieces))
    lens = np.array([pieces[i].size for i in order], dtype=np.uint64)
    offsets = np.zeros(len(pieces) + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    data = np.concatenate([pieces[i] for i in order]) if pieces else np.zeros(0, np.uint8)
    return data, offsets


def repeat_genome(genome_len: int, seed: int = 1, repeat_frac: float = 0.05, n_families: int = 500,
                  fam_min: int = 1_000, fam_max: int = 5_000, copy_lo: float = 10.0, copy_hi: float = 1e4,
                  divergence: float = 0.02) -> np.ndarray:
    """Random genome where ``repeat_frac`` of the bases are copies of repeat families (lengths
    U{fam_min..fam_max}, copy numbers log-uniform in [copy_lo, copy_hi], ``divergence``
    substitutions between copies).  Copy numbers are scaled to fit the repeat budget."""
    rng = np.random.default_rng(seed)
    g = random_genome(genome_len, rng)
    fam_len = rng.integers(fam_min, fam_max + 1, n_families)
    copies = np.exp(rng.uniform(np.log(copy_lo), np.log(copy_hi), n_families))
    budget = repeat_frac * genome_len
    scale = budget / float((fam_len * copies).sum())
    copies = np.maximum(1, np.round(copies * scale)).astype(np.int64)
    for f in range(n_families):
        fam = random_genome(int(fam_len[f]), rng)
        for _ in range(int(copies[f])):
            pos = int(rng.integers(0, genome_len - fam.size))
            cp = fam.copy()
            _apply_substitutions(cp[None, :], divergence, rng)
            g[pos:pos + cp.size] = cp
    return g


def random_sequences(n: int, len_lo: int, len_hi: int, seed: int = 1, genome: np.ndarray | None = None,
                     from_genome_frac: float = 0.5, err: float = 0.01) -> tuple[np.ndarray, np.ndarray]:
    """Sequences with log-uniform lengths in [len_lo, len_hi]; ``from_genome_frac`` of them are
    drawn from ``genome`` with substitutions, the rest are uniform random ACGT."""
    rng = np.random.default_rng(seed)
    lens = np.exp(rng.uniform(np.log(len_lo), np.log(len_hi), n)).astype(np.int64)
    pieces = []
    for L in lens:
        if genome is not None and rng.random() < from_genome_frac and genome.size > L:
            st = int(rng.integers(0, genome.size - L + 1))
            r = genome[st:st + L].copy()
            if rng.random() < 0.5:
                r = 3 - r[::-1]
            _apply_substitutions(r[None, :], err, rng)
        else:
            r = random_genome(int(L), rng)
        pieces.append(LETTERS[r])
    offsets = np.zeros(n + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    data = np.concatenate(pieces) if pieces else np.zeros(0, np.uint8)
    return data, offsets


def split(data: np.ndarray, offsets: np.ndarray) -> list[bytes]:
    """Back to a list of byte strings (small batches only)."""
    return [data[int(offsets[i]):int(offsets[i + 1])].tobytes() for i in range(len(offsets) - 1)]
