"""Host-side mirror of the reference crate's public API (super-counting-bloom 0.1.0, src/api.rs,
src/fastx.rs, src/config.rs, src/error.rs) over the CUDA library's C ABI.

Names, argument meaning and error behaviour follow the Rust API so that a user of the reference
finds the same surface: SuperCountingBloomConfig, CounterBits, SuperCountingBloomBuilder,
SuperCountingBloomIndex, the report types, estimate_spectrum_from_fastx[_pair],
stream_estimates_from_fastx[_pair], write_spectrum and for_each_fastx_record.  FASTA/FASTQ
parsing stays on the host; all insert / query / spectrum work runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import enum
import math
import os
import time
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from . import _lib


# ---------------------------------------------------------------------------------------
# Errors (src/error.rs:4-12)
# ---------------------------------------------------------------------------------------
class SuperCountingBloomError(Exception):
    """Base of the error variants of SuperCountingBloomError."""


class InvalidConfig(SuperCountingBloomError):
    pass


class FastxOpen(SuperCountingBloomError):
    pass


class InvalidIndexFormat(SuperCountingBloomError):
    pass


class ChannelClosed(SuperCountingBloomError):
    pass


class WorkerPanic(SuperCountingBloomError):
    pass


class InternalState(SuperCountingBloomError):
    pass


class Io(SuperCountingBloomError):
    pass


_STATUS_ERRORS = {1: InvalidConfig, 2: FastxOpen, 3: InvalidIndexFormat, 4: ChannelClosed, 5: WorkerPanic,
                  6: InternalState, 7: Io}


def _check(status: int) -> None:
    if status != _lib.SCB_OK:
        raise _STATUS_ERRORS.get(status, InternalState)(_lib.last_error())


# ---------------------------------------------------------------------------------------
# Config (src/config.rs)
# ---------------------------------------------------------------------------------------
class CounterBits(enum.IntEnum):
    Bits8 = 8
    Bits16 = 16
    Bits32 = 32

    def as_u8(self) -> int:
        return int(self)


@dataclass
class SuperCountingBloomConfig:
    """src/config.rs:20-47; defaults k=31 m=21 s=25 h=4, 16-bit counters, 2^30 slots, 2^9/block."""

    k: int = 31
    m: int = 21
    s: int = 25
    n_hashes: int = 4
    counter_bits: CounterBits = CounterBits.Bits16
    counter_slots_exponent: int = 30
    block_slots_exponent: int = 9
    threads: int = field(default_factory=lambda: max(1, os.cpu_count() or 1))
    queue: int = 4096

    def to_c(self) -> _lib.ScbConfig:
        for name in ("k", "m", "s", "n_hashes", "threads", "queue"):
            if int(getattr(self, name)) < 0:
                raise InvalidConfig(f"invalid config: {name} must be non-negative")
        for name in ("counter_slots_exponent", "block_slots_exponent"):
            if not 0 <= int(getattr(self, name)) <= 255:
                raise InvalidConfig(f"invalid config: {name} must fit in u8")
        if int(self.counter_bits) not in (8, 16, 32):
            raise InvalidConfig("invalid config: unsupported counter width")
        return _lib.ScbConfig(int(self.k), int(self.m), int(self.s), int(self.n_hashes), int(self.counter_bits),
                              int(self.counter_slots_exponent), int(self.block_slots_exponent), int(self.threads),
                              int(self.queue))

    @classmethod
    def from_c(cls, c: _lib.ScbConfig) -> "SuperCountingBloomConfig":
        return cls(c.k, c.m, c.s, c.n_hashes, CounterBits(c.counter_bits), c.counter_slots_exponent,
                   c.block_slots_exponent, c.threads, c.queue)

    def validate(self) -> None:
        """src/config.rs:50-92 (+ filter.rs:96-100); raises InvalidConfig."""
        c = self.to_c()
        _check(_lib.load().scb_config_validate(C.byref(c)))

    def counter_slots(self) -> int:
        return 1 << int(self.counter_slots_exponent)

    def block_slots(self) -> int:
        return 1 << int(self.block_slots_exponent)


# ---------------------------------------------------------------------------------------
# Reports (src/api.rs:56-99, src/fastx.rs:21-60)
# ---------------------------------------------------------------------------------------
@dataclass
class AddReport:
    records_processed: int = 0
    records_indexed: int = 0
    inserted_kmers: int = 0
    inserted_smers: int = 0
    add_seconds: float = 0.0


@dataclass
class QueryFastaReport:
    records_processed: int = 0
    total_windows: int = 0
    valid_kmers: int = 0
    positive_estimates: int = 0
    estimate_checksum: int = 0


@dataclass
class SequenceAbundanceSummary:
    name: str
    sequence_len: int
    total_windows: int
    valid_kmers: int
    mean_abundance: float | None
    median_abundance: float | None


@dataclass
class BuildIndexReport:
    index: "SuperCountingBloomIndex"
    chunks: int
    indexed_kmers: int
    inserted_smers: int
    counter_slots: int
    blocks: int
    build_seconds: float


@dataclass
class SuperCountingBloomStats:
    chunks: int = 0
    indexed_kmers: int = 0
    inserted_smers: int = 0
    queried_kmers: int = 0
    distinct_keys: int = 0
    counter_slots: int = 0
    blocks: int = 0
    build_seconds: float = 0.0
    query_seconds: float = 0.0
    spectrum_seconds: float = 0.0
    total_seconds: float = 0.0


@dataclass
class SuperCountingBloomReport:
    spectrum: list
    stats: SuperCountingBloomStats


@dataclass
class StreamEstimateStats:
    chunks: int = 0
    indexed_kmers: int = 0
    inserted_smers: int = 0
    queried_kmers: int = 0
    positive_estimates: int = 0
    estimate_checksum: int = 0
    counter_slots: int = 0
    blocks: int = 0
    build_seconds: float = 0.0
    query_seconds: float = 0.0
    total_seconds: float = 0.0


@dataclass
class StreamEstimateReport:
    stats: StreamEstimateStats


@dataclass
class FilterOnlySpectrumEstimate:
    """src/api.rs:95-99: rows are (abundance, estimated k-mers) for abundance 1..=max_abundance."""
    method: str
    kmer_count_hint: int
    rows: list


# ---------------------------------------------------------------------------------------
# Filter-only spectrum (src/api.rs:337-385, 933-1033): host f64 arithmetic over the counter
# histogram the GPU computes.  The k-mer counts per abundance are the coefficients of the
# logarithm of the counters' generating function (a compound Poisson deconvolution); every
# product, quotient and sum is taken in the reference's order (sums left to right), so the rows
# are the reference's to the last bit.
# ---------------------------------------------------------------------------------------
_FILTER_ONLY_METHOD = "compound_poisson_counter_deconvolution"


def _round_u64(x: float) -> int:
    """Rust `x.round() as u64`: halves away from zero; NaN and negatives give 0."""
    if not x > 0.0:
        return 0
    r = math.floor(x)
    if x - r >= 0.5:
        r += 1
    return min(int(r), (1 << 64) - 1)


def _sum_f64(values: np.ndarray) -> float:
    """Left-to-right f64 sum (Rust's Iterator::sum; numpy's sum and Python's sum round differently)."""
    return float(np.add.accumulate(values)[-1]) if len(values) else 0.0


def _deconvolved_counts(counter_histogram, n_hashes: int, max_abundance: int) -> np.ndarray:
    """src/api.rs:958-1001."""
    if max_abundance == 0:
        return np.zeros(0)
    total = sum(int(c) for _, c in counter_histogram)
    if total == 0:
        return np.zeros(max_abundance)
    prob = np.zeros(max_abundance + 1)
    for abundance, counters in counter_histogram:
        if abundance <= max_abundance:
            prob[abundance] += float(counters) / float(total)
    p0 = float(prob[0])
    if p0 <= 0.0:
        return np.zeros(0)
    norm = prob / p0
    norm[0] = 1.0
    idx = np.arange(max_abundance + 1, dtype=np.float64)
    logc = np.zeros(max_abundance + 1)
    seq = np.empty(max_abundance + 1)
    for a in range(1, max_abundance + 1):
        # a * norm[a] - sum over p = 1 .. a-1 of (p * logc[p]) * norm[a - p], subtracted in order
        seq[0] = idx[a] * norm[a]
        seq[1:a] = (idx[1:a] * logc[1:a]) * norm[a - 1:0:-1]
        logc[a] = float(np.subtract.accumulate(seq[:a])[-1]) / idx[a]
    v = (float(total) * logc[1:]) / float(max(n_hashes, 1))
    return np.where(v > 0.0, v, 0.0)


def _scaled_positive_counter_histogram(counter_histogram, max_abundance: int, kmer_count_hint: int) -> list:
    """src/api.rs:1003-1022: the positive counters' histogram scaled to the hint."""
    positive = float(max(sum(int(c) for a, c in counter_histogram if a > 0), 1))
    by_value = {int(a): int(c) for a, c in counter_histogram}
    return [(a, _round_u64(float(kmer_count_hint) * float(by_value.get(a, 0)) / positive))
            for a in range(1, max_abundance + 1)]


def _filter_only_rows(counter_histogram, n_hashes: int, max_abundance: int, kmer_count_hint: int) -> list:
    """src/api.rs:933-956."""
    dec = _deconvolved_counts(counter_histogram, n_hashes, max_abundance)
    total = _sum_f64(dec)
    if total <= 0.0:
        return _scaled_positive_counter_histogram(counter_histogram, max_abundance, kmer_count_hint)
    scale = float(kmer_count_hint) / total
    return [(a, _round_u64(float(dec[a - 1]) * scale)) for a in range(1, max_abundance + 1)]


# ---------------------------------------------------------------------------------------
# Sequence batches
# ---------------------------------------------------------------------------------------
def pack_sequences(seqs) -> tuple[np.ndarray, np.ndarray]:
    """(bytes uint8, offsets uint64[n+1]) from a list of bytes / str."""
    parts = [s.encode() if isinstance(s, str) else bytes(s) for s in seqs]
    offsets = np.zeros(len(parts) + 1, dtype=np.uint64)
    if parts:
        offsets[1:] = np.cumsum([len(p) for p in parts], dtype=np.uint64)
    data = np.frombuffer(b"".join(parts), dtype=np.uint8) if parts else np.zeros(0, np.uint8)
    if data.size == 0:
        data = np.zeros(1, dtype=np.uint8)
    return np.ascontiguousarray(data), offsets


def _as_batch(data, offsets) -> tuple[np.ndarray, np.ndarray]:
    data = np.ascontiguousarray(data, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    if data.size == 0:
        data = np.zeros(1, dtype=np.uint8)
    return data, offsets


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _is_acgt_mask(a: np.ndarray) -> np.ndarray:
    u = a & 0xDF
    return (u == 65) | (u == 67) | (u == 71) | (u == 84)


def _chunk_stats(data: np.ndarray, offsets: np.ndarray, k: int) -> tuple[int, int]:
    """Number of maximal ACGT runs of length >= k and their k-mer windows (fastx.rs:231-243)."""
    total = int(offsets[-1]) if len(offsets) > 1 else 0
    if total == 0:
        return 0, 0
    ok = _is_acgt_mask(data[:total])
    seqstart = np.zeros(total, dtype=bool)
    s = offsets[:-1][offsets[:-1] < total].astype(np.int64)
    seqstart[s] = True
    prev_ok = np.concatenate(([False], ok[:-1]))
    next_ok = np.concatenate((ok[1:], [False]))
    next_start = np.concatenate((seqstart[1:], [True]))
    run_s = np.flatnonzero(ok & (~prev_ok | seqstart))
    run_e = np.flatnonzero(ok & (~next_ok | next_start)) + 1
    lens = run_e - run_s
    keep = lens >= k
    return int(keep.sum()), int((lens[keep] - k + 1).sum())


# ---------------------------------------------------------------------------------------
# Device context handle
# ---------------------------------------------------------------------------------------
class _Ctx:
    def __init__(self, handle: int):
        self.h = C.c_void_p(handle)

    def close(self):
        if self.h and self.h.value:
            _lib.load().scb_destroy(self.h)
            self.h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _create(cfg: SuperCountingBloomConfig) -> _Ctx:
    c = cfg.to_c()
    out = C.c_void_p(0)
    _check(_lib.load().scb_create(C.byref(c), C.byref(out)))
    return _Ctx(out.value)


def set_strategy(obj, insert: str = "auto", query: str = "auto") -> None:
    """Select the insert / query kernels (plain, fused, staged, grouped or auto)."""
    _check(_lib.load().scb_set_strategy(obj._ctx.h, _lib.STRATEGIES[insert], _lib.STRATEGIES[query]))


# ---------------------------------------------------------------------------------------
# FASTA / FASTQ (host parsing; helicase semantics of records and names)
# ---------------------------------------------------------------------------------------
class _FastxOwner:
    """Holds one native read of a FASTA/FASTQ file (scb_fastx_read); the arrays viewing its memory
    keep it alive, and it is freed with the last of them."""

    def __init__(self, handle):
        self.h = handle

    def __del__(self):
        if self.h:
            try:
                _lib.load().scb_fastx_free(self.h)
            except Exception:  # interpreter shutdown: the process frees its memory anyway
                pass
            self.h = None


def _view(owner: _FastxOwner, addr: int, n: int, ctype, dtype) -> np.ndarray:
    if n == 0 or not addr:
        return np.zeros(0, dtype)
    buf = (ctype * n).from_address(addr)
    buf._owner = owner
    return np.frombuffer(buf, dtype=dtype)


def _fastx_read(path: str) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """Sequences, offsets (n + 1), headers and header offsets of a FASTA/FASTQ file (plain or gzip),
    read by the library's one-pass reader without copies."""
    L = _lib.load()
    h = C.c_void_p()
    _check(L.scb_fastx_read(os.fsencode(path), C.byref(h)))
    owner = _FastxOwner(h)
    sp, op, hp, hop, n = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_uint64()
    _check(L.scb_fastx_sequences(h, C.byref(sp), C.byref(op), C.byref(n)))
    _check(L.scb_fastx_headers(h, C.byref(hp), C.byref(hop)))
    offsets = _view(owner, op.value, n.value + 1, C.c_uint64, np.uint64)
    hoffs = _view(owner, hop.value, n.value + 1, C.c_uint64, np.uint64)
    seqs = _view(owner, sp.value, int(offsets[-1]), C.c_uint8, np.uint8)
    headers = _view(owner, hp.value, int(hoffs[-1]), C.c_uint8, np.uint8)
    return seqs, offsets, headers, hoffs


def _record_name(header: bytes, idx: int) -> str:
    """src/api.rs:917-927: first whitespace-separated token, or record_<idx>."""
    tok = header.split()[0] if header.split() else b""
    return tok.decode(errors="replace") if tok else f"record_{idx}"


def for_each_fastx_record(path: str, visit: Callable[[str, bytes], None]) -> None:
    """src/api.rs:893-915."""
    seqs, offsets, headers, hoffs = _fastx_read(str(path))
    sv, hv = memoryview(seqs), memoryview(headers)
    o, ho = offsets.tolist(), hoffs.tolist()
    for i in range(len(o) - 1):
        visit(_record_name(bytes(hv[ho[i]:ho[i + 1]]), i + 1), bytes(sv[o[i]:o[i + 1]]))


def _read_batch(path: str) -> tuple[np.ndarray, np.ndarray]:
    """All records of a FASTA/FASTQ file as one batch (concatenated sequences, offsets)."""
    seqs, offsets, _, _ = _fastx_read(str(path))
    return seqs, offsets


# ---------------------------------------------------------------------------------------
# Builder (src/api.rs:101-208)
# ---------------------------------------------------------------------------------------
class SuperCountingBloomBuilder:
    def __init__(self, cfg: SuperCountingBloomConfig | None = None):
        cfg = cfg or SuperCountingBloomConfig()
        cfg.validate()
        self._cfg = SuperCountingBloomConfig(**cfg.__dict__)
        self._ctx = _create(self._cfg)
        self._inserted_kmers = 0
        self._inserted_smers = 0

    @classmethod
    def new(cls, cfg: SuperCountingBloomConfig) -> "SuperCountingBloomBuilder":
        return cls(cfg)

    def _insert(self, data: np.ndarray, offsets: np.ndarray) -> tuple[int, int]:
        data, offsets = _as_batch(data, offsets)
        km, sm = C.c_uint64(0), C.c_uint64(0)
        _check(_lib.load().scb_insert_batch(self._ctx.h, _ptr(data), _ptr(offsets), len(offsets) - 1,
                                            C.byref(km), C.byref(sm)))
        self._inserted_kmers += km.value
        self._inserted_smers += sm.value
        return km.value, sm.value

    def add_sequence(self, sequence: bytes | str) -> int:
        """src/api.rs:123-138: returns the k-mer windows inserted."""
        data, offsets = pack_sequences([sequence])
        return self._insert(data, offsets)[0]

    def add_sequences(self, data: np.ndarray, offsets: np.ndarray) -> AddReport:
        """Batch form of add_sequence over concatenated records (one GPU batch)."""
        t0 = time.perf_counter()
        km, sm = self._insert(data, offsets)
        lens = np.diff(np.asarray(offsets, dtype=np.int64))
        rep = AddReport(records_processed=len(lens), inserted_kmers=km, inserted_smers=sm,
                        add_seconds=time.perf_counter() - t0)
        rep.records_indexed = self._records_indexed(data, offsets)
        return rep

    def _records_indexed(self, data, offsets) -> int:
        """Records that inserted at least one k-mer (src/api.rs:640-642)."""
        data, offsets = _as_batch(data, offsets)
        return int(_lib.load().scb_records_indexed(self._ctx.h, _ptr(data), _ptr(offsets), len(offsets) - 1))

    def add_fasta(self, path) -> AddReport:
        """src/api.rs:140-158, 621-666."""
        self._cfg.validate()
        t0 = time.perf_counter()
        data, offsets = _read_batch(str(path))
        rep = self.add_sequences(data, offsets)
        rep.add_seconds = time.perf_counter() - t0
        return rep

    def into_index(self) -> "SuperCountingBloomIndex":
        """src/api.rs:160-177: freezes the device table and hands it to the index."""
        if self._ctx is None:
            raise InternalState("internal state error: builder already consumed")
        _check(_lib.load().scb_freeze(self._ctx.h))
        idx = SuperCountingBloomIndex._from_ctx(self._ctx, self._cfg, self._inserted_kmers)
        self._ctx = None
        return idx

    def inserted_kmers(self) -> int:
        return self._inserted_kmers

    def inserted_smers(self) -> int:
        return self._inserted_smers

    def set_threads(self, threads: int) -> None:
        if threads == 0:
            raise InvalidConfig("invalid config: threads must be positive")
        self._cfg.threads = threads
        _check(_lib.load().scb_set_threads(self._ctx.h, threads))

    def clear_threads(self) -> None:
        self.set_threads(max(1, os.cpu_count() or 1))

    def threads(self) -> int:
        return self._cfg.threads

    def config(self) -> SuperCountingBloomConfig:
        return self._cfg


# ---------------------------------------------------------------------------------------
# Index (src/api.rs:210-386)
# ---------------------------------------------------------------------------------------
class SuperCountingBloomIndex:
    def __init__(self):
        raise TypeError("use SuperCountingBloomBuilder.into_index, build_from_fastx or load")

    @classmethod
    def _from_ctx(cls, ctx: _Ctx, cfg: SuperCountingBloomConfig, inserted_kmers: int) -> "SuperCountingBloomIndex":
        obj = object.__new__(cls)
        obj._ctx = ctx
        obj._cfg = cfg
        obj._inserted_kmers = inserted_kmers
        return obj

    @classmethod
    def build_from_fastx(cls, path, cfg: SuperCountingBloomConfig) -> BuildIndexReport:
        """src/api.rs:211-223 + fastx.rs:206-253, 378-390."""
        cfg.validate()
        t0 = time.perf_counter()
        data, offsets = _read_batch(str(path))
        b = SuperCountingBloomBuilder(cfg)
        km, sm = b._insert(data, offsets)
        chunks, _ = _chunk_stats(data, offsets, int(cfg.k))
        idx = b.into_index()
        return BuildIndexReport(index=idx, chunks=chunks, indexed_kmers=km, inserted_smers=sm,
                                counter_slots=cfg.counter_slots(), blocks=cfg.counter_slots() // cfg.block_slots(),
                                build_seconds=time.perf_counter() - t0)

    def config(self) -> SuperCountingBloomConfig:
        return self._cfg

    def inserted_kmers(self) -> int:
        return self._inserted_kmers

    def save(self, path) -> None:
        """src/api.rs:233-240, 388-414."""
        _check(_lib.load().scb_save(self._ctx.h, str(path).encode()))

    @classmethod
    def load(cls, path) -> "SuperCountingBloomIndex":
        """src/api.rs:242-248, 416-464."""
        out = C.c_void_p(0)
        _check(_lib.load().scb_load(str(path).encode(), C.byref(out)))
        ctx = _Ctx(out.value)
        c = _lib.ScbConfig()
        _check(_lib.load().scb_get_config(ctx.h, C.byref(c)))
        km = C.c_uint64(0)
        _check(_lib.load().scb_get_counts(ctx.h, C.byref(km), None))
        return cls._from_ctx(ctx, SuperCountingBloomConfig.from_c(c), km.value)

    def estimate_batch(self, data: np.ndarray, offsets: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """Per-window abundances of every sequence (windows concatenated) and validity flags."""
        data, offsets = _as_batch(data, offsets)
        L = _lib.load()
        n = len(offsets) - 1
        nw = int(L.scb_count_windows(self._ctx.h, _ptr(offsets), n))
        out = np.zeros(max(nw, 1), dtype=np.uint64)
        valid = np.zeros(max(nw, 1), dtype=np.uint8)
        _check(L.scb_query_batch(self._ctx.h, _ptr(data), _ptr(offsets), n, _ptr(out), _ptr(valid)))
        return out[:nw], valid[:nw]

    def estimate_sequence_abundances(self, sequence: bytes | str) -> list[int | None]:
        """src/api.rs:250-262."""
        data, offsets = pack_sequences([sequence])
        out, valid = self.estimate_batch(data, offsets)
        return [int(v) if ok else None for v, ok in zip(out.tolist(), valid.tolist())]

    def summarize_sequence(self, name: str, sequence: bytes | str) -> SequenceAbundanceSummary:
        """src/api.rs:264-271, 855-891."""
        ab = self.estimate_sequence_abundances(sequence)
        valid = sorted(v for v in ab if v is not None)
        if not valid:
            return SequenceAbundanceSummary(name, len(sequence), len(ab), 0, None, None)
        mean = sum(valid) / len(valid)
        mid = len(valid) // 2
        median = (valid[mid - 1] + valid[mid]) / 2.0 if len(valid) % 2 == 0 else float(valid[mid])
        return SequenceAbundanceSummary(name, len(sequence), len(ab), len(valid), mean, median)

    def query_report(self, data: np.ndarray, offsets: np.ndarray) -> QueryFastaReport:
        data, offsets = _as_batch(data, offsets)
        rep = _lib.ScbReport()
        _check(_lib.load().scb_query_report(self._ctx.h, _ptr(data), _ptr(offsets), len(offsets) - 1,
                                            C.byref(rep)))
        return QueryFastaReport(rep.records_processed, rep.total_windows, rep.valid_kmers,
                                rep.positive_estimates, rep.estimate_checksum & ((1 << 64) - 1))

    def query_fasta(self, path) -> QueryFastaReport:
        """src/api.rs:273-327."""
        data, offsets = _read_batch(str(path))
        return self.query_report(data, offsets)

    def counter_histogram(self) -> list[tuple[int, int]]:
        """src/api.rs:329-335."""
        L = _lib.load()
        rows = C.c_uint64(0)
        _check(L.scb_counter_histogram(self._ctx.h, None, None, 0, C.byref(rows)))
        vals = np.zeros(max(rows.value, 1), np.uint64)
        cnts = np.zeros(max(rows.value, 1), np.uint64)
        _check(L.scb_counter_histogram(self._ctx.h, _ptr(vals), _ptr(cnts), rows.value, C.byref(rows)))
        return list(zip(vals[: rows.value].tolist(), cnts[: rows.value].tolist()))

    def estimate_filter_only_spectrum(self, max_abundance: int, kmer_count_hint: int) -> FilterOnlySpectrumEstimate:
        """src/api.rs:337-348: the k-mer spectrum estimated from the counters alone (no reads)."""
        return self.estimate_filter_only_spectrum_from_counter_histogram(self.counter_histogram(), max_abundance,
                                                                         kmer_count_hint)

    def estimate_filter_only_spectrum_from_counter_histogram(self, counter_histogram, max_abundance: int,
                                                             kmer_count_hint: int) -> FilterOnlySpectrumEstimate:
        """src/api.rs:350-368."""
        rows = _filter_only_rows(counter_histogram, int(self._cfg.n_hashes), int(max_abundance), int(kmer_count_hint))
        return FilterOnlySpectrumEstimate(method=_FILTER_ONLY_METHOD, kmer_count_hint=int(kmer_count_hint), rows=rows)

    def filter_only_count_hint(self) -> int:
        """src/api.rs:370-373: the deconvolved k-mer total (abundances up to 255), at least 1."""
        return self.filter_only_count_hint_from_counter_histogram(self.counter_histogram(), 255)

    def filter_only_count_hint_from_counter_histogram(self, counter_histogram, max_abundance: int) -> int:
        """src/api.rs:375-385."""
        dec = _deconvolved_counts(counter_histogram, int(self._cfg.n_hashes), int(max_abundance))
        return max(_round_u64(_sum_f64(dec)), 1)

    def spectrum_distinct(self, data: np.ndarray, offsets: np.ndarray) -> dict:
        """estimate_distinct_kmers + spectrum_from_estimates (fastx.rs:255-308, 392-410)."""
        data, offsets = _as_batch(data, offsets)
        L = _lib.load()
        n = len(offsets) - 1
        rows, dk, qk = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
        _check(L.scb_spectrum_distinct(self._ctx.h, _ptr(data), _ptr(offsets), n, None, None, 0, C.byref(rows),
                                       C.byref(dk), C.byref(qk)))
        cap = max(rows.value, 1)
        vals = np.zeros(cap, np.uint64)
        cnts = np.zeros(cap, np.uint64)
        _check(L.scb_spectrum_distinct(self._ctx.h, _ptr(data), _ptr(offsets), n, _ptr(vals), _ptr(cnts), cap,
                                       C.byref(rows), C.byref(dk), C.byref(qk)))
        return {"rows": list(zip(vals[: rows.value].tolist(), cnts[: rows.value].tolist())),
                "distinct_keys": dk.value, "queried_kmers": qk.value}

    def table(self) -> np.ndarray:
        """Counter table in .scb file order."""
        L = _lib.load()
        nb = int(L.scb_table_bytes(self._ctx.h))
        buf = np.zeros(nb, dtype=np.uint8)
        _check(L.scb_table_download(self._ctx.h, _ptr(buf), nb))
        return buf.view({8: np.uint8, 16: np.uint16, 32: np.uint32}[int(self._cfg.counter_bits)])

    def batch_stats(self, data, offsets) -> dict:
        data, offsets = _as_batch(data, offsets)
        st = _lib.ScbStats()
        _check(_lib.load().scb_batch_stats(self._ctx.h, _ptr(data), _ptr(offsets), len(offsets) - 1, C.byref(st)))
        return {"windows": st.windows, "super_kmers": st.super_kmers, "smers": st.smers, "sectors": st.sectors}


# ---------------------------------------------------------------------------------------
# Pipeline functions (src/fastx.rs:81-131)
# ---------------------------------------------------------------------------------------
def estimate_spectrum_from_fastx_pair(index_path, query_path, cfg: SuperCountingBloomConfig) -> SuperCountingBloomReport:
    cfg.validate()
    t_total = time.perf_counter()
    rep = SuperCountingBloomIndex.build_from_fastx(index_path, cfg)
    t_q = time.perf_counter()
    data, offsets = _read_batch(str(query_path))
    sp = rep.index.spectrum_distinct(data, offsets)
    t_end = time.perf_counter()
    stats = SuperCountingBloomStats(chunks=rep.chunks, indexed_kmers=rep.indexed_kmers,
                                    inserted_smers=rep.inserted_smers, queried_kmers=sp["queried_kmers"],
                                    distinct_keys=sp["distinct_keys"], counter_slots=rep.counter_slots,
                                    blocks=rep.blocks, build_seconds=rep.build_seconds, query_seconds=t_end - t_q,
                                    spectrum_seconds=0.0, total_seconds=t_end - t_total)
    return SuperCountingBloomReport(spectrum=sp["rows"], stats=stats)


def estimate_spectrum_from_fastx(path, cfg: SuperCountingBloomConfig) -> SuperCountingBloomReport:
    return estimate_spectrum_from_fastx_pair(path, path, cfg)


def stream_estimates_from_fastx_pair(index_path, query_path, cfg: SuperCountingBloomConfig) -> StreamEstimateReport:
    cfg.validate()
    t_total = time.perf_counter()
    rep = SuperCountingBloomIndex.build_from_fastx(index_path, cfg)
    t_q = time.perf_counter()
    data, offsets = _read_batch(str(query_path))
    q = rep.index.query_report(data, offsets)
    t_end = time.perf_counter()
    stats = StreamEstimateStats(chunks=rep.chunks, indexed_kmers=rep.indexed_kmers, inserted_smers=rep.inserted_smers,
                                queried_kmers=q.valid_kmers, positive_estimates=q.positive_estimates,
                                estimate_checksum=q.estimate_checksum, counter_slots=rep.counter_slots,
                                blocks=rep.blocks, build_seconds=rep.build_seconds, query_seconds=t_end - t_q,
                                total_seconds=t_end - t_total)
    return StreamEstimateReport(stats=stats)


def stream_estimates_from_fastx(path, cfg: SuperCountingBloomConfig) -> StreamEstimateReport:
    return stream_estimates_from_fastx_pair(path, path, cfg)


def write_spectrum(spectrum, output=None) -> None:
    """src/spectrum.rs:11-31: TSV with header estimated_count<TAB>kmers."""
    text = "estimated_count\tkmers\n" + "".join(f"{c}\t{n}\n" for c, n in spectrum)
    if output is None:
        import sys

        sys.stdout.write(text)
        return
    try:
        with open(output, "w") as fh:
            fh.write(text)
    except OSError as err:
        raise Io(f"I/O error for '{output}': {err}") from err


# ---------------------------------------------------------------------------------------
# Serving (continuous batching over a device-resident frozen index)
# ---------------------------------------------------------------------------------------
@dataclass
class RequestStats:
    queue_ms: float
    service_ms: float
    total_ms: float
    windows: int


class SuperCountingBloomServer:
    """Request loop over a frozen index: submit() queues a request of sequences and returns a
    ticket immediately; wait(ticket) returns its per-window abundances and validity flags (the
    layout of SuperCountingBloomIndex.estimate_batch).  Requests arriving while others run share
    batches and overlap on the GPU; the device-memory budget bounds the batches in flight."""

    def __init__(self, index: "SuperCountingBloomIndex", memory_budget_bytes: int = 0,
                 max_batch_bytes: int = 64 << 20, max_batch_seqs: int = 0, max_inflight: int = 4,
                 spectrum_keys: int = 0):
        self.index = index
        cfg = _lib.ScbServerConfig(memory_budget_bytes, max_batch_bytes, max_batch_seqs, max_inflight, 0,
                                   spectrum_keys)
        out = C.c_void_p(0)
        _check(_lib.load().scb_server_create(index._ctx.h, C.byref(cfg), C.byref(out)))
        self.h = out
        self._live: dict[int, tuple] = {}

    def submit(self, data: np.ndarray, offsets: np.ndarray) -> int:
        data, offsets = _as_batch(data, offsets)
        n = len(offsets) - 1
        nw = int(_lib.load().scb_count_windows(self.index._ctx.h, _ptr(offsets), n))
        out = np.zeros(max(nw, 1), dtype=np.uint64)
        valid = np.zeros(max(nw, 1), dtype=np.uint8)
        t = C.c_uint64(0)
        _check(_lib.load().scb_server_submit(self.h, _ptr(data), _ptr(offsets), n, _ptr(out), _ptr(valid),
                                             C.byref(t)))
        self._live[t.value] = (data, offsets, out, valid, nw)  # keeps the buffers alive
        return t.value

    def wait(self, ticket: int) -> tuple[np.ndarray, np.ndarray, RequestStats]:
        st = _lib.ScbRequestStats()
        rc = _lib.load().scb_server_wait(self.h, ticket, C.byref(st))
        data, offsets, out, valid, nw = self._live.pop(ticket)
        _check(rc)
        return out[:nw], valid[:nw], RequestStats(st.queue_ms, st.service_ms, st.total_ms, st.windows)

    def summary(self) -> dict:
        s = _lib.ScbServerSummary()
        _check(_lib.load().scb_server_get_summary(self.h, C.byref(s)))
        return {"requests": s.requests, "windows": s.windows, "batches": s.batches, "p50_ms": s.p50_ms,
                "p99_ms": s.p99_ms, "mean_ms": s.mean_ms, "max_ms": s.max_ms, "span_s": s.span_s, "slots": s.slots}

    def reset_stats(self) -> None:
        _check(_lib.load().scb_server_reset_stats(self.h))

    def spectrum(self) -> dict:
        """The whole stream's distinct-k-mer spectrum (src/fastx.rs:255-308, 392-410) over every
        sequence answered since creation or the last reset_stats (needs spectrum_keys > 0)."""
        L = _lib.load()
        rows, dk, qk = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
        _check(L.scb_server_spectrum(self.h, None, None, 0, C.byref(rows), C.byref(dk), C.byref(qk)))
        vals = np.zeros(max(rows.value, 1), np.uint64)
        cnts = np.zeros(max(rows.value, 1), np.uint64)
        _check(L.scb_server_spectrum(self.h, _ptr(vals), _ptr(cnts), rows.value, C.byref(rows), C.byref(dk),
                                     C.byref(qk)))
        return {"rows": list(zip(vals[: rows.value].tolist(), cnts[: rows.value].tolist())),
                "distinct_keys": dk.value, "queried_kmers": qk.value}

    def close(self) -> None:
        if self.h and self.h.value:
            _lib.load().scb_server_destroy(self.h)
            self.h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
