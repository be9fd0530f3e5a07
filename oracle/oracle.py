"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE).

The oracle is a plain-C restatement of the reference crate super-counting-bloom 0.1.0
(scb_oracle.c) plus a multi-threaded port with the reference's structure (scb_cpu_port.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use this module, and
only as the checker / the timed CPU path -- never as the product.

Parity status: bit-exact restatement of the reference's in-repo arithmetic; the arithmetic of
the absent third-party crates (packed-seq 4.4.2, simd-minimizers 2.3.1, seq-hash 0.1.2) is
restated from their published descriptions -- parity unpinned for those parts.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np

MASK64 = (1 << 64) - 1

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libscb_oracle.so")


class OraConfig(C.Structure):
    _fields_ = [
        ("k", C.c_uint64), ("m", C.c_uint64), ("s", C.c_uint64), ("n_hashes", C.c_uint64),
        ("counter_bits", C.c_uint8), ("counter_slots_exponent", C.c_uint8),
        ("block_slots_exponent", C.c_uint8), ("threads", C.c_uint64), ("queue", C.c_uint64),
    ]


class OraReport(C.Structure):
    _fields_ = [
        ("records_processed", C.c_uint64), ("total_windows", C.c_uint64),
        ("valid_kmers", C.c_uint64), ("positive_estimates", C.c_uint64),
        ("estimate_checksum", C.c_uint64),
    ]

    def as_tuple(self):
        return (self.records_processed, self.total_windows, self.valid_kmers,
                self.positive_estimates, self.estimate_checksum)


def build() -> str:
    """Compile the oracle with its Makefile (gcc / g++)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        u8p, u64p, u32p = C.POINTER(C.c_uint8), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)
        vp = C.c_void_p
        L.ora_validate.argtypes = [C.POINTER(OraConfig), C.c_char_p, C.c_size_t]
        L.ora_xorshift_u64.restype = C.c_uint64
        L.ora_xorshift_u64.argtypes = [C.c_uint64]
        L.ora_mmer_hash.restype = C.c_uint32
        L.ora_mmer_hash.argtypes = [u8p, C.c_size_t, C.c_size_t]
        L.ora_canonical_kmer.restype = C.c_uint64
        L.ora_canonical_kmer.argtypes = [u8p, C.c_size_t, C.c_size_t]
        L.ora_read_kmer.restype = C.c_uint64
        L.ora_read_kmer.argtypes = [u8p, C.c_size_t, C.c_size_t]
        L.ora_read_revcomp_kmer.restype = C.c_uint64
        L.ora_read_revcomp_kmer.argtypes = [u8p, C.c_size_t, C.c_size_t]
        L.ora_super_kmers.restype = C.c_size_t
        L.ora_super_kmers.argtypes = [u8p, C.c_size_t, C.c_size_t, C.c_size_t, u32p, u64p]
        L.ora_filter_new.restype = vp
        L.ora_filter_new.argtypes = [C.POINTER(OraConfig)]
        L.ora_filter_free.argtypes = [vp]
        L.ora_filter_clear.argtypes = [vp]
        L.ora_filter_table.restype = vp
        L.ora_filter_table.argtypes = [vp]
        L.ora_filter_table_bytes.restype = C.c_uint64
        L.ora_filter_table_bytes.argtypes = [vp]
        L.ora_filter_inserted_kmers.restype = C.c_uint64
        L.ora_filter_inserted_kmers.argtypes = [vp]
        L.ora_filter_inserted_smers.restype = C.c_uint64
        L.ora_filter_inserted_smers.argtypes = [vp]
        L.ora_insert_packed.restype = C.c_uint64
        L.ora_insert_packed.argtypes = [vp, u8p, C.c_size_t]
        L.ora_estimate_packed.argtypes = [vp, u8p, C.c_size_t, u64p]
        L.ora_insert_batch.argtypes = [vp, u8p, u64p, C.c_uint64, u64p, u64p]
        L.ora_query_batch.argtypes = [vp, u8p, u64p, C.c_uint64, u64p, u8p]
        L.ora_query_report.argtypes = [vp, u8p, u64p, C.c_uint64, C.POINTER(OraReport)]
        L.ora_spectrum_distinct.restype = C.c_uint64
        L.ora_spectrum_distinct.argtypes = [vp, u8p, u64p, C.c_uint64, u64p, u64p, C.c_uint64,
                                            u64p, u64p, u64p]
        L.ora_counter_histogram.restype = C.c_uint64
        L.ora_counter_histogram.argtypes = [vp, u64p, u64p, C.c_uint64]
        L.ora_save.argtypes = [vp, C.c_char_p]
        L.ora_load.restype = vp
        L.ora_load.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t]
        L.ora_batch_window_minimizers.argtypes = [u8p, u64p, C.c_uint64, C.c_uint64, C.c_uint64, u32p]
        L.ora_batch_sector_stats.argtypes = [C.POINTER(OraConfig), u8p, u64p, C.c_uint64, u64p, u64p, u64p]
        L.ora_port_build_and_stream_query.argtypes = [vp, u8p, u64p, C.c_uint64, C.c_uint64, C.c_uint64,
                                                      u64p, u64p, C.POINTER(OraReport),
                                                      C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib = L
    return _lib


def _u8(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def _u64(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _u32(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def make_config(k=31, m=21, s=25, n_hashes=4, counter_bits=16, counter_slots_exponent=30,
                block_slots_exponent=9, threads=1, queue=4096) -> OraConfig:
    return OraConfig(k, m, s, n_hashes, counter_bits, counter_slots_exponent,
                     block_slots_exponent, threads, queue)


def validate(cfg: OraConfig) -> str | None:
    buf = C.create_string_buffer(256)
    rc = lib().ora_validate(C.byref(cfg), buf, 256)
    return buf.value.decode() if rc else None


def pack_batch(seqs: list[bytes]) -> tuple[np.ndarray, np.ndarray]:
    """Concatenate sequences into (bytes, offsets[n+1])."""
    offsets = np.zeros(len(seqs) + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum([len(s) for s in seqs], dtype=np.uint64)
    data = np.frombuffer(b"".join(seqs), dtype=np.uint8).copy() if seqs else np.zeros(0, np.uint8)
    if data.size == 0:
        data = np.zeros(1, dtype=np.uint8)  # keep a valid pointer
    return data, offsets


def codes_of(seq: bytes) -> np.ndarray:
    a = np.frombuffer(seq, dtype=np.uint8)
    return ((a >> 1) & 3).astype(np.uint8)


def xorshift_u64(x: int) -> int:
    return int(lib().ora_xorshift_u64(C.c_uint64(x)))


def super_kmers(seq: bytes, k: int, m: int) -> tuple[list[int], list[int]]:
    codes = codes_of(seq)
    n = max(len(seq) - k + 1, 1)
    starts = np.zeros(n, dtype=np.uint32)
    mins = np.zeros(n, dtype=np.uint64)
    cnt = lib().ora_super_kmers(_u8(codes), len(seq), k, m, _u32(starts), _u64(mins))
    return starts[:cnt].tolist(), mins[:cnt].tolist()


def canonical_kmer(seq: bytes, length: int, pos: int) -> int:
    codes = codes_of(seq)
    return int(lib().ora_canonical_kmer(_u8(codes), length, pos))


@dataclass
class QueryReport:
    records_processed: int
    total_windows: int
    valid_kmers: int
    positive_estimates: int
    estimate_checksum: int


class OracleFilter:
    """The oracle's mutable / frozen filter (one object; the table is in .scb file order)."""

    def __init__(self, cfg: OraConfig | None = None, _handle=None):
        L = lib()
        if _handle is not None:
            self.h = _handle
        else:
            self.h = L.ora_filter_new(C.byref(cfg))
            if not self.h:
                raise ValueError(validate(cfg) or "oracle allocation failed")
        self.cfg = cfg

    def close(self):
        if self.h:
            lib().ora_filter_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clear(self):
        """All counters and totals back to zero on the same (already touched) allocation."""
        lib().ora_filter_clear(self.h)

    def table_view(self) -> np.ndarray:
        """The table's bytes without a copy (valid while the filter lives)."""
        L = lib()
        nbytes = L.ora_filter_table_bytes(self.h)
        return np.frombuffer((C.c_uint8 * nbytes).from_address(L.ora_filter_table(self.h)), dtype=np.uint8)

    @property
    def counter_bits(self) -> int:
        return self.cfg.counter_bits

    def table(self) -> np.ndarray:
        L = lib()
        nbytes = L.ora_filter_table_bytes(self.h)
        ptr = L.ora_filter_table(self.h)
        dt = {8: np.uint8, 16: np.uint16, 32: np.uint32}[self.counter_bits]
        raw = (C.c_uint8 * nbytes).from_address(ptr)
        return np.frombuffer(raw, dtype=np.uint8).view(dt).copy()

    def table_bytes(self) -> bytes:
        return self.table().tobytes()

    @property
    def inserted_kmers(self) -> int:
        return int(lib().ora_filter_inserted_kmers(self.h))

    @property
    def inserted_smers(self) -> int:
        return int(lib().ora_filter_inserted_smers(self.h))

    def insert_packed(self, seq: bytes) -> int:
        codes = codes_of(seq) if seq else np.zeros(1, np.uint8)
        return int(lib().ora_insert_packed(self.h, _u8(codes), len(seq)))

    def estimate_packed(self, seq: bytes) -> list[int]:
        k = self.cfg.k
        if len(seq) < k:
            return []
        codes = codes_of(seq)
        out = np.zeros(len(seq) + 1 - k, dtype=np.uint64)
        lib().ora_estimate_packed(self.h, _u8(codes), len(seq), _u64(out))
        return out.tolist()

    def insert_batch_arrays(self, data: np.ndarray, offsets: np.ndarray) -> tuple[int, int]:
        km, sm = C.c_uint64(0), C.c_uint64(0)
        lib().ora_insert_batch(self.h, _u8(data), _u64(offsets), len(offsets) - 1, C.byref(km), C.byref(sm))
        return km.value, sm.value

    def insert_batch(self, seqs: list[bytes]) -> tuple[int, int]:
        data, offsets = pack_batch(seqs)
        return self.insert_batch_arrays(data, offsets)

    def query_batch_arrays(self, data: np.ndarray, offsets: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        k = self.cfg.k
        lens = np.diff(offsets.astype(np.int64))
        total = int(np.where(lens >= k, lens + 1 - k, 0).sum())
        out = np.zeros(max(total, 1), dtype=np.uint64)
        valid = np.zeros(max(total, 1), dtype=np.uint8)
        lib().ora_query_batch(self.h, _u8(data), _u64(offsets), len(offsets) - 1, _u64(out), _u8(valid))
        return out[:total], valid[:total]

    def query_batch(self, seqs: list[bytes]) -> tuple[np.ndarray, np.ndarray]:
        data, offsets = pack_batch(seqs)
        return self.query_batch_arrays(data, offsets)

    def estimate_sequence_abundances(self, seq: bytes) -> list[int | None]:
        out, valid = self.query_batch([seq])
        return [int(v) if ok else None for v, ok in zip(out, valid)]

    def query_report_arrays(self, data, offsets) -> QueryReport:
        rep = OraReport()
        lib().ora_query_report(self.h, _u8(data), _u64(offsets), len(offsets) - 1, C.byref(rep))
        return QueryReport(*rep.as_tuple())

    def query_report(self, seqs: list[bytes]) -> QueryReport:
        data, offsets = pack_batch(seqs)
        return self.query_report_arrays(data, offsets)

    def spectrum_distinct_arrays(self, data, offsets):
        L = lib()
        dk, qk, mm = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
        n = len(offsets) - 1
        rows = L.ora_spectrum_distinct(self.h, _u8(data), _u64(offsets), n, None, None, 0,
                                       C.byref(dk), C.byref(qk), C.byref(mm))
        vals = np.zeros(max(rows, 1), np.uint64)
        cnts = np.zeros(max(rows, 1), np.uint64)
        L.ora_spectrum_distinct(self.h, _u8(data), _u64(offsets), n, _u64(vals), _u64(cnts), rows,
                                C.byref(dk), C.byref(qk), C.byref(mm))
        return {
            "rows": list(zip(vals[:rows].tolist(), cnts[:rows].tolist())),
            "distinct_keys": dk.value,
            "queried_kmers": qk.value,
            "mismatches": mm.value,
        }

    def spectrum_distinct(self, seqs: list[bytes]):
        data, offsets = pack_batch(seqs)
        return self.spectrum_distinct_arrays(data, offsets)

    def counter_histogram(self) -> list[tuple[int, int]]:
        L = lib()
        rows = L.ora_counter_histogram(self.h, None, None, 0)
        vals = np.zeros(max(rows, 1), np.uint64)
        cnts = np.zeros(max(rows, 1), np.uint64)
        L.ora_counter_histogram(self.h, _u64(vals), _u64(cnts), rows)
        return list(zip(vals[:rows].tolist(), cnts[:rows].tolist()))

    def save(self, path: str):
        if lib().ora_save(self.h, path.encode()):
            raise OSError(f"oracle save failed: {path}")

    @classmethod
    def load(cls, path: str) -> "OracleFilter":
        buf = C.create_string_buffer(256)
        h = lib().ora_load(path.encode(), buf, 256)
        if not h:
            raise ValueError(buf.value.decode())
        obj = cls(_handle=h)
        # read back the config from the file header
        with open(path, "rb") as fh:
            head = fh.read(63)
        import struct
        k, m, s, nh = struct.unpack_from("<4Q", head, 12)
        bits, cse, bse = struct.unpack_from("<3B", head, 44)
        thr, q = struct.unpack_from("<2Q", head, 47)
        obj.cfg = make_config(k, m, s, nh, bits, cse, bse, thr, q)
        return obj

    def port_build_and_stream_query(self, data, offsets, threads, queue=4096):
        km, sm = C.c_uint64(0), C.c_uint64(0)
        rep = OraReport()
        bs, qs = C.c_double(0), C.c_double(0)
        lib().ora_port_build_and_stream_query(self.h, _u8(data), _u64(offsets), len(offsets) - 1,
                                              threads, queue, C.byref(km), C.byref(sm), C.byref(rep),
                                              C.byref(bs), C.byref(qs))
        return {"inserted_kmers": km.value, "inserted_smers": sm.value,
                "report": QueryReport(*rep.as_tuple()), "build_s": bs.value, "query_s": qs.value}


def window_minimizers(data: np.ndarray, offsets: np.ndarray, k: int, m: int) -> np.ndarray:
    out = np.zeros(max(int(offsets[-1]), 1), dtype=np.uint32)
    lib().ora_batch_window_minimizers(_u8(data), _u64(offsets), len(offsets) - 1, k, m, _u32(out))
    return out[: int(offsets[-1])]


def sector_stats(cfg: OraConfig, data, offsets) -> tuple[int, int, int]:
    a, b, c = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
    lib().ora_batch_sector_stats(C.byref(cfg), _u8(data), _u64(offsets), len(offsets) - 1,
                                 C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


# ---------------------------------------------------------------------------------------
# Filter-only spectrum (src/api.rs:337-385, 933-1033): host f64 arithmetic over a counter
# histogram, restated step for step (plain loops, sums left to right) so that every rounding is
# the reference's.  The checker of scbf_b200.api's vectorised form.
# ---------------------------------------------------------------------------------------
def rust_round_u64(x: float) -> int:
    """`x.round() as u64`: nearest integer with halves away from zero; NaN and negatives give 0,
    values past u64 saturate."""
    if not x > 0.0:
        return 0
    r = math.floor(x)
    if x - r >= 0.5:
        r += 1
    return min(int(r), (1 << 64) - 1)


def filter_only_deconvolved_counts(counter_histogram, n_hashes: int, max_abundance: int) -> list[float]:
    """src/api.rs:958-1001 (deconvolved_counts): k-mer counts per abundance 1..=max_abundance from
    the logarithm of the counters' generating function (compound Poisson)."""
    if max_abundance == 0:
        return []
    total = 0
    for _, counters in counter_histogram:
        total += counters
    if total == 0:
        return [0.0] * max_abundance
    prob = [0.0] * (max_abundance + 1)
    for abundance, counters in counter_histogram:
        if abundance <= max_abundance:
            prob[abundance] += float(counters) / float(total)
    p0 = prob[0]
    if p0 <= 0.0:
        return []
    norm = [0.0] * (max_abundance + 1)
    norm[0] = 1.0
    for a in range(1, max_abundance + 1):
        norm[a] = prob[a] / p0
    logc = [0.0] * (max_abundance + 1)
    for a in range(1, max_abundance + 1):
        coef = float(a) * norm[a]
        for p in range(1, a):
            coef -= float(p) * logc[p] * norm[a - p]
        logc[a] = coef / float(a)
    h = float(max(n_hashes, 1))
    out = []
    for a in range(1, max_abundance + 1):
        v = float(total) * logc[a] / h
        out.append(v if v > 0.0 else 0.0)  # f64::max(v, 0.0), NaN -> 0
    return out


def _sum_left(values) -> float:
    t = 0.0
    for v in values:
        t += v
    return t


def filter_only_scaled_positive(counter_histogram, max_abundance: int, kmer_count_hint: int) -> list[tuple[int, int]]:
    """src/api.rs:1003-1022 (scaled_positive_counter_histogram)."""
    positive = 0
    for abundance, counters in counter_histogram:
        if abundance > 0:
            positive += counters
    positive_f = float(max(positive, 1))
    by_value = {}
    for abundance, counters in counter_histogram:
        by_value[abundance] = counters
    return [(a, rust_round_u64(float(kmer_count_hint) * float(by_value.get(a, 0)) / positive_f))
            for a in range(1, max_abundance + 1)]


def filter_only_spectrum(counter_histogram, n_hashes: int, max_abundance: int,
                         kmer_count_hint: int) -> list[tuple[int, int]]:
    """src/api.rs:933-956 (estimate_filter_only_spectrum_from_counter_histogram)."""
    dec = filter_only_deconvolved_counts(counter_histogram, n_hashes, max_abundance)
    total = _sum_left(dec)
    if total <= 0.0:
        return filter_only_scaled_positive(counter_histogram, max_abundance, kmer_count_hint)
    scale = float(kmer_count_hint) / total
    return [(a, rust_round_u64(dec[a - 1] * scale)) for a in range(1, max_abundance + 1)]


def filter_only_count_hint(counter_histogram, n_hashes: int, max_abundance: int = 255) -> int:
    """src/api.rs:375-385 (filter_only_count_hint_from_counter_histogram)."""
    s = _sum_left(filter_only_deconvolved_counts(counter_histogram, n_hashes, max_abundance))
    return max(rust_round_u64(s), 1)


# ---------------------------------------------------------------------------------------
# FASTA/FASTQ records (src/api.rs:893-915): the line-by-line reader, the checker of the library's
# one-pass reader (scb_fastx_read).  Lines end at b"\n" and lose trailing b"\r" / b"\n"; b">" or
# b"@" opens a record; a FASTQ record's sequence runs to a b"+" line and the next line (its
# qualities) is skipped; lines before the first header are ignored; gzip input is inflated.
# ---------------------------------------------------------------------------------------
def fastx_records(path: str):
    """Yields (header without its marker, sequence) per record."""
    import gzip

    with open(path, "rb") as probe:
        gz = probe.read(2) == b"\x1f\x8b"
    with (gzip.open(path, "rb") if gz else open(path, "rb")) as fh:
        header = None
        seq: list[bytes] = []
        fastq_state = 0
        for raw in fh:
            line = raw.rstrip(b"\r\n")
            if fastq_state == 2:
                fastq_state = 0
                continue
            if fastq_state == 1:
                if line.startswith(b"+"):
                    fastq_state = 2
                else:
                    seq.append(line)
                continue
            if line.startswith(b">") or line.startswith(b"@"):
                if header is not None:
                    yield header, b"".join(seq)
                header = line[1:]
                seq = []
                fastq_state = 1 if line.startswith(b"@") else 0
            elif header is not None:
                seq.append(line)
        if header is not None:
            yield header, b"".join(seq)


# ---------------------------------------------------------------------------------------
# Sampled spectrum (src/bin/sampled_spectrum.rs:182-223, 263-305): reservoir sampling of the
# valid k-mer windows, restated as the sequential loop (the checker of the vectorised sampler).
# ---------------------------------------------------------------------------------------
def _splitmix_next(state: int) -> tuple[int, int]:
    state = (state + 0x9E3779B97F4A7C15) & MASK64
    v = state
    v = ((v ^ (v >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    v = ((v ^ (v >> 27)) * 0x94D049BB133111EB) & MASK64
    return state, v ^ (v >> 31)


def reservoir_sample_kmers(sequences, k: int, capacity: int, seed: int) -> tuple[list[bytes], int]:
    """The sampled k-mers (upper case, in reservoir slot order) and the number of windows seen."""
    kmers: list[bytes] = []
    seen = 0
    state = seed & MASK64
    for seq in sequences:
        if len(seq) < k:
            continue
        runs, start = [], None
        for i, b in enumerate(seq):
            ub = b - 32 if 97 <= b <= 122 else b  # to_ascii_uppercase
            if ub in (65, 67, 71, 84):
                if start is None:
                    start = i
            elif start is not None:
                runs.append((start, i))
                start = None
        if start is not None:
            runs.append((start, len(seq)))
        for a, e in runs:
            if e - a < k:
                continue
            for off in range(a, e - k + 1):
                seen += 1
                if len(kmers) < capacity:
                    slot = len(kmers)
                else:
                    state, v = _splitmix_next(state)
                    r = v % seen
                    slot = r if r < capacity else None
                if slot is not None:
                    km = seq[off:off + k].upper()
                    if slot == len(kmers):
                        kmers.append(km)
                    else:
                        kmers[slot] = km
    return kmers, seen
