"""Generic packed-sequence filters on the GPU backend (src/filter.rs:57-75, 118-571).

The reference's low-level types take a 2-bit packed sequence (packed_seq::PackedSeq) and a
config, and are generic over the counter type C (u8 / u16 / u32):

    SuperCountingBloom<C>::new(&cfg)                        -> mutable filter
        insert_packed_sequence(seq, &cfg) -> u64            inserted s-mers (filter.rs:199-237)
        freeze() -> FrozenSuperCountingBloom<C>             (filter.rs:147-163)
        counter_slots(), blocks(), counter_histogram()
    FrozenSuperCountingBloom<C>
        estimate_abundances_packed_sequence(seq, &cfg) -> Vec<C>        (filter.rs:337-369)
        stream_estimate_packed_sequence(seq, &cfg) -> (queried, checksum) (filter.rs:371-405)
        estimate_packed_sequence(seq, &cfg, &mut HashMap) -> queried     (filter.rs:302-335)
        counter_slots(), blocks(), counter_histogram()
    canonical_kmer(seq, len, pos), xorshift_u64(x)          (filter.rs:622-635)

Here the counters live in the device table of one C-ABI context (the counter type picks
counter_bits), and every call runs through libscb_b200.so.  A packed sequence holds only the four
base codes (PackedSeqVec.from_ascii maps every byte to (byte >> 1) & 3, as packed-seq does), so
each window is valid; the filter passes it to the library as the letters of those codes.

    from scbf_b200.filter import SuperCountingBloom, PackedSeqVec
    bloom = SuperCountingBloom[np.uint16].new(cfg)
    seq = PackedSeqVec.from_ascii(b"ACGTACGT...")
    bloom.insert_packed_sequence(seq, cfg)
    frozen = bloom.freeze()
    frozen.estimate_abundances_packed_sequence(seq, cfg)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .api import CounterBits, InternalState, InvalidConfig, SuperCountingBloomConfig, _check, _create

_LETTERS = np.frombuffer(b"ACTG", np.uint8)  # code -> letter: A=0, C=1, T=2, G=3
_COUNTER_BITS = {np.uint8: 8, np.uint16: 16, np.uint32: 32}
MASK64 = (1 << 64) - 1


class PackedSeqVec:
    """A 2-bit packed DNA sequence (packed_seq::PackedSeqVec): codes 0..3 = A, C, T, G."""

    def __init__(self, codes: np.ndarray):
        self.codes = np.ascontiguousarray(codes, dtype=np.uint8) & 3

    @classmethod
    def from_ascii(cls, sequence: bytes | str) -> "PackedSeqVec":
        if isinstance(sequence, str):
            sequence = sequence.encode()
        return cls((np.frombuffer(sequence, np.uint8) >> 1) & 3)

    def __len__(self) -> int:
        return int(self.codes.size)

    def len(self) -> int:
        return len(self)

    def as_slice(self) -> "PackedSeqVec":
        return self

    def to_ascii(self) -> bytes:
        return _LETTERS[self.codes].tobytes()


def xorshift_u64(x: int) -> int:
    """src/filter.rs:629-635: SplitMix64 finaliser with the golden-ratio increment."""
    x = (x + 0x9E3779B97F4A7C15) & MASK64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & MASK64
    return x ^ (x >> 31)


def _kmer_values(codes: np.ndarray, length: int) -> tuple[np.ndarray, np.ndarray]:
    """Forward and reverse-complement values of every length-`length` window (base t of the
    window at bits 2t; the reverse complement reads the complements, code ^ 2, backwards)."""
    n = codes.size + 1 - length
    fw = np.zeros(max(n, 0), np.uint64)
    rc = np.zeros(max(n, 0), np.uint64)
    c = codes.astype(np.uint64)
    for t in range(length):
        fw |= c[t:t + n] << np.uint64(2 * t)
        rc |= (c[length - 1 - t:length - 1 - t + n] ^ np.uint64(2)) << np.uint64(2 * t)
    return fw, rc


def canonical_kmer(sequence: PackedSeqVec, length: int, pos: int) -> int:
    """src/filter.rs:622-627: min of the window's value and its reverse complement's."""
    if not 0 < length <= 32 or pos + length > len(sequence):
        raise ValueError("window outside the sequence")
    fw, rc = _kmer_values(sequence.codes[pos:pos + length], length)
    return int(min(fw[0], rc[0]))


def canonical_kmers(sequence: PackedSeqVec, length: int) -> np.ndarray:
    """canonical_kmer of every window, in order."""
    fw, rc = _kmer_values(sequence.codes, length)
    return np.minimum(fw, rc)


def _counter_type(counter, cfg: SuperCountingBloomConfig):
    if counter is None:
        return {8: np.uint8, 16: np.uint16, 32: np.uint32}[int(cfg.counter_bits)]
    t = np.dtype(counter).type
    if t not in _COUNTER_BITS:
        raise InvalidConfig("invalid config: counter type must be u8, u16 or u32")
    return t


class _Generic:
    """`Cls[np.uint16]` selects the counter type, like `SuperCountingBloom::<u16>`."""

    counter = None

    def __class_getitem__(cls, counter):
        t = np.dtype(counter).type
        if t not in _COUNTER_BITS:
            raise TypeError("counter type must be np.uint8, np.uint16 or np.uint32")
        return type(f"{cls.__name__}[{np.dtype(t).name}]", (cls,), {"counter": t})


class SuperCountingBloom(_Generic):
    """The mutable filter (src/filter.rs:57-65, 118-237) on a device table."""

    def __init__(self, cfg: SuperCountingBloomConfig, counter=None):
        cfg.validate()
        self._type = _counter_type(counter if counter is not None else self.counter, cfg)
        self._cfg = SuperCountingBloomConfig(**{**cfg.__dict__, "counter_bits": CounterBits(_COUNTER_BITS[self._type])})
        self._ctx = _create(self._cfg)

    @classmethod
    def new(cls, cfg: SuperCountingBloomConfig) -> "SuperCountingBloom":
        return cls(cfg)

    def _live(self):
        if self._ctx is None:
            raise InternalState("internal state error: filter already frozen")
        return self._ctx

    def insert_packed_sequence(self, sequence: PackedSeqVec, cfg: SuperCountingBloomConfig) -> int:
        """Inserts every s-mer of every super-k-mer (filter.rs:199-237); returns the s-mers
        inserted, 0 for a sequence shorter than k."""
        ctx = self._live()
        if len(sequence) < cfg.k:
            return 0
        data = sequence.to_ascii()
        buf = np.frombuffer(data, np.uint8)
        offsets = np.array([0, buf.size], np.uint64)
        km, sm = C.c_uint64(0), C.c_uint64(0)
        _check(_lib.load().scb_insert_batch(ctx.h, buf.ctypes.data, offsets.ctypes.data, 1, C.byref(km),
                                            C.byref(sm)))
        return sm.value

    insert_packed_dna = insert_packed_sequence

    def freeze(self) -> "FrozenSuperCountingBloom":
        ctx = self._live()
        _check(_lib.load().scb_freeze(ctx.h))
        frozen = object.__new__(FrozenSuperCountingBloom)
        frozen._ctx, frozen._cfg, frozen._type = ctx, self._cfg, self._type
        self._ctx = None
        return frozen

    def counter_slots(self) -> int:
        return 1 << int(self._cfg.counter_slots_exponent)

    def blocks(self) -> int:
        return 1 << (int(self._cfg.counter_slots_exponent) - int(self._cfg.block_slots_exponent))

    def counter_histogram(self) -> list[tuple[int, int]]:
        return _histogram(self._live())


class FrozenSuperCountingBloom(_Generic):
    """The read-only filter (src/filter.rs:67-75, 239-571) on a device table."""

    def __init__(self):
        raise TypeError("use SuperCountingBloom.freeze")

    def _batch(self, sequence: PackedSeqVec):
        buf = np.frombuffer(sequence.to_ascii(), np.uint8)
        return buf, np.array([0, buf.size], np.uint64)

    def estimate_abundances_packed_sequence(self, sequence: PackedSeqVec, cfg: SuperCountingBloomConfig) -> np.ndarray:
        """One estimate per k-mer window, of the counter type (filter.rs:337-369)."""
        if len(sequence) < cfg.k:
            return np.zeros(0, self._type)
        buf, offsets = self._batch(sequence)
        n = len(sequence) + 1 - int(cfg.k)
        out = np.zeros(n, np.uint64)
        valid = np.zeros(n, np.uint8)
        _check(_lib.load().scb_query_batch(self._ctx.h, buf.ctypes.data, offsets.ctypes.data, 1, out.ctypes.data,
                                           valid.ctypes.data))
        return out.astype(self._type)

    estimate_abundances_packed_dna = estimate_abundances_packed_sequence

    def stream_estimate_packed_sequence(self, sequence: PackedSeqVec, cfg: SuperCountingBloomConfig) -> tuple[int, int]:
        """(windows queried, wrapping sum of their estimates) without per-window output
        (filter.rs:371-405)."""
        if len(sequence) < cfg.k:
            return 0, 0
        buf, offsets = self._batch(sequence)
        rep = _lib.ScbReport()
        _check(_lib.load().scb_query_report(self._ctx.h, buf.ctypes.data, offsets.ctypes.data, 1, C.byref(rep)))
        return rep.valid_kmers, rep.estimate_checksum & MASK64

    stream_estimate_packed_dna = stream_estimate_packed_sequence

    def estimate_packed_sequence(self, sequence: PackedSeqVec, cfg: SuperCountingBloomConfig,
                                 estimates: dict) -> int:
        """Adds each window's canonical k-mer -> estimate to `estimates` where the key is new
        (HashMap::entry(key).or_insert, filter.rs:407-460); returns the windows queried."""
        if len(sequence) < cfg.k:
            return 0
        ab = self.estimate_abundances_packed_sequence(sequence, cfg)
        keys = canonical_kmers(sequence, int(cfg.k))
        for key, est in zip(keys.tolist(), ab.tolist()):
            estimates.setdefault(key, est)
        return int(ab.size)

    estimate_packed_dna = estimate_packed_sequence

    def counter_slots(self) -> int:
        return 1 << int(self._cfg.counter_slots_exponent)

    def blocks(self) -> int:
        return 1 << (int(self._cfg.counter_slots_exponent) - int(self._cfg.block_slots_exponent))

    def counter_histogram(self) -> list[tuple[int, int]]:
        return _histogram(self._ctx)


def _histogram(ctx) -> list[tuple[int, int]]:
    L = _lib.load()
    rows = C.c_uint64(0)
    _check(L.scb_counter_histogram(ctx.h, None, None, 0, C.byref(rows)))
    vals = np.zeros(max(rows.value, 1), np.uint64)
    cnts = np.zeros(max(rows.value, 1), np.uint64)
    _check(L.scb_counter_histogram(ctx.h, vals.ctypes.data, cnts.ctypes.data, rows.value, C.byref(rows)))
    return list(zip(vals[: rows.value].tolist(), cnts[: rows.value].tolist()))
