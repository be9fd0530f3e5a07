"""Generic packed-sequence filters (src/filter.rs:57-75, 118-571) on the GPU backend.

Host helpers (packing, canonical_kmer, xorshift_u64) are checked against the oracle on CPU; the
reference's backend matrix (tests/backend_matrix.rs:95-235: u8/u16/u32 x four (k, m, s) cases x
five properties) and oracle parity of every estimate run on the GPU.
"""
import numpy as np
import pytest

# tests/backend_matrix.rs:8-20 (n_hashes 3, 2^16 slots, 2^6 per block) and 127-235
CASES = [
    (9, 5, 7, b"ACGTACGTACGTACGTACGTACGTACGT"),
    (9, 5, 9, b"ACGTACGTACGTACGTACGTACGTACGT"),
    (11, 5, 8, b"ACGTTGCATGTCAGTACGATCGTACGTTAGC"),
    (13, 7, 9, b"TGCATGCAACGTACGTTGCATGCAACGTACGT"),
]
TYPES = [np.uint8, np.uint16, np.uint32]


def _cfg(k, m, s, t):
    import scbf_b200 as scb

    return scb.SuperCountingBloomConfig(k=k, m=m, s=s, n_hashes=3,
                                        counter_bits=scb.CounterBits({np.uint8: 8, np.uint16: 16, np.uint32: 32}[t]),
                                        counter_slots_exponent=16, block_slots_exponent=6, threads=2, queue=4)


def test_host_helpers_match_oracle(oracle_mod):
    from scbf_b200.filter import PackedSeqVec, canonical_kmer, canonical_kmers, xorshift_u64

    rng = np.random.default_rng(3)
    for x in [0, 1, 2**63, 2**64 - 1] + rng.integers(0, 2**63, 20).tolist():
        assert xorshift_u64(int(x)) == oracle_mod.xorshift_u64(int(x))
    seq = rng.choice(np.frombuffer(b"ACGTacgt", np.uint8), 300).tobytes()
    p = PackedSeqVec.from_ascii(seq)
    assert np.array_equal(p.codes, oracle_mod.codes_of(seq))
    for length in (1, 5, 21, 31, 32):
        keys = canonical_kmers(p, length)
        assert keys.size == len(seq) + 1 - length
        for pos in (0, 7, len(seq) - length):
            assert int(keys[pos]) == canonical_kmer(p, length, pos) == oracle_mod.canonical_kmer(seq, length, pos)
    # filter.rs:748-756: a k-mer and its reverse complement share the canonical value
    assert canonical_kmer(PackedSeqVec.from_ascii(b"ACGTAC"), 6, 0) == canonical_kmer(PackedSeqVec.from_ascii(b"GTACGT"), 6, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("t", TYPES)
@pytest.mark.parametrize("case", CASES)
def test_backend_matrix_on_gpu(oracle_mod, case, t):
    from scbf_b200.filter import PackedSeqVec, SuperCountingBloom, canonical_kmers

    k, m, s, text = case
    cfg = _cfg(k, m, s, t)
    seq = PackedSeqVec.from_ascii(text)
    n = len(seq) + 1 - k

    def frozen(repeats):
        bloom = SuperCountingBloom[t].new(cfg)
        for _ in range(repeats):
            assert bloom.insert_packed_sequence(seq.as_slice(), cfg) > 0
        return bloom.freeze()

    # positive estimates (backend_matrix.rs:39-46)
    once = frozen(1)
    est = once.estimate_abundances_packed_sequence(seq.as_slice(), cfg)
    assert est.dtype == t and est.size == n and (est > 0).all()
    # vector length (48-57)
    twice = frozen(2)
    assert twice.estimate_abundances_packed_sequence(seq.as_slice(), cfg).size == n
    # stream == (len, wrapping sum of the vector) (58-69)
    thrice = frozen(3)
    vec = thrice.estimate_abundances_packed_sequence(seq.as_slice(), cfg)
    assert thrice.stream_estimate_packed_sequence(seq.as_slice(), cfg) == (vec.size, int(vec.astype(np.uint64).sum()))
    # map query (71-79)
    estimates = {}
    assert twice.estimate_packed_sequence(seq.as_slice(), cfg, estimates) == n
    assert estimates and all(v > 0 for v in estimates.values())
    assert set(estimates) == set(canonical_kmers(seq, k).tolist())
    # repeated inserts raise estimates (81-93)
    more = frozen(4).estimate_abundances_packed_sequence(seq.as_slice(), cfg)
    assert more.size == est.size and (more >= est).all()

    # every estimate and counter equals the oracle's after the same inserts
    bits = {np.uint8: 8, np.uint16: 16, np.uint32: 32}[t]
    for repeats, fz in ((1, once), (3, thrice)):
        o = oracle_mod.OracleFilter(oracle_mod.make_config(k, m, s, 3, bits, 16, 6, 2, 4))
        for _ in range(repeats):
            o.insert_packed(text)
        assert fz.estimate_abundances_packed_sequence(seq, cfg).astype(np.uint64).tolist() == o.estimate_packed(text)
        assert fz.counter_histogram() == o.counter_histogram()


@pytest.mark.gpu
def test_generic_filter_short_sequence_and_freeze_rules():
    import scbf_b200 as scb
    from scbf_b200.filter import PackedSeqVec, SuperCountingBloom

    cfg = _cfg(9, 5, 7, np.uint16)
    bloom = SuperCountingBloom[np.uint16].new(cfg)
    assert bloom.insert_packed_sequence(PackedSeqVec.from_ascii(b"ACGTACG"), cfg) == 0  # shorter than k
    assert bloom.counter_slots() == 1 << 16 and bloom.blocks() == 1 << 10
    assert bloom.counter_histogram() == [(0, 1 << 16)]
    fz = bloom.freeze()
    with pytest.raises(scb.InternalState):
        bloom.insert_packed_sequence(PackedSeqVec.from_ascii(b"ACGTACGTACGT"), cfg)
    assert fz.estimate_abundances_packed_sequence(PackedSeqVec.from_ascii(b"ACG"), cfg).size == 0
    assert fz.stream_estimate_packed_sequence(PackedSeqVec.from_ascii(b"ACGTACGTACGT"), cfg) == (4, 0)
