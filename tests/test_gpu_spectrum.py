"""Distinct-k-mer spectrum (src/fastx.rs:255-308, 392-410) on the GPU against the oracle.

The grouped spectrum apply deduplicates the canonical k-mers of each bucket's only work item in a
shared-memory set (every occurrence of a canonical k-mer has the same minimizer, so it lands in
the same bucket) and histograms the estimates in shared memory; split buckets go through the
global set.  The fused tile kernel inserts every key into the global set.  Both must give the
oracle's rows, distinct-key and queried-window counts.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scb():
    import scbf_b200

    return scbf_b200


def _index(scb, seqs, bits, slot_exp=20, strategy="auto", k=31, m=21, s=25, h=4, block_exp=9):
    from scbf_b200 import api

    cfg = scb.SuperCountingBloomConfig(k=k, m=m, s=s, n_hashes=h, counter_bits=scb.CounterBits(bits),
                                       counter_slots_exponent=slot_exp, block_slots_exponent=block_exp)
    b = scb.SuperCountingBloomBuilder(cfg)
    data, offsets = scb.pack_sequences(seqs)
    b.add_sequences(data, offsets)
    idx = b.into_index()
    api.set_strategy(idx, strategy, strategy)
    return idx, data, offsets


def _oracle(oracle_mod, data, offsets, bits, slot_exp=20, k=31, m=21, s=25, h=4, block_exp=9):
    o = oracle_mod.OracleFilter(oracle_mod.make_config(k, m, s, h, bits, slot_exp, block_exp))
    o.insert_batch_arrays(data, offsets)
    sp = o.spectrum_distinct_arrays(data, offsets)
    assert sp["mismatches"] == 0
    return sp


def _reads(seed, n, lo, hi, dup=3):
    rng = np.random.default_rng(seed)
    base = []
    for _ in range(n):
        L = int(rng.integers(lo, hi + 1))
        s = rng.choice(np.frombuffer(b"ACGT", np.uint8), L)
        s[rng.random(L) < 0.005] = ord("N")
        base.append(s.tobytes())
    return base + base[: n // dup] + [b"", b"ACGT", b"N" * 40]


@pytest.mark.parametrize("bits", [8, 16, 32])
@pytest.mark.parametrize("strategy", ["grouped", "fused"])
def test_spectrum_matches_oracle(scb, oracle_mod, bits, strategy):
    seqs = _reads(40 + bits, 3000, 100, 2000)
    idx, data, offsets = _index(scb, seqs, bits, strategy=strategy)
    ref = _oracle(oracle_mod, data, offsets, bits)
    got = idx.spectrum_distinct(data, offsets)
    assert got["rows"] == ref["rows"]
    assert (got["distinct_keys"], got["queried_kmers"]) == (ref["distinct_keys"], ref["queried_kmers"])


@pytest.mark.parametrize("geom", [(9, 5, 7, 3, 16, 6), (13, 7, 9, 3, 16, 6), (21, 11, 21, 5, 22, 10)])
def test_grouped_spectrum_other_geometries(scb, oracle_mod, geom):
    k, m, s, h, se, be = geom
    seqs = _reads(70 + k, 1500, 30, 800)
    idx, data, offsets = _index(scb, seqs, 16, slot_exp=se, strategy="grouped", k=k, m=m, s=s, h=h, block_exp=be)
    ref = _oracle(oracle_mod, data, offsets, 16, slot_exp=se, k=k, m=m, s=s, h=h, block_exp=be)
    got = idx.spectrum_distinct(data, offsets)
    assert got["rows"] == ref["rows"] and got["distinct_keys"] == ref["distinct_keys"]


def test_grouped_spectrum_hot_buckets_use_the_global_set(scb, oracle_mod):
    """20 000 copies of three reads split their buckets over several work items, whose keys then
    meet in the global set; the rest of the buckets deduplicate in shared memory."""
    rng = np.random.default_rng(12)
    hot = [rng.choice(np.frombuffer(b"ACGT", np.uint8), 150).tobytes() for _ in range(3)]
    seqs = [hot[i % 3] for i in range(20000)] + _reads(13, 1000, 100, 1500)
    for bits in (8, 16):
        idx, data, offsets = _index(scb, seqs, bits, strategy="grouped")
        ref = _oracle(oracle_mod, data, offsets, bits)
        got = idx.spectrum_distinct(data, offsets)
        assert got["rows"] == ref["rows"] and got["distinct_keys"] == ref["distinct_keys"]


def test_spectrum_values_past_the_dense_histogram(scb, oracle_mod):
    """32-bit counters above 65535 go to the overflow list (and past the shared-memory bins)."""
    rng = np.random.default_rng(14)
    read = rng.choice(np.frombuffer(b"ACGT", np.uint8), 60).tobytes()
    seqs = [read] * 70_000 + _reads(15, 300, 100, 1000)
    for strategy in ("grouped", "fused"):
        idx, data, offsets = _index(scb, seqs, 32, strategy=strategy)
        ref = _oracle(oracle_mod, data, offsets, 32)
        got = idx.spectrum_distinct(data, offsets)
        assert max(v for v, _ in ref["rows"]) >= 70_000
        assert got["rows"] == ref["rows"] and got["distinct_keys"] == ref["distinct_keys"]
