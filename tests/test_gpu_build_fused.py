"""The build + stream query in one apply pass (scb_set_fused_build) against the oracle.

With the grouped strategy for both passes, a bucket's only work item commits its deltas and then
answers its own records' windows from the committed shared-memory block; items of buckets split
over several items (hot buckets) or with more s-mers than the kept probe slots go through a second,
query-only pass.  The report must equal the oracle's insert-then-query (src/filter.rs:199-237,
462-508) whichever path each item takes, with graphs on and off, and equal the two-pass path.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GEOMETRIES = [  # (k, m, s, n_hashes, slot_exp, block_exp)
    (31, 21, 25, 4, 20, 9),   # default geometry, four probes (unrolled path)
    (9, 5, 7, 3, 16, 6),      # three probes (general path)
    (5, 3, 4, 2, 12, 5),      # two probes, tiny blocks
    (31, 1, 1, 6, 18, 11),    # six probes: no probe slots, the two-pass path
    (21, 11, 21, 4, 22, 7),   # s = k: one s-mer per window
]


@pytest.fixture(scope="module")
def scb():
    import scbf_b200

    return scbf_b200


def _random_batch(seed, n, lo, hi):
    rng = np.random.default_rng(seed)
    seqs = []
    for _ in range(n):
        L = int(rng.integers(lo, hi + 1))
        s = rng.choice(np.frombuffer(b"ACGT", np.uint8), L)
        s[rng.random(L) < 0.01] = ord("N")
        seqs.append(s.tobytes())
    return seqs


def _build_stream(scb, geom, bits, data, offsets, graphs=True, fused=True):
    from scbf_b200 import _lib, api

    k, m, s, h, se, be = geom
    cfg = scb.SuperCountingBloomConfig(k=k, m=m, s=s, n_hashes=h, counter_bits=scb.CounterBits(bits),
                                       counter_slots_exponent=se, block_slots_exponent=be)
    b = scb.SuperCountingBloomBuilder(cfg)
    api.set_strategy(b, "grouped", "grouped")
    L = _lib.load()
    assert L.scb_set_graphs(b._ctx.h, 1 if graphs else 0) == 0
    assert L.scb_set_fused_build(b._ctx.h, 1 if fused else 0) == 0
    km, sm = C.c_uint64(0), C.c_uint64(0)
    rep = _lib.ScbReport()
    out = []
    for _ in range(2):  # a second step (after a reset) replays the captured graph
        assert L.scb_reset(b._ctx.h) == 0
        st = L.scb_build_and_stream_query(b._ctx.h, data.ctypes.data, offsets.ctypes.data, len(offsets) - 1,
                                          C.byref(km), C.byref(sm), C.byref(rep))
        assert st == 0, _lib.last_error()
        tab = np.zeros(int(L.scb_table_bytes(b._ctx.h)), np.uint8)
        assert L.scb_table_download(b._ctx.h, tab.ctypes.data, tab.size) == 0
        out.append(((km.value, sm.value), (rep.records_processed, rep.total_windows, rep.valid_kmers,
                                           rep.positive_estimates, rep.estimate_checksum), tab))
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1] and np.array_equal(out[0][2], out[1][2])
    return out[0]


def _oracle(oracle_mod, geom, bits, data, offsets):
    k, m, s, h, se, be = geom
    o = oracle_mod.OracleFilter(oracle_mod.make_config(k, m, s, h, bits, se, be))
    counts = o.insert_batch_arrays(data, offsets)
    q = o.query_report_arrays(data, offsets)
    return counts, (q.records_processed, q.total_windows, q.valid_kmers, q.positive_estimates,
                    q.estimate_checksum), o.table().view(np.uint8)


@pytest.mark.parametrize("bits", [8, 16, 32])
@pytest.mark.parametrize("geom", GEOMETRIES)
def test_fused_build_matches_oracle(scb, oracle_mod, geom, bits):
    seqs = _random_batch(700 + geom[0] + bits, 400, 20, 3000)
    data, offsets = scb.pack_sequences(seqs)
    ref = _oracle(oracle_mod, geom, bits, data, offsets)
    for graphs in (True, False):
        got = _build_stream(scb, geom, bits, data, offsets, graphs=graphs)
        assert got[0] == ref[0] and got[1] == ref[1], graphs
        assert np.array_equal(got[2], ref[2])


@pytest.mark.parametrize("bits", [8, 16])
def test_fused_build_hot_buckets_are_deferred_and_exact(scb, oracle_mod, bits):
    """20 000 copies of three reads fill some buckets far past one work item: those items are split
    (not exclusive), their queries wait for the second pass, and u8 counters saturate."""
    rng = np.random.default_rng(9)
    base = [rng.choice(np.frombuffer(b"ACGT", np.uint8), 150).tobytes() for _ in range(3)]
    seqs = [base[i % 3] for i in range(20000)] + _random_batch(10, 300, 100, 2000) + [b"A" * 500, b"C" * 200]
    data, offsets = scb.pack_sequences(seqs)
    geom = GEOMETRIES[0]
    ref = _oracle(oracle_mod, geom, bits, data, offsets)
    for graphs in (True, False):
        got = _build_stream(scb, geom, bits, data, offsets, graphs=graphs)
        assert got[0] == ref[0] and got[1] == ref[1], graphs
        assert np.array_equal(got[2], ref[2])


def test_fused_build_equals_two_pass_on_short_reads(scb):
    from scbf_b200 import workloads

    data, offsets = workloads.short_reads(genome_len=400_000, n_reads=60_000, read_len=150, seed=5, sub_rate=0.01,
                                          n_rate=0.01)
    geom = (31, 21, 25, 4, 22, 9)
    fused = _build_stream(scb, geom, 16, data, offsets, fused=True)
    two = _build_stream(scb, geom, 16, data, offsets, fused=False)
    assert fused[0] == two[0] and fused[1] == two[1]
    assert np.array_equal(fused[2], two[2])


def test_fused_build_large_exclusive_items_are_deferred_and_exact(scb, oracle_mod):
    """A table of eight blocks: most buckets' only work item holds about 3 000 records (35 000
    s-mers), more probe words than a CTA keeps, so it stores them in item order for the
    query-only pass; the counts, report and table stay the oracle's."""
    from scbf_b200 import workloads

    data, offsets = workloads.short_reads(genome_len=100_000, n_reads=1200, read_len=150, seed=8, sub_rate=0.01,
                                          n_rate=0.0)
    geom = (31, 21, 25, 4, 12, 9)
    ref = _oracle(oracle_mod, geom, 16, data, offsets)
    for graphs in (True, False):
        got = _build_stream(scb, geom, 16, data, offsets, graphs=graphs)
        assert got[0] == ref[0] and got[1] == ref[1], graphs
        assert np.array_equal(got[2], ref[2])
