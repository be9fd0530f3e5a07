"""Bit-exact parity of the CUDA path (through the C ABI) against the CPU oracle.

Integer work: counters, per-window abundances, reports, spectra, counter histograms and .scb
bytes must be identical, for every counter width and the reference tests' geometries.
"""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GEOMETRIES = [  # (k, m, s, n_hashes, slot_exp, block_exp): reference test geometries + default
    (31, 21, 25, 4, 20, 9),
    (9, 5, 7, 3, 16, 6),
    (9, 5, 9, 3, 16, 6),
    (11, 5, 8, 3, 16, 6),
    (13, 7, 9, 3, 16, 6),
    (5, 3, 4, 2, 12, 5),
    (31, 31, 31, 2, 18, 7),
    (31, 1, 1, 6, 18, 11),
    (21, 11, 21, 5, 22, 10),
]


@pytest.fixture(scope="module")
def scb():
    import scbf_b200

    return scbf_b200


def _cfg(scb, k, m, s, h, se, be, bits):
    return scb.SuperCountingBloomConfig(k=k, m=m, s=s, n_hashes=h, counter_bits=scb.CounterBits(bits),
                                        counter_slots_exponent=se, block_slots_exponent=be, threads=3, queue=17)


def _random_batch(seed, n, lo, hi, n_rate=0.02, lower_rate=0.01):
    rng = np.random.default_rng(seed)
    seqs = []
    for _ in range(n):
        L = int(rng.integers(lo, hi + 1))
        s = rng.choice(np.frombuffer(b"ACGT", np.uint8), L)
        if n_rate:
            s[rng.random(L) < n_rate] = ord("N")
        if lower_rate:
            low = rng.random(L) < lower_rate
            s[low] = s[low] | 0x20
        seqs.append(s.tobytes())
    seqs += [b"", b"ACG", b"N" * 40, b"acgtacgtacgtacgtacgtacgtacgtacgtacgtacgtACGT"]
    return seqs


def _pair(scb, oracle_mod, k, m, s, h, se, be, bits, seqs, strategy="auto"):
    from scbf_b200 import api

    cfg = _cfg(scb, k, m, s, h, se, be, bits)
    b = scb.SuperCountingBloomBuilder(cfg)
    api.set_strategy(b, strategy, strategy)
    data, offsets = scb.pack_sequences(seqs)
    rep = b.add_sequences(data, offsets)
    idx = b.into_index()
    o = oracle_mod.OracleFilter(oracle_mod.make_config(k, m, s, h, bits, se, be, 3, 17))
    okm, osm = o.insert_batch_arrays(data, offsets)
    return cfg, idx, o, data, offsets, rep, (okm, osm)


@pytest.mark.parametrize("bits", [8, 16, 32])
@pytest.mark.parametrize("geom", GEOMETRIES)
def test_insert_query_parity(scb, oracle_mod, geom, bits):
    k, m, s, h, se, be = geom
    seqs = _random_batch(1000 + k * 7 + bits, 120, 1, 600)
    cfg, idx, o, data, offsets, rep, (okm, osm) = _pair(scb, oracle_mod, k, m, s, h, se, be, bits, seqs)
    assert (rep.inserted_kmers, rep.inserted_smers) == (okm, osm)
    assert np.array_equal(idx.table(), o.table())
    out, valid = idx.estimate_batch(data, offsets)
    oout, ovalid = o.query_batch_arrays(data, offsets)
    assert np.array_equal(valid, ovalid)
    assert np.array_equal(np.where(valid == 1, out, 0), np.where(ovalid == 1, oout, 0))
    q = idx.query_report(data, offsets)
    oq = o.query_report_arrays(data, offsets)
    assert (q.records_processed, q.total_windows, q.valid_kmers, q.positive_estimates, q.estimate_checksum) == (
        oq.records_processed, oq.total_windows, oq.valid_kmers, oq.positive_estimates, oq.estimate_checksum)
    sp = idx.spectrum_distinct(data, offsets)
    osp = o.spectrum_distinct_arrays(data, offsets)
    assert osp["mismatches"] == 0
    assert sp["rows"] == osp["rows"]
    assert sp["distinct_keys"] == osp["distinct_keys"] and sp["queried_kmers"] == osp["queried_kmers"]
    assert idx.counter_histogram() == o.counter_histogram()


@pytest.mark.parametrize("geom", [GEOMETRIES[0], GEOMETRIES[1], GEOMETRIES[7]])
def test_window_minimizers_match_oracle(scb, oracle_mod, geom):
    from scbf_b200 import _lib
    import ctypes as C

    k, m, s, h, se, be = geom
    seqs = _random_batch(77 + k, 60, 1, 400)
    data, offsets = scb.pack_sequences(seqs)
    b = scb.SuperCountingBloomBuilder(_cfg(scb, k, m, s, h, se, be, 16))
    out = np.zeros(max(int(offsets[-1]), 1), dtype=np.uint32)
    st = _lib.load().scb_debug_window_minimizers(b._ctx.h, data.ctypes.data, offsets.ctypes.data,
                                                   len(offsets) - 1, out.ctypes.data)
    assert st == 0, _lib.last_error()
    ref = oracle_mod.window_minimizers(data, offsets, k, m)
    assert np.array_equal(out[: int(offsets[-1])], ref)


@pytest.mark.parametrize("bits", [8, 16, 32])
def test_strategies_agree(scb, oracle_mod, bits):
    seqs = _random_batch(5 + bits, 300, 100, 2000)
    res = []
    for strategy in ("plain", "fused", "grouped"):
        cfg, idx, o, data, offsets, rep, okms = _pair(scb, oracle_mod, 31, 21, 25, 4, 20, 9, bits, seqs, strategy)
        res.append((idx.table(), idx.estimate_batch(data, offsets), idx.query_report(data, offsets),
                    (rep.inserted_kmers, rep.inserted_smers)))
        assert np.array_equal(idx.table(), o.table())
        assert (rep.inserted_kmers, rep.inserted_smers) == okms
    for other in res[1:]:
        assert np.array_equal(res[0][0], other[0])
        assert np.array_equal(res[0][1][0], other[1][0]) and np.array_equal(res[0][1][1], other[1][1])
        assert res[0][2] == other[2]


@pytest.mark.parametrize("geom", GEOMETRIES)
def test_grouped_parity_all_geometries(scb, oracle_mod, geom):
    k, m, s, h, se, be = geom
    for bits in (8, 16, 32):
        seqs = _random_batch(300 + k + bits, 150, 1, 800)
        cfg, idx, o, data, offsets, rep, okms = _pair(scb, oracle_mod, k, m, s, h, se, be, bits, seqs, "grouped")
        assert (rep.inserted_kmers, rep.inserted_smers) == okms
        assert np.array_equal(idx.table(), o.table())
        q = idx.query_report(data, offsets)
        oq = o.query_report_arrays(data, offsets)
        assert (q.valid_kmers, q.positive_estimates, q.estimate_checksum) == (
            oq.valid_kmers, oq.positive_estimates, oq.estimate_checksum)


@pytest.mark.parametrize("bits", [8, 16, 32])
def test_grouped_hot_buckets_split_and_saturate(scb, oracle_mod, bits):
    """20000 copies of a few reads put far more than one work item's records in the same
    buckets: the split items commit through saturating CAS and must still be exact."""
    rng = np.random.default_rng(4)
    base = [rng.choice(np.frombuffer(b"ACGT", np.uint8), 150).tobytes() for _ in range(3)]
    seqs = [base[i % 3] for i in range(20000)] + _random_batch(8, 50, 100, 300)
    for strategy in ("grouped", "fused"):
        cfg, idx, o, data, offsets, rep, okms = _pair(scb, oracle_mod, 31, 21, 25, 4, 20, 9, bits, seqs, strategy)
        assert (rep.inserted_kmers, rep.inserted_smers) == okms
        assert np.array_equal(idx.table(), o.table())
        q = idx.query_report(data, offsets)
        oq = o.query_report_arrays(data, offsets)
        assert (q.valid_kmers, q.positive_estimates, q.estimate_checksum) == (
            oq.valid_kmers, oq.positive_estimates, oq.estimate_checksum)


def test_save_matches_oracle_bytes_and_roundtrips(scb, oracle_mod):
    seqs = _random_batch(9, 80, 30, 300)
    with tempfile.TemporaryDirectory() as d:
        for bits in (8, 16, 32):
            cfg, idx, o, data, offsets, rep, _ = _pair(scb, oracle_mod, 31, 21, 25, 4, 18, 9, bits, seqs)
            o_path, g_path = os.path.join(d, f"o{bits}.scb"), os.path.join(d, f"g{bits}.scb")
            o.save(o_path)
            idx.save(g_path)
            assert open(o_path, "rb").read() == open(g_path, "rb").read()
            loaded = scb.SuperCountingBloomIndex.load(g_path)
            assert loaded.config() == idx.config()
            assert loaded.inserted_kmers() == idx.inserted_kmers()
            assert loaded.counter_histogram() == idx.counter_histogram()
            q = b"ACGTACGTNNACGTACGTACGTACGTACGTACGTACGTACGTACG" + seqs[0]
            assert loaded.estimate_sequence_abundances(q) == idx.estimate_sequence_abundances(q)
            # the GPU reads the oracle's file too
            from_oracle = scb.SuperCountingBloomIndex.load(o_path)
            assert np.array_equal(from_oracle.table(), o.table())


def test_saturation_u8_and_wider(scb, oracle_mod, known_answers):
    t = known_answers["saturation"]
    c = known_answers["configs"][t["config"]]
    for seq in (t["sequence"], t["pipeline_sequence"]):
        for bits in (8, 16, 32):
            cfg = _cfg(scb, c["k"], c["m"], c["s"], c["n_hashes"], c["counter_slots_exponent"],
                       c["block_slots_exponent"], bits)
            b = scb.SuperCountingBloomBuilder(cfg)
            data, offsets = scb.pack_sequences([seq] * t["repeats"])
            b.add_sequences(data, offsets)
            idx = b.into_index()
            est = idx.estimate_sequence_abundances(seq)
            if bits == 8:
                assert all(v == t["u8_all_equal"] for v in est)
            else:
                assert all(v >= t["wider_floor"] for v in est)
            o = oracle_mod.OracleFilter(oracle_mod.make_config(c["k"], c["m"], c["s"], c["n_hashes"], bits,
                                                               c["counter_slots_exponent"],
                                                               c["block_slots_exponent"]))
            o.insert_batch_arrays(data, offsets)
            assert np.array_equal(idx.table(), o.table())


def test_reference_known_answers_on_gpu(scb, known_answers, tmp_path):
    # src/api.rs:1057-1072, 1095-1111, 1158-1202 and fastx.rs:448-466 through the GPU API
    ka = known_answers
    c = dict(ka["configs"]["api_small"])
    c.pop("_cite")
    cfg = scb.SuperCountingBloomConfig(**{**c, "counter_bits": scb.CounterBits(c["counter_bits"])})
    fa = tmp_path / "r.fa"
    fa.write_bytes(b">r\nACGTACGTACGT\n")
    idx = scb.SuperCountingBloomIndex.build_from_fastx(fa, cfg).index
    ab = idx.estimate_sequence_abundances(ka["invalid_windows"]["query"])
    assert len(ab) == 10 and all(x is not None for x in ab[:2] + ab[8:]) and all(x is None for x in ab[2:8])
    summ = idx.summarize_sequence("query", b"ACGTACGT")
    assert (summ.total_windows, summ.valid_kmers) == (4, 4) and summ.mean_abundance > 0

    t = ka["builder"]
    cfg16 = scb.SuperCountingBloomConfig(**{**c, "counter_bits": scb.CounterBits.Bits16, "threads": 2, "queue": 1})
    b = scb.SuperCountingBloomBuilder(cfg16)
    assert b.threads() == 2
    assert b.add_sequence(t["add_sequence"]) == t["add_sequence_kmers"]
    reads = tmp_path / "b.fa"
    reads.write_bytes(b">r1\nACGTACGTACGT\n>r2\nACGTNNACGTAC\n")
    rep = b.add_fasta(reads)
    assert (rep.records_processed, rep.records_indexed, rep.inserted_kmers) == (2, 2, 10)
    assert b.inserted_kmers() == 14 and b.inserted_smers() > 0
    idx = b.into_index()
    assert idx.inserted_kmers() == 14
    q = idx.query_fasta(reads)
    assert (q.records_processed, q.total_windows, q.valid_kmers) == (2, 16, 10)
    assert q.positive_estimates > 0 and q.estimate_checksum > 0
    p = tmp_path / "i.scb"
    idx.save(p)
    loaded = scb.SuperCountingBloomIndex.load(p)
    assert loaded.inserted_kmers() == 14 and loaded.query_fasta(reads) == q

    sm = ka["fastx_spectrum_smoke"]
    c2 = dict(ka["configs"]["fastx_small"])
    c2.pop("_cite")
    fa2 = tmp_path / "s.fa"
    fa2.write_bytes(b">r1\nACGTACGTACGTACGTACGT\n>r2\nACGTACGTACGTACGTACGT\n")
    for bits in (8, 16, 32):
        cfgb = scb.SuperCountingBloomConfig(**{**c2, "counter_bits": scb.CounterBits(bits)})
        r = scb.estimate_spectrum_from_fastx(fa2, cfgb)
        assert (r.stats.chunks, r.stats.indexed_kmers, r.stats.queried_kmers) == (
            sm["chunks"], sm["indexed_kmers"], sm["queried_kmers"])
        assert r.spectrum
        st = scb.stream_estimates_from_fastx(fa2, cfgb)
        assert st.stats.queried_kmers == sm["queried_kmers"] and st.stats.estimate_checksum > 0


def test_workload_medium_parity(scb, oracle_mod):
    """Seeded short-read workload (config-1 shape at reduced depth) bit-exact vs the oracle."""
    from scbf_b200 import workloads

    data, offsets = workloads.short_reads(genome_len=200_000, n_reads=20_000, read_len=150, seed=1,
                                          sub_rate=0.005, n_rate=0.01)
    for strategy in ("plain", "fused", "grouped"):
        cfg = _cfg(scb, 31, 21, 25, 4, 24, 9, 16)
        b = scb.SuperCountingBloomBuilder(cfg)
        from scbf_b200 import api

        api.set_strategy(b, strategy, strategy)
        rep = b.add_sequences(data, offsets)
        idx = b.into_index()
        if strategy == "plain":
            o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 24, 9))
            okm, osm = o.insert_batch_arrays(data, offsets)
            oq = o.query_report_arrays(data, offsets)
            otab = o.table()
        assert (rep.inserted_kmers, rep.inserted_smers) == (okm, osm)
        assert np.array_equal(idx.table(), otab)
        q = idx.query_report(data, offsets)
        assert (q.valid_kmers, q.positive_estimates, q.estimate_checksum) == (
            oq.valid_kmers, oq.positive_estimates, oq.estimate_checksum)


@pytest.mark.parametrize("strategy", ["auto", "plain", "fused", "grouped"])
def test_build_and_stream_query_matches_separate_calls(scb, oracle_mod, strategy):
    from scbf_b200 import _lib, api, workloads
    import ctypes as C

    data, offsets = workloads.short_reads(genome_len=100_000, n_reads=5_000, read_len=150, seed=3,
                                          sub_rate=0.01, n_rate=0.01)
    cfg = _cfg(scb, 31, 21, 25, 4, 22, 9, 16)
    b = scb.SuperCountingBloomBuilder(cfg)
    api.set_strategy(b, strategy, strategy)
    km, sm = C.c_uint64(0), C.c_uint64(0)
    rep = _lib.ScbReport()
    st = _lib.load().scb_build_and_stream_query(b._ctx.h, data.ctypes.data, offsets.ctypes.data, len(offsets) - 1,
                                                C.byref(km), C.byref(sm), C.byref(rep))
    assert st == 0, _lib.last_error()
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 22, 9))
    okm, osm = o.insert_batch_arrays(data, offsets)
    oq = o.query_report_arrays(data, offsets)
    assert (km.value, sm.value) == (okm, osm)
    assert (rep.valid_kmers, rep.positive_estimates, rep.estimate_checksum) == (
        oq.valid_kmers, oq.positive_estimates, oq.estimate_checksum)
    fresh = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 22, 9))
    res = fresh.port_build_and_stream_query(data, offsets, threads=4)
    assert res["report"].estimate_checksum == rep.estimate_checksum


def test_errors_map_to_reference_variants(scb, tmp_path):
    with pytest.raises(scb.InvalidConfig):
        scb.SuperCountingBloomBuilder(scb.SuperCountingBloomConfig(k=10, m=5, s=7, counter_slots_exponent=16,
                                                                   block_slots_exponent=6))
    bad = tmp_path / "bad.scb"
    bad.write_bytes(b"not an index")
    with pytest.raises(scb.InvalidIndexFormat):
        scb.SuperCountingBloomIndex.load(bad)
    with pytest.raises(scb.Io):
        scb.SuperCountingBloomIndex.load(tmp_path / "missing.scb")
    b = scb.SuperCountingBloomBuilder(scb.SuperCountingBloomConfig(counter_slots_exponent=16))
    with pytest.raises(scb.InvalidConfig):
        b.set_threads(0)
    with pytest.raises(scb.FastxOpen):
        b.add_fasta(tmp_path / "missing.fa")


@pytest.mark.parametrize("strategy", ["plain", "fused", "grouped"])
def test_build_and_stream_query_device_matches_oracle(scb, oracle_mod, strategy):
    import torch

    from scbf_b200 import _lib, api, workloads
    import ctypes as C

    data, offsets = workloads.short_reads(genome_len=150_000, n_reads=8_000, read_len=150, seed=13,
                                          sub_rate=0.01, n_rate=0.01)
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 22, 9))
    okm, osm = o.insert_batch_arrays(data, offsets)
    oq = o.query_report_arrays(data, offsets)
    b = scb.SuperCountingBloomBuilder(_cfg(scb, 31, 21, 25, 4, 22, 9, 16))
    api.set_strategy(b, strategy, strategy)
    L = _lib.load()
    d_data = torch.from_numpy(data).cuda()
    d_off = torch.from_numpy(offsets.view(np.int64)).cuda()
    km, sm = C.c_uint64(0), C.c_uint64(0)
    rep = _lib.ScbReport()
    for _ in range(2):  # a reset between steps gives the same result
        assert L.scb_reset(b._ctx.h) == 0
        st = L.scb_build_and_stream_query_device(b._ctx.h, d_data.data_ptr(), d_off.data_ptr(), len(offsets) - 1,
                                                 int(offsets[-1]), None, C.byref(km), C.byref(sm), C.byref(rep))
        assert st == 0, _lib.last_error()
        assert (km.value, sm.value) == (okm, osm)
        assert (rep.records_processed, rep.total_windows, rep.valid_kmers, rep.positive_estimates,
                rep.estimate_checksum) == (oq.records_processed, oq.total_windows, oq.valid_kmers,
                                           oq.positive_estimates, oq.estimate_checksum)
        out = np.zeros(int(L.scb_table_bytes(b._ctx.h)), dtype=np.uint8)
        assert L.scb_table_download(b._ctx.h, out.ctypes.data, out.size) == 0
        assert np.array_equal(out.view(np.uint16), o.table())


def test_records_indexed_matches_run_definition(scb):
    """AddReport::records_indexed (src/api.rs:640-642): records holding a run of k A/C/G/T bases."""
    seqs = _random_batch(77, 400, 1, 120, n_rate=0.08, lower_rate=0.05)
    seqs += [b"A" * 30 + b"N" + b"C" * 30, b"a" * 31, b"ACGTN" * 20, b"", b"G" * 31 + b"N"]
    data, offsets = scb.pack_sequences(seqs)
    k = 31

    def indexed(s: bytes) -> bool:
        run = 0
        for c in s:
            run = run + 1 if chr(c) in "ACGTacgt" else 0
            if run >= k:
                return True
        return False

    b = scb.SuperCountingBloomBuilder(_cfg(scb, 31, 21, 25, 4, 20, 9, 16))
    rep = b.add_sequences(data, offsets)
    assert rep.records_indexed == sum(indexed(s) for s in seqs)
    assert rep.records_processed == len(seqs)
