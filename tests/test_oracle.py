"""Pins the CPU oracle against the reference crate's own known answers and properties.

Every assertion mirrors one in the reference's tests (file:line in the golden JSON).  The
oracle is then the checker for the CUDA library (tests/test_gpu_*.py).
"""
import os
import struct
import tempfile

import numpy as np
import pytest


def rand_seq(rng, n):
    return rng.choice(np.frombuffer(b"ACGT", np.uint8), int(n)).tobytes()


def cfg_from(o, ka, name, **over):
    c = dict(ka["configs"][name])
    c.pop("_cite", None)
    c.update(over)
    return o.make_config(**c)


def test_xorshift_known_values(oracle_mod):
    # filter.rs:629-635 restated in Python integer arithmetic, independently of the C code.
    def ref(x):
        M = (1 << 64) - 1
        x = (x + 0x9E3779B97F4A7C15) & M
        x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M
        x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M
        return x ^ (x >> 31)

    rng = np.random.default_rng(1)
    for x in [0, 1, 2, (1 << 64) - 1, 0x123456789ABCDEF] + [int(v) for v in rng.integers(0, 2**63, 50)]:
        assert oracle_mod.xorshift_u64(x) == ref(x)
    # SplitMix64 first output from seed 0 is the published value 0xE220A8397B1DCDAF
    assert oracle_mod.xorshift_u64(0) == 0xE220A8397B1DCDAF


def test_canonical_symmetry(oracle_mod, known_answers):
    # filter.rs:748-756
    c = known_answers["canonical_symmetry"]
    a = oracle_mod.canonical_kmer(c["a"].encode(), c["len"], 0)
    b = oracle_mod.canonical_kmer(c["b"].encode(), c["len"], 0)
    assert a == b


def test_canonical_symmetry_random(oracle_mod):
    rng = np.random.default_rng(7)
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    for _ in range(200):
        n = int(rng.integers(1, 33))
        s = rand_seq(rng, n)
        rc = s.translate(comp)[::-1]
        assert oracle_mod.canonical_kmer(s, n, 0) == oracle_mod.canonical_kmer(rc, n, 0)


def test_super_kmers_strand_symmetric(oracle_mod):
    """Each window's block (through its canonical minimizer) must not depend on the strand:
    the minimizer value of window i of s equals that of window n-1-i of revcomp(s)."""
    rng = np.random.default_rng(3)
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    for k, m in [(31, 21), (9, 5), (11, 5), (13, 7), (5, 3), (31, 31), (31, 1)]:
        for _ in range(20):
            s = rand_seq(rng, int(rng.integers(k, 200)))
            rc = s.translate(comp)[::-1]
            nw = len(s) - k + 1

            def per_window(seq):
                st, mins = oracle_mod.super_kmers(seq, k, m)
                out = []
                for i in range(len(st)):
                    end = st[i + 1] if i + 1 < len(st) else nw
                    out += [mins[i]] * (end - st[i])
                return out

            a, b = per_window(s), per_window(rc)
            assert a == b[::-1]


def test_validation_rejections(oracle_mod, known_answers):
    # tests/pipeline_matrix.rs:187-262
    vr = known_answers["validation_rejections"]
    assert oracle_mod.validate(cfg_from(oracle_mod, known_answers, vr["base"])) is None
    for case in vr["cases"]:
        assert oracle_mod.validate(cfg_from(oracle_mod, known_answers, vr["base"], **case)) is not None, case


def test_invalid_windows(oracle_mod, known_answers):
    # api.rs:1057-1072
    t = known_answers["invalid_windows"]
    f = oracle_mod.OracleFilter(cfg_from(oracle_mod, known_answers, t["config"]))
    f.insert_batch([r.encode() for r in t["index_records"]])
    ab = f.estimate_sequence_abundances(t["query"].encode())
    assert len(ab) == t["n_windows"]
    for a, b in t["some_ranges"]:
        assert all(x is not None for x in ab[a:b])
    a, b = t["none_range"]
    assert all(x is None for x in ab[a:b])


def test_summary_windows(oracle_mod, known_answers):
    # api.rs:1095-1111
    t = known_answers["summary"]
    f = oracle_mod.OracleFilter(cfg_from(oracle_mod, known_answers, t["config"]))
    f.insert_batch([r.encode() for r in t["index_records"]])
    ab = f.estimate_sequence_abundances(t["query"].encode())
    assert len(ab) == t["total_windows"]
    valid = [x for x in ab if x is not None]
    assert len(valid) == t["valid_kmers"]
    assert np.mean(valid) > 0 and np.median(valid) > 0


def test_builder_counts(oracle_mod, known_answers):
    # api.rs:1158-1202
    t = known_answers["builder"]
    f = oracle_mod.OracleFilter(cfg_from(oracle_mod, known_answers, t["config"], counter_bits=t["counter_bits"]))
    km, _ = f.insert_batch([t["add_sequence"].encode()])
    assert km == t["add_sequence_kmers"]
    recs = [r.encode() for r in t["fasta_records"]]
    km2, sm2 = f.insert_batch(recs)
    assert km2 == t["add_fasta_inserted_kmers"]
    assert f.inserted_kmers == t["total_inserted_kmers"]
    assert f.inserted_smers > 0
    rep = f.query_report(recs)
    assert rep.records_processed == t["query_records_processed"]
    assert rep.total_windows == t["query_total_windows"]
    assert rep.valid_kmers == t["query_valid_kmers"]
    assert rep.positive_estimates > 0 and rep.estimate_checksum > 0
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "i.scb")
        f.save(p)
        g = oracle_mod.OracleFilter.load(p)
        assert g.inserted_kmers == t["total_inserted_kmers"]
        assert g.query_report(recs) == rep


def test_fastx_spectrum_smoke(oracle_mod, known_answers):
    # fastx.rs:448-466 for all widths
    t = known_answers["fastx_spectrum_smoke"]
    recs = [r.encode() for r in t["records"]]
    for bits in (8, 16, 32):
        f = oracle_mod.OracleFilter(cfg_from(oracle_mod, known_answers, t["config"], counter_bits=bits))
        km, _ = f.insert_batch(recs)
        assert km == t["indexed_kmers"]
        sp = f.spectrum_distinct(recs)
        assert sp["queried_kmers"] == t["queried_kmers"]
        assert sp["rows"] and sp["mismatches"] == 0


def test_pipeline_stream_and_negative(oracle_mod, known_answers):
    # tests/pipeline_matrix.rs:61-117
    t = known_answers["pipeline_stream"]
    recs = [r.encode() for r in t["records"]]
    neg = [r.encode() for r in t["negative_records"]]
    for bits in (8, 16, 32):
        f = oracle_mod.OracleFilter(cfg_from(oracle_mod, known_answers, t["config"], counter_bits=bits))
        km, _ = f.insert_batch(recs)
        assert km == t["indexed_kmers"]
        rep = f.query_report(recs)
        assert rep.valid_kmers == t["queried_kmers"]
        assert rep.positive_estimates == t["positive_estimates"]
        assert rep.estimate_checksum > 0
        nrep = f.query_report(neg)
        assert nrep.valid_kmers == t["queried_kmers"]
        assert rep.estimate_checksum >= nrep.estimate_checksum


def test_saturation(oracle_mod, known_answers):
    # filter.rs:722-746, tests/pipeline_matrix.rs:172-185
    t = known_answers["saturation"]
    for seq in (t["sequence"], t["pipeline_sequence"]):
        s = seq.encode()
        for bits in (8, 16, 32):
            f = oracle_mod.OracleFilter(cfg_from(oracle_mod, known_answers, t["config"], counter_bits=bits))
            for _ in range(t["repeats"]):
                f.insert_packed(s)
            est = f.estimate_packed(s)
            if bits == 8:
                assert all(v == t["u8_all_equal"] for v in est)
            else:
                assert all(v >= t["wider_floor"] for v in est)


def test_backend_matrix(oracle_mod, known_answers):
    # tests/backend_matrix.rs:39-93: positive, length, stream == vector, map count, monotone
    bm = known_answers["backend_matrix"]
    for case in bm["cases"]:
        for bits in (8, 16, 32):
            cfg = oracle_mod.make_config(case["k"], case["m"], case["s"], bm["n_hashes"], bits,
                                         bm["counter_slots_exponent"], bm["block_slots_exponent"], 2, 4)
            s = case["sequence"].encode()
            n = len(s) + 1 - case["k"]
            f1 = oracle_mod.OracleFilter(cfg)
            assert f1.insert_packed(s) > 0
            e1 = f1.estimate_packed(s)
            assert len(e1) == n and all(v > 0 for v in e1)
            f3 = oracle_mod.OracleFilter(cfg)
            for _ in range(3):
                f3.insert_packed(s)
            e3 = f3.estimate_packed(s)
            rep = f3.query_report([s])
            assert (rep.valid_kmers, rep.estimate_checksum) == (len(e3), sum(e3))
            sp = f3.spectrum_distinct([s])
            assert sp["queried_kmers"] == n and sp["mismatches"] == 0
            f4 = oracle_mod.OracleFilter(cfg)
            for _ in range(4):
                f4.insert_packed(s)
            assert all(a >= b for a, b in zip(f4.estimate_packed(s), e1))


def test_save_load_roundtrip_and_format(oracle_mod, known_answers):
    # api.rs:1129-1156 + 1215-1225 + layout of api.rs:388-529
    t = known_answers["index_magic"]
    recs = [b"ACGTACGTACGTACGT", b"TTTTACGTACGTAAAA"]
    with tempfile.TemporaryDirectory() as d:
        for bits in (8, 16, 32):
            cfg = cfg_from(oracle_mod, known_answers, "api_small", counter_bits=bits)
            f = oracle_mod.OracleFilter(cfg)
            f.insert_batch(recs)
            p = os.path.join(d, f"r{bits}.scb")
            f.save(p)
            raw = open(p, "rb").read()
            assert raw[:8].hex() == t["magic_hex"]
            assert struct.unpack_from("<I", raw, 8)[0] == t["version"]
            assert len(raw) == t["header_bytes"] + (1 << cfg.counter_slots_exponent) * bits // 8
            g = oracle_mod.OracleFilter.load(p)
            assert g.counter_histogram() == f.counter_histogram()
            q = b"ACGTACGTNNACGTACGT"
            assert g.estimate_sequence_abundances(q) == f.estimate_sequence_abundances(q)
            assert g.table_bytes() == f.table_bytes()
        bad = os.path.join(d, "bad.scb")
        open(bad, "wb").write(b"not an index")
        with pytest.raises(ValueError, match="magic"):
            oracle_mod.OracleFilter.load(bad)
        # trailing byte rejected (api.rs:599-608)
        raw = open(os.path.join(d, "r8.scb"), "rb").read()
        trail = os.path.join(d, "trail.scb")
        open(trail, "wb").write(raw + b"\0")
        with pytest.raises(ValueError, match="trailing"):
            oracle_mod.OracleFilter.load(trail)


def test_inserted_smers_formula(oracle_mod):
    """inserted s-mers = windows + (k-s) * super-k-mers for each run (filter.rs:224-233)."""
    rng = np.random.default_rng(11)
    cfg = oracle_mod.make_config(31, 21, 25, 4, 16, 20, 9)
    f = oracle_mod.OracleFilter(cfg)
    for _ in range(20):
        s = rand_seq(rng, int(rng.integers(31, 400)))
        st, _ = oracle_mod.super_kmers(s, 31, 21)
        assert f.insert_packed(s) == (len(s) - 30) + 6 * len(st)


def test_port_matches_oracle(oracle_mod):
    """The multi-threaded port (timed CPU baseline) gives the oracle's table and report."""
    from scbf_b200 import workloads

    data, offsets = workloads.short_reads(genome_len=20000, n_reads=800, read_len=150, seed=5,
                                          sub_rate=0.01, n_rate=0.01)
    for bits in (8, 16, 32):
        cfg = oracle_mod.make_config(31, 21, 25, 4, bits, 18, 9)
        a = oracle_mod.OracleFilter(cfg)
        a.insert_batch_arrays(data, offsets)
        rep_a = a.query_report_arrays(data, offsets)
        b = oracle_mod.OracleFilter(cfg)
        res = b.port_build_and_stream_query(data, offsets, threads=4, queue=16)
        assert res["inserted_kmers"] == a.inserted_kmers
        assert res["inserted_smers"] == a.inserted_smers
        assert np.array_equal(a.table(), b.table())
        assert res["report"].valid_kmers == rep_a.valid_kmers
        assert res["report"].positive_estimates == rep_a.positive_estimates
        assert res["report"].estimate_checksum == rep_a.estimate_checksum
