"""The command-line tools (src/bin/build-index.rs, query-index.rs, filter_spectrum.rs,
sampled_spectrum.rs): the reference's arguments and error exits, the sampled spectrum's reservoir
and scaling against the oracle's sequential restatement on the host, and on the GPU the same index
bytes, CSV rows and spectrum as the library calls they wrap."""
import csv
import io
import os
import sys

import numpy as np
import pytest

from scbf_b200 import cli

GEOM = ["-k", "31", "-m", "21", "-s", "25", "-H", "4", "--counter-bits", "16", "--counter-slots-exponent", "20",
        "--block-slots-exponent", "9", "-t", "3", "--queue", "17"]


def _fasta(path, n=300, seed=5):
    rng = np.random.default_rng(seed)
    genome = rng.choice(np.frombuffer(b"ACGT", np.uint8), 30_000).tobytes()
    with open(path, "w") as fh:
        for i, s in enumerate(rng.integers(0, len(genome) - 150, n)):
            read = bytearray(genome[s:s + 150])
            if i % 7 == 0:
                read[40:43] = b"NNN"
            fh.write(f">read_{i} sample,{i}\n{read.decode()}\n")
    return path


def test_invalid_config_exits_with_error(tmp_path, capsys):
    fa = _fasta(tmp_path / "r.fa", n=3)
    assert cli.main(["build-index", str(fa), str(tmp_path / "x.scb"), "-k", "32"]) == 1
    assert "error: invalid config" in capsys.readouterr().err


def test_missing_index_exits_with_error(tmp_path, capsys):
    fa = _fasta(tmp_path / "r.fa", n=3)
    assert cli.main(["query-index", str(tmp_path / "none.scb"), str(fa)]) == 1
    assert capsys.readouterr().err.startswith("error: ")


def test_counter_bits_must_be_a_width():
    with pytest.raises(SystemExit) as e:
        cli.main(["build-index", "a.fa", "b.scb", "--counter-bits", "12"])
    assert e.value.code == 2


def _rows(text):
    return list(csv.reader(io.StringIO(text)))


@pytest.mark.gpu
def test_tools_match_the_library(tmp_path, capsys, oracle_mod):
    import scbf_b200 as scb

    fa = str(_fasta(tmp_path / "reads.fa"))
    out = str(tmp_path / "cli.scb")
    assert cli.main(["build-index", fa, out] + GEOM) == 0
    cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits(16),
                                       counter_slots_exponent=20, block_slots_exponent=9, threads=3, queue=17)
    b = scb.SuperCountingBloomBuilder(cfg)
    b.add_fasta(fa)
    idx = b.into_index()
    ref = str(tmp_path / "api.scb")
    idx.save(ref)
    assert open(out, "rb").read() == open(ref, "rb").read()
    capsys.readouterr()

    csv_path = str(tmp_path / "report.csv")
    assert cli.main(["query-index", out, fa, "--mode", "report", "-o", csv_path]) == 0
    rows = _rows(open(csv_path).read())
    r = idx.query_fasta(fa)
    assert rows[0] == ["records_processed", "total_windows", "valid_kmers", "positive_estimates", "estimate_checksum"]
    assert [int(x) for x in rows[1]] == [r.records_processed, r.total_windows, r.valid_kmers, r.positive_estimates,
                                         r.estimate_checksum]
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 20, 9, 3, 17))
    seqs = []
    scb.for_each_fastx_record(fa, lambda name, s: seqs.append(s))
    data, offsets = scb.pack_sequences(seqs)
    o.insert_batch_arrays(data, offsets)
    oq = o.query_report_arrays(data, offsets)
    assert (r.valid_kmers, r.positive_estimates, r.estimate_checksum) == (oq.valid_kmers, oq.positive_estimates,
                                                                         oq.estimate_checksum)

    assert cli.main(["query-index", out, fa, "--mode", "fast"]) == 0
    rows = _rows(capsys.readouterr().out)
    assert rows[0] == ["sequence", "length", "total_windows", "valid_kmers", "mean_abundance", "median_abundance"]
    want = []
    scb.for_each_fastx_record(fa, lambda name, s: want.append(idx.summarize_sequence(name, s)))
    assert len(rows) == len(want) + 1
    for row, s in zip(rows[1:], want):
        assert row[:4] == [s.name, str(s.sequence_len), str(s.total_windows), str(s.valid_kmers)]
        assert row[4:] == [f"{s.mean_abundance:.6f}" if s.mean_abundance is not None else "",
                           f"{s.median_abundance:.6f}" if s.median_abundance is not None else ""]

    assert cli.main(["query-index", out, fa, "--mode", "slow"]) == 0
    rows = _rows(capsys.readouterr().out)
    want = []
    scb.for_each_fastx_record(fa, lambda name, s: want.extend(
        [name, str(i), "" if v is None else str(v)] for i, v in enumerate(idx.estimate_sequence_abundances(s))))
    assert rows[1:] == want

    hist_path = str(tmp_path / "hist.csv")
    assert cli.main(["filter-spectrum", fa, "--counter-histogram", hist_path, "--max-abundance", "40"] + GEOM) == 0
    rows = _rows(capsys.readouterr().out)
    hist = idx.counter_histogram()
    assert [tuple(int(x) for x in r) for r in _rows(open(hist_path).read())[1:]] == hist
    hint = idx.filter_only_count_hint_from_counter_histogram(hist, 40)
    est = idx.estimate_filter_only_spectrum_from_counter_histogram(hist, 40, hint)
    assert rows[0] == ["estimated_count", "estimated_kmers", "method", "kmer_count_hint"]
    assert rows[1:] == [[str(a), str(n), est.method, str(hint)] for a, n in est.rows]


def _random_batch(rng, n_seqs, k):
    seqs = []
    for _ in range(n_seqs):
        L = int(rng.integers(0, 3 * k))
        s = bytearray(rng.choice(np.frombuffer(b"ACGTacgtNn", np.uint8), L, p=[.2, .2, .2, .2, .04, .04, .04, .04,
                                                                               .02, .02]).tobytes())
        seqs.append(bytes(s))
    return seqs


@pytest.mark.parametrize("k,capacity,seed,chunk", [(5, 1, 1, 64), (7, 4, 0, 5), (9, 37, (1 << 64) - 1, 1 << 24),
                                                   (11, 10**6, 12345, 13), (5, 200, 7, 1000)])
def test_reservoir_sample_matches_sequential_sampler(oracle_mod, k, capacity, seed, chunk):
    """The vectorised reservoir (counter-based SplitMix64 calls, chunked windows) keeps exactly the
    k-mers of the sequential sampler of src/bin/sampled_spectrum.rs, in the same slots."""
    import scbf_b200 as scb

    rng = np.random.default_rng(k * 1000 + capacity)
    seqs = _random_batch(rng, 400, k)
    data, offsets = scb.pack_sequences(seqs)
    kmers, seen = cli.sample_kmers(data, offsets, k, capacity, seed, chunk=chunk)
    want, want_seen = oracle_mod.reservoir_sample_kmers(seqs, k, capacity, seed)
    assert seen == want_seen
    assert [bytes(r) for r in kmers] == want


def test_sampled_rows_match_literal_histogram(oracle_mod):
    """The batch query of the sample and the scaling of sampled_spectrum.rs:225-261, with the
    oracle as the estimator, against per-k-mer queries and Rust rounding."""
    import scbf_b200 as scb

    rng = np.random.default_rng(4)
    genome = rng.choice(np.frombuffer(b"ACGT", np.uint8), 3000).tobytes()
    seqs = [genome[s:s + 60] for s in rng.integers(0, 2940, 300)]
    data, offsets = scb.pack_sequences(seqs)
    o = oracle_mod.OracleFilter(oracle_mod.make_config(11, 7, 9, 3, 8, 14, 6, 1, 4))
    o.insert_batch_arrays(data, offsets)
    kmers, seen = cli.sample_kmers(data, offsets, 11, 500, 3)
    rows, invalid = cli.sampled_rows(kmers, seen, o.query_batch_arrays)
    hist = {}
    for km in kmers:
        v = o.estimate_sequence_abundances(bytes(km))[0]
        hist[v] = hist.get(v, 0) + 1
    scale = float(seen) / float(len(kmers))
    want = []
    for a in sorted(hist):
        lsw = oracle_mod.rust_round_u64(float(hist[a]) * scale)
        want.append((a, hist[a], lsw, 0 if a == 0 else oracle_mod.rust_round_u64(float(lsw) / float(a))))
    assert invalid == 0 and rows == want


def test_sampled_spectrum_rejects_empty_sample(tmp_path, capsys):
    fa = _fasta(tmp_path / "r.fa", n=3)
    assert cli.main(["sampled-spectrum", str(fa), "--sample-size", "0"]) == 1
    assert "error: invalid config: sample_size must be positive" in capsys.readouterr().err
    with pytest.raises(SystemExit):
        cli.main(["sampled-spectrum", str(fa), "--seed", "-1"])
