"""Filter-only spectrum (src/api.rs:337-385, 933-1033): the k-mer spectrum estimated from the
counter histogram alone, by a compound Poisson deconvolution in host f64 arithmetic.

The vectorised host form in scbf_b200.api must give the oracle's step-for-step restatement bit
for bit; the restatement must meet the reference's known answers and the deconvolution's
defining property (counters that are sums of Poisson hits give back the k-mers' abundances); on
the GPU, the index methods over the device's counter histogram must give the oracle's rows.
"""
import math

import numpy as np
import pytest

from scbf_b200 import api


def _cfg(oracle_mod, known_answers, name):
    c = dict(known_answers["configs"][name])
    c.pop("_cite", None)
    return oracle_mod.make_config(**c)


def _histograms(seed=7):
    """Counter histograms of several shapes: decaying (as real tables), sparse, without a zero
    row (no empty counters: the scaled fallback), with values past the maximum, and empty."""
    rng = np.random.default_rng(seed)
    out = [[], [(0, 0), (3, 0)], [(0, 5)], [(2, 7), (5, 1)]]
    for _ in range(24):
        top = int(rng.integers(1, 320))
        values = np.unique(rng.integers(0, top + 1, int(rng.integers(1, 60))))
        lam = float(rng.uniform(0.05, 3.0))
        counts = [int(1e9 * math.exp(-lam * v / 4.0) * float(rng.uniform(0.5, 1.5))) for v in values]
        hist = [(int(v), int(c)) for v, c in zip(values, counts)]
        if rng.random() < 0.8 and (not hist or hist[0][0] != 0):
            hist.insert(0, (0, int(rng.integers(1, 10**10))))
        out.append(hist)
    return out


def _bits(x):
    return np.asarray(x, dtype=np.float64).view(np.uint64)


def test_vectorised_form_matches_restatement_bit_for_bit(oracle_mod):
    rng = np.random.default_rng(3)
    for i, hist in enumerate(_histograms()):
        for max_abundance in (0, 1, 8, int(rng.integers(2, 300))):
            h = int(rng.integers(1, 7))
            dec = api._deconvolved_counts(hist, h, max_abundance)
            ref = oracle_mod.filter_only_deconvolved_counts(hist, h, max_abundance)
            assert len(dec) == len(ref), (i, max_abundance)
            assert np.array_equal(_bits(dec), _bits(ref)), (i, max_abundance, h)
            hint = int(rng.integers(0, 10**9))
            assert api._filter_only_rows(hist, h, max_abundance, hint) == oracle_mod.filter_only_spectrum(
                hist, h, max_abundance, hint), (i, max_abundance, h)
            s = api._sum_f64(dec)
            assert max(api._round_u64(s), 1) == oracle_mod.filter_only_count_hint(hist, h, max_abundance)


def test_rust_rounding():
    # f64::round: halves away from zero; `as u64` clamps negatives and NaN to 0
    cases = {0.0: 0, 0.49999999999999994: 0, 0.5: 1, 1.5: 2, 2.5: 3, 2.4999999999999996: 2, -0.7: 0,
             float("nan"): 0, 1e30: (1 << 64) - 1}
    for x, want in cases.items():
        assert api._round_u64(x) == want, x


def _compound_poisson(rates, n_values):
    """Probabilities of a counter's value when k-mers of abundance a add Poisson(rates[a]) hits
    of a each: the convolution of one Poisson law per abundance, on multiples of a."""
    p = np.zeros(n_values)
    p[0] = 1.0
    for a, lam in rates.items():
        q = np.zeros(n_values)
        for j in range(0, n_values, a):
            n = j // a
            q[j] = math.exp(-lam) * lam ** n / math.factorial(n)
        p = np.convolve(p, q)[:n_values]
    return p


@pytest.mark.parametrize("rates", [{1: 0.8}, {1: 0.5, 3: 0.2}, {2: 0.3, 5: 0.05}])
def test_deconvolution_recovers_abundances(rates):
    total, h = 10**15, 4
    p = _compound_poisson(rates, 60)
    hist = [(v, int(round(total * float(x)))) for v, x in enumerate(p) if round(total * float(x)) > 0]
    n_counters = sum(c for _, c in hist)
    dec = api._deconvolved_counts(hist, h, 12)
    for a in range(1, 13):
        want = n_counters * rates.get(a, 0.0) / h
        assert abs(dec[a - 1] - want) <= 1e-6 * n_counters * max(rates.values()) / h, (a, dec[a - 1], want)


def test_reference_known_answers_on_oracle_table(oracle_mod, known_answers):
    """src/api.rs:1113-1124 on a table the oracle built from the same record."""
    t = known_answers["filter_only_spectrum"]
    cfg = _cfg(oracle_mod, known_answers, t["config"])
    f = oracle_mod.OracleFilter(cfg)
    f.insert_batch([t["index_fasta"].split("\n")[1].encode()])
    hist = f.counter_histogram()
    h = known_answers["configs"][t["config"]]["n_hashes"]
    assert (oracle_mod.filter_only_count_hint(hist, h) > 0) == t["count_hint_positive"]
    rows = oracle_mod.filter_only_spectrum(hist, h, t["max_abundance"], t["kmer_count_hint"])
    assert rows[0][0] == t["first_row_abundance"] and rows[-1][0] == t["last_row_abundance"]
    assert api._filter_only_rows(hist, h, t["max_abundance"], t["kmer_count_hint"]) == rows
    assert api._FILTER_ONLY_METHOD == t["method"]


@pytest.mark.gpu
def test_index_filter_only_spectrum_matches_oracle(oracle_mod, known_answers):
    """The index methods over the GPU's counter histogram give the oracle's rows and hint, for
    the reference test's record and for 2000 random reads."""
    import scbf_b200 as scb

    t = known_answers["filter_only_spectrum"]
    c = dict(known_answers["configs"][t["config"]])
    c.pop("_cite")
    rng = np.random.default_rng(11)
    genome = rng.choice(np.frombuffer(b"ACGT", np.uint8), 20_000).tobytes()
    reads = [genome[s:s + 150] for s in rng.integers(0, len(genome) - 150, 2000)]
    for seqs in ([t["index_fasta"].split("\n")[1].encode()], reads):
        cfg = scb.SuperCountingBloomConfig(k=c["k"], m=c["m"], s=c["s"], n_hashes=c["n_hashes"],
                                           counter_bits=scb.CounterBits(c["counter_bits"]),
                                           counter_slots_exponent=c["counter_slots_exponent"],
                                           block_slots_exponent=c["block_slots_exponent"], threads=c["threads"],
                                           queue=c["queue"])
        b = scb.SuperCountingBloomBuilder(cfg)
        data, offsets = scb.pack_sequences(seqs)
        b.add_sequences(data, offsets)
        idx = b.into_index()
        o = oracle_mod.OracleFilter(_cfg(oracle_mod, known_answers, t["config"]))
        o.insert_batch_arrays(data, offsets)
        hist = o.counter_histogram()
        assert idx.counter_histogram() == hist
        est = idx.estimate_filter_only_spectrum(t["max_abundance"], t["kmer_count_hint"])
        assert est.method == t["method"] and est.kmer_count_hint == t["kmer_count_hint"]
        assert est.rows == oracle_mod.filter_only_spectrum(hist, c["n_hashes"], t["max_abundance"],
                                                          t["kmer_count_hint"])
        assert idx.filter_only_count_hint() == oracle_mod.filter_only_count_hint(hist, c["n_hashes"])
