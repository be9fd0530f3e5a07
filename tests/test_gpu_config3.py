"""Configuration 3: reads of a genome with repeat families, whose high-copy k-mers drive counters
into saturation (u8 at 255), across counter widths and geometries.

A sweep that covers every value of counter_bits {8, 16, 32}, block_slots_exponent 7..11,
n_hashes 2..6 and s {21, 25, 31} runs on a scaled-down repeat genome against the oracle (counters,
counts and report bit-exact; slot exponents 20..24 keep the oracle's tables small).  On the
full-size configuration-3 workload (50 Mbp genome, 30x) with 2^28 u8 and 2^30 u16 slots, the
plain, fused and grouped kernels, three independent implementations, must give byte-identical
tables and reports."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (counter_bits, counter_slots_exponent, block_slots_exponent, n_hashes, s); k = 31, m = 21
SWEEP = [
    (8, 20, 7, 2, 21),
    (8, 22, 9, 4, 25),
    (8, 24, 11, 6, 31),
    (16, 20, 8, 3, 25),
    (16, 22, 10, 5, 31),
    (16, 24, 7, 6, 21),
    (32, 20, 11, 4, 21),
    (32, 22, 8, 2, 31),
    (32, 24, 9, 5, 25),
]


@pytest.fixture(scope="module")
def repeat_reads():
    from scbf_b200 import workloads

    # scaled down (200 kbp, 30x) with fewer, higher-copy families so that u8 counters saturate
    g = workloads.repeat_genome(200_000, seed=3, repeat_frac=0.5, n_families=4, fam_min=1_000, fam_max=3_000,
                                copy_lo=10.0, copy_hi=1e3, divergence=0.02)
    return workloads.short_reads(coverage=30, read_len=150, seed=3, sub_rate=0.01, genome=g)


@pytest.mark.parametrize("geom", SWEEP, ids=[f"u{b}-e{se}-b{be}-h{h}-s{s}" for b, se, be, h, s in SWEEP])
def test_repeat_genome_sweep_matches_oracle(oracle_mod, repeat_reads, geom):
    import scbf_b200 as scb

    bits, se, be, h, s = geom
    data, offsets = repeat_reads
    cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=s, n_hashes=h, counter_bits=scb.CounterBits(bits),
                                       counter_slots_exponent=se, block_slots_exponent=be, threads=3, queue=17)
    b = scb.SuperCountingBloomBuilder(cfg)
    rep = b.add_sequences(data, offsets)
    idx = b.into_index()
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, s, h, bits, se, be, 3, 17))
    okm, osm = o.insert_batch_arrays(data, offsets)
    assert (rep.inserted_kmers, rep.inserted_smers) == (okm, osm)
    table = idx.table()
    assert np.array_equal(table, o.table())
    if bits == 8:
        assert table.max() == 255  # the repeats saturate u8 counters
    q = idx.query_report(data, offsets)
    oq = o.query_report_arrays(data, offsets)
    assert (q.valid_kmers, q.positive_estimates, q.estimate_checksum) == (
        oq.valid_kmers, oq.positive_estimates, oq.estimate_checksum)


@pytest.mark.parametrize("bits,slot_exp", [(8, 28), (16, 30)])
def test_full_config3_strategies_agree(bits, slot_exp):
    import scbf_b200 as scb
    from scbf_b200 import api, workloads

    data, offsets = workloads.config3(seed=1)
    assert int(offsets[-1]) > 1_000_000_000  # the full 1.5 Gbp of reads
    cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits(bits),
                                       counter_slots_exponent=slot_exp, block_slots_exponent=9, threads=3, queue=17)
    tables, reports = {}, {}
    for strategy in ("plain", "fused", "grouped"):
        b = scb.SuperCountingBloomBuilder(cfg)
        api.set_strategy(b, strategy, strategy)
        rep = b.add_sequences(data, offsets)
        idx = b.into_index()
        api.set_strategy(idx, strategy, strategy)
        q = idx.query_report(data, offsets)
        tables[strategy] = idx.table()
        reports[strategy] = (rep.inserted_kmers, rep.inserted_smers, q.valid_kmers, q.positive_estimates,
                             q.estimate_checksum)
        del b, idx
    assert reports["plain"] == reports["fused"] == reports["grouped"]
    assert np.array_equal(tables["plain"], tables["fused"])
    assert np.array_equal(tables["plain"], tables["grouped"])
    if bits == 8:
        assert tables["grouped"].max() == 255
