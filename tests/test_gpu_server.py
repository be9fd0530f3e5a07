"""Serving loop: each request's abundances are identical alone, in a concurrent mix, and when
the device-memory budget forces small batches and split requests -- and equal to the
per-call query path."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def index_and_requests():
    import scbf_b200 as scb
    from scbf_b200 import workloads

    genome = workloads.random_genome(400_000, seed=31)
    data, offsets = workloads.short_reads(n_reads=30_000, read_len=150, seed=32, sub_rate=0.01, n_rate=0.005,
                                          genome=genome)
    cfg = scb.SuperCountingBloomConfig(counter_slots_exponent=22, counter_bits=scb.CounterBits.Bits16)
    b = scb.SuperCountingBloomBuilder(cfg)
    b.add_sequences(data, offsets)
    idx = b.into_index()
    rng = np.random.default_rng(33)
    requests = []
    for i in range(40):
        n = int(np.exp(rng.uniform(0, np.log(300))))
        d, o = workloads.random_sequences(n, 20, 20_000, seed=100 + i, genome=genome)
        if i % 7 == 3:  # runs of N inside some requests
            d = d.copy()
            d[rng.integers(0, d.size, max(1, d.size // 200))] = ord("N")
        requests.append((d, o))
    requests.append(scb.pack_sequences([b"", b"ACGT", b"N" * 50]))
    expected = [idx.estimate_batch(d, o) for d, o in requests]
    return idx, requests, expected


def _check_all(results, expected):
    for (out, valid), (eo, ev) in zip(results, expected):
        assert np.array_equal(valid, ev)
        assert np.array_equal(out, eo)


def test_alone_equals_per_call_query(index_and_requests):
    import scbf_b200 as scb

    idx, requests, expected = index_and_requests
    srv = scb.SuperCountingBloomServer(idx, max_batch_bytes=8 << 20, max_inflight=3)
    results = []
    for d, o in requests:
        t = srv.submit(d, o)
        out, valid, st = srv.wait(t)
        assert st.total_ms >= st.service_ms >= 0
        results.append((out, valid))
    _check_all(results, expected)
    summ = srv.summary()
    assert summ["requests"] == len(requests) and summ["p99_ms"] >= summ["p50_ms"] > 0
    srv.close()


def test_concurrent_mix_equals_alone(index_and_requests):
    import scbf_b200 as scb

    idx, requests, expected = index_and_requests
    srv = scb.SuperCountingBloomServer(idx, max_batch_bytes=4 << 20, max_inflight=4)
    results = [None] * len(requests)
    order = np.random.default_rng(5).permutation(len(requests))

    def client(ids):
        tickets = [(i, srv.submit(*requests[i])) for i in ids]  # submit all, then wait
        for i, t in tickets:
            out, valid, _ = srv.wait(t)
            results[i] = (out, valid)

    threads = [threading.Thread(target=client, args=(order[j::4].tolist(),)) for j in range(4)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    _check_all(results, expected)
    assert srv.summary()["batches"] < len(requests)  # requests shared batches
    srv.close()


def test_memory_budget_admits_one_small_batch_at_a_time(index_and_requests):
    import scbf_b200 as scb

    idx, requests, expected = index_and_requests
    # room for one slot of 256 KiB batches: big requests are split into many pieces
    srv = scb.SuperCountingBloomServer(idx, memory_budget_bytes=4 << 20, max_batch_bytes=256 << 10,
                                       max_inflight=8)
    assert srv.summary()["slots"] == 1
    tickets = [srv.submit(d, o) for d, o in requests]
    results = [srv.wait(t)[:2] for t in tickets]
    _check_all(results, expected)
    srv.close()
    with pytest.raises(scb.InvalidConfig, match="budget"):
        scb.SuperCountingBloomServer(idx, memory_budget_bytes=1 << 20, max_batch_bytes=64 << 20)


def test_whole_stream_spectrum_equals_batch_spectrum(index_and_requests, oracle_mod):
    """A server with spectrum_keys adds every answered window's canonical k-mer to one device set;
    at the end of the stream its spectrum equals the distinct-k-mer spectrum of all the requests'
    sequences at once (src/fastx.rs:255-308, 392-410), which the oracle checks too, and every
    request's abundances equal the per-call query's."""
    import scbf_b200 as scb

    idx, requests, expected = index_and_requests
    srv = scb.SuperCountingBloomServer(idx, max_batch_bytes=2 << 20, max_inflight=4, spectrum_keys=4_000_000)
    tickets = [srv.submit(d, o) for d, o in requests + requests[:5]]  # repeats add no distinct k-mer
    # the same kernel answers the windows and feeds the set: the abundances stay the per-call query's
    _check_all([srv.wait(t)[:2] for t in tickets], expected + expected[:5])
    got = srv.spectrum()
    seqs = [bytes(d[int(o[i]):int(o[i + 1])]) for d, o in requests for i in range(len(o) - 1)]
    data, offsets = scb.pack_sequences(seqs)
    ref = idx.spectrum_distinct(data, offsets)
    assert got["rows"] == ref["rows"] and got["distinct_keys"] == ref["distinct_keys"]
    # every answered valid window is queried once, the five repeated requests' windows again
    assert got["queried_kmers"] == ref["queried_kmers"] + sum(int(expected[i][1].sum()) for i in range(5))
    # the oracle's spectrum of the same reads over the same training set
    from scbf_b200 import workloads

    genome = workloads.random_genome(400_000, seed=31)
    tr, to = workloads.short_reads(n_reads=30_000, read_len=150, seed=32, sub_rate=0.01, n_rate=0.005, genome=genome)
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 22, 9))
    o.insert_batch_arrays(tr, to)
    osp = o.spectrum_distinct_arrays(data, offsets)
    assert osp["mismatches"] == 0 and got["rows"] == osp["rows"]
    srv.reset_stats()
    empty = srv.spectrum()
    assert empty["rows"] == [] and empty["distinct_keys"] == 0
    srv.close()


@pytest.mark.parametrize("bits", [8, 32])
def test_served_estimates_cross_at_the_counters_width(bits):
    """The server copies each window's estimate to the host at the counters' width (2 bytes for 8-
    and 16-bit counters, 4 for 32-bit ones) and widens it to u64 there: results equal the per-call
    query for 8-bit counters (saturated at 255) and 32-bit ones, in batches large enough that the
    copy-out is split over several threads."""
    import scbf_b200 as scb
    from scbf_b200 import workloads

    genome = workloads.random_genome(200_000, seed=41)
    data, offsets = workloads.short_reads(n_reads=40_000, read_len=150, seed=42, sub_rate=0.01, genome=genome)
    cfg = scb.SuperCountingBloomConfig(counter_slots_exponent=18, counter_bits=scb.CounterBits(bits))
    b = scb.SuperCountingBloomBuilder(cfg)
    for _ in range(3 if bits == 8 else 1):  # repeats push u8 counters to saturation
        b.add_sequences(data, offsets)
    idx = b.into_index()
    requests = [workloads.random_sequences(60, 5_000, 30_000, seed=300 + i, genome=genome) for i in range(6)]
    expected = [idx.estimate_batch(d, o) for d, o in requests]
    if bits == 8:
        assert any(int(eo.max()) == 255 for eo, _ in expected)
    srv = scb.SuperCountingBloomServer(idx, max_batch_bytes=4 << 20, max_inflight=2)
    tickets = [srv.submit(d, o) for d, o in requests]
    _check_all([srv.wait(t)[:2] for t in tickets], expected)
    srv.close()
