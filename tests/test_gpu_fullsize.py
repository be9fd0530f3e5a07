"""Bit-exact parity at the full sizes of the benchmark configurations.

- Configuration 1 exactly as specified (1 Mbp genome, 30x of 150 bp reads = 200 000 reads,
  k=31 m=21 s=25 h=4, u16, 2^24 slots, 2^9 slots per block): the whole counter array, the .scb
  bytes, every per-window abundance, the query report, the distinct-k-mer spectrum and the
  counter histogram against the single-threaded oracle.
- Configuration 2 at full size (100 Mbp genome, 13.3 M reads, 2 Gbp, 2^30 u16 slots): the
  inserted k-mer / s-mer counts, the stream-query report and the whole 2 GiB table of the
  build + stream-query entry points (host and device) against the multi-threaded CPU port
  (its own rolling arithmetic, itself checked against the oracle in tests/test_oracle.py).
- The largest tables: 2^31 u16 slots (4 GiB, configuration 4's geometry) and 2^32 u8 / u32 slots
  (4 / 16 GiB, the top of configuration 3's sweep), where byte offsets pass 2^32, with a few
  thousand reads, for every kernel strategy, against the oracle; the tables are compared in
  256 MiB pieces so the host never holds two copies.

Insert follows src/filter.rs:199-237, query src/filter.rs:462-508 and 562-571.
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GIB = 1 << 30


@pytest.fixture(scope="module")
def scb():
    import scbf_b200

    return scbf_b200


def _cfg(scb, bits, slot_exp, block_exp=9, threads=1, queue=4096):
    return scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits(bits),
                                        counter_slots_exponent=slot_exp, block_slots_exponent=block_exp,
                                        threads=threads, queue=queue)


def _report_tuple(r):
    return (r.records_processed, r.total_windows, r.valid_kmers, r.positive_estimates, r.estimate_checksum)


def _assert_table_equal(L, h, ref: np.ndarray, piece=256 << 20):
    """Device table (downloaded piece by piece) equals the reference bytes."""
    from scbf_b200 import _lib

    assert int(L.scb_table_bytes(h)) == ref.size
    buf = np.empty(min(piece, ref.size), np.uint8)
    for off in range(0, ref.size, piece):
        n = min(piece, ref.size - off)
        assert L.scb_table_download_range(h, off, buf.ctypes.data, n) == 0, _lib.last_error()
        if not np.array_equal(buf[:n], ref[off:off + n]):
            bad = (np.flatnonzero(buf[:n] != ref[off:off + n])[:8] + off).tolist()
            raise AssertionError(f"counter bytes differ from the reference at {bad}")


def _host_bytes_available() -> int:
    try:
        import psutil

        return int(psutil.virtual_memory().available)
    except ImportError:
        return 1 << 62


def test_config1_exact_against_oracle(scb, oracle_mod):
    from scbf_b200 import _lib, workloads

    data, offsets = workloads.config1()
    assert len(offsets) - 1 == 200_000 and int(offsets[-1]) == 30_000_000
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 24, 9, 1, 4096))
    okm, osm = o.insert_batch_arrays(data, offsets)
    assert okm == 24_000_000  # 200 000 reads x 120 windows, no N

    b = scb.SuperCountingBloomBuilder(_cfg(scb, 16, 24))
    rep = b.add_sequences(data, offsets)
    assert (rep.inserted_kmers, rep.inserted_smers) == (okm, osm)
    idx = b.into_index()
    L = _lib.load()
    _assert_table_equal(L, idx._ctx.h, o.table_view())

    with tempfile.TemporaryDirectory() as d:
        og, gg = os.path.join(d, "o.scb"), os.path.join(d, "g.scb")
        o.save(og)
        idx.save(gg)
        assert os.path.getsize(gg) == 139 + (2 << 24)
        assert open(og, "rb").read() == open(gg, "rb").read()

    out, valid = idx.estimate_batch(data, offsets)
    oout, ovalid = o.query_batch_arrays(data, offsets)
    assert out.size == 24_000_000
    assert np.array_equal(valid, ovalid) and np.array_equal(out, oout)

    q = idx.query_report(data, offsets)
    oq = o.query_report_arrays(data, offsets)
    assert _report_tuple(q) == _report_tuple(oq)
    assert oq.total_windows == oq.valid_kmers == 24_000_000

    sp = idx.spectrum_distinct(data, offsets)
    osp = o.spectrum_distinct_arrays(data, offsets)
    assert osp["mismatches"] == 0
    assert sp["rows"] == osp["rows"]
    assert (sp["distinct_keys"], sp["queried_kmers"]) == (osp["distinct_keys"], osp["queried_kmers"])
    assert idx.counter_histogram() == o.counter_histogram()

    # the benchmark's entry point (build, freeze, stream-query the same reads) on the same reads
    fresh = scb.SuperCountingBloomBuilder(_cfg(scb, 16, 24))
    km, sm = C.c_uint64(0), C.c_uint64(0)
    r = _lib.ScbReport()
    assert L.scb_build_and_stream_query(fresh._ctx.h, data.ctypes.data, offsets.ctypes.data, len(offsets) - 1,
                                        C.byref(km), C.byref(sm), C.byref(r)) == 0, _lib.last_error()
    assert (km.value, sm.value) == (okm, osm)
    assert _report_tuple(r) == _report_tuple(oq)
    _assert_table_equal(L, fresh._ctx.h, o.table_view())


def test_config2_full_size_against_cpu_port(scb, oracle_mod):
    import torch

    from scbf_b200 import _lib, api, workloads

    if _host_bytes_available() < 12 * GIB:
        pytest.skip("needs about 8 GiB of free host memory")
    data, offsets = workloads.config2()
    n = len(offsets) - 1
    assert n == 13_333_333
    threads = os.cpu_count() or 1
    port = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 30, 9, threads, 4096))
    pres = port.port_build_and_stream_query(data, offsets, threads=threads, queue=4096)
    ref = port.table_view()
    assert pres["inserted_kmers"] > 1_400_000_000
    # the port reports the stream query's own units (src/fastx.rs:310-369): chunks (maximal ACGT
    # runs of at least k bases) and their windows; the C ABI reports QueryFastaReport's: records
    # and all their windows, of which valid_kmers are queried
    chunks, chunk_windows = api._chunk_stats(data, offsets, 31)
    pr = pres["report"]
    assert (pr.records_processed, pr.total_windows, pr.valid_kmers) == (chunks, chunk_windows, chunk_windows)
    lens = np.diff(offsets.astype(np.int64))
    expect = (n, int(np.where(lens >= 31, lens - 30, 0).sum()), pr.valid_kmers, pr.positive_estimates,
              pr.estimate_checksum)

    L = _lib.load()
    b = scb.SuperCountingBloomBuilder(_cfg(scb, 16, 30))
    h = b._ctx.h
    km, sm = C.c_uint64(0), C.c_uint64(0)
    r = _lib.ScbReport()
    # host entry point: pieces copied from host memory while earlier pieces are inserted
    assert L.scb_build_and_stream_query(h, data.ctypes.data, offsets.ctypes.data, n, C.byref(km), C.byref(sm),
                                        C.byref(r)) == 0, _lib.last_error()
    assert (km.value, sm.value) == (pres["inserted_kmers"], pres["inserted_smers"])
    assert _report_tuple(r) == expect
    _assert_table_equal(L, h, ref)

    # device entry point on resident reads (the benchmark's timed call), after a reset
    d_data = torch.from_numpy(data).cuda()
    d_off = torch.from_numpy(offsets.view(np.int64)).cuda()
    assert L.scb_reset(h) == 0
    assert L.scb_build_and_stream_query_device(h, d_data.data_ptr(), d_off.data_ptr(), n, int(offsets[-1]), None,
                                               C.byref(km), C.byref(sm), C.byref(r)) == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert (km.value, sm.value) == (pres["inserted_kmers"], pres["inserted_smers"])
    assert _report_tuple(r) == expect
    _assert_table_equal(L, h, ref)


def _big_table_reads():
    """A few thousand reads: short reads with N runs plus long reads, from a 2 Mbp genome."""
    from scbf_b200 import workloads

    short = workloads.short_reads(genome_len=2_000_000, n_reads=6_000, read_len=150, seed=31, sub_rate=0.01,
                                  n_rate=0.01, n_max_run=10)
    long_ = workloads.random_sequences(12, 1_000, 30_000, seed=32, genome=workloads.random_genome(2_000_000, 31))
    return workloads.interleave([short, long_], seed=33)


@pytest.mark.parametrize("bits,slot_exp", [(16, 31), (8, 32), (32, 32)])
def test_largest_tables_against_oracle(scb, oracle_mod, bits, slot_exp):
    from scbf_b200 import _lib, api

    table_bytes = (1 << slot_exp) * bits // 8
    if _host_bytes_available() < table_bytes + 8 * GIB:
        pytest.skip(f"needs {table_bytes / GIB:.0f} GiB of free host memory for the oracle's table")
    data, offsets = _big_table_reads()
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, bits, slot_exp, 9, 1, 4096))
    okm, osm = o.insert_batch_arrays(data, offsets)
    oout, ovalid = o.query_batch_arrays(data, offsets)
    oq = o.query_report_arrays(data, offsets)
    ref = o.table_view()
    assert ref.size == table_bytes

    L = _lib.load()
    b = scb.SuperCountingBloomBuilder(_cfg(scb, bits, slot_exp))
    h = b._ctx.h
    for strategy in ("plain", "fused", "grouped"):
        assert L.scb_reset(h) == 0
        api.set_strategy(b, strategy, strategy)
        rep = b.add_sequences(data, offsets)
        assert (rep.inserted_kmers, rep.inserted_smers) == (okm, osm), strategy
        _assert_table_equal(L, h, ref)
        assert L.scb_freeze(h) == 0
        idx = scb.SuperCountingBloomIndex._from_ctx(b._ctx, b.config(), okm)
        out, valid = idx.estimate_batch(data, offsets)
        assert np.array_equal(valid, ovalid) and np.array_equal(out, oout), strategy
        assert _report_tuple(idx.query_report(data, offsets)) == _report_tuple(oq), strategy
