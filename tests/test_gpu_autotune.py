"""Autotuner: measured choices change speed only -- counters and estimates stay bit-exact -- and
apply to later contexts of the same geometry."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results_exact_and_caches_by_geometry(oracle_mod):
    import scbf_b200 as scb
    from scbf_b200 import _lib, workloads

    L = _lib.load()
    data, offsets = workloads.short_reads(genome_len=300_000, n_reads=60_000, read_len=150, seed=41,
                                          sub_rate=0.01, n_rate=0.01)
    cfg = scb.SuperCountingBloomConfig(counter_slots_exponent=21, counter_bits=scb.CounterBits.Bits16)
    b = scb.SuperCountingBloomBuilder(cfg)
    t = _lib.ScbTuning()
    assert L.scb_autotune(b._ctx.h, data.ctypes.data, offsets.ctypes.data, len(offsets) - 1, C.byref(t)) == 0, \
        _lib.last_error()
    tuned = t.as_dict()
    assert tuned["candidates"] >= 5 and tuned["insert_large"] in ("plain", "fused", "grouped")
    assert tuned["bucket_records"] in (256, 512, 1024, 2048) and tuned["apply_threads"] in (256, 512)
    # the builder's own table was not touched by the measurements
    raw = np.zeros(int(L.scb_table_bytes(b._ctx.h)), dtype=np.uint8)
    assert L.scb_table_download(b._ctx.h, raw.ctypes.data, raw.size) == 0
    assert not raw.any()
    b.add_sequences(data, offsets)
    idx = b.into_index()
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 21, 9))
    o.insert_batch_arrays(data, offsets)
    assert np.array_equal(idx.table(), o.table())
    q = idx.query_report(data, offsets)
    oq = o.query_report_arrays(data, offsets)
    assert (q.valid_kmers, q.positive_estimates, q.estimate_checksum) == (
        oq.valid_kmers, oq.positive_estimates, oq.estimate_checksum)
    # a new context of the same geometry starts with the tuned choices
    b2 = scb.SuperCountingBloomBuilder(cfg)
    t2 = _lib.ScbTuning()
    assert L.scb_get_tuning(b2._ctx.h, C.byref(t2)) == 0
    d2 = t2.as_dict()
    for key in ("insert_large", "query_large", "bucket_records", "apply_threads", "host_batch_bytes"):
        assert d2[key] == tuned[key]
