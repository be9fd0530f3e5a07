"""scb_query_report_device_noalloc: the query report for callers that cannot allocate device
memory while they run (code inside a CUDA stream capture, real-time serving threads that keep
the allocator out of the request path, hosts with a fixed memory budget).  Its scratch is a
static device array instead of per-call buffers; its report must equal the allocating
scb_query_report_device's, call after call.

Kept in a file collected last, so a run that stops at the first failure has run every other
test first; it needs no state from them and passes alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _report(fn, h, batch):
    from scbf_b200 import _lib

    d, o, n, nbytes = batch
    rep = _lib.ScbReport()
    st = fn(h, d.data_ptr(), o.data_ptr(), n, nbytes, None, C.byref(rep))
    assert st == 0, _lib.last_error()
    return (rep.records_processed, rep.total_windows, rep.valid_kmers, rep.positive_estimates,
            rep.estimate_checksum)


def test_noalloc_report_equals_allocating_report_on_repeated_calls():
    import torch

    import scbf_b200 as scb
    from scbf_b200 import _lib, workloads

    L = _lib.load()
    big = workloads.short_reads(genome_len=300_000, n_reads=40_000, read_len=150, seed=21, sub_rate=0.01,
                                n_rate=0.01)
    small = workloads.short_reads(genome_len=50_000, n_reads=3_000, read_len=150, seed=22, sub_rate=0.02)
    for bits in (8, 16, 32):
        cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits(bits),
                                           counter_slots_exponent=22, block_slots_exponent=9)
        b = scb.SuperCountingBloomBuilder(cfg)
        b.add_sequences(*big)
        idx = b.into_index()
        h = idx._ctx.h
        batches = [(torch.from_numpy(d).cuda(), torch.from_numpy(o.view(np.int64)).cuda(), len(o) - 1, int(o[-1]))
                   for d, o in (big, small)]
        torch.cuda.synchronize()
        expected = [_report(L.scb_query_report_device, h, x) for x in batches]
        assert expected[0][2] > 0 and expected[1][2] > 0
        # two calls in a row on each batch, then alternating: the shared array keeps the previous
        # call's contents, which must not leak into the next report
        for x, ref in zip(batches, expected):
            assert _report(L.scb_query_report_device_noalloc, h, x) == ref
            assert _report(L.scb_query_report_device_noalloc, h, x) == ref
        for x, ref in zip(batches[::-1] + batches, expected[::-1] + expected):
            assert _report(L.scb_query_report_device_noalloc, h, x) == ref


def test_noalloc_rejects_batches_above_its_limit():
    import torch

    import scbf_b200 as scb
    from scbf_b200 import _lib

    L = _lib.load()
    b = scb.SuperCountingBloomBuilder(scb.SuperCountingBloomConfig(counter_slots_exponent=16))
    idx = b.into_index()
    d = torch.zeros(64, dtype=torch.uint8, device="cuda")
    o = torch.zeros(2, dtype=torch.int64, device="cuda")
    rep = _lib.ScbReport()
    st = L.scb_query_report_device_noalloc(idx._ctx.h, d.data_ptr(), o.data_ptr(), 1, (32 << 20) + 1, None,
                                           C.byref(rep))
    assert st == 6
    assert "at most" in _lib.last_error()
