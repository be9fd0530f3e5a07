"""scb_query_report_device_noalloc: the query report for callers that cannot call cudaMalloc
while they run (real-time serving threads that keep allocator latency out of the request path,
hosts with a fixed device-memory budget).  Its scratch is a static device array instead of
per-call buffers; its report must equal the allocating scb_query_report_device's, call after
call, up to the largest batch it takes (32 MiB of sequence bytes) and on a caller's stream.

Kept in a file collected last, so a run that stops at the first failure has run every other
test first; it needs no state from them and passes alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _report(fn, h, batch, stream=None):
    from scbf_b200 import _lib

    d, o, n, nbytes = batch
    rep = _lib.ScbReport()
    st = fn(h, d.data_ptr(), o.data_ptr(), n, nbytes, stream, C.byref(rep))
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


def test_noalloc_largest_batch_and_caller_stream():
    """A batch of exactly 32 MiB fills the array to its last byte; a call on a caller's stream
    (not the default stream) gives the same report."""
    import torch

    import scbf_b200 as scb
    from scbf_b200 import _lib, workloads

    L = _lib.load()
    limit = 32 << 20
    d, o = workloads.short_reads(genome_len=2_000_000, n_reads=223_700, read_len=150, seed=23, sub_rate=0.01,
                                 n_rate=0.01)
    assert int(o[-1]) >= limit
    keep = int(np.searchsorted(o, limit, side="right")) - 1
    o = o[: keep + 1].copy()
    if int(o[-1]) < limit:
        o = np.append(o, np.uint64(limit))  # the last read is cut short at the limit
    d = d[:limit]
    cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits.Bits16,
                                       counter_slots_exponent=24, block_slots_exponent=9)
    b = scb.SuperCountingBloomBuilder(cfg)
    b.add_sequences(d, o)
    idx = b.into_index()
    h = idx._ctx.h
    full = (torch.from_numpy(d).cuda(), torch.from_numpy(o.view(np.int64)).cuda(), len(o) - 1, limit)
    small = (full[0], full[1][:1001], 1000, int(o[1000]))
    torch.cuda.synchronize()
    ref_full = _report(L.scb_query_report_device, h, full)
    ref_small = _report(L.scb_query_report_device, h, small)
    assert ref_full[1] > 0 and ref_full[2] > 0
    side = torch.cuda.Stream()
    for x, ref in ((full, ref_full), (small, ref_small), (full, ref_full)):
        assert _report(L.scb_query_report_device_noalloc, h, x) == ref
        assert _report(L.scb_query_report_device_noalloc, h, x, C.c_void_p(side.cuda_stream)) == ref
    torch.cuda.synchronize()


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
