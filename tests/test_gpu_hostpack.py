"""Host entry points with host packing (the default for uploads of at least 1 MiB): the reads are
packed on the host into the device's 2-bit code and validity layout, in slices of 256 MiB that
alternate between two pinned staging areas, and only those words cross PCIe.  Every result must
equal the same calls with the letters copied and packed on the device, and the configuration-1
reads (30 MB, one slice) must give the oracle's counters, report and spectrum."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scb():
    import scbf_b200

    return scbf_b200


def _run(scb, data, offsets, host_pack, slots=24):
    from scbf_b200 import _lib

    L = _lib.load()
    cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits.Bits16,
                                       counter_slots_exponent=slots, block_slots_exponent=9)
    b = scb.SuperCountingBloomBuilder(cfg)
    h = b._ctx.h
    assert L.scb_set_host_pack(h, 1 if host_pack else 0) == 0
    c0 = C.c_uint64()
    assert L.scb_h2d_bytes(h, C.byref(c0)) == 0
    rep = b.add_sequences(data, offsets)
    c1 = C.c_uint64()
    assert L.scb_h2d_bytes(h, C.byref(c1)) == 0
    idx = b.into_index()
    q = idx.query_report(data, offsets)
    sp = idx.spectrum_distinct(data, offsets)
    return ((rep.inserted_kmers, rep.inserted_smers), idx.table(),
            (q.records_processed, q.total_windows, q.valid_kmers, q.positive_estimates, q.estimate_checksum),
            sp["rows"], sp["distinct_keys"], c1.value - c0.value)


def test_host_packed_uploads_match_the_oracle_on_config1(scb, oracle_mod):
    from scbf_b200 import workloads

    data, offsets = workloads.config1()
    got = _run(scb, data, offsets, True)
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 24, 9, 1, 64))
    assert got[0] == o.insert_batch_arrays(data, offsets)
    assert np.array_equal(got[1], o.table())
    oq = o.query_report_arrays(data, offsets)
    assert got[2] == (oq.records_processed, oq.total_windows, oq.valid_kmers, oq.positive_estimates,
                      oq.estimate_checksum)
    osp = o.spectrum_distinct_arrays(data, offsets)
    assert got[3] == osp["rows"] and got[4] == osp["distinct_keys"]
    n_bytes, n_seqs = int(offsets[-1]), len(offsets) - 1
    assert got[5] < n_bytes // 2 + (n_seqs + 1) * 8  # the insert's upload: 3 bits per base and the offsets


def test_host_packed_slices_equal_letters(scb):
    """A 640 MB batch: three slices of the staging areas (the third partly filled, with the padding
    words), against the same calls with the letters copied."""
    from scbf_b200 import workloads

    data, offsets = workloads.short_reads(genome_len=5_000_000, n_reads=4_300_000, read_len=150, seed=31,
                                          sub_rate=0.01, n_rate=0.01)
    assert int(offsets[-1]) > 2 * (256 << 20)
    packed = _run(scb, data, offsets, True, slots=26)
    letters = _run(scb, data, offsets, False, slots=26)
    assert packed[0] == letters[0] and packed[2] == letters[2]
    assert np.array_equal(packed[1], letters[1])
    assert packed[3] == letters[3] and packed[4] == letters[4]
    assert packed[5] * 2 < letters[5]
