"""CUDA graphs per batch shape: batches of the fused and grouped strategies replay a graph
captured for their shape class.  Replays must give exactly the eager pipeline's (and the
oracle's) counters and reports, one capture must serve several batches of a class, and a batch
whose super-k-mer records outgrow the class's record slots must be redone correctly."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scb():
    import scbf_b200

    return scbf_b200


def _reads(seed, n, lo, hi):
    rng = np.random.default_rng(seed)
    seqs = []
    for _ in range(n):
        L = int(rng.integers(lo, hi + 1))
        s = rng.choice(np.frombuffer(b"ACGT", np.uint8), L)
        s[rng.random(L) < 0.01] = ord("N")
        seqs.append(s.tobytes())
    return seqs


def _class(n_bytes):
    """Byte class of a grouped batch: bytes rounded up to four steps per octave (at least 64 KiB)."""
    if n_bytes <= 1 << 16:
        return 1 << 16
    e = (n_bytes - 1).bit_length() - 1
    step = 1 << (e - 2)
    return -(-n_bytes // step) * step


def _graph_stats(L, h):
    c, r, f = C.c_uint64(), C.c_uint64(), C.c_uint64()
    assert L.scb_graph_stats(h, C.byref(c), C.byref(r), C.byref(f)) == 0
    return c.value, r.value, f.value


def _run_batches(scb, cfg, batches, strategy, graphs):
    """Insert every batch through scb_insert_batch, freeze, report every batch; returns the table,
    the per-batch insert counts and reports, and the graph statistics."""
    from scbf_b200 import _lib, api

    L = _lib.load()
    b = scb.SuperCountingBloomBuilder(cfg)
    api.set_strategy(b, strategy, strategy)
    assert L.scb_set_graphs(b._ctx.h, 1 if graphs else 0) == 0
    counts = [(r.inserted_kmers, r.inserted_smers) for r in (b.add_sequences(d, o) for d, o in batches)]
    idx = b.into_index()
    reports = []
    for d, o in batches:
        q = idx.query_report(d, o)
        reports.append((q.records_processed, q.total_windows, q.valid_kmers, q.positive_estimates,
                        q.estimate_checksum))
    return idx.table(), counts, reports, _graph_stats(L, idx._ctx.h)


@pytest.mark.parametrize("strategy", ["fused", "grouped"])
def test_replays_match_eager_and_oracle(scb, oracle_mod, strategy):
    cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits(16),
                                       counter_slots_exponent=20, block_slots_exponent=9, threads=3, queue=17)
    # batches of 340-370 KB (one byte class) and one of about 90 KB
    batches = [scb.pack_sequences(_reads(s, n, 100, 800)) for s, n in ((1, 760), (2, 800), (3, 840), (4, 200))]
    classes = {_class(int(o[-1])) for _, o in batches}
    assert len(classes) == 2
    t_g, c_g, r_g, (cap, rep, fb) = _run_batches(scb, cfg, batches, strategy, graphs=True)
    t_e, c_e, r_e, (cap_e, rep_e, _) = _run_batches(scb, cfg, batches, strategy, graphs=False)
    assert rep_e == 0 and cap_e == 0
    assert np.array_equal(t_g, t_e)
    assert c_g == c_e and r_g == r_e
    # 4 insert + 4 report batches replayed; grouped graphs are captured per (kind, byte class),
    # fused ones per kind (their kernels take any batch that fits the lane's buffers, which grow
    # in class steps: the largest class came first)
    assert fb == 0 and rep == 8 and cap == (2 * len(classes) if strategy == "grouped" else 2)
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 20, 9, 3, 17))
    for (d, off), (km, sm) in zip(batches, c_g):
        assert o.insert_batch_arrays(d, off) == (km, sm)
    assert np.array_equal(t_g, o.table())
    for (d, off), r in zip(batches, r_g):
        q = o.query_report_arrays(d, off)
        assert r == (q.records_processed, q.total_windows, q.valid_kmers, q.positive_estimates, q.estimate_checksum)


@pytest.mark.parametrize("strategy", ["fused", "grouped"])
def test_build_and_stream_replay_matches_oracle(scb, oracle_mod, strategy):
    import torch

    from scbf_b200 import _lib, api

    L = _lib.load()
    cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits(8),
                                       counter_slots_exponent=22, block_slots_exponent=9, threads=3, queue=17)
    data, offsets = scb.pack_sequences(_reads(11, 1500, 50, 1200))
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 8, 22, 9, 3, 17))
    okm, osm = o.insert_batch_arrays(data, offsets)
    oq = o.query_report_arrays(data, offsets)
    d_data = torch.from_numpy(data).to("cuda")
    d_off = torch.from_numpy(offsets.view(np.int64)).to("cuda")
    km, sm = C.c_uint64(), C.c_uint64()
    rep = _lib.ScbReport()
    ctx = api._create(cfg)
    assert L.scb_set_strategy(ctx.h, _lib.STRATEGIES[strategy], _lib.STRATEGIES[strategy]) == 0
    for step in range(3):  # the first call captures, the next ones replay
        assert L.scb_reset(ctx.h) == 0
        assert L.scb_build_and_stream_query_device(ctx.h, d_data.data_ptr(), d_off.data_ptr(), len(offsets) - 1,
                                                   int(offsets[-1]), None, C.byref(km), C.byref(sm),
                                                   C.byref(rep)) == 0, _lib.last_error()
        assert (km.value, sm.value) == (okm, osm)
        assert (rep.records_processed, rep.total_windows, rep.valid_kmers, rep.positive_estimates,
                rep.estimate_checksum) == (oq.records_processed, oq.total_windows, oq.valid_kmers,
                                           oq.positive_estimates, oq.estimate_checksum)
    raw = np.zeros(int(L.scb_table_bytes(ctx.h)), dtype=np.uint8)
    assert L.scb_table_download(ctx.h, raw.ctypes.data, raw.size) == 0
    assert np.array_equal(raw, o.table().view(np.uint8))
    cap, replays, fb = _graph_stats(L, ctx.h)
    assert cap == 1 and replays == 3 and fb == 0
    ctx.close()


def test_record_overflow_is_redone_exactly(scb):
    """Poly-A reads give one super-k-mer per window (the minimizer position moves with every
    window), far above the class's record estimate: the replay applies nothing, the batch is redone
    eagerly, and the next batch of the class is captured with room for its records."""
    cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits(16),
                                       counter_slots_exponent=24, block_slots_exponent=9, threads=3, queue=17)
    seqs = [b"A" * 100_000 for _ in range(200)] + _reads(5, 300, 100, 400)
    batch = scb.pack_sequences(seqs)
    t_g, c_g, r_g, (cap, rep, fb) = _run_batches(scb, cfg, [batch, batch], "grouped", graphs=True)
    t_e, c_e, r_e, _ = _run_batches(scb, cfg, [batch, batch], "grouped", graphs=False)
    assert np.array_equal(t_g, t_e)
    assert c_g == c_e and r_g == r_e
    assert c_g[0][0] > 19_000_000  # windows: one record each
    # the first insert's replay overflows and is redone eagerly; the record count it saw sizes
    # the next captures (second insert, then the reports), which replace the first graph
    assert fb == 1 and rep == 4 and cap == 3


def test_server_batches_replay_graphs(scb, oracle_mod):
    from scbf_b200 import _lib

    L = _lib.load()
    cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits(16),
                                       counter_slots_exponent=20, block_slots_exponent=9, threads=3, queue=17)
    b = scb.SuperCountingBloomBuilder(cfg)
    ref_data, ref_off = scb.pack_sequences(_reads(21, 400, 100, 1500))
    b.add_sequences(ref_data, ref_off)
    idx = b.into_index()
    requests = [scb.pack_sequences(_reads(100 + i, 20 + 7 * i, 80, 900)) for i in range(12)]
    srv = scb.SuperCountingBloomServer(idx, max_batch_bytes=1 << 18, max_inflight=2)
    tickets = [srv.submit(d, o) for d, o in requests]
    outs = [srv.wait(t) for t in tickets]
    c, r = C.c_uint64(), C.c_uint64()
    assert L.scb_server_graph_stats(srv.h, C.byref(c), C.byref(r)) == 0
    srv.close()
    assert c.value == 2 and r.value >= 2  # one graph per slot, captured when the server starts
    for (d, o), res in zip(requests, outs):
        ab, valid = idx.estimate_batch(d, o)
        assert np.array_equal(res[1], valid)
        assert np.array_equal(np.where(valid == 1, res[0], 0), np.where(valid == 1, ab, 0))


@pytest.mark.parametrize("graphs", [True, False])
def test_build_and_stream_probe_slots_overflow(scb, oracle_mod, graphs):
    """A grouped build + stream query keeps the insert's probe slots for the query; poly-A reads
    (one super-k-mer per window, seven s-mers each) outgrow the slots' capacity, so later work
    items hash again.  Counts, report and table stay exact either way."""
    import torch

    from scbf_b200 import _lib, api

    L = _lib.load()
    cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits(16),
                                       counter_slots_exponent=22, block_slots_exponent=9, threads=3, queue=17)
    data, offsets = scb.pack_sequences([b"A" * 100_000 for _ in range(20)] + _reads(31, 2000, 100, 900))
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 22, 9, 3, 17))
    okm, osm = o.insert_batch_arrays(data, offsets)
    oq = o.query_report_arrays(data, offsets)
    assert osm > 2 * len(data)  # more s-mers than the probe slots hold
    d_data = torch.from_numpy(data.copy()).to("cuda")
    d_off = torch.from_numpy(offsets.view(np.int64).copy()).to("cuda")
    km, sm = C.c_uint64(), C.c_uint64()
    rep = _lib.ScbReport()
    ctx = api._create(cfg)
    assert L.scb_set_strategy(ctx.h, _lib.STRATEGIES["grouped"], _lib.STRATEGIES["grouped"]) == 0
    assert L.scb_set_graphs(ctx.h, 1 if graphs else 0) == 0
    for _ in range(2):
        assert L.scb_reset(ctx.h) == 0
        assert L.scb_build_and_stream_query_device(ctx.h, d_data.data_ptr(), d_off.data_ptr(), len(offsets) - 1,
                                                   int(offsets[-1]), None, C.byref(km), C.byref(sm),
                                                   C.byref(rep)) == 0, _lib.last_error()
        assert (km.value, sm.value) == (okm, osm)
        assert (rep.records_processed, rep.total_windows, rep.valid_kmers, rep.positive_estimates,
                rep.estimate_checksum) == (oq.records_processed, oq.total_windows, oq.valid_kmers,
                                           oq.positive_estimates, oq.estimate_checksum)
    raw = np.zeros(int(L.scb_table_bytes(ctx.h)), dtype=np.uint8)
    assert L.scb_table_download(ctx.h, raw.ctypes.data, raw.size) == 0
    assert np.array_equal(raw, o.table().view(np.uint8))
    ctx.close()


@pytest.mark.parametrize("pinned,long_first,host_pack", [(False, False, True), (True, False, True),
                                                          (True, True, True), (False, False, False),
                                                          (True, True, False)])
def test_host_build_and_stream_in_pieces_matches_oracle(scb, oracle_mod, pinned, long_first, host_pack):
    """The host build + stream query split into pieces (copy of piece p + 1 overlapping the insert
    of piece p, each piece queried on its kept records after the last insert) gives exactly the
    oracle's counts, report and table, from pageable or pinned host memory, with the pieces after
    the first packed on the host (3 bits per base copied) or packed on the device from copied
    letters (the first piece's letters copy while the offsets are validated), also when
    the first sequence is longer than the first piece's bytes copied while the offsets are
    validated.  The bytes copied are the packed layout's, or the letters', plus the offsets."""
    import torch

    from scbf_b200 import _lib, api

    L = _lib.load()
    cfg = scb.SuperCountingBloomConfig(k=31, m=21, s=25, n_hashes=4, counter_bits=scb.CounterBits(16),
                                       counter_slots_exponent=22, block_slots_exponent=9, threads=3, queue=17)
    seqs = _reads(51, 9000, 100, 1200)
    if long_first:  # 700 kB, above the 0.45 MiB first piece of 1 MiB pieces
        seqs = _reads(52, 1, 700_000, 700_000) + seqs
    data, offsets = scb.pack_sequences(seqs)
    o = oracle_mod.OracleFilter(oracle_mod.make_config(31, 21, 25, 4, 16, 22, 9, 3, 17))
    okm, osm = o.insert_batch_arrays(data, offsets)
    oq = o.query_report_arrays(data, offsets)
    if pinned:
        h_data = torch.from_numpy(data.copy()).pin_memory()
        h_off = torch.from_numpy(offsets.view(np.int64).copy()).pin_memory()
        dp, op = h_data.data_ptr(), h_off.data_ptr()
    else:
        h_data, h_off = data, offsets
        dp, op = data.ctypes.data, offsets.ctypes.data
    ctx = api._create(cfg)
    assert L.scb_set_strategy(ctx.h, _lib.STRATEGIES["grouped"], _lib.STRATEGIES["grouped"]) == 0
    assert L.scb_set_piece_bytes(ctx.h, 1 << 20) == 0  # pieces of 0.45 MiB growing to 1 MiB: about eight
    assert L.scb_set_host_pack(ctx.h, 1 if host_pack else 0) == 0
    km, sm = C.c_uint64(), C.c_uint64()
    rep = _lib.ScbReport()
    n_bytes, n_seqs = int(offsets[-1]), len(offsets) - 1
    for _ in range(2):
        assert L.scb_reset(ctx.h) == 0
        b0, b1 = C.c_uint64(), C.c_uint64()
        assert L.scb_h2d_bytes(ctx.h, C.byref(b0)) == 0
        assert L.scb_build_and_stream_query(ctx.h, dp, op, len(offsets) - 1, C.byref(km), C.byref(sm),
                                            C.byref(rep)) == 0, _lib.last_error()
        assert L.scb_h2d_bytes(ctx.h, C.byref(b1)) == 0
        copied = b1.value - b0.value
        if host_pack:  # 3 bits per base plus padding per piece, the offsets of every piece, and the
            # first piece's letters (copied while the offsets are validated; at most 1 MiB here, a
            # longer first sequence packs that piece instead)
            assert n_bytes * 3 // 8 < copied < n_bytes * 3 // 8 + (1 << 20) + 20 * 256 + (n_seqs + 20) * 8
        else:
            # (a first sequence longer than the preloaded first piece copies that piece again)
            assert n_bytes + (n_seqs + 1) * 8 <= copied <= n_bytes + (1 << 20) + (n_seqs + 20) * 8
        assert (km.value, sm.value) == (okm, osm)
        assert (rep.records_processed, rep.total_windows, rep.valid_kmers, rep.positive_estimates,
                rep.estimate_checksum) == (oq.records_processed, oq.total_windows, oq.valid_kmers,
                                           oq.positive_estimates, oq.estimate_checksum)
        cnt_k, cnt_s = C.c_uint64(), C.c_uint64()
        assert L.scb_get_counts(ctx.h, C.byref(cnt_k), C.byref(cnt_s)) == 0
        assert (cnt_k.value, cnt_s.value) == (okm, osm)
    raw = np.zeros(int(L.scb_table_bytes(ctx.h)), dtype=np.uint8)
    assert L.scb_table_download(ctx.h, raw.ctypes.data, raw.size) == 0
    assert np.array_equal(raw, o.table().view(np.uint8))
    del h_data, h_off
    ctx.close()
