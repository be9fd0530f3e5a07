"""Command-line tools over the GPU backend, with the reference's arguments, defaults and output:

    python -m scbf_b200.cli build-index INPUT OUTPUT [geometry]        (src/bin/build-index.rs)
    python -m scbf_b200.cli query-index INDEX QUERY [-o CSV] [--mode report|fast|slow]
                                                                        (src/bin/query-index.rs)
    python -m scbf_b200.cli filter-spectrum INPUT [-o CSV] [--counter-histogram CSV]
        [--max-abundance N] [--kmer-count-hint N] [geometry]            (src/bin/filter_spectrum.rs)
    python -m scbf_b200.cli sampled-spectrum INPUT [-o CSV] [--sample-size N] [--seed S] [geometry]
                                                                        (src/bin/sampled_spectrum.rs)

geometry: -k -m -s -H/--n-hashes --counter-bits {8,16,32} --counter-slots-exponent
--block-slots-exponent -t/--threads --queue.  Errors print "error: ..." and exit 1.
"""
from __future__ import annotations

import argparse
import os
import sys
import time
from typing import IO, Callable

import numpy as np

from . import api


def _add_geometry(p: argparse.ArgumentParser) -> None:
    p.add_argument("-k", "--k", type=int, default=31)
    p.add_argument("-m", "--m", type=int, default=21)
    p.add_argument("-s", "--s", type=int, default=25)
    p.add_argument("-H", "--n-hashes", type=int, default=4)
    p.add_argument("--counter-bits", type=int, choices=(8, 16, 32), default=16)
    p.add_argument("--counter-slots-exponent", type=int, default=30)
    p.add_argument("--block-slots-exponent", type=int, default=9)
    p.add_argument("-t", "--threads", type=int, default=None)
    p.add_argument("--queue", type=int, default=4096)


def _config(a: argparse.Namespace) -> api.SuperCountingBloomConfig:
    """config_from_cli of the reference binaries: threads default to the host's CPUs, at least 1."""
    threads = a.threads if a.threads is not None else (os.cpu_count() or 1)
    return api.SuperCountingBloomConfig(k=a.k, m=a.m, s=a.s, n_hashes=a.n_hashes,
                                        counter_bits=api.CounterBits(a.counter_bits),
                                        counter_slots_exponent=a.counter_slots_exponent,
                                        block_slots_exponent=a.block_slots_exponent, threads=max(threads, 1),
                                        queue=a.queue)


def _open_out(path: str | None) -> IO[str]:
    if path is None:
        return sys.stdout
    try:
        return open(path, "w", newline="")
    except OSError as e:
        raise api.Io(f"{path}: {e}") from e


def _u64(text: str) -> int:
    v = int(text)
    if not 0 <= v < 1 << 64:
        raise argparse.ArgumentTypeError(f"{text} is not an unsigned 64-bit value")
    return v


def _csv_escape(value: str) -> str:
    if any(c in value for c in ',"\n\r'):
        return '"' + value.replace('"', '""') + '"'
    return value


def _optional(value) -> str:
    return "" if value is None else f"{value:.6f}"


def build_index(a: argparse.Namespace) -> None:
    """src/bin/build-index.rs:55-78."""
    builder = api.SuperCountingBloomBuilder(_config(a))
    report = builder.add_fasta(a.input)
    inserted_kmers, inserted_smers = builder.inserted_kmers(), builder.inserted_smers()
    index = builder.into_index()
    index.save(a.output)
    cfg = index.config()
    print(f"records_processed: {report.records_processed}\trecords_indexed: {report.records_indexed}\t"
          f"inserted_kmers: {inserted_kmers}\tinserted_smers: {inserted_smers}\t"
          f"counter_bits: {cfg.counter_bits.as_u8()}\tthreads: {cfg.threads}\tadd_s: {report.add_seconds:.3f}",
          file=sys.stderr)


def query_index(a: argparse.Namespace) -> None:
    """src/bin/query-index.rs:52-139: one aggregate row (report), one row per sequence (fast) or
    one row per k-mer window (slow)."""
    index = api.SuperCountingBloomIndex.load(a.index)
    cfg = index.config()
    print(f"inserted_kmers: {index.inserted_kmers()}\tcounter_bits: {cfg.counter_bits.as_u8()}\t"
          f"threads: {cfg.threads}", file=sys.stderr)
    out = _open_out(a.output)
    try:
        if a.mode == "report":
            r = index.query_fasta(a.query)
            out.write("records_processed,total_windows,valid_kmers,positive_estimates,estimate_checksum\n")
            out.write(f"{r.records_processed},{r.total_windows},{r.valid_kmers},{r.positive_estimates},"
                      f"{r.estimate_checksum}\n")
        elif a.mode == "fast":
            out.write("sequence,length,total_windows,valid_kmers,mean_abundance,median_abundance\n")

            def fast(name, seq):
                s = index.summarize_sequence(name, seq)
                out.write(f"{_csv_escape(s.name)},{s.sequence_len},{s.total_windows},{s.valid_kmers},"
                          f"{_optional(s.mean_abundance)},{_optional(s.median_abundance)}\n")

            api.for_each_fastx_record(a.query, fast)
        else:
            out.write("sequence,kmer_index,abundance\n")

            def slow(name, seq):
                n = _csv_escape(name)
                for i, v in enumerate(index.estimate_sequence_abundances(seq)):
                    out.write(f"{n},{i},{'' if v is None else v}\n")

            api.for_each_fastx_record(a.query, slow)
    finally:
        if out is not sys.stdout:
            out.close()
        else:
            out.flush()


def filter_spectrum(a: argparse.Namespace) -> None:
    """src/bin/filter_spectrum.rs:73-146."""
    build = api.SuperCountingBloomIndex.build_from_fastx(a.input, _config(a))
    print("warning: filter-only spectra are model-based counter-histogram estimates, not a replacement for "
          "key-aware spectra", file=sys.stderr)
    print(f"indexed_kmers: {build.indexed_kmers}\tinserted_smers: {build.inserted_smers}\t"
          f"counter_slots: {build.counter_slots}\tblocks: {build.blocks}\tbuild_s: {build.build_seconds:.3f}",
          file=sys.stderr)
    hist = build.index.counter_histogram()
    if a.counter_histogram is not None:
        with _open_out(a.counter_histogram) as fh:
            fh.write("counter_value,counters\n")
            for value, counters in hist:
                fh.write(f"{value},{counters}\n")
    hint = a.kmer_count_hint
    if hint is None:
        hint = build.index.filter_only_count_hint_from_counter_histogram(hist, a.max_abundance)
    est = build.index.estimate_filter_only_spectrum_from_counter_histogram(hist, a.max_abundance, hint)
    out = _open_out(a.output)
    try:
        out.write("estimated_count,estimated_kmers,method,kmer_count_hint\n")
        for count, kmers in est.rows:
            out.write(f"{count},{kmers},{est.method},{est.kmer_count_hint}\n")
    finally:
        if out is not sys.stdout:
            out.close()
        else:
            out.flush()


# ---------------------------------------------------------------------------------------
# Sampled spectrum (src/bin/sampled_spectrum.rs): a reservoir sample of the valid k-mer windows,
# queried against the index as one batch, scaled to all windows.
# ---------------------------------------------------------------------------------------
_ACGT = np.zeros(256, dtype=bool)
_ACGT[list(b"ACGTacgt")] = True
_GOLDEN, _MIX1, _MIX2 = np.uint64(0x9E3779B97F4A7C15), np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB)


def _splitmix_calls(first: int, n: int, seed: int) -> np.ndarray:
    """Outputs of the sampler's SplitMix64 calls first .. first + n - 1 (1-based): call j mixes
    seed + j * golden (sampled_spectrum.rs:293-300), so any range is computed at once."""
    j = np.arange(first, first + n, dtype=np.uint64)
    state = np.uint64(seed) + j * _GOLDEN
    v = (state ^ (state >> np.uint64(30))) * _MIX1
    v = (v ^ (v >> np.uint64(27))) * _MIX2
    return v ^ (v >> np.uint64(31))


def _valid_windows(data: np.ndarray, offsets: np.ndarray, c0: int, c1: int, k: int) -> np.ndarray:
    """Batch positions g in [c0, c1) whose k bases are A/C/G/T (either case) within one sequence."""
    total = len(data)
    m = min(c1, total - k + 1) - c0  # window starts to test
    if m <= 0:
        return np.zeros(0, np.int64)
    hi = min(c1 + k - 1, total)
    n = hi - c0
    bad = np.zeros(n + 1, np.int32)
    np.cumsum(~_ACGT[data[c0:hi]], out=bad[1:])
    starts = offsets[np.searchsorted(offsets, c0, side="right"):np.searchsorted(offsets, hi, side="left")]
    marks = np.zeros(n + 2, np.int32)  # marks[x]: sequence starts at positions < x (relative)
    np.cumsum(np.bincount(starts.astype(np.int64) - c0, minlength=n + 1)[: n + 1], out=marks[1:])
    ok = (bad[k:k + m] == bad[:m]) & (marks[k:k + m] == marks[1:1 + m])
    return np.nonzero(ok)[0].astype(np.int64) + c0


def sample_kmers(data: np.ndarray, offsets: np.ndarray, k: int, capacity: int, seed: int,
                 chunk: int = 1 << 24) -> tuple[np.ndarray, int]:
    """Reservoir sample of the batch's valid k-mer windows in order (sampled_spectrum.rs:182-223,
    265-282): the first `capacity` fill the slots, window t > capacity replaces slot r when
    r = (SplitMix64 call t - capacity) mod t < capacity.  Returns the sampled k-mers in slot order
    (rows of k upper-case bytes) and the number of windows seen."""
    res = np.zeros(capacity, np.int64)
    filled = seen = 0
    for c0 in range(0, max(len(data), 1), chunk):
        pos = _valid_windows(data, offsets, c0, c0 + chunk, k)
        take = min(len(pos), capacity - filled)
        res[filled:filled + take] = pos[:take]
        filled += take
        seen += take
        rest = pos[take:]
        if len(rest):
            t = np.arange(seen + 1, seen + 1 + len(rest), dtype=np.uint64)
            r = _splitmix_calls(seen + 1 - capacity, len(rest), seed) % t
            sel = r < np.uint64(capacity)
            slots, vals = r[sel].astype(np.int64)[::-1], rest[sel][::-1]
            uniq, last = np.unique(slots, return_index=True)  # the latest replacement of each slot
            res[uniq] = vals[last]
            seen += len(rest)
    kmers = data[res[:filled, None] + np.arange(k)] & np.uint8(0xDF)  # A/C/G/T upper case
    return kmers.reshape(filled, k), seen


def sampled_rows(kmers: np.ndarray, total_windows: int,
                 estimate: Callable[[np.ndarray, np.ndarray], tuple[np.ndarray, np.ndarray]]):
    """Queries the sampled k-mers as one batch (one window each) and scales their abundance
    histogram to all windows (sampled_spectrum.rs:225-261).  Returns the rows (abundance, sampled
    k-mers, linearly scaled windows, estimated distinct k-mers) and the invalid query count."""
    n, k = kmers.shape
    if n == 0:
        return [], 0
    out, valid = estimate(np.ascontiguousarray(kmers).reshape(-1), np.arange(0, (n + 1) * k, k, dtype=np.uint64))
    ok = np.asarray(valid).astype(bool)
    values, counts = np.unique(np.asarray(out)[ok], return_counts=True)
    scale = float(total_windows) / float(max(n, 1))
    rows = []
    for a, c in zip(values.tolist(), counts.tolist()):
        lsw = api._round_u64(float(c) * scale)
        rows.append((a, c, lsw, 0 if a == 0 else api._round_u64(float(lsw) / float(a))))
    return rows, int(n - ok.sum())


def sampled_spectrum(a: argparse.Namespace) -> None:
    """src/bin/sampled_spectrum.rs:97-148."""
    if a.sample_size == 0:
        raise api.InvalidConfig("invalid config: sample_size must be positive")
    build = api.SuperCountingBloomIndex.build_from_fastx(a.input, _config(a))
    print(f"indexed_kmers: {build.indexed_kmers}\tinserted_smers: {build.inserted_smers}\t"
          f"counter_slots: {build.counter_slots}\tblocks: {build.blocks}\tbuild_s: {build.build_seconds:.3f}",
          file=sys.stderr)
    t0 = time.perf_counter()
    data, offsets = api._read_batch(a.input)
    kmers, total = sample_kmers(data, offsets, int(build.index.config().k), a.sample_size, a.seed)
    sample_s = time.perf_counter() - t0
    if total != build.indexed_kmers:
        print(f"warning: sampled valid k-mer windows ({total}) differ from indexed k-mers ({build.indexed_kmers})",
              file=sys.stderr)
    t0 = time.perf_counter()
    rows, invalid = sampled_rows(kmers, total, build.index.estimate_batch)
    query_s = time.perf_counter() - t0
    out = _open_out(a.output)
    try:
        out.write("estimated_count,sampled_kmers,linear_scaled_windows,estimated_distinct_kmers\n")
        for row in rows:
            out.write(",".join(str(x) for x in row) + "\n")
    finally:
        if out is not sys.stdout:
            out.close()
        else:
            out.flush()
    print(f"total_inserted_kmers: {total}\tsampled_kmers: {len(kmers)}\tqueried_kmers: {len(kmers)}\t"
          f"invalid_queries: {invalid}\tsample_s: {sample_s:.3f}\tquery_s: {query_s:.3f}", file=sys.stderr)


def parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser(prog="python -m scbf_b200.cli")
    sub = p.add_subparsers(dest="command", required=True)
    b = sub.add_parser("build-index", help="Build and save a SuperCountingBloom index")
    b.add_argument("input", help="FASTA/FASTQ input used to build the abundance index")
    b.add_argument("output", help="output index path")
    _add_geometry(b)
    b.set_defaults(run=build_index)
    q = sub.add_parser("query-index", help="Load a SuperCountingBloom index and query FASTA/FASTQ")
    q.add_argument("index", help="saved SuperCountingBloom index")
    q.add_argument("query", help="FASTA/FASTQ queried against the saved index")
    q.add_argument("-o", "--output", default=None, help="output CSV path (default: stdout)")
    q.add_argument("--mode", choices=("report", "fast", "slow"), default="fast")
    q.set_defaults(run=query_index)
    f = sub.add_parser("filter-spectrum", help="Experimental filter-only k-mer spectrum estimator")
    f.add_argument("input", help="FASTA/FASTQ input used to build the abundance index")
    f.add_argument("-o", "--output", default=None, help="output CSV path (default: stdout)")
    f.add_argument("--counter-histogram", default=None, help="optional raw counter histogram CSV path")
    f.add_argument("--max-abundance", type=int, default=255)
    f.add_argument("--kmer-count-hint", type=int, default=None)
    _add_geometry(f)
    f.set_defaults(run=filter_spectrum)
    g = sub.add_parser("sampled-spectrum", help="Estimate an abundance spectrum by querying sampled inserted k-mers")
    g.add_argument("input", help="FASTA/FASTQ input used to build the abundance index and sample inserted k-mers")
    g.add_argument("-o", "--output", default=None, help="output CSV path (default: stdout)")
    g.add_argument("--sample-size", type=_u64, default=1_000_000)
    g.add_argument("--seed", type=_u64, default=1)
    _add_geometry(g)
    g.set_defaults(run=sampled_spectrum)
    return p


def main(argv=None) -> int:
    args = parser().parse_args(argv)
    try:
        args.run(args)
    except api.SuperCountingBloomError as e:
        print(f"error: {e}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
