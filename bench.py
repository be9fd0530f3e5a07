#!/usr/bin/env python
"""Benchmark of the SuperCountingBloom build + stream-query path on B200.

One step = the reference's `--stream-query-only` pipeline (src/main.rs:110-127, the command
benchmark/common.py times) on the default-geometry short-read workload: clear the counter table,
insert every read, freeze, then query every read's k-mers into the stream report.  The metric is
indexed k-mers per second over the whole step (whole job, all ranks).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Arms:
  ours       value   : inputs resident in HBM, device entry points, CUDA events on the stream
             e2e     : scb_build_and_stream_query with pinned host inputs (H2D inside the step)
             plain   : the one-launch-per-stage kernels, same measurement as value
  reference  the reference's CPU pipeline (multi-threaded port with its structure: 1024 mutex
             shards, bounded queue, all host threads) on a bounded sample of the same workload.

N > 1 runs N independent replicas (one table and one read set per GPU); value = k-mers of all
ranks / the slowest rank's time.  Rank 0 prints one JSON line.  The single-GPU characterisations
(serving, mixed lengths, spectrum, configuration 1, CPU baseline) run at N = 1 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GEOM = dict(k=31, m=21, s=25, n_hashes=4, counter_bits=16, counter_slots_exponent=30, block_slots_exponent=9)
METRIC = "k-mers/s (build + stream query)"
WORKLOAD = ("default geometry, short reads: 100 Mbp uniform genome, 20x of 150 bp reads (13.3M reads, 2 Gbp), "
            "both strands, 1% substitutions, 1% of bases N in runs of 1-10; k=31 m=21 s=25 h=4, 16-bit "
            "counters, 2^30 slots (2 GiB), 2^9 slots per block")
CPU_SAMPLE_READS = 2_000_000  # the CPU-baseline leg of our arm: one timed run
REF_STEP_READS = 1_000_000  # the reference arm: reads per step


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--scale", type=float, default=1.0, help="genome scale (same coverage) for quick runs")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-mixed", action="store_true", help="skip the mixed-length (config 4) comparison")
    p.add_argument("--no-serve", action="store_true", help="skip the serving (config 5) measurement")
    p.add_argument("--no-spectrum", action="store_true", help="skip the distinct-k-mer spectrum measurement")
    p.add_argument("--no-tune", action="store_true",
                   help="skip the autotuner (untuned defaults: fixed settings for comparing kernel builds)")
    p.add_argument("--profile-case", choices=["plain", "fused", "grouped"], default=None,
                   help="run one insert + query of a small case (for ncu) and exit")
    p.add_argument("--profile-scale", type=float, default=0.1,
                   help="genome scale of the profile case (1.0 = the full 2 Gbp workload)")
    p.add_argument("--profile-slots", type=int, default=GEOM["counter_slots_exponent"],
                   help="counter_slots_exponent of the profile case: scale 0.25 with 2^28 slots keeps the full "
                        "workload's records per block, so its buckets (4 blocks, about 500 records) are the full "
                        "run's")
    return p.parse_args()


class Dist:
    """One process per GPU (torchrun): NCCL over the GPUs, or gloo on a host without one (the
    reference arm and the CPU tests of this launch path)."""

    def __init__(self, gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.dev = "cpu"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            timeout = datetime.timedelta(seconds=600)
            if torch.cuda.is_available():
                torch.cuda.set_device(self.local)
                dist.init_process_group("nccl", timeout=timeout, device_id=torch.device("cuda", self.local))
                self.dev = "cuda"
            else:
                dist.init_process_group("gloo", timeout=timeout)
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self.dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self.dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class Clocks:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
            return
        # the timed region starts once the sampler is running (its first line is out)
        t0 = time.perf_counter()
        while not self.lines and self.proc.poll() is None and time.perf_counter() - t0 < 3.0:
            time.sleep(0.01)
        self.skip = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines[getattr(self, "skip", 0):] or self.lines[-1:]
        for ln in lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def kernel_source_hash() -> str:
    """Hash of the CUDA sources (the kernels a committed ncu capture measured)."""
    import hashlib

    h = hashlib.sha256()
    for name in ("scb_kernels.cu", "scb_kernels.cuh", "scb_device.cuh"):
        with open(os.path.join(ROOT, "scbf_b200", "csrc", name), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def profile_traffic() -> dict | None:
    """Per-kernel DRAM bytes per launch of the grouped step on this workload, from the committed
    one-pass ncu capture (profiles/traffic_grouped_config2.json), with the pipe that limits each
    kernel from the full capture of the small case."""
    p = os.path.join(ROOT, "profiles", "traffic_grouped_config2.json")
    try:
        return json.load(open(p))
    except (OSError, ValueError):
        return None


def workload(rank: int, scale: float):
    from scbf_b200 import workloads

    return workloads.config2(seed=1 + rank, scale=scale)


# ---------------------------------------------------------------------------------------
def cpu_port_run(data, offsets, first: int, reads: int, f) -> tuple[float, int, str]:
    """The CPU port (reference structure: parser thread, bounded queue of 4096, all host threads,
    1024 mutex shards) on reads [first, first + reads) of the workload, on filter f after a clear:
    f's table was touched before, so the timed region holds build + stream query work only."""
    n_total = len(offsets) - 1
    a = first % n_total
    b = min(a + reads, n_total)
    so = (offsets[a:b + 1] - offsets[a]).astype(np.uint64)
    sd = data[int(offsets[a]):int(offsets[b])]
    threads = os.cpu_count() or 1
    f.clear()
    t0 = time.perf_counter()
    r = f.port_build_and_stream_query(sd, so, threads=threads, queue=4096)
    dt = time.perf_counter() - t0
    return dt, r["inserted_kmers"], f"reads {a}..{b}"


def cpu_filter():
    from oracle import oracle

    threads = os.cpu_count() or 1
    f = oracle.OracleFilter(oracle.make_config(GEOM["k"], GEOM["m"], GEOM["s"], GEOM["n_hashes"], GEOM["counter_bits"],
                                               GEOM["counter_slots_exponent"], GEOM["block_slots_exponent"], threads,
                                               4096))
    f.clear()  # first touch of every page of the 2 GiB table, outside any timed region
    return f, threads


def run_reference(args, dist: Dist):
    if dist.rank != 0:
        return
    data, offsets = workload(0, args.scale)
    n_total = len(offsets) - 1
    per_step = min(REF_STEP_READS, n_total)
    f, threads = cpu_filter()
    times, kmers = [], 0
    for step in range(args.warmup + args.steps):
        # consecutive steps take consecutive slices, so the timed steps cover the whole workload
        dt, km, _ = cpu_port_run(data, offsets, step * per_step, per_step, f)
        if step >= args.warmup:
            times.append(dt)
            kmers += km
    f.close()
    total = sum(times)
    value = kmers / total
    sample = (f"{per_step} reads per step, consecutive slices of the workload ({args.steps} timed steps, "
              f"{kmers} k-mers in all); each step clears a pre-touched 2 GiB table outside its timed region")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "k-mers/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": WORKLOAD + (f" (genome scale {args.scale})" if args.scale != 1.0 else ""),
                   "reads": n_total, "bytes": int(offsets[-1]), "sample": sample,
                   "parallelism": f"{threads} host threads", "strategy": "CPU port of the reference pipeline"},
        "cpu_baseline": {"value": value, "unit": "k-mers/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "k-mers/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
STRATEGY_IDS = {"auto": 0, "plain": 1, "fused": 2, "grouped": 4}


def graph_stats(L, h) -> tuple[int, int, int]:
    c, r, f = C.c_uint64(), C.c_uint64(), C.c_uint64()
    assert L.scb_graph_stats(h, C.byref(c), C.byref(r), C.byref(f)) == 0
    return c.value, r.value, f.value


def occupied(n_items: float, n_bins: float) -> float:
    """Expected number of distinct bins hit by n_items uniform draws over n_bins."""
    if n_bins <= 0:
        return 0.0
    return n_bins * -np.expm1(-n_items / n_bins)


def run_ours(args, dist: Dist):
    import torch

    from scbf_b200 import _lib
    from scbf_b200 import api

    torch.cuda.set_device(dist.local)
    L = _lib.load()
    data, offsets = workload(dist.rank, args.scale)
    n_seqs = len(offsets) - 1
    n_bytes = int(offsets[-1])
    cfg = api.SuperCountingBloomConfig(k=GEOM["k"], m=GEOM["m"], s=GEOM["s"], n_hashes=GEOM["n_hashes"],
                                       counter_bits=api.CounterBits(GEOM["counter_bits"]),
                                       counter_slots_exponent=GEOM["counter_slots_exponent"],
                                       block_slots_exponent=GEOM["block_slots_exponent"], threads=1, queue=4096)
    ctx = api._create(cfg)
    h = ctx.h
    d_data = torch.from_numpy(data).to("cuda")
    d_off = torch.from_numpy(offsets.view(np.int64)).to("cuda")
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)

    def check(st):
        if st != 0:
            raise RuntimeError(_lib.last_error())

    km, sm = C.c_uint64(0), C.c_uint64(0)
    rep = _lib.ScbReport()

    def step():
        # stream_estimates_from_fastx on resident reads: clear, build, freeze, stream-query
        check(L.scb_reset(h))
        check(L.scb_build_and_stream_query_device(h, d_data.data_ptr(), d_off.data_ptr(), n_seqs, n_bytes, sp,
                                                  C.byref(km), C.byref(sm), C.byref(rep)))

    def timed(strategy: str, steps: int) -> tuple[float, dict]:
        sid = STRATEGY_IDS[strategy]
        check(L.scb_set_strategy(h, sid, sid))
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        check(L.scb_set_timing(h, 1))
        dist.barrier()
        torch.cuda.synchronize()
        launches0 = L.scb_kernel_launches()
        clocks = Clocks(dist.local)
        clocks.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("timed")  # lets a profiler capture the timed launches only
        ev0.record(stream)
        for _ in range(steps):
            step()
        ev1.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        clk = clocks.stop()
        dist.barrier()
        ms = ev0.elapsed_time(ev1)
        t = _lib.ScbTimings()
        check(L.scb_get_timings(h, C.byref(t)))
        check(L.scb_set_timing(h, 0))
        info = {"clocks": clk, "launches": L.scb_kernel_launches() - launches0}
        for f in ("pack_ms", "insert_ms", "query_ms", "cut_ms", "bucket_ms", "apply_insert_ms", "apply_query_ms"):
            info[f] = getattr(t, f) / steps
        info["report"] = (rep.valid_kmers, rep.positive_estimates, rep.estimate_checksum)
        return dist.max(ms), info

    # workload statistics for the algorithmic bytes (outside any timed region)
    st = _lib.ScbStats()
    check(L.scb_reset(h))
    check(L.scb_batch_stats(h, data.ctypes.data, offsets.ctypes.data, n_seqs, C.byref(st)))

    # autotune on a sample of the workload (first 2 M reads) outside the timed region
    tune = _lib.ScbTuning()
    if args.no_tune:
        check(L.scb_get_tuning(h, C.byref(tune)))
        tuning = dict(tune.as_dict(), sample_reads=0, seconds=0.0)
    else:
        n_tune = min(n_seqs, 2_000_000)
        t_tune = time.perf_counter()
        check(L.scb_autotune(h, data.ctypes.data, offsets.ctypes.data, n_tune, C.byref(tune)))
        tuning = dict(tune.as_dict(), sample_reads=n_tune, seconds=time.perf_counter() - t_tune)

    g0 = graph_stats(L, h)
    ms, info = timed("auto", args.steps)
    g1 = graph_stats(L, h)
    graphs = {"captures": g1[0] - g0[0], "replays": g1[1] - g0[1], "eager_redos": g1[2] - g0[2],
              "note": "every timed step is one graph replay of its batch shape (captured in warm-up)"}
    kmers = km.value
    assert rep.valid_kmers == kmers, (rep.valid_kmers, kmers)
    all_kmers = dist.sum(float(kmers))
    value = all_kmers * args.steps / (ms / 1e3)
    reference_report = info["report"]

    strategies = {}
    for name in ([] if args.no_plain else ["plain", "fused", "grouped"]):
        s_steps = max(1, args.steps // 2)
        sms, sinfo = timed(name, s_steps)
        assert sinfo["report"] == reference_report, (name, sinfo["report"], reference_report)
        strategies[name] = {"value": all_kmers * s_steps / (sms / 1e3), "ms_per_step": sms / s_steps,
                            "insert_ms": sinfo["insert_ms"], "query_ms": sinfo["query_ms"]}
    check(L.scb_set_strategy(h, 0, 0))
    if not args.no_plain:
        # the tuned step with the grouped insert and query as two passes (probe slots stored by the
        # insert, read back by the query) instead of the build apply that answers each exclusive
        # bucket right after its commit
        check(L.scb_set_fused_build(h, 0))
        s_steps = max(1, args.steps // 2)
        sms, sinfo = timed("auto", s_steps)
        check(L.scb_set_fused_build(h, 1))
        assert sinfo["report"] == reference_report, ("two-pass", sinfo["report"], reference_report)
        strategies["auto_two_pass"] = {"value": all_kmers * s_steps / (sms / 1e3), "ms_per_step": sms / s_steps,
                                       "insert_ms": sinfo["insert_ms"], "query_ms": sinfo["query_ms"],
                                       "apply_insert_ms": sinfo["apply_insert_ms"],
                                       "apply_query_ms": sinfo["apply_query_ms"]}
    plain = None
    if "plain" in strategies:
        plain = dict(strategies["plain"], unit="k-mers/s", batched_over_plain=value / strategies["plain"]["value"])

    e2e = None
    if not args.no_e2e:
        p_data = torch.from_numpy(data).pin_memory()
        p_off = torch.from_numpy(offsets.view(np.int64)).pin_memory()
        h2d = C.c_uint64(0)

        def e2e_steps():
            """Timed steps through the host entry point; returns (k-mers/s, bytes copied last step)."""
            times = []
            h2d_before = 0
            for i in range(args.warmup + args.steps):
                check(L.scb_reset(h))
                torch.cuda.synchronize()
                dist.barrier()
                check(L.scb_h2d_bytes(h, C.byref(h2d)))
                h2d_before = h2d.value
                t0 = time.perf_counter()
                check(L.scb_build_and_stream_query(h, p_data.data_ptr(), p_off.data_ptr(), n_seqs, C.byref(km),
                                                   C.byref(sm), C.byref(rep)))
                dt = time.perf_counter() - t0
                if i >= args.warmup:
                    times.append(dist.max(dt))
            assert (rep.valid_kmers, rep.positive_estimates, rep.estimate_checksum) == reference_report
            check(L.scb_h2d_bytes(h, C.byref(h2d)))
            return all_kmers * len(times) / sum(times), h2d.value - h2d_before

        # the letters copied and packed on the device, for comparison; then the default: the reads
        # packed on the host (3 bits per base) while the GPU works on the previous piece
        check(L.scb_set_host_pack(h, 0))
        letters_value, letters_h2d = e2e_steps()
        check(L.scb_set_host_pack(h, 1))
        e2e_value, e2e_h2d = e2e_steps()
        # h2d: the library's own count of the bytes it copied in the last step
        e2e = {"value": e2e_value, "unit": "k-mers/s", "h2d_bytes_per_step": e2e_h2d,
               "d2h_bytes_per_step": 2 * (16 * 8 + 4) + 8, "host_input_bytes_per_step": n_bytes + (n_seqs + 1) * 8,
               "without_host_pack": {"value": letters_value, "h2d_bytes_per_step": letters_h2d}}

    # roofline of the dominant kernel of the timed step.  Algorithmic bytes follow the design the
    # kernel implements: the grouped kernels stage each touched counter block once per bucket, so
    # their minimum traffic is the sorted records (8 B each), the records' 2-bit bases, and each
    # touched block read (and, for the insert, written) once; the direct designs (fused tiles)
    # pay the random-32-byte-sector model (each distinct sector a super-k-mer's probes hit, read
    # and for the insert written, per super-k-mer).
    peak, peak_kind = measured_peaks()
    R = float(st.super_kmers)
    sector_bytes = 32.0 * st.sectors
    packed = n_bytes / 4.0
    model_insert = 2.0 * sector_bytes + packed
    model_query = sector_bytes + packed
    touched = occupied(R, float(1 << (GEOM["counter_slots_exponent"] - GEOM["block_slots_exponent"])))
    block_bytes = (1 << GEOM["block_slots_exponent"]) * (GEOM["counter_bits"] // 8)
    gather = (st.windows + R * (GEOM["k"] - 1)) / 4.0
    staged_insert = 8 * R + gather + 2 * touched * block_bytes
    staged_query = 8 * R + gather + touched * block_bytes
    grouped_step = info["cut_ms"] > 0
    # (time, algorithmic bytes, random-sector model bytes or None, work units, unit name)
    # with the build apply (the default), the insert apply's span is the build apply (insert, commit
    # and the query of every exclusive bucket from shared memory) and the query apply's span only
    # covers the items it deferred (split buckets)
    kernels = {
        "k_apply<build>": (info["apply_insert_ms"], staged_insert, model_insert + model_query, float(st.smers),
                           "s-mer"),
        "k_apply<query, deferred items>": (info["apply_query_ms"], 0.0, None, 0.0, "s-mer"),
        # the cut reads the 2-bit codes and both bitmaps once and writes an 8-byte record and a
        # 16-byte base entry per super-k-mer
        "k_tiles<cut>": (info["cut_ms"], n_bytes / 2 + 24 * R, None, float(st.windows), "window"),
        # pack: ASCII read once, codes (2 bits) and the two bitmaps (1 bit each) written
        "k_pack": (info["pack_ms"], n_bytes * 1.5, None, float(n_bytes), "base"),
        "k_tiles<insert>": (0.0 if grouped_step else info["insert_ms"], model_insert, model_insert,
                            float(st.smers), "s-mer"),
        "k_tiles<report>": (0.0 if grouped_step else info["query_ms"], model_query, model_query,
                            float(st.smers), "s-mer"),
    }
    dom = max((k_ for k_ in kernels if k_ != "k_pack"), key=lambda k_: kernels[k_][0])
    dom_ms, alg, model, units, unit = kernels[dom]
    achieved = alg / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
    prof = profile_traffic() or {}
    kprof = prof.get("kernels", {}).get(dom, {})
    src_hash = kernel_source_hash()
    fresh = bool(kprof) and prof.get("source_hash") == src_hash
    step_bytes = sum(v[1] for v in kernels.values() if v[0] > 0)
    step_s = ms / args.steps / 1e3
    issue = None
    if fresh and kprof.get("warp_instructions_per_unit"):
        # instruction-issue roofline: 4 schedulers x 148 SMs issue one warp instruction per clock
        wipu = kprof["warp_instructions_per_unit"]
        sm_mhz = info["clocks"].get("sm_mhz") or 1965.0
        issue_rate = 4 * 148 * sm_mhz * 1e6
        issue = {"unit": unit, "warp_instructions_per_unit": wipu,
                 "thread_instructions_per_unit": 32 * wipu,
                 "floor_thread_instructions_per_unit": kprof.get("floor_thread_instructions_per_unit"),
                 "floor_note": kprof.get("floor_note"),
                 "issue_bound_ms": units * wipu / issue_rate * 1e3,
                 "frac": (units * wipu / issue_rate) / (dom_ms / 1e3) if dom_ms > 0 else None,
                 "source": prof.get("source_small")}

    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "algorithmic_bytes": alg, "kernel_ms": dom_ms,
                "algorithmic_model": ("grouped design minimum: 8 B record + 2-bit bases per super-k-mer, each "
                                      "touched 1 KiB block read (and written, insert) once"
                                      if dom.startswith("k_apply") else
                                      "direct design: 32 B per distinct sector per super-k-mer (x2 insert) + "
                                      "2-bit reads"),
                # measured DRAM bytes per launch from the committed ncu capture, only while the
                # kernel sources are the ones that capture measured
                "traffic": kprof.get("dram_bytes_per_launch") if fresh else None,
                "traffic_source": (prof.get("source") if fresh else
                                   f"stale or absent (capture of sources {prof.get('source_hash')}, "
                                   f"these are {src_hash})"),
                "traffic_frac": (kprof["dram_bytes_per_launch"] / (dom_ms / 1e3) / 1e9 / peak)
                if fresh and kprof.get("dram_bytes_per_launch") and dom_ms > 0 else None,
                "limiter": kprof.get("limiter") if fresh else None,
                "issue": issue,
                "random_sector_model": None if model is None else {
                    "bytes": model, "frac": model / (dom_ms / 1e3) / 1e9 / peak if dom_ms > 0 else None,
                    "note": "the per-super-k-mer sector model of a direct design; the grouped kernels stage "
                            "each block once per bucket and are not bound by it"},
                # every kernel's algorithmic bytes of one step over the step time: at most the peak
                "step_check": {"algorithmic_bytes": step_bytes, "gbs": step_bytes / step_s / 1e9,
                               "frac": step_bytes / step_s / 1e9 / peak},
                "kernels": {k_: {"ms": v[0], "algorithmic_bytes": v[1],
                                 "frac": (v[1] / (v[0] / 1e3) / 1e9 / peak) if v[0] > 0 else None}
                            for k_, v in kernels.items() if v[0] > 0},
                "sectors_per_superkmer": st.sectors / max(st.super_kmers, 1),
                "super_kmers": st.super_kmers, "smers": st.smers, "windows": st.windows,
                "touched_blocks": touched}

    del d_data, d_off
    spectrum = None
    if not args.no_spectrum:
        spectrum = {"config2": run_spectrum(L, h, data, offsets, st, GEOM["counter_slots_exponent"])}
        # configuration 1: 1 Mbp genome, 30x of 150 bp reads, 2^24 slots (the table fits in L2)
        from scbf_b200 import workloads as wl

        d1, o1 = wl.config1()
        cfg1 = api.SuperCountingBloomConfig(k=GEOM["k"], m=GEOM["m"], s=GEOM["s"], n_hashes=GEOM["n_hashes"],
                                            counter_bits=api.CounterBits(16), counter_slots_exponent=24,
                                            block_slots_exponent=GEOM["block_slots_exponent"], threads=1, queue=4096)
        c1 = api._create(cfg1)
        st1 = _lib.ScbStats()
        check(L.scb_batch_stats(c1.h, d1.ctypes.data, o1.ctypes.data, len(o1) - 1, C.byref(st1)))
        k1, s1 = C.c_uint64(0), C.c_uint64(0)
        check(L.scb_insert_batch(c1.h, d1.ctypes.data, o1.ctypes.data, len(o1) - 1, C.byref(k1), C.byref(s1)))
        check(L.scb_freeze(c1.h))
        spectrum["config1"] = run_spectrum(L, c1.h, d1, o1, st1, 24)
        c1.close()
    config1 = run_config1(L, args) if dist.world == 1 else None
    serving = None
    if not args.no_serve:
        check(L.scb_set_strategy(h, 0, 0))
        serving = run_serving(ctx, args, dist.rank)
    ctx.close()
    mixed = None if args.no_mixed else run_mixed(args, dist)

    cpu = None
    if not args.no_cpu and dist.rank == 0 and dist.world == 1:
        n = min(CPU_SAMPLE_READS, n_seqs)
        f, threads = cpu_filter()
        dt, ckm, _ = cpu_port_run(data, offsets, 0, n, f)
        f.close()
        cpu = {"value": ckm / dt, "unit": "k-mers/s", "cores": threads, "kind": "port",
               "sample": f"first {n} reads ({ckm} k-mers), build + stream query, on a cleared, pre-touched "
                         f"2 GiB table (no page faults in the timed region)"}

    if dist.rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "k-mers/s", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16", "data": "synthetic",
            "config": {"workload": WORKLOAD + (f" (genome scale {args.scale})" if args.scale != 1.0 else ""),
                       "reads": n_seqs, "bytes": n_bytes, "kmers_per_step": kmers,
                       "l2": "inputs larger than L2 (2 GB of reads, 2 GiB table)",
                       "parallelism": f"replicas x{dist.world}", "strategy": "auto"},
            "insert_kmers_per_s": kmers / (info["insert_ms"] / 1e3),
            "query_kmers_per_s": kmers / (info["query_ms"] / 1e3),
            "stage_ms": {k_: info[k_] for k_ in ("pack_ms", "insert_ms", "query_ms", "cut_ms", "bucket_ms",
                                                 "apply_insert_ms", "apply_query_ms")},
            "tuning": tuning, "graphs": graphs,
            "plain": plain, "strategies": strategies, "mixed": mixed, "serve": serving, "config1": config1,
            "e2e": e2e,
            "spectrum": spectrum,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": info["clocks"], "gpu_launches": info["launches"],
        }
        print(json.dumps(line), flush=True)


def run_spectrum(L, h, data, offsets, st, slot_exp: int, reps: int = 2) -> dict:
    """estimate_distinct_kmers + spectrum_from_estimates (src/fastx.rs:255-308, 392-410) on the
    frozen index h over the given reads, through the host entry point scb_spectrum_distinct (reads
    copied to the device inside the call), with the grouped strategy (the spectrum apply) and the
    fused tile kernel (one global key-set insert per window).  Algorithmic bytes of the spectrum
    apply: per super-k-mer its 8-byte record and 2-bit bases, each touched block read once; the
    keys and the histogram stay on the SM (split buckets excepted)."""
    from scbf_b200 import _lib

    n = len(offsets) - 1
    peak, _ = measured_peaks()
    out = {}
    ref_rows = None
    for name in ("grouped", "fused"):
        sid = STRATEGY_IDS[name]
        assert L.scb_set_strategy(h, sid, sid) == 0
        rows, dk, qk = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
        times, dev = [], []
        for _ in range(reps + 1):
            assert L.scb_set_timing(h, 1) == 0
            t0 = time.perf_counter()
            if L.scb_spectrum_distinct(h, data.ctypes.data, offsets.ctypes.data, n, None, None, 0, C.byref(rows),
                                       C.byref(dk), C.byref(qk)) != 0:
                raise RuntimeError(_lib.last_error())
            times.append(time.perf_counter() - t0)
            t = _lib.ScbTimings()
            assert L.scb_get_timings(h, C.byref(t)) == 0
            dev.append(t.pack_ms + t.query_ms)
        assert L.scb_set_timing(h, 0) == 0
        vals, cnts = np.zeros(max(rows.value, 1), np.uint64), np.zeros(max(rows.value, 1), np.uint64)
        L.scb_spectrum_distinct(h, data.ctypes.data, offsets.ctypes.data, n, vals.ctypes.data, cnts.ctypes.data,
                                rows.value, C.byref(rows), C.byref(dk), C.byref(qk))
        got = list(zip(vals[: rows.value].tolist(), cnts[: rows.value].tolist()))
        if ref_rows is None:
            ref_rows = got
        assert got == ref_rows, ("spectrum rows differ between strategies", name)
        wall = min(times[1:])
        dms = min(dev[1:])
        out[name] = {"kmers_per_s": qk.value / wall, "seconds": wall, "device_ms": dms,
                     "device_kmers_per_s": qk.value / (dms / 1e3) if dms > 0 else None}
    assert L.scb_set_strategy(h, 0, 0) == 0
    R = float(st.super_kmers)
    touched = occupied(R, float(1 << (slot_exp - GEOM["block_slots_exponent"])))
    block_bytes = (1 << GEOM["block_slots_exponent"]) * (GEOM["counter_bits"] // 8)
    alg = 8 * R + (st.windows + R * (GEOM["k"] - 1)) / 4.0 + touched * block_bytes + int(offsets[-1]) * 1.5
    gms = out["grouped"]["device_ms"]
    out.update({"queried_kmers": qk.value, "distinct_kmers": dk.value, "rows": rows.value,
                "grouped_over_fused": out["grouped"]["kmers_per_s"] / out["fused"]["kmers_per_s"],
                "roofline": {"bound": "hbm", "algorithmic_bytes": alg, "device_ms": gms,
                             "achieved_gbs": alg / (gms / 1e3) / 1e9 if gms else None,
                             "frac": alg / (gms / 1e3) / 1e9 / peak if gms else None,
                             "model": "pack (1.5 B per base) + per super-k-mer an 8-byte record and its 2-bit "
                                      "bases + each touched block read once; keys and histogram stay in shared "
                                      "memory"}})
    return out


def run_config1(L, args) -> dict:
    """Configuration 1 (1 Mbp genome, 30x of 150 bp reads, 2^24 16-bit slots: the 32 MiB table fits
    in L2), the same build + stream query step on reads resident in HBM, CUDA events on the stream.
    With the counters in L2 the rate is also given as counter updates per second (s-mers x
    n_hashes), the L2-atomic figure the configuration asks for."""
    import torch

    from scbf_b200 import _lib, api
    from scbf_b200 import workloads as wl

    d1, o1 = wl.config1()
    cfg1 = api.SuperCountingBloomConfig(k=GEOM["k"], m=GEOM["m"], s=GEOM["s"], n_hashes=GEOM["n_hashes"],
                                        counter_bits=api.CounterBits(16), counter_slots_exponent=24,
                                        block_slots_exponent=GEOM["block_slots_exponent"], threads=1, queue=4096)
    c1 = api._create(cfg1)
    dd = torch.from_numpy(d1).cuda()
    do = torch.from_numpy(o1.view(np.int64)).cuda()
    n, nb = len(o1) - 1, int(o1[-1])
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    km, sm = C.c_uint64(0), C.c_uint64(0)
    rep = _lib.ScbReport()

    def check(st):
        if st != 0:
            raise RuntimeError(_lib.last_error())

    def step():
        check(L.scb_reset(c1.h))
        check(L.scb_build_and_stream_query_device(c1.h, dd.data_ptr(), do.data_ptr(), n, nb, sp, C.byref(km),
                                                  C.byref(sm), C.byref(rep)))

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    steps = 20
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    c1.close()
    return {"workload": "configuration 1: 1 Mbp uniform genome, 30x of 150 bp reads (200 000 reads), 0.5% "
                        "substitutions; 2^24 16-bit slots (32 MiB, resident in L2)",
            "kmers": km.value, "smers": sm.value, "ms_per_step": ms, "kmers_per_s": km.value / (ms / 1e3),
            "counter_updates_per_s": sm.value * GEOM["n_hashes"] / (ms / 1e3),
            "note": "build + stream query per step, reads resident in HBM; the step includes the table clear"}


def run_serving(ctx, args, rank: int) -> dict:
    """Config-5 shape on the resident config-2 index: requests of sequences, half drawn from the
    indexed genome (1% errors) and half uniform random, arriving as a Poisson process.

    - 1 M-k-mer requests (40 sequences of 25 kbp, the p99 < 10 ms target) at offered rates from
      100 req/s up, until the knee (served k-mers/s below 90% of the offered load, or p99 above
      100 ms), through the continuous-batching server;
    - the same requests and rates through the unbatched path: one scb_query_batch per request,
      in arrival order, no overlap (the plain per-request GPU path);
    - mixed requests, 1-10^5 sequences of log-uniform 100 bp-50 kbp (about 90 Mbp and 820 MB of
      per-window output on average, uncapped), at rates up to their knee;
    - the whole-stream distinct-k-mer spectrum, read from the server's set at the end of the 1 M
      stream and checked against the spectrum of the same sequences in one batch."""
    import threading

    from scbf_b200 import _lib, workloads

    L = _lib.load()
    genome = workloads.random_genome(int(100_000_000 * args.scale), seed=1 + rank)
    rng = np.random.default_rng(17)

    def pool_fixed(count):
        return [workloads.random_sequences(40, 25_000, 25_001, seed=1000 + i, genome=genome) for i in range(count)]

    def pool_mixed(count):
        # its own generator: the pool does not depend on how many rates the sweeps before it ran
        prng = np.random.default_rng(19)
        reqs = []
        for i in range(count):
            n = int(np.exp(prng.uniform(0, np.log(1e5))))
            reqs.append(workloads.random_sequences(n, 100, 50_000, seed=2000 + i, genome=genome))
        return reqs

    def outputs(reqs):
        outs = []
        for d, o in reqs:
            nw = int(L.scb_count_windows(ctx.h, o.ctypes.data, len(o) - 1))
            outs.append((np.empty(max(nw, 1), np.uint64), np.empty(max(nw, 1), np.uint8), nw))
        return outs

    def schedule(rate, seconds, n_pool):
        n_req = max(20, int(round(rate * seconds)))
        return np.cumsum(rng.exponential(1.0 / rate, n_req)), rng.integers(0, n_pool, n_req)

    def summarise(lat_ms, kmers, span_s, rate, extra):
        lat = np.sort(np.asarray(lat_ms))
        return dict({"rate_req_s": rate, "requests": int(lat.size), "p50_ms": float(np.percentile(lat, 50)),
                     "p99_ms": float(np.percentile(lat, 99)), "max_ms": float(lat[-1]),
                     "kmers_per_s": kmers / span_s if span_s > 0 else None,
                     "offered_kmers_per_s": None}, **extra)

    def stream(srv, reqs, outs, rate, seconds):
        """Poisson arrivals into the server; requests of one template share output buffers."""
        arrivals, pick = schedule(rate, seconds, len(reqs))
        L.scb_server_reset_stats(srv)
        tickets = []
        lock = threading.Lock()
        done = threading.Event()

        def waiter():
            i = 0
            while i < len(arrivals):
                with lock:
                    t = tickets[i] if i < len(tickets) else None
                if t is None:
                    time.sleep(0.0001)
                    continue
                L.scb_server_wait(srv, t, None)
                i += 1
            done.set()

        wt = threading.Thread(target=waiter)
        wt.start()
        t0 = time.perf_counter()
        for a_, j in zip(arrivals, pick):
            delay = t0 + a_ - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            d, o = reqs[j]
            ob, vb, _ = outs[j]
            t = C.c_uint64(0)
            if L.scb_server_submit(srv, d.ctypes.data, o.ctypes.data, len(o) - 1, ob.ctypes.data, vb.ctypes.data,
                                   C.byref(t)) != 0:
                raise RuntimeError(_lib.last_error())
            with lock:
                tickets.append(t.value)
        wt.join()
        sm = _lib.ScbServerSummary()
        L.scb_server_get_summary(srv, C.byref(sm))
        mean_k = float(np.mean([outs[j][2] for j in pick]))
        return {"rate_req_s": rate, "requests": sm.requests, "p50_ms": sm.p50_ms, "p99_ms": sm.p99_ms,
                "mean_ms": sm.mean_ms, "max_ms": sm.max_ms,
                "kmers_per_s": sm.windows / sm.span_s if sm.span_s else None,
                "offered_kmers_per_s": rate * mean_k, "batches": sm.batches, "slots": sm.slots,
                "mean_kmers_per_request": mean_k}

    def per_request(reqs, outs, rate, seconds):
        """The unbatched path: requests answered one at a time, in arrival order, each by one
        scb_query_batch call (host buffers, H2D and D2H inside it)."""
        arrivals, pick = schedule(rate, seconds, len(reqs))
        lat, kmers = [], 0
        t0 = time.perf_counter()
        for a_, j in zip(arrivals, pick):
            delay = t0 + a_ - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            d, o = reqs[j]
            ob, vb, nw = outs[j]
            if L.scb_query_batch(ctx.h, d.ctypes.data, o.ctypes.data, len(o) - 1, ob.ctypes.data,
                                 vb.ctypes.data) != 0:
                raise RuntimeError(_lib.last_error())
            lat.append((time.perf_counter() - t0 - a_) * 1e3)
            kmers += nw
        span = time.perf_counter() - t0
        mean_k = float(np.mean([outs[j][2] for j in pick]))
        return summarise(lat, kmers, span, rate, {"offered_kmers_per_s": rate * mean_k,
                                                  "mean_kmers_per_request": mean_k})

    def knee(r):
        return (r["kmers_per_s"] or 0) < 0.9 * r["offered_kmers_per_s"] or r["p99_ms"] > 100.0

    def server(reqs, max_batch_bytes, spectrum_keys=0):
        cfg = _lib.ScbServerConfig(16 << 30, max_batch_bytes, 0, 4, 0, spectrum_keys)
        srv = C.c_void_p(0)
        if L.scb_server_create(ctx.h, C.byref(cfg), C.byref(srv)) != 0:
            raise RuntimeError(_lib.last_error())
        outs = outputs(reqs)
        for (d, o), (ob, vb, _) in zip(reqs, outs):  # warm-up: every template once (graph captures)
            t = C.c_uint64(0)
            L.scb_server_submit(srv, d.ctypes.data, o.ctypes.data, len(o) - 1, ob.ctypes.data, vb.ctypes.data,
                                C.byref(t))
            L.scb_server_wait(srv, t.value, None)
        return srv, outs

    out = {"index": "config-2 frozen index, resident",
           "arrivals": "Poisson; requests drawn from a pool of generated templates (results of one template "
                       "share an output buffer, checked against a direct query after the sweep)"}
    # 1 M-k-mer requests: batched server (with the whole-stream spectrum) vs unbatched
    fixed = pool_fixed(16)
    srv, outs = server(fixed, 16 << 20, spectrum_keys=64 << 20)
    sweep = []
    for rate in (100, 300, 1000, 3000, 10000):
        r = stream(srv, fixed, outs, rate, seconds=2.0)
        sweep.append(r)
        if knee(r):
            break
    # every template's output buffer holds the answer of its last request: it must equal one direct
    # per-window query of the same sequences
    for (d, o), (ob, vb, nw) in zip(fixed, outs):
        eo, ev = np.zeros(max(nw, 1), np.uint64), np.zeros(max(nw, 1), np.uint8)
        if L.scb_query_batch(ctx.h, d.ctypes.data, o.ctypes.data, len(o) - 1, eo.ctypes.data, ev.ctypes.data) != 0:
            raise RuntimeError(_lib.last_error())
        assert np.array_equal(vb[:nw], ev[:nw]) and np.array_equal(np.where(ev[:nw] == 1, ob[:nw], 0),
                                                                   np.where(ev[:nw] == 1, eo[:nw], 0)), "served results"
    t_sp = time.perf_counter()
    rows, dk, qk = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
    if L.scb_server_spectrum(srv, None, None, 0, C.byref(rows), C.byref(dk), C.byref(qk)) != 0:
        raise RuntimeError(_lib.last_error())
    vals, cnts = np.zeros(max(rows.value, 1), np.uint64), np.zeros(max(rows.value, 1), np.uint64)
    L.scb_server_spectrum(srv, vals.ctypes.data, cnts.ctypes.data, rows.value, C.byref(rows), C.byref(dk),
                          C.byref(qk))
    spectrum_ms = (time.perf_counter() - t_sp) * 1e3
    # the same spectrum from one batch of the pool's sequences (each template is in the stream)
    from scbf_b200 import api

    seqs = [bytes(d[int(o[i]):int(o[i + 1])]) for d, o in fixed for i in range(len(o) - 1)]
    bd, bo = api.pack_sequences(seqs)
    ref = api.SuperCountingBloomIndex._from_ctx(ctx, None, 0).spectrum_distinct(bd, bo)
    assert ref["rows"] == list(zip(vals[: rows.value].tolist(), cnts[: rows.value].tolist())), "stream spectrum"
    assert ref["distinct_keys"] == dk.value
    L.scb_server_destroy(srv)
    out["one_mkmer_requests"] = {"server": sweep, "knee_rate_req_s": sweep[-1]["rate_req_s"] if knee(sweep[-1])
                                 else None,
                                 "whole_stream_spectrum": {"distinct_kmers": dk.value, "queried_kmers": qk.value,
                                                           "rows": rows.value, "read_ms": spectrum_ms,
                                                           "equals_one_batch_spectrum": True}}
    plain = []
    for rate in (100, 300, 1000, 3000, 10000):
        r = per_request(fixed, outs, rate, seconds=1.0)
        plain.append(r)
        if knee(r):
            break
    out["one_mkmer_requests"]["per_request_unbatched"] = plain
    # the same server without graph replays, at the highest rate below the knee
    ok = [r["rate_req_s"] for r in sweep if not knee(r)] or [100]
    L.scb_set_graphs(ctx.h, 0)
    srv, outs = server(fixed, 16 << 20)
    out["one_mkmer_requests"]["server_without_graphs"] = stream(srv, fixed, outs, ok[-1], seconds=2.0)
    L.scb_server_destroy(srv)
    L.scb_set_graphs(ctx.h, 1)
    del outs
    # mixed requests, uncapped
    mixed = pool_mixed(12)
    srv, mouts = server(mixed, 64 << 20)
    msweep = []
    # heavy-tailed requests (the largest are hundreds of Mbp): each rate runs at least 40 requests,
    # and the sweep stops once p99 passes 2 s
    for rate in (2, 5, 10, 20, 50):
        r = stream(srv, mixed, mouts, rate, seconds=40.0 / rate)
        msweep.append(r)
        if r["p99_ms"] > 2000.0:
            break
    L.scb_server_destroy(srv)
    out["mixed_requests"] = {"server": msweep, "pool_requests": len(mixed),
                             "pool_mean_bytes": float(np.mean([int(o[-1]) for _, o in mixed])),
                             "pool_max_sequences": int(max(len(o) - 1 for _, o in mixed))}
    return out


MIXED_WORKLOAD = ("mixed lengths: 200 Mbp uniform genome at 15x; 70% of bases from 150 bp reads (1% "
                  "substitutions), 30% from log-normal long reads (median 10 kbp, 1-100 kbp, 5% errors, "
                  "sub:ins:del = 2:1:1); default geometry with 2^31 16-bit slots (4 GiB)")


def run_mixed(args, dist: Dist) -> dict:
    """Config-4 shape: insert then query every read of an uneven-length workload, in device
    batches of at most 1.6 GB, per strategy.  Returns k-mers/s per strategy."""
    import torch

    from scbf_b200 import _lib, api, workloads

    L = _lib.load()
    data, offsets = workloads.config4(seed=7 + dist.rank, scale=args.scale)
    # split into batches of whole reads of at most 1.6 GB
    cuts = [0]
    limit = 1_600_000_000
    while int(offsets[-1]) - int(offsets[cuts[-1]]) > limit:
        cuts.append(int(np.searchsorted(offsets, offsets[cuts[-1]] + limit, side="right")) - 1)
    cuts.append(len(offsets) - 1)
    batches = []
    for a, b in zip(cuts[:-1], cuts[1:]):
        o = (offsets[a:b + 1] - offsets[a]).astype(np.uint64)
        d = data[int(offsets[a]):int(offsets[b])]
        batches.append((torch.from_numpy(d).to("cuda"), torch.from_numpy(o.view(np.int64)).to("cuda"), b - a,
                        int(o[-1])))
    del data
    cfg = api.SuperCountingBloomConfig(k=GEOM["k"], m=GEOM["m"], s=GEOM["s"], n_hashes=GEOM["n_hashes"],
                                       counter_bits=api.CounterBits(16), counter_slots_exponent=31,
                                       block_slots_exponent=GEOM["block_slots_exponent"], threads=1, queue=4096)
    ctx = api._create(cfg)
    h = ctx.h
    km, sm = C.c_uint64(0), C.c_uint64(0)
    rep = _lib.ScbReport()

    def check(st):
        if st != 0:
            raise RuntimeError(_lib.last_error())

    def step():
        check(L.scb_reset(h))
        total = 0
        for d, o, n, nb in batches:
            check(L.scb_insert_batch_device(h, d.data_ptr(), o.data_ptr(), n, nb, None, C.byref(km), C.byref(sm)))
            total += km.value
        check(L.scb_freeze(h))
        chk = 0
        for d, o, n, nb in batches:
            check(L.scb_query_report_device(h, d.data_ptr(), o.data_ptr(), n, nb, None, C.byref(rep)))
            chk = (chk + rep.estimate_checksum) % (1 << 64)
        return total, chk

    out = {"workload": MIXED_WORKLOAD + (f" (genome scale {args.scale})" if args.scale != 1.0 else ""),
           "reads": int(len(offsets) - 1), "bytes": int(offsets[-1]), "batches": len(batches)}
    ref = None
    for name in ("plain", "fused", "grouped", "auto"):
        sid = STRATEGY_IDS[name]
        check(L.scb_set_strategy(h, sid, sid))
        steps = max(1, args.steps // 2)
        for _ in range(min(args.warmup, 2)):
            res = step()
        torch.cuda.synchronize()
        dist.barrier()
        t0 = time.perf_counter()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(steps):
            res = step()
        ev1.record()
        torch.cuda.synchronize()
        ms = dist.max(ev0.elapsed_time(ev1))
        if ref is None:
            ref = res
        assert res == ref, (name, res, ref)
        out[name] = dist.sum(float(res[0])) * steps / (ms / 1e3)
    # the same tuned strategies with every batch launched eagerly (no graph replays)
    check(L.scb_set_strategy(h, 0, 0))
    check(L.scb_set_graphs(h, 0))
    for _ in range(min(args.warmup, 2)):
        step()
    torch.cuda.synchronize()
    dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(max(1, args.steps // 2)):
        res = step()
    ev1.record()
    torch.cuda.synchronize()
    ms = dist.max(ev0.elapsed_time(ev1))
    assert res == ref, ("auto without graphs", res, ref)
    out["auto_without_graphs"] = dist.sum(float(res[0])) * max(1, args.steps // 2) / (ms / 1e3)
    check(L.scb_set_graphs(h, 1))
    out["kmers_per_step"] = ref[0]
    out["batched_over_plain"] = out["auto"] / out["plain"]
    ctx.close()
    return out


def run_profile_case(args):
    """One insert + one stream query with the chosen strategy, for ncu: by default genome scale 0.1
    (200 MB of reads) on the 2 GiB table; with --profile-scale 0.25 --profile-slots 28 (500 MB of
    reads, a 512 MiB table) the workload has the full run's records per block and bucket, so its
    per-unit instruction and DRAM figures scale to the full 2 Gbp step by the units processed."""
    import torch

    from scbf_b200 import _lib, api

    L = _lib.load()
    data, offsets = workload(0, args.profile_scale)
    cfg = api.SuperCountingBloomConfig(k=GEOM["k"], m=GEOM["m"], s=GEOM["s"], n_hashes=GEOM["n_hashes"],
                                       counter_bits=api.CounterBits(GEOM["counter_bits"]),
                                       counter_slots_exponent=args.profile_slots,
                                       block_slots_exponent=GEOM["block_slots_exponent"], threads=1, queue=4096)
    ctx = api._create(cfg)
    sid = STRATEGY_IDS[args.profile_case]
    assert L.scb_set_strategy(ctx.h, sid, sid) == 0
    d_data = torch.from_numpy(data).to("cuda")
    d_off = torch.from_numpy(offsets.view(np.int64)).to("cuda")
    km, sm = C.c_uint64(0), C.c_uint64(0)
    rep = _lib.ScbReport()
    n = len(offsets) - 1
    assert L.scb_build_and_stream_query_device(ctx.h, d_data.data_ptr(), d_off.data_ptr(), n, int(offsets[-1]),
                                               None, C.byref(km), C.byref(sm), C.byref(rep)) == 0, _lib.last_error()
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": args.profile_case, "kmers": km.value, "smers": sm.value,
                      "checksum": rep.estimate_checksum}), flush=True)
    ctx.close()


def main():
    args = parse()
    if args.profile_case:
        run_profile_case(args)
        return
    dist = Dist(args.gpus)
    if dist.world > 1:
        # the single-GPU characterisations (serving, mixed lengths, spectrum, configuration 1) run at
        # N = 1; with N replicas every rank times the step, its strategies and the end-to-end call
        args.no_serve = args.no_mixed = args.no_spectrum = True
    try:
        if args.impl == "reference":
            run_reference(args, dist)
        else:
            run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
