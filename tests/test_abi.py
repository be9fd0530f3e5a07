"""C-ABI checks that need no GPU: the library loads, exports every symbol include/scb.h declares,
validates configs with the reference's rules, and refuses compute without a device."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from scbf_b200 import _lib, build

    build.build()
    return _lib.load()


def _has_gpu() -> bool:
    if shutil.which("nvidia-smi") is None:
        return False
    return subprocess.run(["nvidia-smi", "-L"], capture_output=True).returncode == 0


def test_exports_every_declared_symbol(lib):
    from scbf_b200 import _lib

    declared = _lib.declared_symbols()
    assert len(declared) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing


def test_header_compiles_as_c_and_cpp(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "scb.h"\nint main(void){scb_config c; return scb_config_default(&c) != SCB_OK;}\n')
    for comp, name in (("gcc", "t.c"), ("g++", "t.cpp")):
        f = tmp_path / name
        f.write_text(src.read_text())
        r = subprocess.run([comp, "-c", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(f), "-o",
                            str(tmp_path / (name + ".o"))], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_default_config_matches_reference(lib):
    # src/config.rs:33-47
    from scbf_b200 import _lib

    c = _lib.ScbConfig()
    assert lib.scb_config_default(C.byref(c)) == 0
    assert (c.k, c.m, c.s, c.n_hashes, c.counter_bits, c.counter_slots_exponent, c.block_slots_exponent,
            c.queue) == (31, 21, 25, 4, 16, 30, 9, 4096)
    assert c.threads >= 1


def test_validation_matches_reference(known_answers):
    # tests/pipeline_matrix.rs:187-262 through the C ABI
    import scbf_b200 as s

    vr = known_answers["validation_rejections"]
    base = dict(known_answers["configs"][vr["base"]])
    base.pop("_cite")
    base["counter_bits"] = s.CounterBits(base["counter_bits"])
    s.SuperCountingBloomConfig(**base).validate()
    for case in vr["cases"]:
        with pytest.raises(s.InvalidConfig):
            s.SuperCountingBloomConfig(**{**base, **case}).validate()


def test_validation_messages_are_the_references(lib):
    import scbf_b200 as s

    cases = {
        "k must be in 1..=32": dict(k=0),
        "canonical SIMD minimizers require odd k": dict(k=30, m=21, s=25),
        "n_hashes must be positive": dict(n_hashes=0),
        "block_slots_exponent must be smaller than counter_slots_exponent": dict(block_slots_exponent=30),
        "threads must be positive": dict(threads=0),
        "queue must be positive": dict(queue=0),
    }
    for msg, over in cases.items():
        with pytest.raises(s.InvalidConfig, match=msg):
            s.SuperCountingBloomConfig(**over).validate()


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_fails_loudly(lib):
    import scbf_b200 as s

    with pytest.raises(s.InternalState, match="no CUDA device"):
        s.SuperCountingBloomBuilder(s.SuperCountingBloomConfig(counter_slots_exponent=16))


def test_load_rejects_bad_files_without_device(tmp_path, lib):
    # magic / version / trailing checks happen before any device allocation (api.rs:416-431)
    import scbf_b200 as s

    bad = tmp_path / "bad.scb"
    bad.write_bytes(b"not an index")
    with pytest.raises(s.InvalidIndexFormat, match="magic"):
        s.SuperCountingBloomIndex.load(bad)
    v3 = tmp_path / "v3.scb"
    v3.write_bytes(b"SCBIDX\0\0" + (3).to_bytes(4, "little"))
    with pytest.raises(s.InvalidIndexFormat, match="version"):
        s.SuperCountingBloomIndex.load(v3)


def test_records_and_chunks_host_logic():
    from scbf_b200 import api

    data, offsets = api.pack_sequences([b"ACGTACGTACGT", b"ACGTNNACGTAC", b"", b"ACGT"])
    assert api._chunk_stats(data, offsets, 5) == (2, 8 + 2)
    data, offsets = api.pack_sequences([b"ACGTACGTACGTACGTACGT"] * 2)
    assert api._chunk_stats(data, offsets, 9) == (2, 24)


def test_fastx_parsing(tmp_path):
    # src/api.rs:1074-1093 record names and sequences
    import scbf_b200 as s

    p = tmp_path / "r.fa"
    p.write_bytes(b">contig_1 description\nACGTNN\n>contig_2\nTGCA\nTG\n")
    names, seqs = [], []
    s.for_each_fastx_record(p, lambda n, q: (names.append(n), seqs.append(q)))
    assert names == ["contig_1", "contig_2"] and seqs == [b"ACGTNN", b"TGCATG"]
    fq = tmp_path / "r.fq"
    fq.write_bytes(b"@q1 x\nACGT\n+\nIIII\n@\nGG\n+\nII\n")
    names, seqs = [], []
    s.for_each_fastx_record(fq, lambda n, q: (names.append(n), seqs.append(q)))
    assert names == ["q1", "record_2"] and seqs == [b"ACGT", b"GG"]


def test_workload_generators_shapes():
    from scbf_b200 import workloads

    data, offsets = workloads.short_reads(genome_len=10_000, coverage=30, read_len=150, seed=1,
                                          sub_rate=0.005)
    assert len(offsets) - 1 == 2000 and data.size == 2000 * 150
    assert set(np.unique(data).tolist()) <= set(b"ACGT")
    data, offsets = workloads.short_reads(genome_len=10_000, n_reads=1000, seed=2, n_rate=0.01)
    frac_n = float((data == ord("N")).mean())
    assert 0.005 < frac_n < 0.02
    data, offsets = workloads.mixed_reads(genome_len=200_000, coverage=2, seed=3)
    lens = np.diff(offsets.astype(np.int64))
    assert (lens == 150).any() and lens.max() >= 1000
