"""The library's one-pass FASTA/FASTQ reader (scb_fastx_read) against the oracle's line-by-line
reader (src/api.rs:893-915 record rules): the same records, headers and sequences for hand-made
edge cases, gzip input (several members included) and a seeded fuzz over the characters that
carry the line structure.  Host only: no GPU."""
import gzip

import numpy as np
import pytest

from scbf_b200 import api

CASES = [
    b"",
    b"ACGT\n",
    b">only\n",
    b">a desc\nACGT\nAC\n>b\n\n>c\nGG",
    b"junk before\n>r1\nAC\r\nGT\r\r\n>r2\r\nNNNN\n",
    b"@q1 x\nACGT\n+\nIIII\n@\nGG\n+q\n@@@@\n@q3\nA\nC\n+\n!!\n",
    b"@q\nAC\n+\n@notaheader\n>f\nTT\n",
    b">\n\n\n>x\n>y\nA\n",
    b"\r\n\r\n>z\nA\rC\nG\n",
]


def _native(path):
    seqs, offsets, headers, hoffs = api._fastx_read(str(path))
    o, h = offsets.tolist(), hoffs.tolist()
    return [(headers[h[i]:h[i + 1]].tobytes(), seqs[o[i]:o[i + 1]].tobytes()) for i in range(len(o) - 1)]


@pytest.mark.parametrize("i", range(len(CASES)))
def test_edge_cases_match_oracle(tmp_path, oracle_mod, i):
    p = tmp_path / "r.fx"
    p.write_bytes(CASES[i])
    assert _native(p) == list(oracle_mod.fastx_records(str(p)))


def test_gzip_members(tmp_path, oracle_mod):
    p = tmp_path / "r.fa.gz"
    p.write_bytes(gzip.compress(b">a\nACGT\nAC\n>b\nGG") + gzip.compress(b"TT\n@q\nCC\n+\nII\n"))
    assert _native(p) == list(oracle_mod.fastx_records(str(p)))
    assert _native(p) == [(b"a", b"ACGTAC"), (b"b", b"GGTT"), (b"q", b"CC")]


def test_fuzz_matches_oracle(tmp_path, oracle_mod):
    rng = np.random.default_rng(9)
    alphabet = np.frombuffer(b"ACGTN>@+\r\n\n\n ", np.uint8)
    for t in range(200):
        raw = rng.choice(alphabet, int(rng.integers(0, 400))).tobytes()
        p = tmp_path / f"f{t}.fx"
        p.write_bytes(raw)
        assert _native(p) == list(oracle_mod.fastx_records(str(p))), raw


def test_batch_layout_and_names(tmp_path):
    p = tmp_path / "r.fa"
    p.write_bytes(b">contig_1 description\nACGTNN\n>contig_2\nTGCA\nTG\n>\nA\n")
    data, offsets = api._read_batch(str(p))
    assert data.dtype == np.uint8 and offsets.dtype == np.uint64
    assert data.tobytes() == b"ACGTNNTGCATGA" and offsets.tolist() == [0, 6, 12, 13]
    names, seqs = [], []
    api.for_each_fastx_record(str(p), lambda n, s: (names.append(n), seqs.append(s)))
    assert names == ["contig_1", "contig_2", "record_3"] and seqs == [b"ACGTNN", b"TGCATG", b"A"]


def test_missing_file_or_directory_is_fastx_open(tmp_path):
    with pytest.raises(api.FastxOpen):
        api._fastx_read(str(tmp_path / "none.fa"))
    with pytest.raises(api.FastxOpen):
        api._fastx_read(str(tmp_path))
