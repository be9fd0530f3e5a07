"""Host 2-bit packing (scb_hostpack.cpp) produces kernel (a)'s layout exactly: codes of 16 bases per
32-bit word, base g at bits 2*(g%16), code = (byte >> 1) & 3; one validity bit per base for
A/C/G/T in either case; 16 zero words after both arrays.  Checked against a numpy statement of
the layout on edge lengths, every byte value and several thread counts (no GPU needed)."""
import ctypes as C

import numpy as np
import pytest


@pytest.fixture(scope="module")
def pack():
    from scbf_b200 import _lib, build

    build.build()
    L = C.CDLL(_lib.LIB_PATH)
    fn = L.scb_internal_host_pack
    fn.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint]
    return fn


def _layout(a: np.ndarray):
    n = a.size
    g = (n + 31) // 32
    b = np.zeros(g * 32, np.uint8)
    b[:n] = a
    code = ((b >> 1) & 3).astype(np.uint64)
    u = b & 0xDF
    ok = ((u == 65) | (u == 67) | (u == 71) | (u == 84)).astype(np.uint64)
    codes = np.zeros(2 * g + 16, np.uint32)
    valid = np.zeros(g + 16, np.uint32)
    codes[: 2 * g] = (code.reshape(-1, 16) << (2 * np.arange(16)).astype(np.uint64)).sum(axis=1).astype(np.uint32)
    valid[:g] = (ok.reshape(-1, 32) << np.arange(32).astype(np.uint64)).sum(axis=1).astype(np.uint32)
    return codes, valid


@pytest.mark.parametrize("n", [0, 1, 5, 31, 32, 33, 100, 1000, 4097, (1 << 20) + 7])
def test_host_pack_matches_layout(pack, n):
    rng = np.random.default_rng(n)
    a = rng.integers(0, 256, n, dtype=np.uint8)
    mix = rng.choice(np.frombuffer(b"ACGTacgtNn", np.uint8), n)
    a = np.where(rng.random(n) < 0.8, mix, a).astype(np.uint8)
    g = (n + 31) // 32
    ref = _layout(a)
    for threads in (1, 3, 8):
        codes = np.full(2 * g + 16, 0xDEADBEEF, np.uint32)
        valid = np.full(g + 16, 0xDEADBEEF, np.uint32)
        pack(a.ctypes.data, n, codes.ctypes.data, valid.ctypes.data, threads)
        assert np.array_equal(codes, ref[0]) and np.array_equal(valid, ref[1])


def test_host_pack_every_byte_value(pack):
    a = np.arange(256, dtype=np.uint8).repeat(3)
    ref = _layout(a)
    g = (a.size + 31) // 32
    codes, valid = np.zeros(2 * g + 16, np.uint32), np.zeros(g + 16, np.uint32)
    pack(a.ctypes.data, a.size, codes.ctypes.data, valid.ctypes.data, 1)
    assert np.array_equal(codes, ref[0]) and np.array_equal(valid, ref[1])
