"""libccs's device cube math, built for the host (tests/emul), against the CPU oracle and the
reference's golden vectors: the kernels' exact index / unrank / move / decode arithmetic is
checked on every CPU test run, before any GPU time is spent."""

from __future__ import annotations

import ctypes
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from cuda_cube_solver.cubie import MOVES_HTM, CubieState, compose
from cuda_cube_solver import native
from cuda_cube_solver.device import state_words

KINDS = ["304", "s4", "d4f", "a4t", "d4t", "d4", "a4"]


@pytest.fixture(scope="module")
def emul():
    subprocess.run(["make", "-C", str(ROOT / "tests" / "emul")], check=True, capture_output=True)
    lib = ctypes.CDLL(str(ROOT / "_build" / "emul" / "libccs_emul.so"))
    lib.emul_index.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                               ctypes.c_void_p]
    lib.emul_unrank.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    lib.emul_lower_bound.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    return lib


def _index(lib, kind, words, move=-1):
    words = np.ascontiguousarray(words, np.uint32)
    out = np.zeros(len(words), np.uint64)
    out_w = np.zeros_like(words)
    assert lib.emul_index(kind.encode(), words.ctypes.data, len(words), move, out.ctypes.data, out_w.ctypes.data) == 0
    return out, out_w


@pytest.mark.parametrize("name", KINDS)
def test_device_index_matches_reference_and_oracle(emul, oracle, host_golden, name):
    words = np.array([r["words"] for r in host_golden["states"]], np.uint32)
    idx, _ = _index(emul, name, words)
    assert np.array_equal(idx, [r["index"][name] for r in host_golden["states"]])
    oracle.set_kind(name)
    rng = np.random.default_rng(7)
    n = oracle.n_entries()
    rand = oracle.unrank(rng.integers(0, n, 3000, dtype=np.uint64))
    for m in [-1, 0, 5, 10, 17, -2, -9, -19]:
        got, _ = _index(emul, name, rand, m)
        assert np.array_equal(got, oracle.index(rand, m)), m


@pytest.mark.parametrize("name", KINDS)
def test_device_unrank_matches_oracle(emul, oracle, name):
    oracle.set_kind(name)
    n = oracle.n_entries()
    idx = np.concatenate([[0, n - 1], np.random.default_rng(8).integers(0, n, 5000, dtype=np.uint64)]).astype(np.uint64)
    out = np.zeros((len(idx), 5), np.uint32)
    assert emul.emul_unrank(name.encode(), idx.ctypes.data, len(idx), out.ctypes.data) == 0
    assert np.array_equal(out, oracle.unrank(idx))


def test_device_moves_match_host_model(emul, host_golden):
    words = np.array([r["words"] for r in host_golden["states"][:60]], np.uint32)
    from cuda_cube_solver.device import unpack_words

    states = unpack_words(words)
    for m in range(18):
        _, right = _index(emul, "d4t", words, m)
        _, left = _index(emul, "d4t", words, -2 - m)
        assert np.array_equal(right, state_words([compose(s, MOVES_HTM[m]) for s in states]))
        assert np.array_equal(left, state_words([compose(MOVES_HTM[m], s) for s in states]))


def test_device_decoders_match_oracle(emul, oracle):
    rng = np.random.default_rng(2)
    depth = rng.integers(5, 14, 124 * 155 * 4).astype(np.uint8)
    blk = oracle.encode_block(depth)
    b3 = oracle.encode_b3(depth, blk)
    idx = rng.integers(0, len(depth), 4000, dtype=np.uint64)
    for fmt, table in ((0, blk), (1, b3)):
        out = np.zeros(len(idx), np.uint32)
        t32 = np.ascontiguousarray(table).view(np.uint32)
        assert emul.emul_lower_bound(t32.ctypes.data, fmt, idx.ctypes.data, len(idx), out.ctypes.data) == 0
        # the oracle decodes by state; decode the same entries through a direct formula
        if fmt == 0:
            want = [blk[(i // 124) * 32] + ((int.from_bytes(blk[(i // 124) * 32:(i // 124) * 32 + 32].tobytes(), "little")
                                              >> (8 + 2 * (i % 124))) & 3) for i in idx.tolist()]
        else:
            want = []
            for i in idx.tolist():
                sec = b3[(i // 155) * 32:(i // 155) * 32 + 32]
                j = i % 155
                d = (int(sec[1 + j // 5]) // 3 ** (j % 5)) % 3
                m, cut = int(sec[0]) & 63, int(sec[0]) >> 6
                want.append(m if d == 0 else m + cut + d)
        assert out.tolist() == want


@pytest.mark.parametrize("name", ["304", "s4", "d4f", "a4t", "d4t", "d4", "a4"])
@pytest.mark.parametrize("fmt", [0, 1])
def test_search_sector_arithmetic_matches_64_bit_division(emul, name, fmt):
    """The search computes the sector of entry cls * NE + e in 32-bit arithmetic; it must equal
    the 64-bit quotient and remainder by the entries per sector, edge cases included."""

    nec, entries = native.kind_info(name)
    ne = entries // 9930
    rng = np.random.default_rng(7)
    cls = np.concatenate([[0, 0, 9929, 9929, 1, 4965], rng.integers(0, 9930, 4000)]).astype(np.uint32)
    e = np.concatenate([[0, ne - 1, 0, ne - 1, ne - 1, ne // 2], rng.integers(0, ne, 4000)]).astype(np.uint32)
    out = np.zeros((len(cls), 2), np.uint64)
    emul.emul_split_sector.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_void_p]
    assert emul.emul_split_sector(name.encode(), fmt, cls.ctypes.data, e.ctypes.data, len(cls), out.ctypes.data) == 0
    per = 155 if fmt else 124
    idx = cls.astype(np.uint64) * np.uint64(ne) + e.astype(np.uint64)
    assert np.array_equal(out[:, 0], idx // np.uint64(per))
    assert np.array_equal(out[:, 1], idx % np.uint64(per))
