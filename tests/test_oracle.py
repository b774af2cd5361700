"""The CPU oracle itself, pinned before it is trusted: its index, unrank and encoders against the
reference's golden vectors and against straightforward Python restatements."""

from __future__ import annotations

import random

import numpy as np
import pytest

from cuda_cube_solver import coords, kinds
from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves, compose
from cuda_cube_solver.device import state_words, unpack_words

KINDS = ["304", "s4", "d4f", "a4t", "d4t", "d4", "a4"]


@pytest.mark.parametrize("name", KINDS)
def test_oracle_index_matches_reference_vectors(oracle, host_golden, name):
    oracle.set_kind(name)
    words = np.array([r["words"] for r in host_golden["states"]], np.uint32)
    want = np.array([r["index"][name] for r in host_golden["states"]], np.uint64)
    assert np.array_equal(oracle.index(words), want)


@pytest.mark.parametrize("name", KINDS)
def test_oracle_unrank_roundtrip_and_edges(oracle, name):
    oracle.set_kind(name)
    n = oracle.n_entries()
    assert n == kinds.N_CLASSES * kinds.get(name).n_edge
    rng = np.random.default_rng(5)
    idx = np.concatenate([[0, n - 1], rng.integers(0, n, 20000, dtype=np.uint64)]).astype(np.uint64)
    assert np.array_equal(oracle.index(oracle.unrank(idx)), idx)


def test_oracle_moves_match_host_model(oracle):
    oracle.set_kind("d4t")
    rng = random.Random(2)
    states = [apply_moves(CubieState(), [MOVES_HTM[rng.randrange(18)] for _ in range(30)]) for _ in range(40)]
    words = state_words(states)
    kind = kinds.get("d4t")
    for m in range(18):
        right = [compose(s, MOVES_HTM[m]) for s in states]
        left = [compose(MOVES_HTM[m], s) for s in states]
        assert np.array_equal(oracle.index(words, m), [coords.table_index(*coords.pack(s), kind) for s in right])
        assert np.array_equal(oracle.index(words, -2 - m), [coords.table_index(*coords.pack(s), kind) for s in left])


def _py_block(depth):
    out = bytearray()
    for b in range(0, len(depth), 124):
        chunk = depth[b:b + 124]
        mn = min(chunk)
        bits = mn
        for j, d in enumerate(chunk):
            bits |= min(d - mn, 3) << (8 + 2 * j)
        out += bits.to_bytes(32, "little")
    return bytes(out)


def _py_b3(depth, blk):
    out = bytearray()
    for b in range(0, len(depth), 155):
        vals = []
        for x in range(b, min(b + 155, len(depth))):
            m124, d = blk[(x // 124) * 32], depth[x]
            vals.append(d if d - m124 < 3 else next(v for v in range(m124 + 3, m124 + 6) if v % 3 == d % 3))
        m = min(vals)
        score = lambda c: sum(m if v <= m + c else (m + c + 1 if v == m + c + 1 else m + c + 2) for v in vals)  # noqa
        best = max(range(4), key=lambda c: (score(c), -c))
        digits = [0 if v <= m + best else (1 if v == m + best + 1 else 2) for v in vals] + [0] * (155 - len(vals))
        out.append(m | best << 6)
        for q in range(31):
            out.append(sum(digits[5 * q + k] * 3 ** k for k in range(5)))
    return bytes(out)


def test_oracle_encoders_match_python_restatement(oracle):
    rng = np.random.default_rng(9)
    for n in (124 * 155, 124 * 155 + 37, 1000):
        depth = rng.integers(6, 15, n).astype(np.uint8)
        depth[rng.integers(0, n, 30)] = 3  # far-from-minimum entries exercise the residue rule
        blk = oracle.encode_block(depth)
        assert bytes(blk) == _py_block(depth.tolist())
        b3 = oracle.encode_b3(depth, blk)
        assert bytes(b3) == _py_b3(depth.tolist(), bytes(blk))


def test_oracle_ida_star_with_trivial_bounds(oracle):
    """With an all-zero (admissible) table IDA* is a plain iterative deepening: its lengths are the
    optimal lengths of short scrambles, which a breadth-first enumeration gives exactly."""

    oracle.set_kind("304")
    from cuda_cube_solver.solver import frames

    dist = {CubieState(): 0}
    frontier = [CubieState()]
    for d in range(1, 4):
        nxt = []
        for s in frontier:
            for mv in MOVES_HTM:
                t = compose(s, mv)
                if t not in dist:
                    dist[t] = d
                    nxt.append(t)
        frontier = nxt
    rng = random.Random(4)
    states = [apply_moves(CubieState(), [MOVES_HTM[rng.randrange(18)] for _ in range(rng.randrange(1, 4))])
              for _ in range(25)]
    fr = np.stack([state_words(frames(s)).reshape(30) for s in states])
    zeros = np.zeros(kinds.PRESET_BY_NAME["304"].table_bytes, np.uint8)  # every bound 0 (pages stay unmapped)
    lengths, moves, nodes, probes = oracle.solve_many(zeros, "block", fr, threads=4)
    for s, L, mv in zip(states, lengths, moves):
        assert L == dist[s]
        assert apply_moves(s, [MOVES_HTM[m] for m in mv[:L]]) == CubieState()


def test_base3_from_the_mod3_and_block_tables(oracle):
    """The reference's base-3 file is a function of its mod-3 and 2-bit block tables
    (build_b3_table, table.py:52-79): recovering each entry's value from the pair (the block offset
    below 3, else the smallest value >= minimum + 3 with the mod-3 residue) and encoding it gives
    the same bytes as encoding from the exact depths; the mod-3 words hold depth mod 3, sixteen
    two-bit entries per little-endian uint32, 3 past the end."""

    rng = np.random.default_rng(21)
    n = 155 * 40 + 17
    base = np.repeat(rng.integers(4, 14, -(-n // 124)), 124)[:n]
    depth = (base + rng.choice([0, 0, 1, 1, 2, 3, 4, 5, 6, 9], n)).astype(np.uint8)
    blk = oracle.encode_block(depth)
    direct = oracle.encode_b3(depth, blk)

    padded = np.full(-(-n // 16) * 16, 3, np.uint32)
    padded[:n] = depth % 3
    mod3 = (padded.reshape(-1, 16) << (2 * np.arange(16, dtype=np.uint32))).sum(axis=1).astype(np.uint32)
    assert int((mod3[-1] >> (2 * (n % 16))) & 3) == 3  # past the end

    x = np.arange(n)
    words = blk.view(np.uint32).reshape(-1, 8)
    sec, j = x // 124, x % 124
    pos = 8 + 2 * j
    m = (words[sec, 0] & 0xFF).astype(np.int64)
    off = ((words[sec, pos // 32] >> (pos % 32).astype(np.uint32)) & 3).astype(np.int64)
    r = ((mod3[x // 16] >> (2 * (x % 16)).astype(np.uint32)) & 3).astype(np.int64)
    lo = m + 3
    value = np.where(off < 3, m + off, lo + (r - lo) % 3)
    assert np.all(value[depth <= m + 5] == depth[depth <= m + 5])
    assert np.array_equal(oracle.encode_b3(value.astype(np.uint8), blk), direct)
