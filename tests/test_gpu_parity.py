"""GPU parity of the cube math: libccs index / unrank / moves / lower bounds against the CPU oracle
and the reference's golden vectors, bit-exact, for the 304 table and the six group kinds."""

from __future__ import annotations

import random

import numpy as np
import pytest

from conftest import resident_handle
from cuda_cube_solver import native
from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves, compose
from cuda_cube_solver.device import state_words

pytestmark = pytest.mark.gpu
KINDS = ["304", "s4", "d4f", "a4t", "d4t", "d4", "a4"]


def _random_words(n, seed, max_len=40):
    rng = np.random.default_rng(seed)
    # Random legal states fast: compose random moves in bulk through the oracle's host model.
    states = []
    r = random.Random(seed)
    for _ in range(n):
        states.append(apply_moves(CubieState(), [MOVES_HTM[r.randrange(18)] for _ in range(r.randrange(max_len))]))
    return state_words(states), states


@pytest.fixture(scope="module")
def handle():
    h = native.Handle()
    yield h
    h.close()


@pytest.fixture(scope="module")
def sample():
    return _random_words(3000, 11)


@pytest.mark.parametrize("name", KINDS)
def test_index_matches_reference_and_oracle(handle, oracle, host_golden, sample, name):
    handle.set_kind(name)
    oracle.set_kind(name)
    golden_words = np.array([r["words"] for r in host_golden["states"]], np.uint32)
    want = np.array([r["index"][name] for r in host_golden["states"]], np.uint64)
    got, _ = handle.index(golden_words)
    assert np.array_equal(got, want)
    words, _ = sample
    got, _ = handle.index(words)
    assert np.array_equal(got, oracle.index(words))


@pytest.mark.parametrize("name", KINDS)
def test_unrank_matches_oracle_and_roundtrips(handle, oracle, name):
    handle.set_kind(name)
    oracle.set_kind(name)
    n = oracle.n_entries()
    rng = np.random.default_rng(hash(name) & 0xFFFF)
    idx = np.concatenate([[0, n - 1], rng.integers(0, n, 100000, dtype=np.uint64)]).astype(np.uint64)
    st = handle.unrank(idx)
    assert np.array_equal(st, oracle.unrank(idx))
    back, _ = handle.index(st)
    assert np.array_equal(back, idx)


def test_right_and_left_moves(handle, oracle, sample):
    handle.set_kind("d4t")
    oracle.set_kind("d4t")
    words, states = sample
    words, states = words[:300], states[:300]
    for m in range(18):
        idx, out = handle.index(words, m)
        assert np.array_equal(out, state_words([compose(s, MOVES_HTM[m]) for s in states]))
        assert np.array_equal(idx, oracle.index(words, m))
        idx, out = handle.index(words, -2 - m)
        assert np.array_equal(out, state_words([compose(MOVES_HTM[m], s) for s in states]))
        assert np.array_equal(idx, oracle.index(words, -2 - m))


def test_lower_bounds_and_root_bounds_match_oracle(oracle, sample):
    from cuda_cube_solver.solver import frames

    h = resident_handle("304")
    oracle.set_kind("304")
    table = h.table_copy()
    words, states = sample
    assert np.array_equal(h.lower_bound(words), oracle.lower_bound(table, "block", words))
    fr = state_words([f for s in states[:500] for f in frames(s)])
    got = h.root_bounds(words[:500])
    assert np.array_equal(got.reshape(-1), oracle.lower_bound(table, "block", fr))
