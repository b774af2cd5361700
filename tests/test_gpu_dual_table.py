"""Two resident tables: d4 attached beside d4t, picked per cube, in one batched launch and in the
continuous-batching server.  Every cube's length is the same optimal length whichever table
searches it."""

from __future__ import annotations

import time

import numpy as np
import pytest

from conftest import resident_handle
from cuda_cube_solver import native
from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves
from cuda_cube_solver.device import state_words
from cuda_cube_solver.solver import GpuSolver, flipped_edges, parse_moves

pytestmark = pytest.mark.gpu


def _states(cubes):
    return [apply_moves(CubieState(), [MOVES_HTM[m] for m in parse_moves(c["scramble"])]) for c in cubes]


@pytest.fixture(scope="module")
def dual():
    h = native.Handle()
    h.build_table("d4t", "block", None, keep_resident=1)
    h.build_table("d4", "block", None, keep_resident=2)
    yield h
    h.close()


def test_second_table_is_the_d4_table(dual, lengths_golden):
    """Completed iterations enumerate the same tree under the same bounds, so their node counts
    match a handle that holds d4 alone exactly."""

    words = state_words(_states(lengths_golden["random1000"][:4]))
    opts = native.solve_opts(timeout_s=300)
    via_second = dual.solve(words, opts, np.ones(4, np.uint8))
    alone = resident_handle("d4").solve(words, opts)
    for a, b in zip(via_second, alone):
        assert a.length == b.length
        assert list(a.iter_nodes[: a.length]) == list(b.iter_nodes[: b.length])


def test_mixed_table_ids_give_reference_lengths(dual, lengths_golden):
    cubes = lengths_golden["random1000"][:96] + [lengths_golden["superflip"]]
    states = _states(cubes)
    words = state_words(states)
    ids = (np.arange(len(states)) % 2).astype(np.uint8)
    res = dual.solve(words, native.solve_opts(timeout_s=600), ids)
    assert [r.length for r in res] == [c["length"] for c in cubes]
    for s, r in zip(states, res):
        assert apply_moves(s, [MOVES_HTM[m] for m in r.moves[: r.length]]) == CubieState()
    # the same cubes with the ids swapped
    res2 = dual.solve(words, native.solve_opts(timeout_s=600), 1 - ids)
    assert [r.length for r in res2] == [r.length for r in res]


def test_flip_rule_in_the_solver(dual, lengths_golden):
    solver = GpuSolver(kind="d4t", handle=dual)
    solver.second_kind = "d4"
    cubes = lengths_golden["random1000"][:40] + [lengths_golden["superflip"]]
    states = _states(cubes)
    ids = solver.table_ids(state_words(states))
    assert ids[-1] == 1 and flipped_edges(state_words(states[-1:]))[0] == 12
    sols = solver.solve(states)
    assert [len(s.moves) for s in sols] == [c["length"] for c in cubes]


def test_server_with_table_ids(dual, lengths_golden):
    cubes = lengths_golden["random1000"][100:148]
    words = state_words(_states(cubes))
    dual.server_start(16)
    try:
        ids = {dual.server_submit(words[i], i % 2): i for i in range(len(cubes))}
        got, t0 = {}, time.time()
        while len(got) < len(cubes) and time.time() - t0 < 300:
            for rid, r in dual.server_poll(64):
                got[ids[rid]] = r
            time.sleep(0.002)
    finally:
        dual.server_stop()
    assert sorted(got) == list(range(len(cubes)))
    assert [got[i].length for i in range(len(cubes))] == [c["length"] for c in cubes]


def test_table_id_errors(dual):
    words = state_words([CubieState()])
    with pytest.raises(native.CcsError, match="not 0 or 1"):
        dual.solve(words, None, np.array([2], np.uint8))
    lone = resident_handle("d4t")
    with pytest.raises(native.CcsError, match="second table"):
        lone.solve(words, None, np.array([1], np.uint8))
