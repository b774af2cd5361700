"""GPU solving: every solution solves its cube and its length is optimal -- equal to the CPU
oracle's exhaustive IDA* on small scrambles and to the reference's reported optimal lengths on
its random, distance-20 and superflip positions."""

from __future__ import annotations

import random

import numpy as np
import pytest

from conftest import resident_handle
from cuda_cube_solver import native
from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves
from cuda_cube_solver.device import state_words
from cuda_cube_solver.solver import GpuSolver, frames, parse_moves

pytestmark = pytest.mark.gpu


def small_scrambles(n=200, seed=0):
    """Seeded 8-12 move HTM scrambles, no two consecutive turns of the same face."""

    rng = random.Random(seed)
    out = []
    for _ in range(n):
        length, seq = rng.randint(8, 12), []
        while len(seq) < length:
            m = rng.randrange(18)
            if seq and m // 3 == seq[-1] // 3:
                continue
            seq.append(m)
        out.append(seq)
    return out


def _state(moves):
    return apply_moves(CubieState(), [MOVES_HTM[m] for m in moves])


def _check_solutions(states, results):
    for s, r in zip(states, results):
        assert r.status == 0
        assert apply_moves(s, [MOVES_HTM[m] for m in r.moves[: r.length]]) == CubieState()


def test_small_scrambles_on_304_match_oracle(oracle):
    h = resident_handle("304")
    scr = small_scrambles()
    states = [_state(s) for s in scr]
    res = h.solve(state_words(states), native.solve_opts(timeout_s=300))
    _check_solutions(states, res)
    assert all(r.length <= len(s) for r, s in zip(res, scr))
    oracle.set_kind("304")
    table = h.table_copy()
    fr = np.stack([state_words(frames(s)).reshape(30) for s in states])
    lengths, _, _, _ = oracle.solve_many(table, "block", fr)
    assert [r.length for r in res] == lengths.tolist()  # all 200 against the exhaustive CPU search


def test_random_cubes_match_reference_lengths(lengths_golden):
    h = resident_handle("d4t")
    cubes = lengths_golden["random1000"]
    states = [_state(parse_moves(c["scramble"])) for c in cubes]
    res = h.solve(state_words(states), native.solve_opts(timeout_s=600))
    _check_solutions(states, res)
    assert [r.length for r in res] == [c["length"] for c in cubes]
    _, probes, _ = h.last_solve_stats()
    assert probes == sum(r.probes for r in res)


def test_distance20_and_hard_positions(lengths_golden):
    h = resident_handle("d4")
    cubes = lengths_golden["distance20"] + [lengths_golden["superflip"], lengths_golden["hard19"]]
    states = [_state(parse_moves(c["scramble"])) for c in cubes]
    res = h.solve(state_words(states), native.solve_opts(timeout_s=900))
    _check_solutions(states, res)
    assert [r.length for r in res] == [c["length"] for c in cubes]


def test_solved_cube_and_public_api(lengths_golden):
    h = resident_handle("d4t")
    solver = GpuSolver(kind="d4t", handle=h)
    sols = solver.solve([CubieState(), _state(parse_moves(lengths_golden["random1000"][1]["scramble"]))])
    assert sols[0].moves == [] and sols[0].nodes == 0
    assert len(sols[1].moves) == lengths_golden["random1000"][1]["length"]
    assert sols[1].iteration_nodes and sols[1].iteration_nodes[-1][0] == len(sols[1].moves)
    h6, words = solver.root_h([CubieState()])
    assert h6.tolist() == [[0] * 6] and words.shape == (1, 30)


def test_illegal_state_is_rejected():
    h = resident_handle("304")
    bad = state_words([CubieState(ep=(1, 0) + tuple(range(2, 12)))])
    with pytest.raises(native.CcsError, match="not a legal position"):
        h.solve(bad)


@pytest.mark.parametrize("variant", [1, 2], ids=["throughput", "lookahead"])
def test_work_stealing_keeps_lengths_and_iteration_nodes(lengths_golden, variant):
    """Donated subtrees are searched exactly once: with stealing on (and forced often by a small
    minimum depth) every completed iteration has the same node count as without it, the lengths
    equal the reference's, and subtrees were in fact donated (also by the lookahead kernel, whose
    stashed siblings stay with the donor)."""

    h = resident_handle("d4")
    # fewer than 32 cubes and no deeper prefixes: prefix lengths then do not depend on timing
    cubes = lengths_golden["distance20"][:4] + [lengths_golden["hard19"]] + lengths_golden["random1000"][:26]
    states = [_state(parse_moves(c["scramble"])) for c in cubes]
    words = state_words(states)
    base = dict(timeout_s=900, variant=variant, deeper_at=(1e18, 1e18))
    off = h.solve(words, native.solve_opts(steal=-1, **base))
    assert h.last_solve_donations() == 0
    for depth in (3, 1):  # (slack 1: donations of small subtrees too, many of them)
        on = h.solve(words, native.solve_opts(steal=0, steal_depth=depth, steal_min_nodes=-1, **base))
        assert h.last_solve_donations() > 0
        _check_solutions(states, on)
        assert [r.length for r in on] == [r.length for r in off] == [c["length"] for c in cubes]
        for a, b in zip(on, off):  # every iteration before the last one was searched in full
            assert list(a.iter_nodes[: a.length]) == list(b.iter_nodes[: b.length])


def test_launch_shapes_agree(lengths_golden):
    """The 128 x 4 and 512 x 1 launch shapes (and the others) give the reference's lengths."""

    h = resident_handle("d4t")
    cubes = lengths_golden["random1000"][300:364]
    words = state_words([_state(parse_moves(c["scramble"])) for c in cubes])
    for variant in (1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11):
        res = h.solve(words, native.solve_opts(timeout_s=600, variant=variant))
        assert [r.length for r in res] == [c["length"] for c in cubes], variant
    h2d, d2h = h.last_solve_io_bytes()
    assert h2d > 64 * 416 and d2h > 64 * 416


def test_head_rotation_keeps_lengths_and_iteration_nodes(lengths_golden):
    """Live ring entries moved from the head to the tail (rotate 1, here with a 64-entry window so
    that entries move all the time) serve the same iterations: the lengths equal the reference's
    and every completed iteration has the node count of a search without rotation."""

    h = resident_handle("d4t")
    cubes = lengths_golden["random1000"][400:431]  # fewer than 32: prefix lengths do not depend on timing
    words = state_words([_state(parse_moves(c["scramble"])) for c in cubes])
    base = dict(timeout_s=600, variant=3, deeper_at=(1e18, 1e18), steal=-1, spread=64)
    plain = h.solve(words, native.solve_opts(rotate=-1, **base))
    moved = h.solve(words, native.solve_opts(rotate=1, **base))
    assert [r.length for r in moved] == [r.length for r in plain] == [c["length"] for c in cubes]
    for a, b in zip(moved, plain):
        assert list(a.iter_nodes[: a.length]) == list(b.iter_nodes[: b.length])


def test_lone_superflip_with_stealing(lengths_golden):
    """A lone hard cube spreads over the GPU through donated subtrees: the superflip on d4t."""

    h = resident_handle("d4t")
    c = lengths_golden["superflip"]
    words = state_words([_state(parse_moves(c["scramble"]))])
    res = h.solve(words, native.solve_opts(timeout_s=900, variant=1))
    assert res[0].length == c["length"]
    assert h.last_solve_donations() > 0


def test_autotuned_settings_give_the_same_lengths(lengths_golden):
    """The autotuner's choice (a short descent on its own sample) changes speed only: the tuned
    solver returns the reference's optimal lengths."""

    h = resident_handle("d4t")
    solver = GpuSolver(kind="d4t", handle=h)
    sample = [_state(parse_moves(c["scramble"])) for c in lengths_golden["random1000"][700:764]]
    result = solver.autotune(sample, save=False, budget_s=20.0)
    assert result["trials"] >= 1 and solver.tuned == result["config"]
    cubes = lengths_golden["random1000"][764:828]
    sols = solver.solve([_state(parse_moves(c["scramble"])) for c in cubes])
    assert [len(s.moves) for s in sols] == [c["length"] for c in cubes]
