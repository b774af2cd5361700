"""ccs_solve_noalloc, the solve entry point that allocates nothing (for callers whose device memory
belongs to a pool or allocator of their own and who cannot cudaMalloc at solve time), checked
against ccs_solve on the same cubes, twice in a row, through the C ABI.  The file is collected
last, so a run that stops at the first failure has run every other test before it."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import resident_handle
from cuda_cube_solver import native
from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves
from cuda_cube_solver.device import state_words
from cuda_cube_solver.solver import parse_moves, verify_solutions

pytestmark = pytest.mark.gpu


def _words(cubes):
    return state_words([apply_moves(CubieState(), [MOVES_HTM[m] for m in parse_moves(c["scramble"])])
                        for c in cubes])


def test_no_alloc_matches_solve_twice(lengths_golden):
    """Same optimal lengths and, for every completed iteration, the same node counts as ccs_solve
    (fewer than 32 cubes, so prefix lengths depend on node counts only); the second call reuses
    the array the first one left behind."""

    h = resident_handle("d4t")
    opts = native.solve_opts(timeout_s=600, deeper_at=(1e18, 1e18))
    for first, count in ((0, 24), (24, 20)):
        cubes = lengths_golden["random1000"][first:first + count]
        words = _words(cubes)
        ref = h.solve(words, opts)
        got = h.solve_noalloc(words, opts)
        assert [r.status for r in got] == [0] * count
        assert [r.length for r in got] == [r.length for r in ref] == [c["length"] for c in cubes]
        assert verify_solutions(words, [list(r.moves[: r.length]) for r in got])
        for a, b in zip(got, ref):
            assert list(a.iter_nodes[: a.length]) == list(b.iter_nodes[: b.length])


def test_no_alloc_full_batch_and_limits(lengths_golden):
    h = resident_handle("d4t")
    cap = native.NOALLOC_MAX_CUBES
    cubes = lengths_golden["random1000"][200:200 + cap]
    words = _words(cubes)
    got = h.solve_noalloc(words, native.solve_opts(timeout_s=600))
    assert [r.length for r in got] == [c["length"] for c in cubes]
    assert verify_solutions(words, [list(r.moves[: r.length]) for r in got])
    with pytest.raises(native.CcsError, match=f"at most {cap}"):
        h.solve_noalloc(np.repeat(words[:1], cap + 1, axis=0))
    with pytest.raises(native.CcsError, match="base_plen 5"):
        h.solve_noalloc(words[:1], native.solve_opts(base_plen=5))
    assert h.solve_noalloc(words[:0]) == []


def test_no_alloc_prefix_length_one_many_cubes(lengths_golden):
    """base_plen = 1 with 32 or more cubes in flight: the shallow rule takes the next iteration's
    prefix length below 1, which is clamped to 1 (a wrapped length would ask for prefix lists the
    array does not hold and stall the search).  The allocating path gives the same lengths."""

    h = resident_handle("d4t")
    cubes = lengths_golden["random1000"][500:540]
    words = _words(cubes)
    opts = native.solve_opts(base_plen=1, timeout_s=600)
    got = h.solve_noalloc(words, opts)
    ref = h.solve(words, opts)
    assert [r.length for r in got] == [r.length for r in ref] == [c["length"] for c in cubes]
    assert verify_solutions(words, [list(r.moves[: r.length]) for r in got])


def test_no_alloc_two_threads_one_device(lengths_golden):
    """Two handles on one device (d4t and 304 tables) share its array; the library runs their calls
    one at a time, so two threads calling together both get their own cubes' results."""

    import threading

    from cuda_cube_solver import workloads

    h1 = resident_handle("d4t")
    h2 = resident_handle("304")
    w1 = _words(lengths_golden["random1000"][600:630])
    w2 = state_words([workloads.scramble_state(s) for s in workloads.small_scrambles(40, seed=7)])
    opts = native.solve_opts(timeout_s=600)
    want = [[r.length for r in h1.solve(w1, opts)], [r.length for r in h2.solve(w2, opts)]]
    out = [None, None]

    def run(i, h, w):
        out[i] = h.solve_noalloc(w, opts)

    for _ in range(2):
        threads = [threading.Thread(target=run, args=(0, h1, w1)), threading.Thread(target=run, args=(1, h2, w2))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for i, w in enumerate((w1, w2)):
            assert [r.length for r in out[i]] == want[i]
            assert verify_solutions(w, [list(r.moves[: r.length]) for r in out[i]])
