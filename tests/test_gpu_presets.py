"""GPU solves on every preset the reference ships: the base-3 format (the reference's FMT=1
decode, kernels.cu:412-422) and the s4, d4f, a4t and a4 kinds (kinds.py:158-173) give the
reference's optimal lengths on its random cubes (the optimal length does not depend on the
table), and every solution solves its cube."""

from __future__ import annotations

import pytest

from cuda_cube_solver import native
from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves
from cuda_cube_solver.device import state_words
from cuda_cube_solver.solver import parse_moves

pytestmark = pytest.mark.gpu

PRESETS = [("s4", "b3"), ("d4f", "b3"), ("a4t", "b3"), ("a4t", "block"), ("d4t", "b3"), ("a4", "b3"),
           ("a4", "block"), ("d4", "b3")]


@pytest.mark.parametrize("kind,fmt", PRESETS, ids=[f"{k}-{f}" for k, f in PRESETS])
def test_preset_solves_match_reference_lengths(lengths_golden, kind, fmt):
    cubes = lengths_golden["random1000"][400:432]
    states = [apply_moves(CubieState(), [MOVES_HTM[m] for m in parse_moves(c["scramble"])]) for c in cubes]
    h = native.Handle()
    try:
        h.build_table(kind, fmt, None, keep_resident=True)
        for variant in (1, 2):  # the throughput and the lookahead kernels of this kind and format
            res = h.solve(state_words(states), native.solve_opts(timeout_s=900, variant=variant))
            assert [r.length for r in res] == [c["length"] for c in cubes]
            for s, r in zip(states, res):
                assert apply_moves(s, [MOVES_HTM[m] for m in r.moves[: r.length]]) == CubieState()
    finally:
        h.close()
