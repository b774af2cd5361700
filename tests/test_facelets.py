"""Facelet parsing and printing (the reference's facelets.py interface and error messages)."""

from __future__ import annotations

import random

import pytest

from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves
from cuda_cube_solver.facelets import FaceletError, is_facelet_string, parse_facelets, to_facelets

SOLVED = "U" * 9 + "R" * 9 + "F" * 9 + "D" * 9 + "L" * 9 + "B" * 9


def _states(n, seed):
    rng = random.Random(seed)
    return [apply_moves(CubieState(), [MOVES_HTM[rng.randrange(18)] for _ in range(rng.randrange(1, 40))])
            for _ in range(n)]


def test_solved_round_trip():
    assert parse_facelets(SOLVED) == CubieState()
    assert to_facelets(CubieState()) == SOLVED


def test_random_round_trip():
    for state in _states(200, 1):
        assert parse_facelets(to_facelets(state)) == state


def test_whitespace_and_colour_letters():
    state = _states(1, 3)[0]
    s = to_facelets(state)
    colours = s.translate(str.maketrans("URFDLB", "WRGYOB"))
    assert is_facelet_string(colours)
    assert parse_facelets(colours) == state
    assert parse_facelets(" ".join(s[i:i + 9] for i in range(0, 54, 9))) == state


def test_known_position():
    # R U applied to solved, read off by hand from the layout: U face's right column came from F.
    state = apply_moves(CubieState(), [MOVES_HTM[3], MOVES_HTM[0]])
    s = to_facelets(state)
    assert s[4::9] == "URFDLB"
    assert parse_facelets(s) == state


def _move_stickers(s, pairs):
    out = list(s)
    for target, source in pairs:
        out[target] = s[source]
    return "".join(out)


@pytest.mark.parametrize("mutate, message", [
    (lambda s: s[:53], "54 stickers"),
    (lambda s: s.replace("U", "R", 1), "has 8 stickers"),
    (lambda s: _move_stickers(s, [(8, 9), (9, 20), (20, 8)]), "twisted"),
    (lambda s: _move_stickers(s, [(5, 10), (10, 5)]), "flipped"),
    (lambda s: _move_stickers(s, [(5, 7), (10, 19), (7, 5), (19, 10)]), "swapped"),
    (lambda s: s[:13] + "U" + s[14:], "centre stickers must all differ"),
])
def test_illegal_cubes(mutate, message):
    with pytest.raises(FaceletError, match=message):
        parse_facelets(mutate(SOLVED))
