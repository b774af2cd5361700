"""Seeded synthetic cube sets for the benchmark configurations.

* ``small_scrambles``: random HTM scrambles of 8-12 moves, no two consecutive turns of the same
  face (``random.Random(seed)``), solvable by an exhaustive CPU search.
* ``uniform_cubes``: positions drawn uniformly from the cube group (``np.random.default_rng(seed)``):
  a random corner and edge permutation (edges 10 and 11 swapped when the parities differ), seven
  random twists and eleven random flips, the last orientation of each closing its sum.
* ``superflip``: every edge flipped in place.
"""

from __future__ import annotations

import random

import numpy as np

from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves, permutation_parity


def small_scrambles(n: int = 200, seed: int = 0) -> list[list[int]]:
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


def scramble_state(moves: list[int]) -> CubieState:
    return apply_moves(CubieState(), [MOVES_HTM[m] for m in moves])


def uniform_cubes(n: int, seed: int = 1) -> list[CubieState]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        cp = [int(x) for x in rng.permutation(8)]
        ep = [int(x) for x in rng.permutation(12)]
        if permutation_parity(cp) != permutation_parity(ep):
            ep[10], ep[11] = ep[11], ep[10]
        co = [int(x) for x in rng.integers(0, 3, 7)]
        eo = [int(x) for x in rng.integers(0, 2, 11)]
        co.append((-sum(co)) % 3)
        eo.append(sum(eo) % 2)
        out.append(CubieState(tuple(cp), tuple(co), tuple(ep), tuple(eo)))
    return out


def superflip() -> CubieState:
    return CubieState(eo=(1,) * 12)
