"""Seeded synthetic cube sets for the benchmark configurations.

* ``small_scrambles``: random HTM scrambles of 8-12 moves, no two consecutive turns of the same
  face (``random.Random(seed)``), solvable by an exhaustive CPU search.
* ``uniform_cubes``: positions drawn uniformly from the cube group (``np.random.default_rng(seed)``):
  a random corner and edge permutation (edges 10 and 11 swapped when the parities differ), seven
  random twists and eleven random flips, the last orientation of each closing its sum.
* ``superflip``: every edge flipped in place.
* ``batched_mix``: the batched configuration -- 4,096 uniform cubes of seed 2 in which 5% (205)
  are replaced by hard positions: uniform cubes of the seed-20 stream whose optimal length is at
  least 19 (their stream positions are listed in ``data/hard20.json``, written by
  ``data/make_hard20.py`` from GPU solves and checked against the reference's kernels) and the
  superflip, at positions drawn by ``np.random.default_rng(4)``.
"""

from __future__ import annotations

import json
import random
from pathlib import Path

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


HARD20 = Path(__file__).with_name("data") / "hard20.json"


def hard20() -> dict:
    """The seed-20 stream's cubes of optimal length >= 19: stream indices and lengths."""

    return json.loads(HARD20.read_text())


def batched_mix(n: int = 4096, seed: int = 2, hard_frac: float = 0.05) -> tuple[list[CubieState], dict[int, int]]:
    """``n`` uniform cubes of ``seed`` with ``round(hard_frac * n)`` of them replaced by hard
    positions (the first ones of ``hard20()`` and, last, the superflip).  Returns the cubes and
    {position: known optimal length} of the hard ones."""

    cubes = uniform_cubes(n, seed=seed)
    n_hard = int(round(hard_frac * n))
    if n_hard == 0:
        return cubes, {}
    info = hard20()
    if n_hard - 1 > len(info["indices"]):
        raise ValueError(f"{n_hard - 1} hard cubes asked for; data/hard20.json lists {len(info['indices'])}")
    stream = uniform_cubes(info["indices"][n_hard - 2] + 1, seed=20) if n_hard > 1 else []
    hard = [(stream[i], L) for i, L in zip(info["indices"][: n_hard - 1], info["lengths"])] + [(superflip(), 20)]
    where = np.random.default_rng(4).choice(n, size=len(hard), replace=False)
    known = {}
    for pos, (cube, length) in zip(where, hard):
        cubes[int(pos)] = cube
        known[int(pos)] = length
    return cubes, known


def coordinate_model_rate(kind: str, seconds: float, seed: int = 0) -> tuple[int, float]:
    """Table indexes the host Python coordinate model computes in about ``seconds`` in this
    process, one cube at a time: the six frames of a cube (``prefixes.frames``) and the table index
    of each (``coords.table_index``), as the reference's root bound does in Python
    (``solver.py:58-64``, ``coords.py:347``).  Returns (indexes, elapsed seconds)."""

    import time

    from cuda_cube_solver import coords, kinds
    from cuda_cube_solver.prefixes import frames

    k = kinds.get(kind)
    cubes = uniform_cubes(64, seed=seed)
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        for f in frames(cubes[(done // 6) % len(cubes)]):
            coords.table_index(*coords.pack(f), kind=k)
            done += 1
    return done, time.perf_counter() - t0

