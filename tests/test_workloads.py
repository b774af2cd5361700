"""Seeded synthetic inputs: legality and determinism of the benchmark cube sets."""

from __future__ import annotations

import numpy as np

from cuda_cube_solver import serving, workloads
from cuda_cube_solver.cubie import CubieState


def test_uniform_cubes_are_legal_and_seeded():
    a = workloads.uniform_cubes(300, seed=1)
    assert all(s.is_legal() for s in a)
    assert a == workloads.uniform_cubes(300, seed=1)
    assert a != workloads.uniform_cubes(300, seed=2)
    # both parities occur: the edge swap keeps permutations legal without biasing them
    from cuda_cube_solver.cubie import permutation_parity

    assert {permutation_parity(s.cp) for s in a} == {0, 1}


def test_small_scrambles_have_no_repeated_faces():
    for seq in workloads.small_scrambles(200, seed=0):
        assert 8 <= len(seq) <= 12
        assert all(a // 3 != b // 3 for a, b in zip(seq, seq[1:]))


def test_superflip():
    s = workloads.superflip()
    assert s.is_legal() and s != CubieState() and all(o == 1 for o in s.eo)


def test_poisson_arrivals():
    t = serving.poisson_arrivals(20000, 100.0, seed=3)
    assert np.all(np.diff(t) > 0)
    assert abs(len(t) / t[-1] - 100.0) < 3.0


def test_flipped_edges_and_the_table_rule():
    from cuda_cube_solver.device import state_words
    from cuda_cube_solver.solver import FLIP_RULE, flipped_edges

    cubes = [CubieState(), workloads.superflip()] + workloads.uniform_cubes(64, seed=5)
    n = flipped_edges(state_words(cubes))
    assert n[0] == 0 and n[1] == 12
    assert all(x % 2 == 0 for x in n)  # edge flips have even parity
    assert (n >= FLIP_RULE).sum() >= 1 and FLIP_RULE == 12
