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


def test_batched_mix_workload():
    """The batched configuration: 4,096 uniform cubes of seed 2 with 205 (5%) replaced by hard
    positions -- 204 seed-20 cubes of known optimal length >= 19 (lengths confirmed by the
    reference's kernels when the fixture was made) and the superflip."""

    from cuda_cube_solver import workloads

    info = workloads.hard20()
    assert info["reference_equal"] and len(info["indices"]) >= 204
    assert all(L >= 19 for L in info["lengths"])
    cubes, known = workloads.batched_mix(4096, seed=2)
    assert len(cubes) == 4096 and len(known) == 205
    assert all(c.is_legal() for c in cubes)
    assert sorted(known.values()).count(20) >= 1 and min(known.values()) >= 19
    assert workloads.superflip() in [cubes[i] for i in known]
    again, known2 = workloads.batched_mix(4096, seed=2)
    assert again == cubes and known2 == known
    uniform, none = workloads.batched_mix(64, seed=2, hard_frac=0.0)
    assert none == {} and uniform == workloads.uniform_cubes(64, seed=2)


def test_bfs_roofline_arithmetic():
    import sys

    from conftest import ROOT

    sys.path.insert(0, str(ROOT))
    import bench

    passes = [{"depth": 1, "forward": True, "found": 2, "random_reads": 10, "claims": 6, "seconds": 0.5},
              {"depth": 2, "forward": False, "found": 5, "random_reads": 100, "claims": 0, "seconds": 1.5}]
    r = bench.bfs_roofline(passes, entries=1000, peak_gbs=1.0, ceiling=50.0)
    assert r["dominant_pass"] == {"depth": 2, "dir": "bwd", "seconds": 1.5} and r["dominant_share"] == 0.75
    assert r["passes"][0]["algorithmic_gb"] == (1000 + 32 * 16) / 1e9
    assert abs(r["random_rate_over_dram_random_ceiling"] - (100 / 1.5) / 50.0) < 1e-12
