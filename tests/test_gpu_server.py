"""Continuous-batching server: cubes submitted while others are on the GPU are admitted into free
slots, and every result is the same alone and in the mix (same optimal length; the move sequence
may differ)."""

from __future__ import annotations

import time

import pytest

from conftest import resident_handle
from cuda_cube_solver import native
from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves
from cuda_cube_solver.device import state_words
from cuda_cube_solver.solver import parse_moves

pytestmark = pytest.mark.gpu


def test_server_results_match_alone(lengths_golden):
    h = resident_handle("d4t")
    cubes = lengths_golden["random1000"][:120]
    states = [apply_moves(CubieState(), [MOVES_HTM[m] for m in parse_moves(c["scramble"])]) for c in cubes]
    words = state_words(states)
    alone = [h.solve(words[i:i + 1])[0].length for i in range(0, 120, 12)]
    h.server_start(32)
    try:
        ids = {}
        for i in range(120):  # bursts: more requests than slots, submitted while others search
            ids[h.server_submit(words[i])] = i
            if i % 40 == 39:
                time.sleep(0.05)
        got = {}
        t0 = time.time()
        while len(got) < 120 and time.time() - t0 < 300:
            for rid, r in h.server_poll(64):
                got[ids[rid]] = r
            time.sleep(0.002)
        assert len(got) == 120
        for i, r in got.items():
            assert r.status == 0
            assert r.length == cubes[i]["length"]
            assert apply_moves(states[i], [MOVES_HTM[m] for m in r.moves[: r.length]]) == CubieState()
        assert [got[i].length for i in range(0, 120, 12)] == alone
    finally:
        h.server_stop()
    with pytest.raises(native.CcsError, match="not running"):
        h.server_poll(1)


def test_server_admits_by_device_memory(lengths_golden):
    """With a device-memory budget the server never holds more cubes in flight than the budget
    leaves room for beside its fixed footprint, and still solves every request; a budget below the
    fixed footprint is refused."""

    h = resident_handle("d4t")
    cubes = lengths_golden["random1000"][120:180]
    states = [apply_moves(CubieState(), [MOVES_HTM[m] for m in parse_moves(c["scramble"])]) for c in cubes]
    words = state_words(states)
    with pytest.raises(native.CcsError, match="alone take"):
        h.server_start_budget(1 << 20)
    # find the fixed footprint, then allow exactly 6 cubes beside it
    h.server_start_budget(64 << 30)
    mem = h.server_memory()
    h.server_stop()
    budget = mem["fixed_bytes"] + 6 * mem["bytes_per_cube"]
    assert mem["fixed_bytes"] > h.table_bytes() and mem["bytes_per_cube"] == 456
    assert h.server_start_budget(budget) == 6
    try:
        ids = {h.server_submit(words[i]): i for i in range(len(cubes))}
        got = {}
        t0 = time.time()
        while len(got) < len(cubes) and time.time() - t0 < 300:
            for rid, r in h.server_poll(64):
                got[ids[rid]] = r
            time.sleep(0.002)
        mem = h.server_memory()
    finally:
        h.server_stop()
    assert [got[i].length for i in range(len(cubes))] == [c["length"] for c in cubes]
    assert mem["budget_bytes"] == budget and 1 <= mem["peak_in_flight"] <= 6
