"""The CLI and ``open_solver`` end to end on the GPU: ``build-table`` writes the reference's file,
``solve`` (batched) and ``solve --stream`` (the continuous-batching server) print the reference's
``<line> <length> <moves>`` lines (__main__.py:98-134) with its optimal lengths, and
``open_solver`` builds a missing table on first use (solver.py:95-115)."""

from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys

import pytest

from conftest import GOLDEN, ROOT
from cuda_cube_solver import kinds
from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves
from cuda_cube_solver.solver import open_solver, parse_moves

pytestmark = pytest.mark.gpu


def _cli(args, stdin: str = "", timeout: int = 900) -> subprocess.CompletedProcess:
    env = dict(os.environ, PYTHONPATH=str(ROOT / "cuda-cube-solver_b200"))
    return subprocess.run([sys.executable, "-m", "cuda_cube_solver", *args], input=stdin, capture_output=True,
                          text=True, timeout=timeout, env=env)


@pytest.fixture(scope="module")
def tables_304(tmp_path_factory):
    out = tmp_path_factory.mktemp("tables")
    r = _cli(["build-table", "--table", "304", "--out", str(out)])
    assert r.returncode == 0, r.stderr
    return out


def test_build_table_writes_the_reference_file(tables_304):
    path = tables_304 / "prune-ud-304-blk.bin"
    assert path.stat().st_size == kinds.PRESET_BY_NAME["304"].table_bytes
    digest = hashlib.sha256(path.read_bytes()).hexdigest()
    assert digest == json.loads((GOLDEN / "ref_table_sha256.json").read_text())["304"]["reference_sha256"]


@pytest.mark.parametrize("stream", [False, True], ids=["batched", "stream"])
def test_solve_prints_reference_lengths(tables_304, lengths_golden, stream):
    cubes = lengths_golden["random1000"][:12]
    text = "# a comment line\n" + "".join(c["scramble"] + "\n" for c in cubes) + "R Q\n"
    args = ["solve", "--tables", str(tables_304), "--table", "304", "--no-build"] + (["--stream"] if stream else [])
    r = _cli(args, text)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert lines[-1] == "14 error unknown move 'Q'"
    got = {}
    for line in lines[:-1]:
        number, length, *moves = line.split()
        got[int(number)] = (int(length), moves)
    assert sorted(got) == list(range(2, 14))
    for i, c in enumerate(cubes):
        length, moves = got[i + 2]
        assert length == c["length"] == len(moves)
        state = apply_moves(CubieState(), [MOVES_HTM[m] for m in parse_moves(c["scramble"])])
        assert apply_moves(state, [MOVES_HTM[m] for m in parse_moves(" ".join(moves))]) == CubieState()


def test_open_solver_builds_a_missing_table(tmp_path, lengths_golden):
    messages = []
    solver = open_solver(tmp_path, table="304", log=messages.append)
    try:
        assert (tmp_path / "prune-ud-304-blk.bin").exists()
        assert any("building table 304" in m for m in messages)
        cubes = lengths_golden["random1000"][12:16]
        sols = solver.solve([apply_moves(CubieState(), [MOVES_HTM[m] for m in parse_moves(c["scramble"])])
                             for c in cubes])
        assert [len(s.moves) for s in sols] == [c["length"] for c in cubes]
    finally:
        solver.close()
