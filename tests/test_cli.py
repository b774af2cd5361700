"""CLI parsing and error lines (host side; the GPU solve path is covered by the GPU tests)."""

from __future__ import annotations

import io
import sys

import pytest

from cuda_cube_solver import __main__ as cli
from cuda_cube_solver.facelets import to_facelets
from cuda_cube_solver.workloads import scramble_state


def test_parse_lines_mixed_input():
    state = scramble_state([0, 3, 6])
    lines = ["# comment", "", "R U F2", to_facelets(state), "R X", "UUUU", to_facelets(state)[:-1] + "Q"]
    cubes, errors = cli.parse_lines(lines)
    assert [n for n, _ in cubes] == [3, 4]
    assert cubes[1][1] == state
    assert errors[0] == (5, "5 error unknown move 'X'")
    assert errors[1][0] == 6 and "unknown move" in errors[1][1]
    assert errors[2][0] == 7 and errors[2][1].startswith("7 error")


def test_solve_with_only_invalid_lines_prints_errors_in_order(monkeypatch, capsys):
    monkeypatch.setattr(sys, "stdin", io.StringIO("R Q\n\n# x\nU2 Z'\n"))
    cli.main(["solve", "--table", "d4t"])
    out = capsys.readouterr().out.splitlines()
    assert out == ["1 error unknown move 'Q'", "4 error unknown move \"Z'\""]


def test_unknown_table_and_mode_exit():
    with pytest.raises(SystemExit, match="unknown table"):
        cli.main(["solve", "--table", "999"])
    with pytest.raises(SystemExit, match="only --mode step"):
        cli.main(["solve", "--mode", "bidir"])
