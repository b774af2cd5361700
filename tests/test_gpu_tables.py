"""GPU table builds: per-depth counts equal the reference's known answers, the histogram
self-check holds, and the files are byte-identical to the CPU oracle's independent build
(tests/golden/table_sha256.json) -- the reference's table format, bit for bit."""

from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

from conftest import GOLDEN, resident_handle
from cuda_cube_solver import kinds, native
from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves
from cuda_cube_solver.device import state_words

pytestmark = pytest.mark.gpu


def _sha(a: np.ndarray) -> str:
    return hashlib.sha256(a.tobytes()).hexdigest()


def _sha_golden():
    p = GOLDEN / "table_sha256.json"
    return json.loads(p.read_text()) if p.exists() else {}


def _ref_sha():
    """Digests of the tables the reference's own kernels build on a B200 (baseline/ref_table_sha.py)."""

    p = GOLDEN / "ref_table_sha256.json"
    return json.loads(p.read_text()) if p.exists() else {}


def test_304_counts_and_bytes(depth_golden):
    h = resident_handle("304")
    assert h.build_counts == depth_golden["304"]["depth_counts"]
    assert h.table_bytes() == kinds.PRESET_BY_NAME["304"].table_bytes
    digest = _sha(h.table_copy())
    assert digest == _sha_golden()["304"]["block_sha256"]  # the CPU oracle's independent build
    assert digest == _ref_sha()["304"]["reference_sha256"]  # the reference's own kernels
    passes = h.last_build_passes()  # per-pass counters behind the build's roofline
    assert [p["found"] for p in passes] == h.build_counts[1:]
    assert all(p["random_reads"] > 0 and p["seconds"] > 0 for p in passes)
    assert any(p["forward"] and p["claims"] >= p["found"] for p in passes)


@pytest.mark.parametrize("name", ["d4t", "d4"])
def test_big_group_tables_counts_and_bytes(depth_golden, name):
    h = resident_handle(name)
    assert h.build_counts == depth_golden[name]["depth_counts"]
    assert sum(h.build_counts) == depth_golden[name]["entries"]
    assert h.table_bytes() == kinds.PRESET_BY_NAME[name].table_bytes
    ref = _ref_sha().get(name)
    if ref:
        assert _sha(h.table_copy()) == ref["reference_sha256"]


def test_s4_b3_counts_and_bytes(depth_golden):
    h = native.Handle()
    try:
        counts, _ = h.build_table("s4", "b3", None, keep_resident=True)
        assert counts == depth_golden["s4"]["depth_counts"]
        assert h.table_bytes() == kinds.PRESET_BY_NAME["s4-b3"].table_bytes
        assert _sha(h.table_copy()) == _sha_golden()["s4"]["b3_sha256"]  # the CPU oracle's independent build
    finally:
        h.close()


@pytest.mark.parametrize("preset", ["s4-b3", "d4f-b3", "a4t-b3", "a4t", "d4t-b3", "a4-b3", "a4", "d4-b3"])
def test_every_preset_is_byte_identical_to_the_reference(preset):
    """Each remaining preset built here has the sha256 of the table the reference's own kernels
    build on a B200 (the 304, d4t and d4 tables are checked above)."""

    p = kinds.PRESET_BY_NAME[preset]
    ref = _ref_sha()[preset]
    h = native.Handle()
    try:
        counts, _ = h.build_table(p.kind, p.format, None, keep_resident=True)
        assert counts == ref["reference_counts"]
        assert h.table_bytes() == p.table_bytes == ref["bytes"]
        assert _sha(h.table_copy()) == ref["reference_sha256"]
    finally:
        h.close()


def test_file_roundtrip_and_size_check(tmp_path):
    h = resident_handle("304")
    path = tmp_path / "prune-ud-304-blk.bin"
    table = h.table_copy()
    table.tofile(path)
    h2 = native.Handle()
    try:
        h2.load_table("304", "block", path)
        assert _sha(h2.table_copy()) == _sha(table)  # the double-buffered load is byte exact
        words = np.array([[0x03020100, 0x07060504, 0x03020100, 0x07060504, 0x0B0A0908]], np.uint32)
        assert h2.lower_bound(words).tolist() == [0]
        # the same file attached as a second table answers like the first
        h2.attach_table("304", "block", path)
        cubes = state_words([CubieState(), apply_moves(CubieState(), [MOVES_HTM[m] for m in (0, 4, 8, 13, 2, 16)])])
        first = h2.solve(cubes, native.solve_opts(timeout_s=120))
        second = h2.solve(cubes, native.solve_opts(timeout_s=120), np.ones(2, np.uint8))
        assert [r.length for r in first] == [r.length for r in second]
        # a table written by the build (double-buffered device -> file) equals its device copy
        out = tmp_path / "built-304.bin"
        h3 = native.Handle()
        try:
            h3.build_table("304", "block", out, keep_resident=True)
            assert _sha(np.fromfile(out, np.uint8)) == _sha(h3.table_copy()) == _sha(table)
        finally:
            h3.close()
        bad = tmp_path / "short.bin"
        table[:1000].tofile(bad)
        with pytest.raises(native.CcsError, match="size 1000"):
            h2.load_table("304", "block", bad)
        with pytest.raises(native.CcsError, match="not found"):
            h2.load_table("304", "block", tmp_path / "missing.bin")
    finally:
        h2.close()
