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


def _block_histogram(words: np.ndarray, n_entries: int, n_bins: int = 32) -> np.ndarray:
    """Host count of a 2-bit block table's entries per decoded value (minimum + offset)."""

    sec = words.reshape(-1, 8)
    m = (sec[:, 0] & 0xFF).astype(np.int64)
    cnt = np.zeros((len(sec), 4), np.int32)
    last = n_entries - (len(sec) - 1) * 124  # entries in the last sector
    for i in range(8):
        j0 = 16 * i - 4  # entry at bit 0 of word i
        full = sum(1 << (2 * t) for t in range(16) if 0 <= j0 + t < 124)
        tail = sum(1 << (2 * t) for t in range(16) if 0 <= j0 + t < last)
        valid = np.full(len(sec), full, np.uint32)
        valid[-1] = tail
        lo, hi = sec[:, i] & valid, (sec[:, i] >> 1) & valid
        cnt[:, 1] += np.bitwise_count(lo & ~hi)
        cnt[:, 2] += np.bitwise_count(hi & ~lo)
        cnt[:, 3] += np.bitwise_count(lo & hi)
    cnt[:, 0] = 124 - cnt[:, 1:].sum(axis=1)
    cnt[-1, 0] -= 124 - last
    out = np.zeros(n_bins, np.int64)
    for k in range(4):
        out += np.bincount(np.minimum(m + k, n_bins - 1), weights=cnt[:, k], minlength=n_bins).astype(np.int64)
    return out


def _b3_histogram(data: np.ndarray, n_entries: int, n_bins: int = 32) -> np.ndarray:
    """Host count of a base-3 table's entries per decoded value (digit 0 -> m, 1 -> m + cut + 1,
    2 -> m + cut + 2)."""

    sec = data.reshape(-1, 32)
    lut = np.zeros((256, 3), np.uint8)  # digits 0 / 1 / 2 among a byte's five
    for b in range(243):
        for k in range(5):
            lut[b, (b // 3 ** k) % 3] += 1
    cnt = np.zeros((len(sec), 3), np.int32)
    for q in range(1, 32):
        cnt += lut[sec[:, q]]
    last = n_entries - (len(sec) - 1) * 155
    cnt[-1, 0] -= 155 - last  # digits past the end are 0
    m = (sec[:, 0] & 63).astype(np.int64)
    cut = (sec[:, 0] >> 6).astype(np.int64)
    out = np.zeros(n_bins, np.int64)
    for k, base in enumerate((m, m + cut + 1, m + cut + 2)):
        out += np.bincount(np.minimum(base, n_bins - 1), weights=cnt[:, k], minlength=n_bins).astype(np.int64)
    return out


def test_reference_table_files_and_helpers(tmp_path, depth_golden):
    """table.build (mod-3 and block files of one BFS), build_b3_table (base 3 from those two files),
    save_device and histogram on the 304 kind, against the CPU oracle's digests and host decodes."""

    from cuda_cube_solver import table

    golden = _sha_golden()["304"]
    h = native.Handle()
    try:
        mod3 = table.build(tmp_path, "304", log=None, handle=h)
        meta = json.loads(mod3.with_suffix(".json").read_text())
        n = meta["entries"]
        assert meta["depth_counts"] == depth_golden["304"]["depth_counts"]
        blk = tmp_path / "prune-ud-304-blk.bin"
        assert _sha(np.fromfile(blk, np.uint8)) == golden["block_sha256"]

        # mod-3 file: residues in 2 bits, 3 past the end; its value counts are the depth counts
        # folded mod 3 (the reference's build self-check, table.py:146-149)
        words = np.fromfile(mod3, np.uint32)
        assert len(words) == (n + 15) // 16
        lo, hi = words & np.uint32(0x55555555), (words >> 1) & np.uint32(0x55555555)
        got = [int(np.bitwise_count(~lo & ~hi & np.uint32(0x55555555)).sum()), int(np.bitwise_count(lo & ~hi).sum()),
               int(np.bitwise_count(hi & ~lo).sum()), int(np.bitwise_count(lo & hi).sum())]
        counts = meta["depth_counts"]
        want = [sum(counts[d] for d in range(r, len(counts), 3)) for r in range(3)] + [len(words) * 16 - n]
        assert got == want
        # where the block table is exact (offset < 3) its value has the mod-3 file's residue
        bw = np.fromfile(blk, np.uint32).reshape(-1, 8)
        x = np.random.default_rng(5).integers(0, n, 200_000, dtype=np.int64)
        sec, j = x // 124, x % 124
        pos = 8 + 2 * j
        off = (bw[sec, pos // 32] >> (pos % 32).astype(np.uint32)) & 3
        r = (words[x // 16] >> (2 * (x % 16)).astype(np.uint32)) & 3
        exact = off < 3
        assert exact.any()
        assert np.array_equal(((bw[sec, 0] & 0xFF) + off)[exact] % 3, r[exact])

        b3 = table.build_b3_table(tmp_path, "304", handle=h, log=lambda *_: None)
        b3_bytes = np.fromfile(b3, np.uint8)
        assert _sha(b3_bytes) == golden["b3_sha256"]  # the same file as the depth-array encoder's

        h.load_table("304", "block", blk)
        out = tmp_path / "saved-blk.bin"
        table.save_device(h, out)
        assert _sha(np.fromfile(out, np.uint8)) == golden["block_sha256"]
        bins = table.histogram(h)
        assert sum(bins) == n
        assert bins == _block_histogram(bw.reshape(-1), n).tolist()
        assert bins[0] == counts[0]  # the solved entry's block is exact at depth 0

        h.load_table("304", "b3", b3)
        bins3 = table.histogram(h)
        assert sum(bins3) == n
        assert bins3 == _b3_histogram(b3_bytes, n).tolist()

        with pytest.raises(native.CcsError, match="no table 1"):
            table.save_device(h, tmp_path / "none.bin", table=1)
        with pytest.raises(native.CcsError, match="n_bins"):
            h.table_histogram(0, 0)
        with pytest.raises(native.CcsError, match="no file to write"):
            h.build_table_files("304")
        short = tmp_path / "short-mod3.bin"
        words[:1000].tofile(short)
        with pytest.raises(native.CcsError, match="size 4000"):
            table.write_b3(short, blk, "304", tmp_path / "x-b3.bin", handle=h)
    finally:
        h.close()


def test_building_another_kind_leaves_the_resident_table_usable(tmp_path):
    """A build that keeps nothing (ccs_build_table with keep_resident 0, ccs_build_table_files)
    leaves the loaded table answering with its own kind's constants."""

    h = native.Handle()
    try:
        h.build_table("304", "block", None, keep_resident=True)
        rng = np.random.default_rng(11)
        states = [apply_moves(CubieState(), [MOVES_HTM[int(m)] for m in rng.integers(0, 18, 14)]) for _ in range(64)]
        words = state_words(states)
        before = h.lower_bound(words).tolist()
        h.build_table("s4", "b3", None, keep_resident=False)
        assert h.lower_bound(words).tolist() == before
        h.build_table_files("s4", b3_path=tmp_path / "prune-ud-s4-b3.bin")
        assert h.lower_bound(words).tolist() == before
    finally:
        h.close()
