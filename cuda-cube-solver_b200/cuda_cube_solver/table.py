"""Building and loading the pruning tables (the reference's ``table.py``).

The BFS, its self-checks and the block / base-3 / mod-3 encoders run in libccs on the GPU
(``ccs_build_table``, ``ccs_build_table_files``); this module keeps the reference's entry points
and file conventions: ``build`` writes the mod-3 and block files plus a ``.json`` meta
(``table.py:140-167``), ``build_b3_table`` / ``write_b3`` turn those two files into the base-3
file (``table.py:52-79``), ``build_preset`` writes only the solving file (through ``.tmp`` and a
rename) plus the preset's meta (``table.py:170-200``, ``kinds.py:223-225``), ``save_device`` and
``histogram`` act on a table resident in a handle (``table.py:20-25,132-137``).
"""

from __future__ import annotations

import json
import time
from pathlib import Path

from cuda_cube_solver import kinds, native

BLOCK_ENTRIES = 124
B3_ENTRIES = 155
N_CORNER_CLASSES = 9930  # corner coordinates (twist x 8C4) up to the 16 UD symmetries
CHUNK_WORDS = 1 << 26


def block_words(n_entries: int) -> int:
    return -(-n_entries // BLOCK_ENTRIES) * 8


def b3_words(n_entries: int) -> int:
    return -(-n_entries // B3_ENTRIES) * 8


def _kind_name(kind) -> str:
    name = kind if isinstance(kind, str) else kind.name
    if not isinstance(kind, str) and isinstance(kind, kinds.GroupKind) and kind.name not in kinds.GROUP_KINDS:
        native.register_group_kind(kind.name, [(list(p), list(f)) for p, f in kind.gens_list])
    return name


def generate(handle: native.Handle, kind, table_format: str = "block", out_path=None, keep_resident: bool = False,
             log=print) -> tuple[list[int], float]:
    """Build a table on the GPU: returns (per-depth entry counts, seconds).  With ``out_path`` the
    solving file is written; with ``keep_resident`` it stays loaded in ``handle``."""

    return handle.build_table(_kind_name(kind), table_format, out_path, keep_resident, log=log)


def load_device(handle: native.Handle, path: Path, kind, table_format: str = "block") -> None:
    """Load a solving table file into the handle's device memory (size checked)."""

    handle.load_table(_kind_name(kind), table_format, path)


def build_preset(out_dir: Path, preset: kinds.Preset, log=print, handle: native.Handle | None = None) -> Path:
    """Generate a ``kinds.Preset`` table and write only its solving file (block or base 3)."""

    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    h = handle or native.Handle()
    t = time.perf_counter()
    path = out_dir / preset.file
    counts, _ = generate(h, preset.kind, preset.format, out_path=path, log=log)
    kinds.write_meta(path.with_suffix(".json"), preset, counts, time.perf_counter() - t)
    return path


def save_device(handle: native.Handle, path: Path, table: int = 0) -> None:
    """Write a resident table (0, or 1 for the second table) to ``path`` in chunks through pinned
    staging, so host memory stays small (``table.py:20-25`` writes a device array the same way)."""

    handle.save_table(path, table)


def histogram(handle: native.Handle, table: int = 0, n_bins: int = 32) -> list[int]:
    """Entries of a resident table per stored lower bound, counted on the GPU.

    The reference's ``histogram`` (``table.py:132-137``) counts the four 2-bit values of its mod-3
    table; the tables resident here are solving tables, so the bins are their decoded bounds:
    exact below a 2-bit block's minimum + 3 ("at least" there), and for base 3 "at least" at the
    cut.  The bins sum to the kind's entry count; the last bin also holds larger values."""

    return handle.table_histogram(table, n_bins)


def write_b3(mod3_path: Path, block_path: Path, kind, path: Path, handle: native.Handle | None = None) -> None:
    """Base-3 file of ``kind`` from its mod-3 and block files, encoded on the GPU (``table.py:66-79``
    takes the two tables as device arrays; here they are the files, read onto the device in
    chunks with their sizes checked)."""

    h = handle or native.Handle()
    h.encode_b3_file(_kind_name(kind), mod3_path, block_path, path)


def build_b3_table(table_dir: Path, kind="304", handle: native.Handle | None = None, log=print) -> Path:
    """``prune-ud-<kind>-b3.bin`` from the ``prune-ud-<kind>.bin`` (mod 3) and
    ``prune-ud-<kind>-blk.bin`` files of ``table_dir``, both of which must exist (``table.py:52-63``)."""

    table_dir = Path(table_dir)
    name = _kind_name(kind)
    path = table_dir / f"prune-ud-{name}-b3.bin"
    write_b3(table_dir / f"prune-ud-{name}.bin", table_dir / f"prune-ud-{name}-blk.bin", name, path, handle)
    log(f"{path}: {path.stat().st_size / 1e9:.2f} GB")
    return path


def build(out_dir: Path, kind="304", log=print, handle: native.Handle | None = None) -> Path:
    """One BFS of ``kind`` writing ``prune-ud-<kind>.bin`` (depth mod 3, sixteen 2-bit entries per
    little-endian uint32), ``prune-ud-<kind>-blk.bin`` (the 2-bit block table) and the ``.json``
    meta with the per-depth counts (``table.py:140-167``).  The build's self-check is the
    exact-depth histogram against the per-pass counts, on the GPU, before anything is encoded.
    Returns the mod-3 file's path."""

    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    h = handle or native.Handle()
    name = _kind_name(kind)
    path = out_dir / f"prune-ud-{name}.bin"
    blk = out_dir / f"prune-ud-{name}-blk.bin"
    t = time.perf_counter()
    counts, _ = h.build_table_files(name, block_path=blk, mod3_path=path, log=log)
    _, n_entries = native.kind_info(name)
    meta = {
        "kind": name,
        "coordinate": f"UD corner class (twist x 8C4 under the 16 UD symmetries) x {n_entries // N_CORNER_CLASSES:,} "
                      f"edge coordinates of kind {name}",
        "entries": n_entries,
        "classes": N_CORNER_CLASSES,
        "encoding": "2-bit distance mod 3, 16 entries per little-endian uint32",
        "block_table": f"{blk.name}: per 32-byte sector, u8 minimum depth then 124 two-bit offsets (3 = at least +3)",
        "depth_counts": counts,
        "seconds": round(time.perf_counter() - t, 1),
    }
    path.with_suffix(".json").write_text(json.dumps(meta, indent=2) + "\n")
    return path
