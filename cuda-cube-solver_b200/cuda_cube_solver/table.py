"""Building and loading the pruning tables (the reference's ``table.py``).

The BFS, its self-checks and the block / base-3 encoders run in libccs on the GPU
(``ccs_build_table``); this module keeps the reference's entry points and file conventions:
``build_preset`` writes only the solving file (through ``.tmp`` and a rename) plus the ``.json``
meta with the per-depth counts (``table.py:170-200``, ``kinds.py:223-225``).
"""

from __future__ import annotations

import time
from pathlib import Path

from cuda_cube_solver import kinds, native

BLOCK_ENTRIES = 124
B3_ENTRIES = 155
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
