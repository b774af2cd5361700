"""Optimal HTM solver: IDA* on the GPU with a resident pruning table (the reference's ``solver.py``).

Same public surface as the reference (``solver.py:1-325``): ``open_solver``, ``GpuSolver`` with
``solve`` and ``root_h``, ``Solution``, ``TableNotFound``, ``NoTableFits``, ``frames``,
``canonical_prefixes``, ``allowed``, ``parse_moves``.  The search itself runs in libccs: one
persistent launch takes every cube of a ``solve`` call through its IDA* bounds on the device
(no host round trip per bound), and a host check verifies every returned solution.
"""

from __future__ import annotations

import re
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from cuda_cube_solver import coords, kinds, native
from cuda_cube_solver.cubie import MOVE_NAMES_HTM, MOVES_HTM, CubieState, apply_moves
from cuda_cube_solver.device import state_words
from cuda_cube_solver.prefixes import allowed, canonical_prefixes, frames  # noqa: F401  (public surface)


@dataclass
class Solution:
    moves: list[int]
    nodes: int
    seconds: float
    iteration_nodes: list[tuple[int, int]] = field(default_factory=list)  # (bound, nodes)
    probes: int = 0

    def text(self) -> str:
        return " ".join(MOVE_NAMES_HTM[m] for m in self.moves)


class TableNotFound(FileNotFoundError):
    """A pruning table file is missing."""


class NoTableFits(RuntimeError):
    """No table preset fits in the GPU memory budget."""


def _table_file(tables: Path, name: str) -> Path:
    path = tables / name
    if not path.exists():
        m = re.fullmatch(r"prune-ud-(\d+|[a-z0-9]+)(?:-blk)?(-b3)?\.bin", name)
        hint = f"; build it with `cuda-cube-solver build-table --table {m[1]}{m[2] or ''} --out {tables}`" if m else ""
        raise TableNotFound(f"{path} not found{hint}")
    return path


def open_solver(tables: Path = Path("tables"), memory="auto", table: str | None = None, build: bool = True,
                log=print) -> "GpuSolver":
    """A solver with the fastest table preset that fits ``memory`` (GB, or "auto": the free device
    memory), or the preset named ``table`` (see ``kinds.PRESETS``).  A missing table is built first
    unless ``build`` is False."""

    from cuda_cube_solver import table as tables_mod

    tables = Path(tables)
    if tables.suffix == ".bin":
        tables = tables.parent
    preset = kinds.pick(tables, memory, table)[0]
    if preset is None:
        raise NoTableFits("no table fits in that GPU memory (the smallest, 304, needs 1.8 GB)")
    if not (tables / preset.file).exists():
        if not build:
            raise TableNotFound(f"{tables / preset.file} not found")
        log(f"building table {preset.name} ({preset.table_bytes / 1e9:.2f} GB) in {tables}/")
        log(f"wrote {tables_mod.build_preset(tables, preset, log=lambda m: log(f'  {m}'))}")
    return GpuSolver(tables, kind=preset.kind, table_format=preset.format)


class GpuSolver:
    """IDA* solver over a solving table resident on the GPU.

    ``prefix_len``: prefix length of the work items of a cube's first iterations; an iteration of
    at least ``deeper_prefix_at[i]`` nodes makes the next one use one move more.  ``grid`` is the
    number of blocks of the persistent launch (default: the library's choice for the kernel
    variant); ``block`` is accepted for compatibility (the kernel's block size is fixed per variant).
    ``handle``: an already open ``native.Handle`` holding the table (``table_format`` and ``kind``
    must then describe it), e.g. one that built it with ``keep_resident``.
    """

    def __init__(self, tables: Path = Path("tables"), prefix_len: int = 4, grid: int | None = None, block: int = 256,
                 inverse: bool = True, collect_stats: bool = False, mode: str = "step",
                 extra_tables: int = 2, step_extra: int = 0, table_format: str = "block",
                 step_defines: tuple[str, ...] = (), kind="d4t",
                 deeper_prefix_at: tuple[float, ...] | None = None, extra_kind=None,
                 handle: native.Handle | None = None, device: int = 0):
        # The reference's keywords (solver.py:119-123) are all accepted; those of its experimental
        # search modes (extra tables, extra kinds, NVRTC defines) are not built and are refused
        # with ValueError like the reference refuses invalid combinations (solver.py:145-148).
        # ``extra_tables`` only matters for mode="multi", which is refused below.
        if mode != "step" or not inverse:
            raise ValueError("only the step search with inverse frames is built (mode='step', inverse=True)")
        if step_extra:
            raise ValueError("step_extra tables (208 + 112/304 lookups) are not built; use a kind preset")
        if step_defines:
            raise ValueError("step_defines (NVRTC kernel defines) do not apply: the kernels are compiled for sm_100a")
        if extra_kind is not None:
            raise ValueError("extra_kind (a second lookup table per node) is not built; attach_second() keeps a "
                             "second table resident and picks one per cube")
        tables = Path(tables)
        if tables.suffix == ".bin":
            tables = tables.parent
        self.kind = kinds.get(kind) if isinstance(kind, str) else kind
        self.table_format = table_format
        if table_format not in native.FORMATS:
            raise ValueError(f"unknown table format {table_format!r}")
        self.prefix_len = prefix_len
        # Given explicitly, the thresholds mean what they mean in the reference (no few-cube
        # division); by default the library also deepens prefixes sooner for a lone hard cube.
        self.exact_thresholds = deeper_prefix_at is not None
        if deeper_prefix_at is None:
            deeper_prefix_at = (5e7, 3e9)
        self.deeper_prefix_at = tuple(deeper_prefix_at) + (float("inf"),) * (2 - len(deeper_prefix_at))
        self.collect_stats = collect_stats
        if handle is None:
            handle = native.Handle(device)
            fname = f"prune-ud-{self.kind.name}-{'b3' if table_format == 'b3' else 'blk'}.bin"
            try:
                handle.load_table(self.kind.name, table_format, _table_file(tables, fname))
            except native.CcsError as exc:
                raise ValueError(str(exc)) if exc.code == native.CCS_E_FILE else exc
        self.handle = handle
        sms = native.ctypes.c_int()
        native.check(native.lib.ccs_device_sms(handle.device, native.ctypes.byref(sms)))
        self.sms = sms.value
        self.grid = grid  # None: the library's default for the kernel variant
        self.block = block
        self.last_kernel_ms = 0.0
        self.last_probes = 0
        self.variant = 0  # search kernel variant (libccs); 0 lets the library choose by batch size
        self.tuned: dict | None = None  # settings chosen by autotune(); else the cached ones
        self.tuned_bucket: str | None = None  # the batch-size bucket they were measured on
        self.use_autotune = True
        self.second_kind: str | None = None  # kind of the attached second table (table id 1)
        self.flip_rule = FLIP_RULE

    def attach_second(self, kind: str = "d4", path: Path | None = None, log=None) -> None:
        """Keep a second table of ``kind`` resident beside the first (loaded from ``path``, else
        built on the GPU).  Cubes with at least ``flip_rule`` flipped edges are then searched with it."""

        if path is None:
            self.handle.build_table(kind, self.table_format, None, keep_resident=2, log=log)
        else:
            self.handle.attach_table(kind, self.table_format, path)
        self.second_kind = kind

    def table_ids(self, words: np.ndarray) -> np.ndarray | None:
        """Per cube 0 (first table) or 1 (second table, when attached) by the flip-count rule."""

        if self.second_kind is None:
            return None
        return (flipped_edges(words) >= self.flip_rule).astype(np.uint8)

    @classmethod
    def build_resident(cls, kind: str = "d4t", table_format: str = "block", log=None, device: int = 0,
                       second_kind: str | None = None, **kw):
        """Build ``kind`` on the GPU and solve with it straight from device memory (no file);
        ``second_kind`` also builds a second resident table (see ``attach_second``)."""

        h = native.Handle(device)
        counts, secs = h.build_table(kind, table_format, None, keep_resident=True, log=log)
        solver = cls(kind=kind, table_format=table_format, handle=h, **kw)
        solver.build_counts, solver.build_seconds = counts, secs
        if second_kind:
            solver.attach_second(second_kind, log=log)
        return solver

    def _opts(self, timeout_s: float = 0.0, n: int = 0) -> native.SolveOpts:
        blocks_per_sm = max(1, round(self.grid / self.sms)) if self.grid else 0
        o = native.solve_opts(self.prefix_len, self.deeper_prefix_at[:2], blocks_per_sm, 0, timeout_s,
                              variant=self.variant, few_divisor=1 if self.exact_thresholds else 0)
        from cuda_cube_solver import autotune

        # tuned settings hold for the batch-size bucket they were measured on (a setting chosen
        # for thousands of cubes is not the one for a lone cube); other sizes keep the defaults
        tuned = self.tuned if self.tuned is not None and autotune.batch_bucket(n or 1) == self.tuned_bucket else None
        if tuned is None and self.use_autotune:
            tuned = autotune.lookup(self.table_name, n or 1, self.handle.device)
        if tuned:
            o.variant, o.base_plen, o.spread = tuned["variant"], tuned["base_plen"], tuned["spread"]
            o.move_min, o.move_age = tuned["move"]
            o.probe_min = tuned.get("probe_min", 0)
            o.steal_depth = tuned.get("steal_depth", 0)
        return o

    @property
    def table_name(self) -> str:
        return self.kind.name if self.table_format == "block" else f"{self.kind.name}-b3"

    def autotune(self, sample: list[CubieState], log=None, save: bool = True, budget_s: float = 0.0,
                 target_n: int | None = None) -> dict:
        """Measure the kernel settings on ``sample`` and use the best from now on (within
        ``budget_s`` seconds when it is > 0) for batches of ``target_n`` cubes' size bucket
        (default: the sample's own size)."""

        from cuda_cube_solver import autotune

        result = autotune.tune(self.handle, sample, self.table_name, log=log, budget_s=budget_s)
        n = target_n or len(sample)
        self.tuned = result["config"]
        self.tuned_bucket = autotune.batch_bucket(n)
        if save:
            autotune.save(result, self.table_name, n, self.handle.device)
        return result

    def root_h(self, states: list[CubieState]) -> tuple[np.ndarray, np.ndarray]:
        words = state_words(states)
        frame_words = state_words([f for s in states for f in frames(s)]).reshape(len(states), 30)
        return self.handle.root_bounds(words), frame_words

    def solve(self, states: list[CubieState], log=None) -> list[Solution]:
        if not states:
            return []
        words = state_words(states)
        t0 = time.perf_counter()
        results = self.handle.solve(words, self._opts(n=len(states)), self.table_ids(words))
        self.last_kernel_ms, self.last_probes, _ = self.handle.last_solve_stats()
        out = []
        for state, r in zip(states, results):
            if r.status != 0:
                raise AssertionError(f"search failed with status {r.status}")
            moves = list(r.moves[: r.length])
            hist = [(b, int(r.iter_nodes[b])) for b in range(24) if r.iter_nodes[b]]
            out.append(Solution(moves, int(r.nodes), float(r.seconds), hist, int(r.probes)))
        if log:
            log(f"{time.perf_counter() - t0:8.2f}s solved {len(out)}/{len(states)}")
        if not verify_solutions(words, [sol.moves for sol in out]):
            raise AssertionError("solution does not solve the cube")
        return out

    def close(self) -> None:
        self.handle.close()


# Cubes with this many flipped edges or more go to the second table when one is attached.  Measured
# on one B200 with d4t and d4 resident: the superflip (all 12 edges flipped) takes 13.5 G probes on
# d4 against 72.7 G on d4t (5.1x faster), while uniform cubes with 10 flipped edges are still
# faster on d4t (127 vs 103 cubes/s), so only fully flipped positions switch.
FLIP_RULE = 12


def flipped_edges(words: np.ndarray) -> np.ndarray:
    """Number of flipped edges of each packed state (n, 5): bit 4 of the twelve edge bytes."""

    b = np.ascontiguousarray(words, np.uint32).reshape(-1, 5).view(np.uint8).reshape(-1, 20)
    return ((b[:, 8:] >> 4) & 1).sum(axis=1)


def verify_solutions(words: np.ndarray, solutions: list[list[int]]) -> bool:
    """True if every move list takes its packed state (n, 5) to solved (the reference's host
    self-check, solver.py:317-319, vectorised over cubes)."""

    b = np.ascontiguousarray(words, np.uint32).reshape(-1, 5).view(np.uint8).reshape(-1, 20)
    corners, edges = b[:, :8].copy(), b[:, 8:].copy()
    longest = max((len(m) for m in solutions), default=0)
    for j in range(longest):
        col = np.array([m[j] if j < len(m) else -1 for m in solutions])
        for mv in np.unique(col[col >= 0]):
            rows = col == mv
            corners[rows], edges[rows] = coords.apply_move(corners[rows], edges[rows], int(mv))
    solved = np.concatenate([np.arange(8, dtype=np.uint8)[None], np.arange(12, dtype=np.uint8)[None]], axis=1)
    return bool((np.concatenate([corners, edges], axis=1) == solved).all())


def parse_moves(text: str) -> list[int]:
    index = {name: i for i, name in enumerate(MOVE_NAMES_HTM)}
    return [index[tok] for tok in text.split()]
