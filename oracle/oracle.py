"""ctypes binding of the CPU oracle (``oracle/ccs_oracle.c``).  TEST INFRASTRUCTURE ONLY.

Used by tests/ as the checker, by ``__graft_entry__.smoke`` and by bench.py's CPU baseline; the
package never imports it.  The oracle gets its constant tables from the package's Python host
model (moves, U-D symmetry actions, corner classes, E-content classes), which tests pin to the
reference's own host model through tests/golden fixtures.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libccs_oracle.so"


def build() -> Path:
    if not LIB.exists() or LIB.stat().st_mtime < (HERE / "ccs_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), str(LIB.relative_to(HERE))], check=True, capture_output=True)
    return LIB


def _host():
    sys.path.insert(0, str(HERE.parent / "cuda-cube-solver_b200"))
    from cuda_cube_solver import coords, cubie, geometry

    return coords, cubie, geometry


class Oracle:
    """One loaded oracle (process-wide state in the C library: one kind at a time)."""

    def __init__(self):
        self.lib = ctypes.CDLL(str(build()))
        coords, cubie, geometry = _host()
        mv = cubie.MOVES_HTM
        self._keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a.ctypes.data_as(ctypes.c_void_p)

        _, edge_syms = coords.ud_actions()
        syms = geometry.ud_symmetries()
        sym_mul = np.zeros((16, 16), np.uint8)
        for t in range(16):
            for s in range(16):
                prod = syms[t].matrix @ syms[s].matrix
                sym_mul[t, s] = next(i for i, u in enumerate(syms) if np.array_equal(u.matrix, prod))
        rot = geometry.move_map(geometry.axis_rotation())
        frame_move = np.array([list(range(18)), rot, [rot[rot[m]] for m in range(18)]], np.uint8)
        cc = coords.corner_classes()
        self.lib.orc_init(arr([m.cp for m in mv], np.uint8), arr([m.co for m in mv], np.uint8),
                          arr([m.ep for m in mv], np.uint8), arr([m.eo for m in mv], np.uint8),
                          arr([e.perm for e in edge_syms], np.uint8), arr([e.flip for e in edge_syms], np.uint8),
                          arr(sym_mul, np.uint8), arr(frame_move, np.uint8),
                          arr(cc.classidx, np.uint32), arr(cc.rep, np.uint32), arr(cc.stab, np.uint16))
        self.lib.orc_n_entries.restype = ctypes.c_uint64
        self.lib.orc_encode_block.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        self.lib.orc_encode_b3.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        self.lib.orc_solve_many.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p]
        self.kind = None

    def set_kind(self, name: str) -> None:
        sys.path.insert(0, str(HERE.parent / "cuda-cube-solver_b200"))
        from cuda_cube_solver import kinds

        k = kinds.get(name)
        if name == "304":
            self.lib.orc_set_kind(2, 1, None, None)
        else:
            gc = np.ascontiguousarray(k.gen[0], np.uint16)
            gr = np.ascontiguousarray(k.gen[1], np.uint16)
            self._keep += [gc, gr]
            self.lib.orc_set_kind(1, k.nec, gc.ctypes.data_as(ctypes.c_void_p), gr.ctypes.data_as(ctypes.c_void_p))
        self.kind = name

    def n_entries(self) -> int:
        return int(self.lib.orc_n_entries())

    def index(self, words: np.ndarray, move: int = -1) -> np.ndarray:
        words = np.ascontiguousarray(words, np.uint32).reshape(-1, 5)
        out = np.zeros(len(words), np.uint64)
        self.lib.orc_index(words.ctypes.data_as(ctypes.c_void_p), len(words), move,
                           out.ctypes.data_as(ctypes.c_void_p))
        return out

    def unrank(self, idx: np.ndarray) -> np.ndarray:
        idx = np.ascontiguousarray(idx, np.uint64).reshape(-1)
        out = np.zeros((len(idx), 5), np.uint32)
        self.lib.orc_unrank(idx.ctypes.data_as(ctypes.c_void_p), len(idx), out.ctypes.data_as(ctypes.c_void_p))
        return out

    def lower_bound(self, table: np.ndarray, fmt: str, words: np.ndarray) -> np.ndarray:
        words = np.ascontiguousarray(words, np.uint32).reshape(-1, 5)
        out = np.zeros(len(words), np.uint32)
        self.lib.orc_lower_bound(table.ctypes.data_as(ctypes.c_void_p), 1 if fmt == "b3" else 0,
                                 words.ctypes.data_as(ctypes.c_void_p), len(words), out.ctypes.data_as(ctypes.c_void_p))
        return out

    def bfs(self, threads: int | None = None) -> tuple[np.ndarray, list[int]]:
        n = self.n_entries()
        depth = np.empty(n, np.uint8)
        counts = np.zeros(64, np.uint64)
        nd = self.lib.orc_bfs(depth.ctypes.data_as(ctypes.c_void_p), threads or os.cpu_count() or 1,
                              counts.ctypes.data_as(ctypes.c_void_p), 64)
        if nd < 0:
            raise RuntimeError(f"oracle BFS failed ({nd})")
        return depth, [int(c) for c in counts[:nd]]

    def encode_block(self, depth: np.ndarray) -> np.ndarray:
        out = np.empty(-(-len(depth) // 124) * 32, np.uint8)
        self.lib.orc_encode_block(depth.ctypes.data_as(ctypes.c_void_p), len(depth), out.ctypes.data_as(ctypes.c_void_p))
        return out

    def encode_b3(self, depth: np.ndarray, blk: np.ndarray) -> np.ndarray:
        out = np.empty(-(-len(depth) // 155) * 32, np.uint8)
        self.lib.orc_encode_b3(depth.ctypes.data_as(ctypes.c_void_p), blk.ctypes.data_as(ctypes.c_void_p), len(depth),
                               out.ctypes.data_as(ctypes.c_void_p))
        return out

    def solve_many(self, table: np.ndarray, fmt: str, frames: np.ndarray, threads: int | None = None,
                   budget_s: float = 0.0):
        """Solve cubes given their six frames (n, 30) on host threads; returns (lengths, moves,
        nodes, probes) with length -1 for cubes cut off by ``budget_s``."""

        frames = np.ascontiguousarray(frames, np.uint32).reshape(-1, 30)
        n = len(frames)
        lengths = np.zeros(n, np.int32)
        moves = np.zeros((n, 24), np.uint8)
        nodes = np.zeros(n, np.uint64)
        probes = np.zeros(n, np.uint64)
        self.lib.orc_solve_many(table.ctypes.data_as(ctypes.c_void_p), 1 if fmt == "b3" else 0,
                                frames.ctypes.data_as(ctypes.c_void_p), n, threads or os.cpu_count() or 1,
                                float(budget_s), lengths.ctypes.data_as(ctypes.c_void_p),
                                moves.ctypes.data_as(ctypes.c_void_p), nodes.ctypes.data_as(ctypes.c_void_p),
                                probes.ctypes.data_as(ctypes.c_void_p))
        return lengths, moves, nodes, probes
