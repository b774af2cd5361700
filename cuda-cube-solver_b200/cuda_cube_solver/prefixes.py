"""The host side of the search's frames and work split, without the library: ``frames`` (the six
search frames of a cube, solver.py:58-64 of the reference), ``allowed`` and
``canonical_prefixes`` (the canonical move order and the work items' prefixes, solver.py:33-48).
``cuda_cube_solver.solver`` re-exports them; code that must not load libccs (the reference-GPU
runner, the CPU baseline) imports them from here."""

from __future__ import annotations

from functools import lru_cache

import numpy as np

from cuda_cube_solver.cubie import CubieState
from cuda_cube_solver.geometry import axis_rotation


def allowed(last: int, move: int) -> bool:
    """Canonical order: never the same face twice in a row, opposite faces only as U-D, R-L, F-B."""

    if last < 0:
        return True
    lf, mf = last // 3, move // 3
    return mf != lf and not (lf >= 3 and mf == lf - 3)


@lru_cache(maxsize=None)
def canonical_prefixes(length: int) -> np.ndarray:
    """All canonical move sequences of ``length``, lexicographic (each sequence's children in move order)."""

    seqs = [()]
    for _ in range(length):
        seqs = [s + (m,) for s in seqs for m in range(18) if allowed(s[-1] if s else -1, m)]
    return np.array(seqs, dtype=np.uint8).reshape(len(seqs), length)


def frames(state: CubieState) -> list[CubieState]:
    """The three axis frames of ``state`` (turned so each axis becomes U-D) followed by their inverses."""

    rot = axis_rotation()
    once = rot.conjugate(state)
    axes = [state, once, rot.conjugate(once)]
    return axes + [f.inverse() for f in axes]
