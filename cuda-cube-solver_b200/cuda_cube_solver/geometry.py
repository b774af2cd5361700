"""The 48 cube symmetries and their action on cubie states.

A symmetry is a signed 3x3 permutation matrix ``M`` acting on sticker slots (a slot is a
cubie position plus the normal of one of its faces).  Conjugation ``g -> M g M^-1`` acts on a
state seen as a slot -> home-slot map; it is valid for reflections too.

Follows the reference's ``src/cuda_cube_solver/geometry.py:1-148``: the same enumeration order
of the 48 matrices (every permutation of the axes, every sign pattern, identity moved first),
the 16 that keep the U-D axis, and the 120-degree turn about the URF diagonal that maps R to U
to F (``axis_rotation``).  Symmetry indices are part of the table index (the corner class
stores the first symmetry reaching the class representative), so the order is kept.
"""

from __future__ import annotations

from functools import lru_cache
from itertools import permutations, product

import numpy as np

from cuda_cube_solver.cubie import CORNER_NAMES, EDGE_NAMES, FACE_NORMAL, MOVES_HTM, CubieState


def _center(name: str) -> tuple[int, ...]:
    return tuple(int(sum(FACE_NORMAL[f][a] for f in name)) for a in range(3))


# Slot 3*i + k (corners) / 2*i + k (edges): position i, the face of letter k of its name.
CORNER_SLOTS = [(_center(n), FACE_NORMAL[f]) for n in CORNER_NAMES for f in n]
EDGE_SLOTS = [(_center(n), FACE_NORMAL[f]) for n in EDGE_NAMES for f in n]
_CORNER_SLOT = {s: i for i, s in enumerate(CORNER_SLOTS)}
_EDGE_SLOT = {s: i for i, s in enumerate(EDGE_SLOTS)}


def cubie_to_slots(state: CubieState) -> tuple[np.ndarray, np.ndarray]:
    """Slot -> home slot of the sticker sitting there (24 corner slots, 24 edge slots)."""

    corners = np.empty(24, dtype=np.int64)
    edges = np.empty(24, dtype=np.int64)
    for i, (c, o) in enumerate(zip(state.cp, state.co)):
        for k in range(3):
            corners[3 * i + (k + o) % 3] = 3 * c + k
    for i, (e, o) in enumerate(zip(state.ep, state.eo)):
        for k in range(2):
            edges[2 * i + (k + o) % 2] = 2 * e + k
    return corners, edges


def slots_to_cubie(corners: np.ndarray, edges: np.ndarray) -> CubieState:
    cp = tuple(int(corners[3 * i]) // 3 for i in range(8))
    co = tuple((3 - int(corners[3 * i]) % 3) % 3 for i in range(8))
    ep = tuple(int(edges[2 * i]) // 2 for i in range(12))
    eo = tuple(int(edges[2 * i]) % 2 for i in range(12))
    return CubieState(cp, co, ep, eo)


class Symmetry:
    """A cube symmetry as permutations of the corner and edge sticker slots."""

    def __init__(self, matrix: np.ndarray):
        self.matrix = np.asarray(matrix, dtype=np.int64)
        self.det = int(round(np.linalg.det(self.matrix)))

        def image(slot):
            c, n = slot
            return tuple(int(x) for x in self.matrix @ np.array(c)), tuple(int(x) for x in self.matrix @ np.array(n))

        self.corner = np.array([_CORNER_SLOT[image(s)] for s in CORNER_SLOTS])
        self.edge = np.array([_EDGE_SLOT[image(s)] for s in EDGE_SLOTS])
        self.corner_inv = np.argsort(self.corner)
        self.edge_inv = np.argsort(self.edge)

    def preserves_ud(self) -> bool:
        return abs(int(self.matrix[1, 1])) == 1

    def conjugate_slots(self, corners: np.ndarray, edges: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """``M g M^-1`` on slot maps; a trailing axis of 24 slots, any leading axes."""

        return self.corner[corners[..., self.corner_inv]], self.edge[edges[..., self.edge_inv]]

    def conjugate(self, state: CubieState) -> CubieState:
        return slots_to_cubie(*self.conjugate_slots(*cubie_to_slots(state)))


@lru_cache(maxsize=1)
def all_symmetries() -> tuple[Symmetry, ...]:
    mats = []
    for perm in permutations(range(3)):
        for signs in product((1, -1), repeat=3):
            m = np.zeros((3, 3), dtype=np.int64)
            for row, col in enumerate(perm):
                m[row, col] = signs[row]
            mats.append(m)
    eye = next(i for i, m in enumerate(mats) if np.array_equal(m, np.eye(3, dtype=np.int64)))
    order = [eye] + [i for i in range(len(mats)) if i != eye]
    return tuple(Symmetry(mats[i]) for i in order)


@lru_cache(maxsize=1)
def ud_symmetries() -> tuple[Symmetry, ...]:
    """The 16 symmetries that keep the U-D axis, identity first."""

    syms = tuple(s for s in all_symmetries() if s.preserves_ud())
    assert len(syms) == 16
    return syms


@lru_cache(maxsize=1)
def axis_rotation() -> Symmetry:
    """The 120-degree turn about the URF diagonal: x -> y -> z -> x (R -> U -> F -> R)."""

    return Symmetry(np.array([[0, 0, 1], [1, 0, 0], [0, 1, 0]], dtype=np.int64))


def compose_slots(a: tuple[np.ndarray, np.ndarray], b: tuple[np.ndarray, np.ndarray]):
    """Slot-level ``compose(a, b)``: apply ``b`` after ``a``."""

    return a[0][b[0]], a[1][b[1]]


def move_map(sym: Symmetry) -> list[int]:
    """For every HTM move ``m``, the index of ``M m M^-1``; raises if the set is not closed."""

    lookup = {mv: i for i, mv in enumerate(MOVES_HTM)}
    return [lookup[sym.conjugate(MOVES_HTM[m])] for m in range(18)]


def validate() -> None:
    for mv in MOVES_HTM:
        assert slots_to_cubie(*cubie_to_slots(mv)) == mv
    for sym in all_symmetries():
        assert sorted(move_map(sym)) == list(range(18))
    assert move_map(axis_rotation())[0] // 3 in (1, 2, 4, 5)
