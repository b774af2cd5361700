"""Cubie-level model of the 3x3 cube: states, the 18 half-turn-metric moves, composition.

Same conventions as the reference model (``src/cuda_cube_solver/cubie.py:1-201``):

* ``cp[i]`` is the corner cubie at corner position ``i`` and ``co[i]`` the slot (0..2, in the
  position's name order, clockwise) that holds that cubie's U/D sticker;
* ``ep[i]`` / ``eo[i]`` likewise for edges, ``eo[i]`` being the slot of the cubie's first sticker;
* ``compose(a, b)`` is "apply transform ``b`` after state ``a``":
  ``cp[i] = a.cp[b.cp[i]]``, ``co[i] = a.co[b.cp[i]] + b.co[i] (mod 3)``.

The reference lists the six face quarter turns as literal tables (``cubie.py:58-95``).  Here
they are derived from 3D geometry instead: a face turn rotates every cubie whose centre lies on
that face by -90 degrees about the face normal, and the permutation and orientation follow from
where each position and sticker normal goes.  ``tests/test_host_model.py`` checks the derived
moves against the reference's tables (golden fixture).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Iterable, Sequence

CORNER_NAMES = ("URF", "UFL", "ULB", "UBR", "DFR", "DLF", "DBL", "DRB")
EDGE_NAMES = ("UR", "UF", "UL", "UB", "DR", "DF", "DL", "DB", "FR", "FL", "BL", "BR")
FACE_NAMES = ("U", "R", "F", "D", "L", "B")

# Face normals in x = R, y = U, z = F coordinates.
FACE_NORMAL = {
    "U": (0, 1, 0), "R": (1, 0, 0), "F": (0, 0, 1),
    "D": (0, -1, 0), "L": (-1, 0, 0), "B": (0, 0, -1),
}
_NORMAL_FACE = {v: k for k, v in FACE_NORMAL.items()}


def permutation_parity(permutation: Sequence[int]) -> int:
    """0 for an even permutation, 1 for odd (counted by inversions)."""

    n = len(permutation)
    return sum(permutation[i] > permutation[j] for i in range(n) for j in range(i + 1, n)) & 1


@dataclass(frozen=True, slots=True)
class CubieState:
    cp: tuple[int, ...] = tuple(range(8))
    co: tuple[int, ...] = (0,) * 8
    ep: tuple[int, ...] = tuple(range(12))
    eo: tuple[int, ...] = (0,) * 12

    def then(self, transform: "CubieState") -> "CubieState":
        return compose(self, transform)

    def inverse(self) -> "CubieState":
        cinv = [0] * 8
        einv = [0] * 12
        for pos, cub in enumerate(self.cp):
            cinv[cub] = pos
        for pos, cub in enumerate(self.ep):
            einv[cub] = pos
        return CubieState(
            tuple(cinv),
            tuple((3 - self.co[cinv[i]]) % 3 for i in range(8)),
            tuple(einv),
            tuple(self.eo[einv[i]] for i in range(12)),
        )

    def is_legal(self) -> bool:
        return (
            sorted(self.cp) == list(range(8))
            and sorted(self.ep) == list(range(12))
            and all(0 <= v < 3 for v in self.co)
            and all(0 <= v < 2 for v in self.eo)
            and sum(self.co) % 3 == 0
            and sum(self.eo) % 2 == 0
            and permutation_parity(self.cp) == permutation_parity(self.ep)
        )


IDENTITY = CubieState()


def compose(a: CubieState, b: CubieState) -> CubieState:
    """The state reached by applying transform ``b`` after state ``a``."""

    return CubieState(
        tuple(a.cp[j] for j in b.cp),
        tuple((a.co[j] + o) % 3 for j, o in zip(b.cp, b.co)),
        tuple(a.ep[j] for j in b.ep),
        tuple((a.eo[j] + o) % 2 for j, o in zip(b.ep, b.eo)),
    )


def power(transform: CubieState, exponent: int) -> CubieState:
    result = IDENTITY
    for _ in range(exponent % 4):
        result = compose(result, transform)
    return result


# --- face turns from geometry -----------------------------------------------------------


def _center(name: str) -> tuple[int, int, int]:
    return tuple(sum(FACE_NORMAL[f][axis] for f in name) for axis in range(3))


def _rotate_cw(face: str, v: tuple[int, int, int]) -> tuple[int, int, int]:
    """Rotate ``v`` by a clockwise quarter turn of ``face`` (seen from outside the cube)."""

    n = FACE_NORMAL[face]
    # Clockwise seen from +n is the rotation by -90 degrees about n: v -> v x n for a unit axis n
    # (Rodrigues with sin = -1, cos = 0), plus the component along n, which stays.
    dot = sum(a * b for a, b in zip(v, n))
    cross = (v[1] * n[2] - v[2] * n[1], v[2] * n[0] - v[0] * n[2], v[0] * n[1] - v[1] * n[0])
    return tuple(dot * n[i] + cross[i] for i in range(3))


def _face_turn(face: str) -> CubieState:
    """The clockwise quarter turn of ``face`` as a transform (the state it makes from solved)."""

    normal = FACE_NORMAL[face]

    def build(names: tuple[str, ...], modulus: int):
        where = {_center(n): i for i, n in enumerate(names)}
        perm = list(range(len(names)))
        orient = [0] * len(names)
        for p, name in enumerate(names):
            c = _center(name)
            if sum(a * b for a, b in zip(c, normal)) <= 0:
                continue  # not in the turning layer
            q = where[_rotate_cw(face, c)]
            perm[q] = p  # position q now holds the cubie from p
            # The cubie's first sticker (index 0 of its name) lands on face rot(normal of name[0]).
            lands = _NORMAL_FACE[_rotate_cw(face, FACE_NORMAL[name[0]])]
            orient[q] = names[q].index(lands) % modulus
        return tuple(perm), tuple(orient)

    cp, co = build(CORNER_NAMES, 3)
    ep, eo = build(EDGE_NAMES, 2)
    return CubieState(cp, co, ep, eo)


FACE_QUARTERS: tuple[CubieState, ...] = tuple(_face_turn(f) for f in FACE_NAMES)

MOVE_NAMES_HTM: tuple[str, ...] = tuple(f + s for f in FACE_NAMES for s in ("", "2", "'"))
MOVES_HTM: tuple[CubieState, ...] = tuple(power(FACE_QUARTERS[f], t) for f in range(6) for t in (1, 2, 3))
MOVE_NAMES_QTM: tuple[str, ...] = tuple(f + s for f in FACE_NAMES for s in ("", "'"))
MOVES_QTM: tuple[CubieState, ...] = tuple(power(FACE_QUARTERS[f], t) for f in range(6) for t in (1, 3))

FIXED_CORNER_FACES = (0, 1, 2)  # U, R, F leave DBL fixed.
MOVE_NAMES_2_HTM: tuple[str, ...] = tuple(f + s for f in ("U", "R", "F") for s in ("", "2", "'"))
MOVES_2_HTM: tuple[CubieState, ...] = tuple(power(FACE_QUARTERS[f], t) for f in FIXED_CORNER_FACES for t in (1, 2, 3))
MOVE_NAMES_2_QTM: tuple[str, ...] = tuple(f + s for f in ("U", "R", "F") for s in ("", "'"))
MOVES_2_QTM: tuple[CubieState, ...] = tuple(power(FACE_QUARTERS[f], t) for f in FIXED_CORNER_FACES for t in (1, 3))


def apply_moves(state: CubieState, moves: Iterable[CubieState]) -> CubieState:
    for move in moves:
        state = compose(state, move)
    return state


def pack_state(state: CubieState) -> tuple[int, int]:
    """Two 64-bit words: ``lo`` = cp nibbles | co 2-bit fields << 32 | eo bits << 48, ``hi`` = ep nibbles
    (the reference's ``cubie.pack_state``)."""

    lo = sum(v << (4 * i) for i, v in enumerate(state.cp))
    lo |= sum(v << (32 + 2 * i) for i, v in enumerate(state.co))
    lo |= sum(v << (48 + i) for i, v in enumerate(state.eo))
    hi = sum(v << (4 * i) for i, v in enumerate(state.ep))
    return lo, hi


def unpack_state(lo: int, hi: int) -> CubieState:
    return CubieState(
        tuple((lo >> (4 * i)) & 15 for i in range(8)),
        tuple((lo >> (32 + 2 * i)) & 3 for i in range(8)),
        tuple((hi >> (4 * i)) & 15 for i in range(12)),
        tuple((lo >> (48 + i)) & 1 for i in range(12)),
    )


def apply_packed(lo: int, hi: int, move: CubieState) -> tuple[int, int]:
    return pack_state(compose(unpack_state(lo, hi), move))
