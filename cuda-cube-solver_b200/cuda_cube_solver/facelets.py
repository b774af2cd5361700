"""54-sticker facelet strings <-> cubie states.

The layout of the ``kociemba`` package and Cube Explorer: faces in the order U, R, F, D, L, B,
nine stickers each, every face read row by row from its top-left sticker as seen when looking at
it, with U viewed with B at the top, D viewed with F at the top and the side faces with U at the
top.  Any six distinct symbols may be used: the centres define which symbol is which face.

Same interface and error messages as the reference's ``src/cuda_cube_solver/facelets.py:1-113``
(the CLI prints them).  The sticker index of every cubie slot is derived here from the face
grids in 3D rather than listed.
"""

from __future__ import annotations

from collections import Counter

from cuda_cube_solver.cubie import CORNER_NAMES, EDGE_NAMES, FACE_NORMAL, CubieState, permutation_parity

FACES = "URFDLB"
CORNER_FACES = CORNER_NAMES
EDGE_FACES = EDGE_NAMES

# (right, down) directions of each face's 3x3 grid as seen from outside.
_GRID = {
    "U": ((1, 0, 0), (0, 0, 1)),
    "R": ((0, 0, -1), (0, -1, 0)),
    "F": ((1, 0, 0), (0, -1, 0)),
    "D": ((1, 0, 0), (0, 0, -1)),
    "L": ((0, 0, 1), (0, -1, 0)),
    "B": ((-1, 0, 0), (0, -1, 0)),
}


def _sticker_index() -> dict[tuple[tuple[int, ...], str], int]:
    """(cubie centre, face letter) -> facelet index."""

    out = {}
    for f, face in enumerate(FACES):
        n = FACE_NORMAL[face]
        right, down = _GRID[face]
        for r in range(3):
            for c in range(3):
                centre = tuple(n[a] + right[a] * (c - 1) + down[a] * (r - 1) for a in range(3))
                out[(centre, face)] = 9 * f + 3 * r + c
    return out


def _slots(names: tuple[str, ...]) -> tuple[tuple[int, ...], ...]:
    index = _sticker_index()
    rows = []
    for name in names:
        centre = tuple(sum(FACE_NORMAL[f][a] for f in name) for a in range(3))
        rows.append(tuple(index[(centre, f)] for f in name))
    return tuple(rows)


# Sticker indices of each corner position (U/D sticker first, then clockwise) and edge position.
CORNER_FACELETS = _slots(CORNER_NAMES)
EDGE_FACELETS = _slots(EDGE_NAMES)


class FaceletError(ValueError):
    """The string does not describe a legal cube."""


def is_facelet_string(text: str) -> bool:
    s = "".join(text.split())
    return len(s) == 54 and len(set(s)) == 6


def _piece_lookups() -> tuple[dict, dict]:
    """What a slot shows, mapped to the piece and orientation that show it: for every corner
    cubie and twist the three stickers read in slot order, for every edge cubie and flip the two."""

    corners = {}
    for cubie, name in enumerate(CORNER_NAMES):
        for twist in range(3):
            shown = [""] * 3
            for k in range(3):
                shown[(k + twist) % 3] = name[k]
            corners[tuple(shown)] = (cubie, twist)
    edges = {}
    for cubie, name in enumerate(EDGE_NAMES):
        edges[name] = (cubie, 0)
        edges[name[::-1]] = (cubie, 1)
    return corners, edges


_CORNER_SEEN, _EDGE_SEEN = _piece_lookups()


def parse_facelets(text: str) -> CubieState:
    """Cubie state of a 54-sticker string; raises ``FaceletError`` if it is not a legal cube.

    Stickers are renamed by the centre they match, each slot's stickers are looked up in the table
    of what every piece shows in every orientation, and the result must be a legal cube.  The
    error messages are the reference's (facelets.py:44-98), which callers may match."""

    s = "".join(text.split())
    if len(s) != 54:
        raise FaceletError(f"expected 54 stickers, got {len(s)}")
    centres = [s[4 + 9 * f] for f in range(6)]
    if len(set(centres)) != 6:
        raise FaceletError("the six centre stickers must all differ")
    face_of = dict(zip(centres, FACES))
    unknown = next((c for c in s if c not in face_of), None)
    if unknown is not None:
        raise FaceletError(f"sticker {unknown!r} matches no centre")
    faces = "".join(face_of[c] for c in s)
    counts = Counter(faces)
    short = next((f for f in FACES if counts[f] != 9), None)
    if short is not None:
        raise FaceletError(f"face {short} has {counts[short]} stickers, expected 9")

    corners = []
    for pos, slots in enumerate(CORNER_FACELETS):
        shown = tuple(faces[i] for i in slots)
        if not set(shown) & {"U", "D"}:
            raise FaceletError(f"corner at {CORNER_NAMES[pos]} has no U or D sticker")
        if shown not in _CORNER_SEEN:
            raise FaceletError(f"corner at {CORNER_NAMES[pos]} has impossible colours {''.join(shown)}")
        corners.append(_CORNER_SEEN[shown])
    edges = []
    for pos, (a, b) in enumerate(EDGE_FACELETS):
        shown = faces[a] + faces[b]
        if shown not in _EDGE_SEEN:
            raise FaceletError(f"edge at {EDGE_NAMES[pos]} has impossible colours {shown}")
        edges.append(_EDGE_SEEN[shown])

    cp, co = (list(x) for x in zip(*corners))
    ep, eo = (list(x) for x in zip(*edges))
    checks = ((len(set(cp)) == 8, "some corner appears twice"), (len(set(ep)) == 12, "some edge appears twice"),
              (sum(co) % 3 == 0, "a corner is twisted (corner orientations do not sum to 0 mod 3)"),
              (sum(eo) % 2 == 0, "an edge is flipped (edge orientations do not sum to 0 mod 2)"),
              (permutation_parity(cp) == permutation_parity(ep),
               "two pieces are swapped (corner and edge permutation parities differ)"))
    for ok, message in checks:
        if not ok:
            raise FaceletError(message)
    return CubieState(tuple(cp), tuple(co), tuple(ep), tuple(eo))


def to_facelets(state: CubieState) -> str:
    """54-sticker string (face letters) of a cubie state."""

    out = list("".join(f * 9 for f in FACES))
    for pos, slots in enumerate(CORNER_FACELETS):
        name = CORNER_NAMES[state.cp[pos]]
        for k in range(3):
            out[slots[(k + state.co[pos]) % 3]] = name[k]
    for pos, slots in enumerate(EDGE_FACELETS):
        name = EDGE_NAMES[state.ep[pos]]
        for k in range(2):
            out[slots[(k + state.eo[pos]) % 2]] = name[k]
    return "".join(out)
