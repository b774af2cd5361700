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


def parse_facelets(text: str) -> CubieState:
    """Cubie state of a 54-sticker string; raises ``FaceletError`` if it is not a legal cube."""

    s = "".join(text.split())
    if len(s) != 54:
        raise FaceletError(f"expected 54 stickers, got {len(s)}")
    centres = [s[4 + 9 * f] for f in range(6)]
    if len(set(centres)) != 6:
        raise FaceletError("the six centre stickers must all differ")
    face_of = {c: FACES[f] for f, c in enumerate(centres)}
    try:
        faces = [face_of[c] for c in s]
    except KeyError as exc:
        raise FaceletError(f"sticker {exc.args[0]!r} matches no centre") from None
    for f in FACES:
        if faces.count(f) != 9:
            raise FaceletError(f"face {f} has {faces.count(f)} stickers, expected 9")

    cp, co = [], []
    for pos, slots in enumerate(CORNER_FACELETS):
        st = [faces[i] for i in slots]
        twist = next((k for k in range(3) if st[k] in "UD"), None)
        if twist is None:
            raise FaceletError(f"corner at {CORNER_NAMES[pos]} has no U or D sticker")
        rest = (st[(twist + 1) % 3], st[(twist + 2) % 3])
        cubie = next((j for j, nm in enumerate(CORNER_NAMES) if nm[0] == st[twist] and (nm[1], nm[2]) == rest), None)
        if cubie is None:
            raise FaceletError(f"corner at {CORNER_NAMES[pos]} has impossible colours {''.join(st)}")
        cp.append(cubie)
        co.append(twist)

    ep, eo = [], []
    for pos, (a, b) in enumerate(EDGE_FACELETS):
        pair = faces[a] + faces[b]
        if pair in EDGE_NAMES:
            ep.append(EDGE_NAMES.index(pair))
            eo.append(0)
        elif pair[::-1] in EDGE_NAMES:
            ep.append(EDGE_NAMES.index(pair[::-1]))
            eo.append(1)
        else:
            raise FaceletError(f"edge at {EDGE_NAMES[pos]} has impossible colours {pair}")

    if sorted(cp) != list(range(8)):
        raise FaceletError("some corner appears twice")
    if sorted(ep) != list(range(12)):
        raise FaceletError("some edge appears twice")
    if sum(co) % 3:
        raise FaceletError("a corner is twisted (corner orientations do not sum to 0 mod 3)")
    if sum(eo) % 2:
        raise FaceletError("an edge is flipped (edge orientations do not sum to 0 mod 2)")
    if permutation_parity(cp) != permutation_parity(ep):
        raise FaceletError("two pieces are swapped (corner and edge permutation parities differ)")
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
