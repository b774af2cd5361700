"""Coordinates of the pruning-table quotient, host side (vectorised numpy).

Every table entry is a right coset ``H g`` of a subgroup ``H`` that contains all U and D turns,
so the coordinates only keep what left multiplication by ``H`` preserves, relative to the U-D
axis:

* corners: twist (3^7) and which positions hold D-layer corners (8C4 = 70), i.e. the raw
  corner coordinate ``twist * 70 + ccomb`` (153,090 values), reduced by the 16 U-D symmetries
  to 9,930 classes;
* edges: which positions hold E-slice edges (12C4 = 495) and an edge factor chosen by the table
  kind (``EdgeKind`` here, ``kinds.GroupKind`` for the preset groups).

A table index is ``corner_class * n_edge + edge_coord(M_s g M_s^-1)``, where ``s`` is the
symmetry that carries the raw corner coordinate to its class representative.

Packed byte formats are the ones the kernels use: corner byte ``cp | co << 3``, edge byte
``ep | eo << 4``.  Restates ``src/cuda_cube_solver/coords.py:1-363`` of the reference (numbering
of combinations, permutations and classes kept identical, since they fix the table layout);
the edge coordinate is computed here for whole arrays of states at once.
"""

from __future__ import annotations

from dataclasses import dataclass
from functools import lru_cache
from itertools import combinations, permutations

import numpy as np

from cuda_cube_solver.cubie import MOVES_HTM, CubieState
from cuda_cube_solver.geometry import Symmetry, ud_symmetries

N_TWIST = 3**7
N_CCOMB = 70
N_CORNER_RAW = N_TWIST * N_CCOMB
N_SLICE = 495
N_EORDER = 24
N_EO8 = 256
N_EDGE = N_SLICE * N_EORDER * N_EO8


def _combination_tables(bits: int, choose: int) -> tuple[np.ndarray, np.ndarray]:
    """Rank of every ``bits``-bit mask with ``choose`` bits set (lexicographic order of the sorted
    bit positions, as ``itertools.combinations`` lists them), 0xFFFF elsewhere, and its inverse."""

    rank = np.full(1 << bits, 0xFFFF, dtype=np.uint16)
    unrank = np.array([sum(1 << i for i in c) for c in combinations(range(bits), choose)], dtype=np.uint16)
    rank[unrank] = np.arange(len(unrank), dtype=np.uint16)
    return rank, unrank


CCOMB_RANK, CCOMB_UNRANK = _combination_tables(8, 4)
SLICE_RANK, SLICE_UNRANK = _combination_tables(12, 4)

# E-order: the 2-bit labels (cubie & 3) of the four E edges in position order, first position in
# the low bits; ranked in ``itertools.permutations`` order.
PERMS4 = list(permutations(range(4)))
EORDER_UNRANK = np.array([sum(v << (2 * j) for j, v in enumerate(p)) for p in PERMS4], dtype=np.uint8)
EORDER_RANK = np.full(256, 0xFF, dtype=np.uint8)
EORDER_RANK[EORDER_UNRANK] = np.arange(24, dtype=np.uint8)
TWIST_WEIGHTS = 3 ** np.arange(7)


@dataclass(frozen=True)
class EdgeKind:
    """An edge coordinate named like vcube/nxopt tables ("208", "112", "304").

    ``ep``: 1 = E-slice positions only, 2 = plus the order of the E edges, 3 = plus which non-E
    positions hold U-layer edges.  ``eo``: 4 = flips of the E edges, 8 = flips of the non-E
    edges, 12 = all flips.
    """

    ep: int
    eo: int

    @property
    def n_ep(self) -> int:
        return {1: 1, 2: 24, 3: 70}[self.ep]

    @property
    def n_eo(self) -> int:
        return {4: 16, 8: 256, 12: 2048}[self.eo]

    @property
    def n_edge(self) -> int:
        return N_SLICE * self.n_ep * self.n_eo

    @property
    def name(self) -> str:
        return f"{self.ep}{self.eo:02d}"

    @property
    def defines(self) -> tuple[str, ...]:
        return (f"EDGE_EP={self.ep}", f"EDGE_EO={self.eo}")

    @classmethod
    def parse(cls, name: str) -> "EdgeKind":
        kind = cls(int(name[0]), int(name[1:]))
        kind.n_ep, kind.n_eo  # raises KeyError for unsupported variants
        return kind


K208 = EdgeKind(2, 8)
K304 = EdgeKind(3, 4)


def pack(state: CubieState) -> tuple[np.ndarray, np.ndarray]:
    corners = np.array([p | (o << 3) for p, o in zip(state.cp, state.co)], dtype=np.uint8)
    edges = np.array([p | (o << 4) for p, o in zip(state.ep, state.eo)], dtype=np.uint8)
    return corners, edges


def unpack(corners: np.ndarray, edges: np.ndarray) -> CubieState:
    return CubieState(tuple(int(c) & 7 for c in corners), tuple(int(c) >> 3 for c in corners),
                      tuple(int(e) & 15 for e in edges), tuple(int(e) >> 4 for e in edges))


def corner_raw(corners: np.ndarray) -> np.ndarray:
    """``twist * 70 + ccomb`` for packed corners of shape (..., 8)."""

    c = np.asarray(corners).astype(np.int64)
    twist = (c[..., :7] >> 3) @ TWIST_WEIGHTS
    dmask = (((c >> 2) & 1) << np.arange(8)).sum(axis=-1)
    return twist * N_CCOMB + CCOMB_RANK[dmask].astype(np.int64)


def corners_from_raw(raw) -> np.ndarray:
    """The representative packed corners of raw coordinates: twists from the digits (the last
    one closing the sum), U cubies 0..3 in the non-D positions and D cubies 4..7 in the D
    positions, each in position order."""

    raw = np.asarray(raw, dtype=np.int64)
    twist, ccomb = np.divmod(raw, N_CCOMB)
    digits = (twist[..., None] // TWIST_WEIGHTS) % 3
    co = np.concatenate([digits, (-digits.sum(axis=-1, keepdims=True)) % 3], axis=-1)
    is_d = (CCOMB_UNRANK[ccomb].astype(np.int64)[..., None] >> np.arange(8)) & 1
    cp = np.where(is_d == 1, 3 + np.cumsum(is_d, axis=-1), np.cumsum(1 - is_d, axis=-1) - 1)
    return (cp | (co << 3)).astype(np.uint8)


@dataclass(frozen=True)
class EdgeParts:
    """The pieces every edge coordinate is built from, for arrays of packed edges."""

    emask: np.ndarray   # 12-bit: positions holding E-slice edges
    eorder: np.ndarray  # labels (cubie & 3) of the E edges in position order, 2 bits each
    eo_e: np.ndarray    # flips of the E edges in position order
    umask: np.ndarray   # over the 8 non-E positions in order: holds a U-layer edge
    eo_n: np.ndarray    # flips of the non-E edges in position order
    eo12: np.ndarray    # flips of positions 0..10


def edge_parts(edges: np.ndarray) -> EdgeParts:
    e = np.asarray(edges).astype(np.int64)
    is_e = (e >> 3) & 1
    not_e = 1 - is_e
    flip = (e >> 4) & 1
    erank = np.cumsum(is_e, axis=-1) - is_e
    nrank = np.cumsum(not_e, axis=-1) - not_e
    pos = np.arange(12)
    return EdgeParts(
        emask=(is_e << pos).sum(axis=-1),
        eorder=(is_e * ((e & 3) << (2 * erank))).sum(axis=-1),
        eo_e=(is_e * (flip << erank)).sum(axis=-1),
        umask=(not_e * ((e & 15) < 4) << nrank).sum(axis=-1),
        eo_n=(not_e * (flip << nrank)).sum(axis=-1),
        eo12=(flip[..., :11] << pos[:11]).sum(axis=-1),
    )


def edge_coord(edges: np.ndarray, kind: EdgeKind = K208) -> np.ndarray:
    """Edge coordinate for packed edges of shape (..., 12)."""

    p = edge_parts(edges)
    ep = {1: np.zeros_like(p.emask), 2: EORDER_RANK[p.eorder].astype(np.int64),
          3: CCOMB_RANK[p.umask].astype(np.int64)}[kind.ep]
    eo = {4: p.eo_e, 8: p.eo_n, 12: p.eo12}[kind.eo]
    return (SLICE_RANK[p.emask].astype(np.int64) * kind.n_ep + ep) * kind.n_eo + eo


def _place_edges(emask: int, eorder: int, umask: int, flips_of) -> np.ndarray:
    """Representative packed edges: E positions get 8 | label in order, non-E positions get U
    cubies 0.. where ``umask`` (over non-E positions) is set and D cubies 4.. elsewhere."""

    out = np.zeros(12, dtype=np.uint8)
    ne = no = nu = nd = 0
    for i in range(12):
        if (emask >> i) & 1:
            b = 8 | ((eorder >> (2 * ne)) & 3)
            flip = flips_of(i, True, ne)
            ne += 1
        else:
            if (umask >> no) & 1:
                b, nu = nu, nu + 1
            else:
                b, nd = 4 + nd, nd + 1
            flip = flips_of(i, False, no)
            no += 1
        out[i] = b | (flip << 4)
    return out


def edges_from_coord(coord: int, kind: EdgeKind = K208) -> np.ndarray:
    """Representative packed edges of an edge coordinate (the kernels' ``unrank``)."""

    rest, eo = divmod(int(coord), kind.n_eo)
    srank, ep = divmod(rest, kind.n_ep)
    eorder = int(EORDER_UNRANK[ep]) if kind.ep == 2 else 0xE4
    umask = int(CCOMB_UNRANK[ep]) if kind.ep == 3 else 0x0F

    def flips_of(i, is_e, rank):
        if kind.eo == 4:
            return (eo >> rank) & 1 if is_e else 0
        if kind.eo == 8:
            return 0 if is_e else (eo >> rank) & 1
        return (eo >> i) & 1 if i < 11 else bin(eo).count("1") & 1

    return _place_edges(int(SLICE_UNRANK[srank]), eorder, umask, flips_of)


# --- symmetry action on packed states -------------------------------------------------


@dataclass(frozen=True)
class EdgeSym:
    """Cubie-level edge action of a symmetry: position ``p`` goes to ``perm[p]`` (cubie labels
    likewise); ``flip[p]`` is 1 where the symmetry swaps the two sticker slots of ``p``."""

    perm: np.ndarray
    perm_inv: np.ndarray
    flip: np.ndarray


@dataclass(frozen=True)
class CornerSym:
    perm: np.ndarray
    perm_inv: np.ndarray
    shift: np.ndarray   # slot index that slot 0 of position p maps to
    reflect: bool       # reflections reverse the cyclic order of the slots


def edge_sym(sym: Symmetry) -> EdgeSym:
    perm = sym.edge[0::2] // 2
    return EdgeSym(perm, np.argsort(perm), sym.edge[0::2] % 2)


def corner_sym(sym: Symmetry) -> CornerSym:
    perm = sym.corner[0::3] // 3
    return CornerSym(perm, np.argsort(perm), sym.corner[0::3] % 3, sym.det < 0)


# Names of the reference's helpers (``coords._edge_sym`` / ``coords._corner_sym``).
_edge_sym = edge_sym
_corner_sym = corner_sym


def conj_edges(edges: np.ndarray, es: EdgeSym) -> np.ndarray:
    """Packed-edge ``M g M^-1``: the new position ``P(p)`` holds cubie ``P(c)`` with flip
    ``o ^ flip[p] ^ flip[c]`` (vectorised over leading axes)."""

    src = np.asarray(edges)[..., es.perm_inv].astype(np.int64)
    cubie = src & 15
    o = (src >> 4) ^ es.flip[es.perm_inv] ^ es.flip[cubie]
    return (es.perm[cubie] | (o << 4)).astype(np.uint8)


def conj_corners(corners: np.ndarray, cs: CornerSym) -> np.ndarray:
    """Packed-corner ``M g M^-1``: sticker ``k`` of cubie ``c`` sits in slot ``k + o`` of ``p``;
    the symmetry sends slot ``j`` of ``p`` to slot ``shift[p] +/- j`` of ``P(p)`` and renames the
    sticker to ``shift[c] +/- k``, so the new twist is ``shift[p] +/- o - shift[c]``."""

    src = np.asarray(corners)[..., cs.perm_inv].astype(np.int64)
    cubie = src & 7
    sign = -1 if cs.reflect else 1
    o = (cs.shift[cs.perm_inv] + sign * (src >> 3) - cs.shift[cubie]) % 3
    return (cs.perm[cubie] | (o << 3)).astype(np.uint8)


@lru_cache(maxsize=1)
def ud_actions() -> tuple[tuple[CornerSym, ...], tuple[EdgeSym, ...]]:
    syms = ud_symmetries()
    return tuple(corner_sym(s) for s in syms), tuple(edge_sym(s) for s in syms)


@dataclass(frozen=True)
class CornerClasses:
    classidx: np.ndarray  # raw -> class << 4 | sym, with conj(sym, raw) = rep(class)
    rep: np.ndarray       # class -> representative raw (the smallest raw of its orbit)
    stab: np.ndarray      # class -> 16-bit mask of the symmetries fixing the representative


@lru_cache(maxsize=1)
def corner_classes() -> CornerClasses:
    """Orbits of the raw corner coordinate under the 16 U-D symmetries.  Class ids follow the
    order of the orbit minima; the symmetry stored per raw is the first one (in
    ``ud_symmetries`` order) reaching the minimum."""

    corner_syms, _ = ud_actions()
    states = corners_from_raw(np.arange(N_CORNER_RAW))
    images = np.stack([corner_raw(conj_corners(states, cs)) for cs in corner_syms])  # (16, N)
    orbit_min = images.min(axis=0)
    reps = np.unique(orbit_min)
    class_of = np.full(N_CORNER_RAW, -1, dtype=np.int64)
    class_of[reps] = np.arange(len(reps))
    first_sym = np.argmax(images == orbit_min[None, :], axis=0)
    classidx = (class_of[orbit_min] << 4 | first_sym).astype(np.uint32)
    fixes = images[:, reps] == reps[None, :]
    stab = (fixes.astype(np.uint32) << np.arange(16, dtype=np.uint32)[:, None]).sum(axis=0)
    return CornerClasses(classidx, reps.astype(np.uint32), stab.astype(np.uint16))


def table_index(corners: np.ndarray, edges: np.ndarray, kind=K208):
    """Table index of packed states (single or arrays).  ``kind`` is an ``EdgeKind`` or a
    ``kinds.GroupKind`` (anything with ``n_edge`` and ``edge_coord``)."""

    cc = corner_classes()
    _, edge_syms = ud_actions()
    packed = cc.classidx[corner_raw(corners)].astype(np.int64)
    cls, sym = packed >> 4, packed & 15
    edges = np.asarray(edges)
    conj = np.empty(edges.shape, dtype=np.uint8)
    flat_e = edges.reshape(-1, 12)
    flat_s = np.asarray(sym).reshape(-1)
    flat_c = conj.reshape(-1, 12)
    for s in np.unique(flat_s):
        rows = flat_s == s
        flat_c[rows] = conj_edges(flat_e[rows], edge_syms[int(s)])
    coord_fn = kind.edge_coord if hasattr(kind, "edge_coord") else (lambda e: edge_coord(e, kind))
    out = cls * kind.n_edge + coord_fn(conj)
    return int(out) if np.ndim(out) == 0 else out


def apply_move(corners: np.ndarray, edges: np.ndarray, move: int):
    """Right-multiply packed states by HTM move ``move`` (vectorised over leading axes)."""

    m = MOVES_HTM[move]
    c = np.asarray(corners)[..., list(m.cp)]
    o = ((c >> 3) + np.array(m.co)) % 3
    e = np.asarray(edges)[..., list(m.ep)] ^ (np.array(m.eo, dtype=np.uint8) << 4)
    return ((c & 7) | (o << 3)).astype(np.uint8), e.astype(np.uint8)
