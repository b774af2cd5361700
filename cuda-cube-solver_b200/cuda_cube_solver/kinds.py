"""Table kinds and the memory ladder of table presets.

A table entry is a right coset of a subgroup H that contains all U and D turns: corner class
(9,930) x E-slice positions (495) x an edge factor.  A ``GroupKind`` keeps the flips of the 8
non-E edges and the E-edge content (labels in position order with their flips, an element of
the signed permutation group B4) up to a relabelling group L <= B4.  L must be normalised by the
relabelling the 16 U-D symmetries induce, or symmetry reduction would be wrong.

Same interface as ``src/cuda_cube_solver/kinds.py:1-225`` of the reference.  The numbering of
the E-content classes (``GroupKind.gen``) and the preset list fix the table layout and the drop-in
names, so both are kept identical; the classes are found here as orbits of the generators'
relabelling maps on the 384 contents (no group enumeration), and the preset chooser scans the
ladder from the fastest preset down.
"""

from __future__ import annotations

import json
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from cuda_cube_solver import coords

N_CONTENT = 24 * 16  # E contents: 24 label orders x 16 flip patterns


def _content_index(order: np.ndarray, flips: np.ndarray) -> np.ndarray:
    """Content number ``rank(order) * 16 + flips`` of label orders (..., 4) and flip bits (..., 4)."""

    code = (order.astype(np.int64) << (2 * np.arange(4))).sum(axis=-1)
    return coords.EORDER_RANK[code].astype(np.int64) * 16 + (flips.astype(np.int64) << np.arange(4)).sum(axis=-1)


# Every content as (labels in position order, flips by position): row c of each table.
_ORDERS = np.array([coords.PERMS4[c >> 4] for c in range(N_CONTENT)], dtype=np.int64)
_FLIPS = np.array([[(c >> i) & 1 for i in range(4)] for c in range(N_CONTENT)], dtype=np.int64)


def relabel_action(perm, flips) -> np.ndarray:
    """The relabelling ``label x -> perm[x]``, flipping the label's edge when ``flips[x]``, as a
    map of the 384 contents (int array: content -> relabelled content)."""

    perm, flips = np.asarray(perm, np.int64), np.asarray(flips, np.int64)
    return _content_index(perm[_ORDERS], _FLIPS ^ flips[_ORDERS])


def _symmetry_actions() -> list[np.ndarray]:
    """The relabellings of the E cubies (8..11) induced by the 16 U-D symmetries, as content maps."""

    return [relabel_action([int(es.perm[8 + x]) - 8 for x in range(4)], [int(es.flip[8 + x]) for x in range(4)])
            for es in coords.ud_actions()[1]]


def _orbits(actions: list[np.ndarray]) -> np.ndarray:
    """Orbit id of every content under the group the content maps generate, the orbits numbered
    by their smallest content.  Union-find over the generators' edges: the group is finite, so
    closing under the generators closes under the group."""

    root = np.arange(N_CONTENT)

    def find(x: int) -> int:
        while root[x] != x:
            root[x] = root[root[x]]
            x = root[x]
        return x

    for a in actions:
        for c in range(N_CONTENT):
            u, v = find(c), find(int(a[c]))
            if u != v:
                root[max(u, v)] = min(u, v)  # the smaller content stays the root
    roots = np.array([find(c) for c in range(N_CONTENT)])
    minima = np.unique(roots)  # sorted: orbit ids follow the orbit minima
    return np.searchsorted(minima, roots)


class GroupKind:
    """Edge factor: non-E flips (256) x E content (384) up to a relabelling group L <= B4.

    ``gen = (gen_class[384], gen_rep[2, 384])``: the class of every content (order rank * 16 +
    flips by position), and a representative content per class for each E-flip parity.  L is
    given by generators; it acts on contents by relabelling, and its classes are the orbits of
    that action.
    """

    ep = 9
    eo = 1

    def __init__(self, name: str, gens):
        self.name = name
        self.gens_list = [(tuple(p), tuple(f)) for p, f in gens]
        actions = [relabel_action(p, f) for p, f in self.gens_list]
        orbit = _orbits(actions)
        # Symmetry reduction conjugates the content by a U-D symmetry's relabelling s; that is only
        # well defined if s carries L-orbits onto L-orbits (s L s^-1 = L: the orbits are L's right
        # cosets, and a subgroup is the coset of the identity).  Orbits are closed under the
        # generators, so it suffices that s(c) and s(g(c)) share an orbit for every generator g.
        for s in _symmetry_actions():
            for a in actions:
                if not np.array_equal(orbit[s], orbit[s[a]]):
                    raise ValueError(f"{name}: group not normalised by the UD symmetries; symmetry reduction would be wrong")
        parity = _FLIPS.sum(axis=1) & 1
        n_orbits = int(orbit.max()) + 1
        gen_class = np.zeros(N_CONTENT, np.uint16)
        gen_rep = np.zeros((2, N_CONTENT), np.uint16)
        keeps_parity = all(sum(f) % 2 == 0 for _, f in self.gens_list)
        if keeps_parity:
            # Every relabelling keeps the E-flip parity, which the non-E flips then determine: the
            # classes are numbered within each parity (in order of their smallest content), and a
            # class's representative is its smallest content.
            orbit_parity = np.zeros(n_orbits, np.int64)
            orbit_parity[orbit] = parity
            rank = np.zeros(n_orbits, np.int64)
            for p in (0, 1):
                ids = np.flatnonzero(orbit_parity == p)
                rank[ids] = np.arange(len(ids))
                first = np.array([np.flatnonzero(orbit == i)[0] for i in ids], dtype=np.int64)
                gen_rep[p, : len(ids)] = first
            gen_class[:] = rank[orbit]
            self.nec = n_orbits // 2
        else:
            # Classes hold both parities: per parity, a class's representative is its largest
            # content of that parity.
            gen_class[:] = orbit
            for p in (0, 1):
                sel = np.flatnonzero(parity == p)
                gen_rep[p, orbit[sel]] = sel  # ascending contents: the last write is the largest
            self.nec = n_orbits
        self.n_edge = coords.N_SLICE * 256 * self.nec
        self.defines = ("EDGE_EP=9", "EDGE_EO=1", f"GEN_NEC={self.nec}")
        self.gen = (gen_class, gen_rep)

    def edge_coord(self, edges: np.ndarray) -> np.ndarray:
        """Edge coordinate ``(slice * 256 + non-E flips) * nec + class(E content)`` of packed edges."""

        p = coords.edge_parts(edges)
        content = coords.EORDER_RANK[p.eorder].astype(np.int64) * 16 + p.eo_e
        return ((coords.SLICE_RANK[p.emask].astype(np.int64) * 256 + p.eo_n) * self.nec
                + self.gen[0][content].astype(np.int64))

    def edges_from_coord(self, coord: int) -> np.ndarray:
        """Representative packed edges of an edge coordinate (the kernels' ``unrank``)."""

        rest, c = divmod(int(coord), self.nec)
        srank, nflips = divmod(rest, 256)
        content = int(self.gen[1][bin(nflips).count("1") & 1, c])
        eorder, eflips = int(coords.EORDER_UNRANK[content >> 4]), content & 15

        def flips_of(i, is_e, rank):
            return (eflips >> rank) & 1 if is_e else (nflips >> rank) & 1

        return coords._place_edges(int(coords.SLICE_UNRANK[srank]), eorder, 0x0F, flips_of)


# research/subgroups names: s4 = g1-49, d4f = g1-43, a4t = g1-31, d4t = g1-27, d4 = g1-26, a4 = g1-30.
GROUP_KINDS = {
    "s4": [((0, 1, 3, 2), (0, 0, 0, 0)), ((0, 2, 1, 3), (0, 0, 0, 0)), ((1, 0, 2, 3), (0, 0, 0, 0))],
    "d4f": [((0, 1, 2, 3), (1, 1, 1, 1)), ((0, 3, 2, 1), (0, 0, 0, 0)), ((1, 0, 3, 2), (0, 0, 0, 0))],
    "a4t": [((0, 2, 3, 1), (0, 1, 1, 0)), ((1, 0, 3, 2), (1, 1, 1, 1))],
    "d4t": [((0, 3, 2, 1), (0, 0, 0, 0)), ((1, 0, 3, 2), (1, 1, 1, 1))],
    "d4": [((1, 2, 3, 0), (0, 0, 0, 0)), ((0, 3, 2, 1), (0, 0, 0, 0))],
    "a4": [((0, 2, 3, 1), (0, 0, 0, 0)), ((1, 0, 3, 2), (0, 0, 0, 0))],
}

_KIND_CACHE: dict[str, object] = {}


def get(name: str):
    """A kind by table name: a ``GroupKind`` above, or a ``coords.EdgeKind`` name like "304"."""

    if name not in _KIND_CACHE:
        _KIND_CACHE[name] = GroupKind(name, GROUP_KINDS[name]) if name in GROUP_KINDS else coords.EdgeKind.parse(name)
    return _KIND_CACHE[name]


N_CLASSES = 9930
B3_ENTRIES = 155
BLOCK_ENTRIES = 124


@dataclass(frozen=True)
class Preset:
    """A solving table: a kind in block format (2-bit offsets) or base 3 (denser, a little slower)."""

    kind: str
    format: str          # "block" or "b3"
    cubes_per_s: float   # the reference's figure: 1,000 random cubes, RTX 5060 Ti 16 GB
    superflip_s: float   # the reference's figure for the superflip, same card
    auto: bool = True    # chosen by --memory; False: only by name

    @property
    def name(self) -> str:
        return self.kind if self.format == "block" else f"{self.kind}-b3"

    @property
    def file(self) -> str:
        return f"prune-ud-{self.kind}-{'blk' if self.format == 'block' else 'b3'}.bin"

    @property
    def entries(self) -> int:
        return N_CLASSES * get(self.kind).n_edge

    @property
    def table_bytes(self) -> int:
        """Size of the solving table (file and device memory)."""

        per = BLOCK_ENTRIES if self.format == "block" else B3_ENTRIES
        return -(-self.entries // per) * 32

    @property
    def build_bytes(self) -> int:
        """Peak device memory of building it here: one exact-depth byte per entry (padded to 16)
        and the encoded block table, plus the base-3 table while it is encoded from the block one."""

        depth = -(-self.entries // 16) * 16
        block = -(-self.entries // BLOCK_ENTRIES) * 32
        return depth + block + (self.table_bytes if self.format == "b3" else 0)


# The memory ladder, smallest first: each step is faster on random cubes and bigger.
PRESETS = [
    Preset("304", "block", 6.0, 44.6),
    Preset("s4", "b3", 13.1, 6.2),
    Preset("d4f", "b3", 16.9, 77.7),
    Preset("a4t", "b3", 21.8, 27.1),
    Preset("a4t", "block", 24.1, 11.5),
    Preset("d4t", "b3", 35.2, 47.5),
    Preset("d4t", "block", 37.5, 16.0),
    # Robust alternatives, only by name: the same groups without the twist keep the E-slice
    # edges' flips exactly (faster on flip-heavy positions such as the superflip).
    Preset("a4", "b3", 20.7, 4.0, auto=False),
    Preset("a4", "block", 22.2, 4.2, auto=False),
    Preset("d4", "b3", 31.6, 3.2, auto=False),
    Preset("d4", "block", 33.3, 3.2, auto=False),
]
PRESET_BY_NAME = {p.name: p for p in PRESETS}

# Solving needs some device memory besides the table (search buffers, corner tables).
SOLVE_MARGIN = 400 << 20


def built(preset: Preset, tables: Path) -> bool:
    return (Path(tables) / preset.file).exists()


def choose(tables: Path, memory: int, build_memory: int | None = None,
           to_build: bool = False) -> tuple[Preset | None, Preset | None]:
    """The fastest preset whose table fits in ``memory`` bytes and is either built already or can
    be built in ``build_memory`` bytes (default ``memory``); and, when a faster one would fit but
    can't be built here, that one (else None).  ``to_build``: tables already built don't count."""

    build_memory = memory if build_memory is None else build_memory
    blocked = None
    for p in reversed([q for q in PRESETS if q.auto]):  # fastest first
        if p.table_bytes + SOLVE_MARGIN > memory:
            continue
        if (not to_build and built(p, tables)) or p.build_bytes + SOLVE_MARGIN <= build_memory:
            return p, blocked
        blocked = blocked or p
    return None, blocked


def free_device_memory() -> int:
    """Free memory on the current GPU, from the native library."""

    from cuda_cube_solver import native

    return native.mem_info()[0]


def pick(tables: Path, memory="auto", name: str | None = None,
         to_build: bool = False) -> tuple[Preset | None, Preset | None]:
    """``choose`` for a ``memory`` budget in GB or "auto" (the free device memory; a larger budget
    is cut to it), or the preset ``name``."""

    if name:
        if name not in PRESET_BY_NAME:
            raise ValueError(f"unknown table {name!r}; choose from {', '.join(PRESET_BY_NAME)}")
        return PRESET_BY_NAME[name], None
    free = free_device_memory()
    budget = free if memory == "auto" else min(free, int(float(memory) * 1e9))
    return choose(tables, budget, free, to_build)


def describe(tables: Path) -> list[str]:
    """The preset table of ``cuda-cube-solver tables``: size, speed, build memory, file status."""

    head = f"{'preset':8} {'VRAM':>8} {'cubes/s':>8} {'superflip':>10} {'build VRAM':>11}  file"
    rows = [head]
    for p in PRESETS:
        notes = ("" if built(p, tables) else "  (not built)") + ("" if p.auto else "  (only with --table)")
        rows.append(f"{p.name:8} {p.table_bytes / 1e9:6.2f}GB {p.cubes_per_s:8.1f} {p.superflip_s:9.1f}s "
                    f"{p.build_bytes / 1e9:9.1f}GB  {p.file}{notes}")
    return rows


def write_meta(path: Path, preset: Preset, counts: list[int], seconds: float) -> None:
    """The ``.json`` beside a table file: preset, entries, per-depth counts, build seconds."""

    meta = {"preset": preset.name, "entries": preset.entries, "depth_counts": counts, "seconds": round(seconds, 1)}
    Path(path).write_text(json.dumps(meta, indent=2) + "\n")
