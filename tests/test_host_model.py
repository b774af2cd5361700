"""Host model (cubie / geometry / coords / kinds / solver helpers) against the reference.

Mirrors the reference's tests/test_cuda_cube_solver.py host-only tests and checks every table the
host model derives against tests/golden/host_model.json (made from the reference's own code).
"""

from __future__ import annotations

import hashlib
import random

import numpy as np
import pytest

from cuda_cube_solver import coords, cubie, geometry, kinds, solver
from cuda_cube_solver.cubie import MOVES_HTM, CubieState, apply_moves, compose
from cuda_cube_solver.device import state_words


def _random_states(n: int, seed: int) -> list[CubieState]:
    rng = random.Random(seed)
    return [apply_moves(CubieState(), [MOVES_HTM[rng.randrange(18)] for _ in range(rng.randrange(40))]) for _ in range(n)]


def test_moves_match_reference(host_golden):
    for mine, ref in zip(cubie.MOVES_HTM, host_golden["moves"]):
        assert (list(mine.cp), list(mine.co), list(mine.ep), list(mine.eo)) == (ref["cp"], ref["co"], ref["ep"], ref["eo"])
    assert list(cubie.MOVE_NAMES_HTM) == host_golden["move_names"]


def test_all_48_symmetries_preserve_the_move_set(host_golden):
    geometry.validate()
    assert len(geometry.all_symmetries()) == 48
    assert [s.matrix.tolist() for s in geometry.ud_symmetries()] == host_golden["ud_sym_matrices"]
    assert geometry.move_map(geometry.axis_rotation()) == host_golden["axis_move_map"]


def test_packed_conjugation_matches_sticker_conjugation():
    for sym in geometry.all_symmetries():
        cs, es = coords.corner_sym(sym), coords.edge_sym(sym)
        for state in _random_states(5, 1):
            want = coords.pack(sym.conjugate(state))
            corners, edges = coords.pack(state)
            assert np.array_equal(coords.conj_corners(corners, cs), want[0])
            assert np.array_equal(coords.conj_edges(edges, es), want[1])


def test_corner_classes_match_reference(host_golden):
    cc = coords.corner_classes()
    assert len(cc.rep) == 9930
    assert cc.stab[0] & 1
    sha = host_golden["corner_classes_sha256"]
    assert hashlib.sha256(cc.classidx.astype(np.uint32).tobytes()).hexdigest() == sha["classidx"]
    assert hashlib.sha256(cc.rep.astype(np.uint32).tobytes()).hexdigest() == sha["rep"]
    assert hashlib.sha256(cc.stab.astype(np.uint16).tobytes()).hexdigest() == sha["stab"]


@pytest.mark.parametrize("name", sorted(kinds.GROUP_KINDS))
def test_group_kind_classes_match_reference(name, host_golden):
    k = kinds.get(name)
    ref = host_golden["group_kinds"][name]
    assert k.nec == ref["nec"]
    assert k.gen[0].tolist() == ref["gen_class"]
    assert k.gen[1].tolist() == ref["gen_rep"]


@pytest.mark.parametrize("name", ["304", "s4", "d4f", "a4t", "d4t", "d4", "a4"])
def test_table_index_matches_reference(name, host_golden):
    kind = kinds.get(name)
    for row in host_golden["states"]:
        state = apply_moves(CubieState(), [MOVES_HTM[m] for m in row["moves"]])
        c, e = coords.pack(state)
        assert coords.table_index(c, e, kind) == row["index"][name]
        assert state_words([state])[0].tolist() == row["words"]


def test_frames_and_facelets_match_reference(host_golden):
    from cuda_cube_solver.device import unpack_words
    from cuda_cube_solver.facelets import to_facelets

    for row in host_golden["frames"]:
        state = unpack_words(np.array(row["words"], np.uint32))[0]
        assert state_words(solver.frames(state)).tolist() == row["frames"]
    for row in host_golden["facelets"]:
        state = unpack_words(np.array(row["words"], np.uint32))[0]
        assert to_facelets(state) == row["facelets"]


def test_canonical_prefix_counts(host_golden):
    assert [len(solver.canonical_prefixes(n)) for n in range(6)] == host_golden["canonical_prefix_counts"]
    assert len(solver.canonical_prefixes(4)) == 43254


KINDS = [coords.EdgeKind(2, 8), coords.EdgeKind(1, 12), coords.EdgeKind(3, 4), coords.EdgeKind(3, 8)]


@pytest.mark.parametrize("kind", KINDS, ids=lambda k: k.name)
def test_edge_coord_roundtrip(kind):
    rng = random.Random(7)
    for coord in [0, kind.n_edge - 1] + [rng.randrange(kind.n_edge) for _ in range(300)]:
        assert coords.edge_coord(coords.edges_from_coord(coord, kind), kind) == coord


@pytest.mark.parametrize("kind", KINDS, ids=lambda k: k.name)
def test_quotient_action_is_well_defined(kind):
    for state in _random_states(30, 3):
        corners, edges = coords.pack(state)
        rep_c = coords.corners_from_raw(coords.corner_raw(corners))
        rep_e = coords.edges_from_coord(coords.edge_coord(edges, kind), kind)
        for m in range(18):
            a = coords.apply_move(corners, edges, m)
            b = coords.apply_move(rep_c, rep_e, m)
            assert coords.corner_raw(a[0]) == coords.corner_raw(b[0])
            assert coords.edge_coord(a[1], kind) == coords.edge_coord(b[1], kind)


@pytest.mark.parametrize("name", sorted(kinds.GROUP_KINDS))
def test_group_kind_roundtrip_and_cosets(name):
    """Representatives invert the edge coordinate, and the index is constant on cosets: relabelling
    the E edges by a group element and the non-E edges arbitrarily keeps it, also after any move."""

    kind = kinds.get(name)
    rng = random.Random(name)
    for coord in [0, kind.n_edge - 1] + [rng.randrange(kind.n_edge) for _ in range(300)]:
        assert int(kind.edge_coord(kind.edges_from_coord(coord))) == coord

    def relabel(state):
        # a random group element: a random word in the generators, applied one letter at a time
        others = list(range(8))
        rng.shuffle(others)
        ep = tuple(c if c >= 8 else others[c] for c in state.ep)
        eo = state.eo
        for _ in range(rng.randrange(1, 6)):
            kp, kf = rng.choice(kind.gens_list)
            eo = tuple(o ^ kf[c - 8] if c >= 8 else o for c, o in zip(ep, eo))
            ep = tuple(8 + kp[c - 8] if c >= 8 else c for c in ep)
        return CubieState(state.cp, state.co, ep, eo)

    for state in _random_states(15, 17):
        other = relabel(state)
        for m in [None] + list(range(18)):
            a = state if m is None else compose(state, MOVES_HTM[m])
            b = other if m is None else compose(other, MOVES_HTM[m])
            assert coords.table_index(*coords.pack(a), kind) == coords.table_index(*coords.pack(b), kind)


def test_preset_choice(tmp_path):
    names = lambda pair: tuple(p.name if p else None for p in pair)  # noqa: E731
    # a 16 GB budget on a GPU with 180 GB free: the d4t build (38 GB) fits beside it
    assert names(kinds.choose(tmp_path, int(16e9), int(180e9))) == ("d4t", None)
    assert names(kinds.choose(tmp_path, int(8e9), int(180e9))) == ("d4t-b3", None)
    # on a 16 GB GPU the d4t table would fit but its build does not: s4-b3 (14.7 GB to build)
    assert names(kinds.choose(tmp_path, int(16e9))) == ("s4-b3", "d4t")
    assert names(kinds.choose(tmp_path, int(8e9))) == ("304", "d4t-b3")
    (tmp_path / "prune-ud-d4t-b3.bin").touch()
    assert names(kinds.choose(tmp_path, int(8e9))) == ("d4t-b3", None)
    assert names(kinds.choose(tmp_path, int(1e9))) == (None, None)
    assert names(kinds.choose(tmp_path, int(8e9), to_build=True)) == ("304", "d4t-b3")


def test_preset_sizes():
    by = kinds.PRESET_BY_NAME
    assert by["d4t"].entries == 30_199_910_400
    assert by["d4t"].table_bytes == 7_793_525_280
    assert by["d4t-b3"].table_bytes == 6_234_820_224
    assert by["304"].table_bytes == 1_420_694_720
    # this library's build: 30,199,910,400 depth bytes + the 7,793,525,280-byte block table
    assert by["d4t"].build_bytes == 30_199_910_400 + 7_793_525_280
    assert by["d4t-b3"].build_bytes == 30_199_910_400 + 7_793_525_280 + 6_234_820_224


def test_group_kind_must_be_normalised_by_the_symmetries():
    with pytest.raises(ValueError, match="not normalised"):
        kinds.GroupKind("swap01", [((1, 0, 2, 3), (0, 0, 0, 0))])
    with pytest.raises(ValueError, match="not normalised"):
        kinds.GroupKind("flip01", [((0, 1, 2, 3), (1, 1, 0, 0))])


def test_inverse_and_legality():
    for state in _random_states(50, 9):
        assert state.is_legal()
        assert compose(state, state.inverse()) == CubieState()
    assert not CubieState(ep=(1, 0) + tuple(range(2, 12))).is_legal()
