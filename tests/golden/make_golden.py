"""Generate the golden fixtures of tests/golden/ from the reference checkout.

    python tests/golden/make_golden.py /path/to/reference

Imports the reference's own Python host model (``src/cuda_cube_solver``) in this process and
reads its data files, then writes:

* ``host_model.json``: the 18 HTM move tables, the 16 U-D symmetry matrices, the axis-frame move
  map, sha256 of the corner classes (classidx / rep / stab), the E-content class tables of the
  six group kinds, 304 / 208 table indices of seeded random states (reference
  ``coords.table_index``), group-kind indices of the same states computed from the reference's
  conjugation and class tables with the edge formula of its kernels.cu:181-196, search frames
  (``solver.frames``) and facelet strings (``facelets.to_facelets``) of some states;
* ``depth_counts.json``: per-depth entry counts of every preset kind from the reference's
  research/subgroups/results.jsonl (the table build's known answers);
* ``optimal_lengths.json``: scrambles from the reference's data/ files with the optimal lengths
  the reference reported for them (data/cuda-cube-solver_1000.txt and friends).
"""

from __future__ import annotations

import hashlib
import json
import random
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).parent


def main(ref: Path) -> None:
    sys.path.insert(0, str(ref / "src"))
    from cuda_cube_solver import coords, cubie, facelets, geometry, kinds, solver

    rng = random.Random(20261203)
    states = []
    for _ in range(300):
        moves = [rng.randrange(18) for _ in range(rng.randrange(40))]
        states.append((moves, cubie.apply_moves(cubie.CubieState(), [cubie.MOVES_HTM[m] for m in moves])))

    def words(s):
        c, e = coords.pack(s)
        return np.concatenate([c, e]).astype(np.uint8).view(np.uint32).tolist()

    cc = coords.corner_classes()
    _, edge_syms = coords.ud_actions()

    def group_index(kind, s):
        c, e = coords.pack(s)
        packed = int(cc.classidx[int(coords.corner_raw(c))])
        ce = coords.conj_edges(e, edge_syms[packed & 15])
        emask = eorder = eo_e = eo_n = ne = no = 0
        for i in range(12):
            b = int(ce[i])
            if b & 8:
                emask |= 1 << i
                eorder |= (b & 3) << (2 * ne)
                eo_e |= (b >> 4) << ne
                ne += 1
            else:
                eo_n |= (b >> 4) << no
                no += 1
        cls = int(kind.gen[0][int(coords.EORDER_RANK[eorder]) * 16 + eo_e])
        edge = (int(coords.SLICE_RANK[emask]) * 256 + eo_n) * kind.nec + cls
        return (packed >> 4) * kind.n_edge + edge

    host = {
        "moves": [{"cp": m.cp, "co": m.co, "ep": m.ep, "eo": m.eo} for m in cubie.MOVES_HTM],
        "move_names": list(cubie.MOVE_NAMES_HTM),
        "ud_sym_matrices": [s.matrix.tolist() for s in geometry.ud_symmetries()],
        "axis_move_map": geometry.move_map(geometry.axis_rotation()),
        "corner_classes_sha256": {
            "classidx": hashlib.sha256(cc.classidx.astype(np.uint32).tobytes()).hexdigest(),
            "rep": hashlib.sha256(cc.rep.astype(np.uint32).tobytes()).hexdigest(),
            "stab": hashlib.sha256(cc.stab.astype(np.uint16).tobytes()).hexdigest(),
        },
        "group_kinds": {name: {"nec": kinds.get(name).nec, "gen_class": kinds.get(name).gen[0].tolist(),
                               "gen_rep": kinds.get(name).gen[1].tolist()} for name in kinds.GROUP_KINDS},
        "canonical_prefix_counts": [len(solver.canonical_prefixes(n)) for n in range(6)],
        "states": [],
    }
    for moves, s in states:
        c, e = coords.pack(s)
        row = {"moves": moves, "words": words(s),
               "index": {"304": int(coords.table_index(c, e, coords.EdgeKind(3, 4))),
                         "208": int(coords.table_index(c, e, coords.EdgeKind(2, 8)))}}
        for name in kinds.GROUP_KINDS:
            row["index"][name] = group_index(kinds.get(name), s)
        host["states"].append(row)
    host["frames"] = [{"words": words(s), "frames": [words(f) for f in solver.frames(s)]} for _, s in states[:40]]
    host["facelets"] = [{"words": words(s), "facelets": facelets.to_facelets(s)} for _, s in states[:60]]
    (HERE / "host_model.json").write_text(json.dumps(host, separators=(",", ":")) + "\n")

    # Depth counts of the preset kinds (research/subgroups names, kinds.py:98).
    subgroup = {"304": "g2-49", "s4": "g1-49", "d4f": "g1-43", "a4t": "g1-31", "d4t": "g1-27", "d4": "g1-26", "a4": "g1-30"}
    rows = {}
    for line in (ref / "research/subgroups/results.jsonl").read_text().splitlines():
        r = json.loads(line)
        rows[r["kind"]] = r
    counts = {name: {"subgroup_name": sname, "entries": rows[sname]["entries"], "depth_counts": rows[sname]["depth_counts"],
                     "block_exact": rows[sname].get("block_exact")} for name, sname in subgroup.items()}
    (HERE / "depth_counts.json").write_text(json.dumps(counts, indent=1) + "\n")

    def solved_file(path):
        out = {}
        for line in (ref / path).read_text().splitlines():
            parts = line.split()
            if len(parts) >= 3:
                out[int(parts[0])] = int(parts[2])
        return out

    scr = [l.strip() for l in (ref / "data/random1000.txt").read_text().splitlines() if l.strip()]
    lens = solved_file("data/cuda-cube-solver_1000.txt")
    d4_lens = solved_file("data/d4/random1000.txt")
    first100 = solved_file("data/single_cube/cuda-cube-solver_first100.txt")
    d20 = [l.strip() for l in (ref / "data/distance20/random10.moves.txt").read_text().splitlines() if l.strip()]
    d20_lens = solved_file("data/distance20/cuda-cube-solver_random10.txt")
    sf = (ref / "data/distance20/superflip.txt").read_text().strip()
    f19 = (ref / "data/other_gpu/19f.txt").read_text().strip()
    opt = {
        "random1000": [{"scramble": s, "length": lens[i]} for i, s in enumerate(scr)],
        "random1000_d4_agree": all(d4_lens.get(i) == lens[i] for i in lens),
        "first100_agree": all(first100[i] == lens[i] for i in first100),
        "distance20": [{"scramble": s, "length": d20_lens[i]} for i, s in enumerate(d20)],
        "superflip": {"scramble": sf, "length": solved_file("data/distance20/cuda-cube-solver_superflip.txt")[0]},
        "hard19": {"scramble": " ".join(f19.split()), "length": solved_file("data/other_gpu/cuda-cube-solver_19f.txt")[0]},
    }
    (HERE / "optimal_lengths.json").write_text(json.dumps(opt, indent=0) + "\n")
    print("wrote", *(p.name for p in HERE.glob("*.json")))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout>")
    main(Path(sys.argv[1]))
