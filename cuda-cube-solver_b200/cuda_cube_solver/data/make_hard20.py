"""Writes hard20.json: the positions of the seed-20 uniform cube stream whose optimal length is at
least 19, the hard positions of the batched configuration (4,096 uniform cubes of seed 2 with 5%
replaced by hard ones: these and the superflip).

    python cuda-cube-solver_b200/cuda_cube_solver/data/make_hard20.py [--count 224] [--reference]

Solves the stream ``workloads.uniform_cubes(n, seed=20)`` on the GPU with libccs (d4t table built
on the device) in chunks until ``--count`` cubes of length >= 19 are found, and records their
stream indices and lengths.  ``--reference`` also solves the selected cubes with the reference's
own kernels.cu (baseline/ref_gpu.py, d4t built by its own BFS kernels) and records those lengths,
which must be equal.  Needs a GPU.
"""

from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[2]
sys.path.insert(0, str(HERE.parents[1]))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=224)
    ap.add_argument("--chunk", type=int, default=2048)
    ap.add_argument("--reference", action="store_true")
    ap.add_argument("--out", default=str(HERE / "hard20.json"))
    args = ap.parse_args()

    from cuda_cube_solver import native, workloads
    from cuda_cube_solver.device import state_words

    h = native.Handle(0)
    h.build_table("d4t", "block", None, keep_resident=True)
    found: list[tuple[int, int]] = []
    histogram: dict[int, int] = {}
    n = 0
    t0 = time.perf_counter()
    while len(found) < args.count:
        n += args.chunk
        cubes = workloads.uniform_cubes(n, seed=20)[n - args.chunk:]
        res = h.solve(state_words(cubes), native.solve_opts(timeout_s=900))
        for i, r in enumerate(res):
            assert r.status == 0
            histogram[r.length] = histogram.get(r.length, 0) + 1
            if r.length >= 19:
                found.append((n - args.chunk + i, r.length))
    found = found[: args.count]
    scanned = found[-1][0] + 1
    out = {"stream": "workloads.uniform_cubes(n, seed=20)", "min_length": 19, "scanned": scanned,
           "indices": [i for i, _ in found], "lengths": [L for _, L in found],
           "length_histogram_of_solved_chunks": {str(k): v for k, v in sorted(histogram.items())},
           "seconds": round(time.perf_counter() - t0, 1)}
    h.close()
    if args.reference:
        sys.path.insert(0, str(ROOT / "baseline"))
        import ref_gpu

        drv = ref_gpu.Driver(0)
        tables = ref_gpu.RefTables(drv, "d4t")
        ptr, _, _, _ = tables.build("block")
        solver = ref_gpu.RefSolver(drv, tables, ptr, "block")
        cubes = workloads.uniform_cubes(scanned, seed=20)
        sel = [cubes[i] for i in out["indices"]]
        ref_lengths = []
        for k in range(0, len(sel), 100):
            ref_lengths += [len(moves) for moves, _, _ in solver.solve(sel[k:k + 100])]
        out["reference_lengths"] = ref_lengths
        out["reference_equal"] = ref_lengths == out["lengths"]
    Path(args.out).write_text(json.dumps(out, indent=1) + "\n")
    print(f"{len(found)} cubes of length >= 19 in the first {scanned} of the stream; wrote {args.out}")


if __name__ == "__main__":
    main()
