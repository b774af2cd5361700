"""Generate tests/golden/table_sha256.json with the CPU oracle (oracle/ccs_oracle.c).

    python tests/golden/make_table_sha.py 304 [s4 ...]

For each kind: exact BFS on the host's cores, the per-depth counts (which must equal the
reference's research/subgroups/results.jsonl counts in depth_counts.json), and the sha256 of
the 2-bit block file and of the base-3 file the reference would write for it.  The GPU tests
compare the tables libccs builds against these digests.
"""

from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1] / "oracle"))

from oracle import Oracle  # noqa: E402


def main(names: list[str]) -> None:
    out_path = HERE / "table_sha256.json"
    out = json.loads(out_path.read_text()) if out_path.exists() else {}
    golden = json.loads((HERE / "depth_counts.json").read_text())
    o = Oracle()
    for name in names:
        o.set_kind(name)
        t = time.time()
        depth, counts = o.bfs()
        bfs_s = time.time() - t
        if counts != golden[name]["depth_counts"]:
            raise SystemExit(f"{name}: oracle depth counts {counts} differ from the reference's")
        blk = o.encode_block(depth)
        b3 = o.encode_b3(depth, blk)
        out[name] = {"entries": len(depth), "depth_counts": counts,
                     "block_sha256": hashlib.sha256(blk.tobytes()).hexdigest(), "block_bytes": int(blk.nbytes),
                     "b3_sha256": hashlib.sha256(b3.tobytes()).hexdigest(), "b3_bytes": int(b3.nbytes),
                     "oracle_bfs_seconds": round(bfs_s, 1)}
        print(name, out[name], flush=True)
        del depth, blk, b3
        out_path.write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main(sys.argv[1:] or ["304"])
