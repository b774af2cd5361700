"""Build preset tables with the reference's own kernels and with libccs on this GPU, and record
both sha256 digests in tests/golden/ref_table_sha256.json (the reference's table files are not
distributed, so their bytes are pinned by running its code here).

    python baseline/ref_table_sha.py [--out FILE] [preset ...]     (default: every preset)
"""

from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent / "cuda-cube-solver_b200"))

import ref_gpu  # noqa: E402
from cuda_cube_solver import kinds, native  # noqa: E402

OUT = HERE.parent / "tests" / "golden" / "ref_table_sha256.json"


def sha_device(drv, ptr, nbytes) -> str:
    h = hashlib.sha256()
    chunk = 1 << 28
    buf = np.empty(chunk, np.uint8)
    for off in range(0, nbytes, chunk):
        n = min(chunk, nbytes - off)
        view = buf[:n]
        drv.d2h(view, ptr + off)
        h.update(view.tobytes())
    return h.hexdigest()


def main(names, out_path: Path = OUT):
    out = json.loads(out_path.read_text()) if out_path.exists() else {}
    drv = ref_gpu.Driver(0)
    for name in names:
        p = kinds.PRESET_BY_NAME[name]
        t = ref_gpu.RefTables(drv, p.kind)
        ptr, nbytes, counts, secs = t.build(p.format)
        ref_sha = sha_device(drv, ptr, nbytes)
        drv.free(ptr)
        h = native.Handle()
        mine_counts, mine_s = h.build_table(p.kind, p.format, None, keep_resident=True)
        mine = h.table_copy()
        mine_sha = hashlib.sha256(mine.tobytes()).hexdigest()
        h.close()
        out[name] = {"bytes": nbytes, "reference_sha256": ref_sha, "reference_counts": counts,
                     "reference_build_s": round(secs, 2), "libccs_sha256": mine_sha, "libccs_build_s": round(mine_s, 2),
                     "identical": ref_sha == mine_sha and counts == mine_counts}
        print(name, out[name], flush=True)
        out_path.write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    args = sys.argv[1:]
    dest = OUT
    if args[:1] == ["--out"]:
        dest, args = Path(args[1]), args[2:]
    main(args or [p.name for p in kinds.PRESETS], dest)
