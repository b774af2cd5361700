"""Generate baseline/ref_blobs/ from the reference checkout's own Python host code.

    python baseline/make_ref_blobs.py /path/to/reference

The reference's kernels read a constant blob (its ``Tables`` struct) and its search reads
``SearchConst``; both are built by its Python host (``device.build_tables``, device.py:22-112,
and ``solver.search_const``, solver.py:51-55).  The GPU box cannot import the reference, so the
blobs are generated here and committed as data: one ``<kind>.bin`` per table kind and
``search_const.bin``, with their sha256 in ``manifest.json``.
"""

from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main(ref: Path) -> None:
    sys.path.insert(0, str(ref / "src"))
    from cuda_cube_solver import device, kinds, solver

    out = HERE / "ref_blobs"
    out.mkdir(exist_ok=True)
    manifest = {}
    for name in ["304", "s4", "d4f", "a4t", "d4t", "d4", "a4"]:
        kind = kinds.get(name)
        blob = device.build_tables(getattr(kind, "gen", None))
        (out / f"{name}.bin").write_bytes(blob)
        manifest[name] = {"bytes": len(blob), "sha256": hashlib.sha256(blob).hexdigest()}
    sc = solver.search_const()
    (out / "search_const.bin").write_bytes(sc)
    manifest["search_const"] = {"bytes": len(sc), "sha256": hashlib.sha256(sc).hexdigest()}
    (out / "manifest.json").write_text(json.dumps(manifest, indent=1) + "\n")
    print(manifest)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python baseline/make_ref_blobs.py <reference checkout>")
    main(Path(sys.argv[1]))
