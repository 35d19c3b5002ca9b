"""Write tests/golden/ref_host_golden.json: outputs of the reference's own
BVHRT-Core code (its Morton, sort call, Karras, refit, ATRBVH, TRBVH and
collapse kernels and host classes, compiled from the reference tree by oracle/build.py
for the host execution model of oracle/ref_cpu/) on the seeded test cases.

Each record holds digests of the tree arrays, the SAH, and for collapsed runs
the per-leaf triangle lists and the collapsed SAH, so that the oracle can be
checked against the reference where the reference's library is not present.
Usage (where the reference tree is present): python tests/golden/make_ref_host_golden.py
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from oracle import build as ob  # noqa: E402
from tests._util import CASES, collapsed_digests, digest, scene_case, tree_digests  # noqa: E402

OUT = ROOT / "tests" / "golden" / "ref_host_golden.json"
SMALL = [c for c in CASES if c not in ("c1", "clu65536")]
# (case, optimiser, treelet, iterations, morton bits, collapse)
RUNS = ([(c, "lbvh", 0, 0, 30, True) for c in SMALL] + [(c, "lbvh", 0, 0, 63, False) for c in SMALL]
        + [(c, "atrbvh", t, i, 30, (t, i) == (9, 2)) for c in SMALL
           for t, i in [(3, 1), (5, 1), (7, 3), (9, 2), (12, 2), (16, 1), (20, 1)]]
        + [(c, "lbvh", 0, 0, 30, True) for c in ("c1", "clu65536")]
        + [(c, "lbvh", 0, 0, 63, False) for c in ("c1", "clu65536")]
        + [(c, "atrbvh", 9, 2, 30, True) for c in ("c1", "clu65536")]
        + [("c1", "atrbvh", 5, 1, 30, False), ("c1", "atrbvh", 7, 3, 30, False)]
        + [(c, "trbvh", 7, i, 30, i == 3) for c in SMALL for i in (1, 2, 3)]
        + [("c1", "trbvh", 7, 3, 30, True), ("clu65536", "trbvh", 7, 2, 30, False)])


def main() -> None:
    lib = ob.build_reference_host()
    if lib is None:
        raise SystemExit("the reference tree is not present")
    records = []
    for case, opt, ts, it, bits, col in RUNS:
        v = scene_case(case)
        mn, mx = O.scene_aabb(v)
        t0 = time.perf_counter()
        t, c, _ = O.ref_host_run(v, mn, mx, use64=bits == 63, optimizer={"lbvh": 0, "atrbvh": 1, "trbvh": 2}[opt],
                                 treelet=ts, iterations=it, collapse=col)
        keys, idx = O.ref_host_morton(v, mn, mx, bits)
        rec = {"case": case, "optimizer": opt, "treelet": ts, "iterations": it, "bits": bits,
               "morton_keys": digest(keys), "morton_indices": digest(idx),
               "tree": tree_digests(t.parent, t.left, t.right, t.data, t.bbox_min, t.bbox_max, t.area),
               "sah": float(O.ref_host_lib().ref_host_sah(t.n, O._ptr(t.area), 1.2, 1.0))}
        if c is not None:
            rec["collapsed"] = collapsed_digests(c.left, c.right, c.data, c.triangle_count, c.triangle_indices,
                                                 len(v))
            rec["collapsed_sah"] = c.sah
        records.append(rec)
        print(case, opt, ts, it, bits, rec["sah"], f"{time.perf_counter() - t0:.1f}s", flush=True)
    doc = {"generator": "tests/golden/make_ref_host_golden.py",
           "reference_build": "oracle/_ref/libbvhrt_ref_host.so: BVHRT-Core/src/{LBVH,AgglomerativeTreelet,"
                              "TRBVH,TreeCollapser}.cu and the host classes, compiled from the reference tree by "
                              "oracle/build.py for the host execution model (oracle/ref_cpu/)",
           "records": records}
    OUT.write_text(json.dumps(doc, indent=1))


if __name__ == "__main__":
    main()
