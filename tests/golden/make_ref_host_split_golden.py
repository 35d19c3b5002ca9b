"""Write tests/golden/ref_host_split_golden.json: outputs of the reference's own
triangle-splitting LBVH kernels (BVHRT-Core/src/LBVH.cu:99-161 primitive-box
Morton codes, 320-428 tree with data and routing indices, 572-669 leaf and
node boxes; compiled from the reference tree by oracle/build.py for the host
execution model of oracle/ref_cpu/) on the fragments that the triangle-
splitting step (restated in oracle/atr_oracle.cpp) makes from seeded cases.

The reference has no splitting step of its own, so its kernels get the
fragments as input; each record holds the fragment digests and the tree
digests and SAH.  Usage (where the reference tree is present):
python tests/golden/make_ref_host_split_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from oracle import build as ob  # noqa: E402
from tests._util import digest, scene_case, tree_digests  # noqa: E402

OUT = ROOT / "tests" / "golden" / "ref_host_split_golden.json"
# (case, split ratio, Morton bits)
RUNS = [(c, r, b) for c in ("u17", "u1000", "u4097", "dupes3000", "flat2000", "same64", "sliver20000")
        for r in (0.0, 0.3, 1.0) for b in (30, 63)] + [("c1", 0.3, 30), ("sliver262144", 0.3, 30)]


def main() -> None:
    if ob.build_reference_host() is None:
        raise SystemExit("the reference tree is not present")
    records = []
    for case, ratio, bits in RUNS:
        v = scene_case(case)
        mn, mx = O.scene_aabb(v)
        b0, b1, d = O.split_triangles(v, ratio)
        t = O.ref_host_lbvh_split(b0, b1, d, mn, mx, bits == 63)
        rec = {"case": case, "split_ratio": ratio, "bits": bits, "primitives": int(len(d)),
               "fragments": {"bmin": digest(np.ascontiguousarray(b0[:, :3])),
                             "bmax": digest(np.ascontiguousarray(b1[:, :3])), "data": digest(d)},
               "tree": tree_digests(t.parent, t.left, t.right, t.data, t.bbox_min, t.bbox_max, t.area),
               "sah": float(O.ref_host_lib().ref_host_sah(t.n, O._ptr(t.area), 1.2, 1.0))}
        records.append(rec)
        print(case, ratio, bits, len(v), "->", len(d), rec["sah"], flush=True)
    doc = {"generator": "tests/golden/make_ref_host_split_golden.py",
           "reference_build": "oracle/_ref/libbvhrt_ref_host.so: BVHRT-Core/src/LBVH.cu (primitive-box kernels), "
                              "compiled from the reference tree by oracle/build.py for the host execution model",
           "records": records}
    OUT.write_text(json.dumps(doc, indent=1))


if __name__ == "__main__":
    main()
