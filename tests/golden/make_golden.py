"""Generate tests/golden/ref_golden.json from the reference's own CUDA build.

Runs oracle/_ref/libbvhrt_ref.so (the reference's BVHRT-Core sources compiled
by oracle/build.py with -fmad=false) on a B200 over the seeded cases of
tests/_util.py and records digests of its output arrays, its SAH values and
its collapsed leaves.  The CPU test test_oracle_matches_reference_golden then
pins the oracle to these records.  A second run of every case, and a run of
the default-contraction build, record whether the reference is repeatable.

Usage (on a GPU machine): python tests/golden/make_golden.py OUT.json
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from tests._util import collapsed_digests, scene_case, tree_digests  # noqa: E402

RUNS = [
    # name, case, bits, optimizer, treelet, iterations, collapse
    ("u17-lbvh", "u17", 30, "none", 0, 0, True),
    ("u100-atr9", "u100", 30, "atrbvh", 9, 2, True),
    ("u1000-atr9", "u1000", 30, "atrbvh", 9, 2, True),
    ("u4097-atr7", "u4097", 30, "atrbvh", 7, 3, True),
    ("clu4096-atr9", "clu4096", 30, "atrbvh", 9, 2, True),
    ("dupes3000-atr9", "dupes3000", 30, "atrbvh", 9, 2, True),
    ("flat2000-atr5", "flat2000", 30, "atrbvh", 5, 1, True),
    ("same64-atr9", "same64", 30, "atrbvh", 9, 2, True),
    ("c1-lbvh30", "c1", 30, "none", 0, 0, True),
    ("c1-lbvh63", "c1", 63, "none", 0, 0, False),
    ("c1-atr9x2", "c1", 30, "atrbvh", 9, 2, True),
    ("c1-atr5x1", "c1", 30, "atrbvh", 5, 1, False),
    ("c1-atr7x3", "c1", 30, "atrbvh", 7, 3, False),
    ("c1-trbvh7x3", "c1", 30, "trbvh", 7, 3, True),
    ("u1000-trbvh7x2", "u1000", 30, "trbvh", 7, 2, True),
    ("clu65536-atr9x2", "clu65536", 30, "atrbvh", 9, 2, True),
    ("clu65536-trbvh7x3", "clu65536", 30, "trbvh", 7, 3, False),
]


def run_one(name, case, bits, opt, treelet, iters, collapse, fmad=False):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    code = {"none": 0, "atrbvh": 1, "trbvh": 2}[opt]
    t, c, times = O.ref_run(v, mn, mx, use64=bits == 63, optimizer=code, treelet=treelet, iterations=iters,
                            collapse=collapse, fmad=fmad)
    rec = {"name": name, "case": case, "bits": bits, "optimizer": opt, "treelet": treelet, "iterations": iters,
           "tree": tree_digests(t.parent, t.left, t.right, t.data, t.bbox_min, t.bbox_max, t.area),
           "sah": float(O.sah(t)), "ref_ms": [float(x) for x in times]}
    if c is not None:
        rec["collapsed"] = collapsed_digests(c.left, c.right, c.data, c.triangle_count, c.triangle_indices, len(v))
        rec["collapse_sah"] = float(c.sah)
    return rec


def main(out: str) -> None:
    cases = []
    notes = {"repeat_mismatch": [], "fmad_mismatch": []}
    for r in RUNS:
        rec = run_one(*r)
        again = run_one(*r)
        if again["tree"] != rec["tree"]:
            notes["repeat_mismatch"].append(r[0])
        fm = run_one(*r, fmad=True)
        if fm["tree"] != rec["tree"]:
            notes["fmad_mismatch"].append(r[0])
        cases.append(rec)
        print(r[0], "sah", rec["sah"], "ms", rec["ref_ms"], flush=True)
    doc = {"generator": "tests/golden/make_golden.py", "reference_build": "oracle/_ref/libbvhrt_ref.so (-fmad=false)",
           "cases": cases, "notes": notes}
    Path(out).parent.mkdir(parents=True, exist_ok=True)
    Path(out).write_text(json.dumps(doc, indent=1))
    print(json.dumps(notes))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(ROOT / "tests" / "golden" / "ref_golden.json"))
