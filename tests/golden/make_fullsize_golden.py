"""Write tests/golden/fullsize_oracle.json: the oracle's outputs on the
benchmark workloads at their full sizes, as digests and SAH values.

  c2  clustered scene, 4,194,304 triangles (seed 0): LBVH 30-bit +
      ATRBVH(9,2) tree, collapsed tree (uncapped), Compact2 arrays, closest-hit
      results of the 1920x1080 pinhole primary rays.
  c3  unit-cube scene, 16,777,216 triangles (seed 0): LBVH, TRBVH(7,3) and
      ATRBVH(5/7/9 x 1-3) trees with their SAH and collapsed SAH.

Everything comes from the oracle (CPU, OpenMP) and the checker's own scene and
ray generators; the script needs no GPU and nothing from the product library.
Usage: python tests/golden/make_fullsize_golden.py [--only c2|c3]
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from tests._util import collapsed_digests, digest, tree_digests  # noqa: E402

OUT = ROOT / "tests" / "golden" / "fullsize_oracle.json"
C2_TRIS, C3_TRIS = 4194304, 16777216
C3_VARIANTS = [("lbvh", 0, 0), ("trbvh", 7, 3)] + [("atrbvh", t, i) for t in (5, 7, 9) for i in (1, 2, 3)]


def tdig(t):
    return tree_digests(t.parent, t.left, t.right, t.data, t.bbox_min, t.bbox_max, t.area)


def make_c2(threads: int) -> dict:
    v = O.gen_scene(O.SCENE_CLUSTERED, C2_TRIS, 0)
    mn, mx = O.scene_aabb(v)
    base, _, _ = O.build_lbvh(v, mn, mx, threads=threads)
    t = O.atrbvh(base, 9, 2, threads=threads)
    c = O.collapse(t)
    cp = O.flatten(c, v)
    rays = O.gen_rays_pinhole(1920, 1080)
    res = O.trace(cp, rays, threads=threads)
    return {"workload": "clustered scene 4,194,304 triangles, seed 0; LBVH 30-bit + ATRBVH(9,2), collapse "
                        "(Ci 1.2, Ct 1.0, uncapped), Compact2, 1920x1080 pinhole primary rays",
            "scene": digest(v), "lbvh_tree": tdig(base), "lbvh_sah": O.sah(base),
            "tree": tdig(t), "tree_sah": O.sah(t),
            "collapsed": collapsed_digests(c.left, c.right, c.data, c.triangle_count, c.triangle_indices, len(v)),
            "collapsed_sah": c.sah,
            "compact2": {"nodes": digest(cp.nodes), "woop": digest(cp.woop), "tri_index": digest(cp.tri_index),
                         "num_nodes": int(len(cp.nodes)), "num_woop": int(len(cp.woop))},
            "primary_rays": digest(rays),
            "primary_hits": {"ids": digest(res[:, 0]), "t": digest(res[:, 1]), "hit_count": int((res[:, 0] >= 0).sum())}}


def make_c3(threads: int) -> dict:
    v = O.gen_scene(O.SCENE_UNIFORM, C3_TRIS, 0)
    mn, mx = O.scene_aabb(v)
    base, _, _ = O.build_lbvh(v, mn, mx, threads=threads)
    rows = {}
    for name, ts, it in C3_VARIANTS:
        t0 = time.perf_counter()
        if name == "lbvh":
            t = base
        elif name == "trbvh":
            t = O.trbvh(base, ts, it, threads=threads)
        else:
            t = O.atrbvh(base, ts, it, threads=threads)
        c = O.collapse(t)
        key = name if name == "lbvh" else f"{name}_{ts}_{it}"
        rows[key] = {"tree": tdig(t), "sah": O.sah(t), "collapsed_sah": c.sah}
        print(key, rows[key]["sah"], f"{time.perf_counter() - t0:.1f}s", flush=True)
    return {"workload": "unit-cube scene 16,777,216 triangles (vertex offsets N(0, 0.005^2)), seed 0; LBVH 30-bit "
                        "then each optimiser on the same LBVH; collapse Ci 1.2, Ct 1.0, uncapped",
            "scene": digest(v), "variants": rows}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["c2", "c3"])
    args = ap.parse_args()
    threads = O.max_threads()
    doc = json.loads(OUT.read_text()) if OUT.exists() else {}
    doc["generator"] = "tests/golden/make_fullsize_golden.py (oracle on the host cores)"
    if args.only in (None, "c2"):
        doc["c2"] = make_c2(threads)
        print("c2 tree sah", doc["c2"]["tree_sah"], "collapsed", doc["c2"]["collapsed_sah"], flush=True)
    if args.only in (None, "c3"):
        doc["c3"] = make_c3(threads)
    OUT.write_text(json.dumps(doc, indent=1))


if __name__ == "__main__":
    main()
