"""The oracle pinned to the reference's own code, on the CPU.

oracle/_ref/libbvhrt_ref_host.so is the reference's BVHRT-Core sources (its
LBVH, ATRBVH, TRBVH and collapse kernels and its host classes) compiled from the
reference tree by oracle/build.py for a host execution model in which every
CUDA thread is a fiber (oracle/ref_cpu/).  tests/golden/ref_host_golden.json
records its outputs on the seeded cases (tests/golden/make_ref_host_golden.py).

  * the oracle reproduces every record bit for bit (always runs);
  * where the library is present, it reproduces the records, and the
    reference's __host__ __device__ arithmetic (Morton codes, surface areas)
    and SoABVHTree::SAH equal the oracle's on adversarial inputs.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from tests._util import collapsed_digests, digest, scene_case, tree_digests

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "ref_host_golden.json").read_text())
needs_ref = pytest.mark.skipif(not O.ref_host_available(),
                               reason="the reference's host-model library is built only where its tree is present")


def _tdig(t):
    return tree_digests(t.parent, t.left, t.right, t.data, t.bbox_min, t.bbox_max, t.area)


def _oracle_run(rec):
    v = scene_case(rec["case"])
    mn, mx = O.scene_aabb(v)
    t, _, _ = O.build_lbvh(v, mn, mx, bits=rec["bits"], threads=0)
    if rec["optimizer"] == "atrbvh":
        t = O.atrbvh(t, rec["treelet"], rec["iterations"], threads=0)
    elif rec["optimizer"] == "trbvh":
        t = O.trbvh(t, rec["treelet"], rec["iterations"], threads=0)
    return v, mn, mx, t


def test_oracle_matches_reference_records():
    """Morton keys, LBVH (30- and 63-bit), ATRBVH (treelet 3-20), TRBVH
    (treelet 7, 1-3 iterations) and collapse of the oracle equal the
    reference's own outputs on every recorded case, multi-block inputs of up to
    65,536 triangles included."""
    assert len(GOLD["records"]) >= 100
    for rec in GOLD["records"]:
        v, mn, mx, t = _oracle_run(rec)
        what = f"{rec['case']} {rec['optimizer']}({rec['treelet']},{rec['iterations']}) {rec['bits']}-bit"
        assert digest(O.morton(v, mn, mx, rec["bits"])) == rec["morton_keys"], what
        assert _tdig(t) == rec["tree"], what
        assert np.float32(O.sah(t)) == np.float32(rec["sah"]), what
        if "collapsed" in rec:
            c = O.collapse(t)
            assert np.float32(c.sah) == np.float32(rec["collapsed_sah"]), what
            assert collapsed_digests(c.left, c.right, c.data, c.triangle_count, c.triangle_indices, len(v)) == \
                rec["collapsed"], what


@needs_ref
def test_reference_library_reproduces_records():
    """The reference's host-model build gives the recorded outputs again
    (small cases and the 65,536-triangle LBVH; the 65,536-triangle ATRBVH
    runs are covered by the records)."""
    for rec in GOLD["records"]:
        if rec["case"] in ("c1", "clu65536") and rec["optimizer"] != "lbvh":
            continue
        v = scene_case(rec["case"])
        mn, mx = O.scene_aabb(v)
        t, c, _ = O.ref_host_run(v, mn, mx, use64=rec["bits"] == 63,
                                 optimizer={"lbvh": 0, "atrbvh": 1, "trbvh": 2}[rec["optimizer"]], treelet=rec["treelet"],
                                 iterations=rec["iterations"], collapse="collapsed" in rec)
        what = f"{rec['case']} {rec['optimizer']}({rec['treelet']},{rec['iterations']})"
        assert _tdig(t) == rec["tree"], what
        keys, idx = O.ref_host_morton(v, mn, mx, rec["bits"])
        assert digest(keys) == rec["morton_keys"] and digest(idx) == rec["morton_indices"], what
        if c is not None:
            assert np.float32(c.sah) == np.float32(rec["collapsed_sah"]), what


def _adversarial_coords() -> list[float]:
    f = np.float32
    vals = [0.0, -0.0, 1.0, 0.5, 1023 / 1024, 1 / 1024, 2097151 / 2097152, 1 / 2097152,
            np.nextafter(f(1), f(0)), np.nextafter(f(1), f(2)), np.nextafter(f(0), f(1)),
            np.nextafter(f(0), f(-1)), 1e-40, -1e-40, 1.17549435e-38, -3.0, 7.0, 1e30,
            float("inf"), float("-inf"), float("nan")]
    rng = np.random.default_rng(7)
    vals += rng.uniform(-0.1, 1.1, 40).astype(np.float32).tolist()
    vals += (rng.integers(0, 1024, 20) / 1024.0).astype(np.float32).tolist()
    return [float(np.float32(x)) for x in vals]


@needs_ref
def test_reference_morton_and_expand_bits_match_oracle():
    """calculateMortonCode / calculateMortonCode64 / expandBits
    (Commons.cuh:481-510, 606-662) against the oracle's restatement on points
    at and around the quantisation edges, outside the unit cube, denormal,
    infinite and NaN, and every 10-bit input of expandBits."""
    L, R = O.lib(), O.ref_host_lib()
    for v in range(1024):
        assert L.orc_expand_bits(v) == R.ref_host_expand_bits(v), v
    cs = _adversarial_coords()
    rng = np.random.default_rng(3)
    for _ in range(4000):
        x, y, z = (cs[int(i)] for i in rng.integers(0, len(cs), 3))
        assert L.orc_morton30_point(x, y, z) == R.ref_host_morton30_point(x, y, z), (x, y, z)
        assert L.orc_morton63_point(x, y, z) == R.ref_host_morton63_point(x, y, z), (x, y, z)


@needs_ref
def test_reference_areas_match_oracle():
    """calculateBoundingBoxSurfaceArea (float3, float4 and array forms) and
    calculateBoundingBoxAndSurfaceArea (Commons.cuh:99-194) bit for bit on
    zero-extent, inverted, denormal, huge and random boxes."""
    L, R = O.lib(), O.ref_host_lib()
    cs = [c for c in _adversarial_coords() if not np.isnan(c)]
    rng = np.random.default_rng(11)
    boxes = []
    for _ in range(3000):
        a = np.array([cs[int(i)] for i in rng.integers(0, len(cs), 3)] + [0], np.float32)
        b = np.array([cs[int(i)] for i in rng.integers(0, len(cs), 3)] + [0], np.float32)
        boxes.append((np.minimum(a, b), np.maximum(a, b)))
        boxes.append((b, a))  # inverted on some axes
    flat = np.array([0.25, 0.5, 0.75, 0], np.float32)
    boxes.append((flat, flat.copy()))
    boxes.append((np.array([0, 0, 0, 0], np.float32), np.array([1e-45, 1, 1, 0], np.float32)))

    def bits(x):
        return np.float32(x).view(np.uint32)

    for k, (mn, mx) in enumerate(boxes):
        want = bits(L.orc_box_area(O._ptr(mn), O._ptr(mx)))
        for f in (R.ref_host_box_area3, R.ref_host_box_area4, R.ref_host_box_area_arr):
            got = bits(f(O._ptr(mn), O._ptr(mx)))
            assert got == want or (np.isnan(np.float32(got).view(np.float32)) and np.isnan(want.view(np.float32))), k
        mn2, mx2 = boxes[(7 * k + 3) % len(boxes)]
        want = bits(L.orc_union_area(O._ptr(mn), O._ptr(mx), O._ptr(mn2), O._ptr(mx2)))
        for f in (R.ref_host_union_area3, R.ref_host_union_area4):
            got = bits(f(O._ptr(mn), O._ptr(mx), O._ptr(mn2), O._ptr(mx2)))
            assert got == want or (np.isnan(got.view(np.float32)) and np.isnan(want.view(np.float32))), k


@needs_ref
def test_reference_sah_matches_oracle():
    """SoABVHTree::SAH (SoABVHTree.cpp:50-74) against orc_sah: the trees of
    every small case, and random area arrays spanning many magnitudes."""
    L, R = O.lib(), O.ref_host_lib()
    for rec in GOLD["records"]:
        if rec["case"] in ("c1", "clu65536"):
            continue
        _, _, _, t = _oracle_run(rec)
        for ci, ct in ((1.2, 1.0), (1.0, 1.0), (0.5, 2.0)):
            assert np.float32(R.ref_host_sah(t.n, O._ptr(t.area), ci, ct)) == \
                np.float32(L.orc_sah(t.n, O._ptr(t.area), 0, ci, ct))
    rng = np.random.default_rng(5)
    for n in (2, 3, 17, 1000, 4097):
        area = np.exp(rng.uniform(-30, 30, 2 * n - 1)).astype(np.float32)
        assert np.float32(R.ref_host_sah(n, O._ptr(area), 1.2, 1.0)) == \
            np.float32(L.orc_sah(n, O._ptr(area), 0, 1.2, 1.0))


GOLD_SPLIT = json.loads((Path(__file__).resolve().parent / "golden" / "ref_host_split_golden.json").read_text())


def test_oracle_split_build_matches_reference_records():
    """The oracle's triangle-splitting LBVH (primitive-box Morton codes, tree,
    boxes) equals the reference's own primitive-box kernels
    (LBVH.cu:99-161, 320-428, 572-669) on the recorded fragment sets; the
    fragments themselves are the splitting step's (restated in the oracle)."""
    assert len(GOLD_SPLIT["records"]) >= 40
    for rec in GOLD_SPLIT["records"]:
        v = scene_case(rec["case"])
        mn, mx = O.scene_aabb(v)
        b0, b1, d = O.split_triangles(v, rec["split_ratio"])
        what = f"{rec['case']} split {rec['split_ratio']} {rec['bits']}-bit"
        assert len(d) == rec["primitives"], what
        assert digest(np.ascontiguousarray(b0[:, :3])) == rec["fragments"]["bmin"], what
        assert digest(np.ascontiguousarray(b1[:, :3])) == rec["fragments"]["bmax"], what
        assert digest(d) == rec["fragments"]["data"], what
        t = O.build_lbvh_split(b0, b1, d, mn, mx, rec["bits"], threads=0)
        assert _tdig(t) == rec["tree"], what
        assert np.float32(O.sah(t)) == np.float32(rec["sah"]), what


@needs_ref
def test_reference_split_kernels_reproduce_records():
    """The reference's host-model primitive-box kernels give the recorded
    trees again."""
    for rec in GOLD_SPLIT["records"]:
        v = scene_case(rec["case"])
        mn, mx = O.scene_aabb(v)
        b0, b1, d = O.split_triangles(v, rec["split_ratio"])
        t = O.ref_host_lbvh_split(b0, b1, d, mn, mx, rec["bits"] == 63)
        assert _tdig(t) == rec["tree"], f"{rec['case']} split {rec['split_ratio']} {rec['bits']}-bit"


def test_split_ratio_zero_is_the_plain_lbvh():
    """Without splits every triangle is one primitive with its own box, and the
    primitive-box build equals the plain LBVH."""
    for case in ("u1000", "clu4096", "dupes3000"):
        v = scene_case(case)
        mn, mx = O.scene_aabb(v)
        b0, b1, d = O.split_triangles(v, 0.0)
        assert np.array_equal(d, np.arange(len(v), dtype=np.uint32))
        t = O.build_lbvh_split(b0, b1, d, mn, mx, 30)
        base, _, _ = O.build_lbvh(v, mn, mx)
        assert _tdig(t) == _tdig(base), case


def test_split_fragments_cover_their_triangles():
    """Fragments of a triangle lie inside the triangle's box, and their union
    is the triangle's box (the clipped pieces cover the triangle)."""
    v = scene_case("sliver20000")
    b0, b1, d = O.split_triangles(v, 1.0)
    tmn = v[:, :, :3].min(axis=1)
    tmx = v[:, :, :3].max(axis=1)
    assert (b0[:, :3] >= tmn[d]).all() and (b1[:, :3] <= tmx[d]).all()
    assert (b0[:, :3] <= b1[:, :3]).all()
    umn = np.full_like(tmn, np.inf)
    umx = np.full_like(tmx, -np.inf)
    np.minimum.at(umn, d, b0[:, :3])
    np.maximum.at(umx, d, b1[:, :3])
    assert np.allclose(umn, tmn, atol=1e-6) and np.allclose(umx, tmx, atol=1e-6)
