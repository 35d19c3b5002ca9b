"""ORACLE -- test infrastructure only.

ctypes access to the CPU restatement (liboracle.so, from atr_oracle.cpp).
Only tests/, __graft_entry__.smoke() and the CPU-baseline legs of bench.py use
this package, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"

_p = C.c_void_p
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            from . import build
            build.build_oracle()
        _lib = C.CDLL(str(ORACLE_LIB))
        L = _lib
        L.orc_max_threads.restype = C.c_int
        L.orc_scene_aabb.argtypes = [_p, C.c_uint32, _p, _p]
        L.orc_morton.argtypes = [_p, C.c_uint32, _p, _p, _p, _p, C.c_int]
        L.orc_sort_pairs32.argtypes = [_p, _p, C.c_uint32, C.c_int]
        L.orc_sort_pairs64.argtypes = [_p, _p, C.c_uint32]
        L.orc_karras.argtypes = [_p, _p, _p, C.c_uint32, _p, _p, _p, _p, C.c_int]
        L.orc_refit.argtypes = [_p, C.c_uint32, _p, _p, _p, _p, _p, _p, _p, C.c_int]
        L.orc_build_lbvh.argtypes = [_p, C.c_uint32, _p, _p, C.c_int, _p, _p, _p, _p, _p, _p, _p, _p, _p,
                                     C.c_int]
        L.orc_build_lbvh.restype = C.c_int
        for f in (L.orc_atrbvh, L.orc_trbvh):
            f.argtypes = [C.c_uint32, _p, _p, _p, _p, _p, _p, _p, C.c_int, C.c_int, C.c_float, C.c_float,
                          C.c_int]
            f.restype = C.c_int
        L.orc_sah.argtypes = [C.c_uint32, _p, C.c_int, C.c_float, C.c_float]
        L.orc_sah.restype = C.c_float
        L.orc_collapse.argtypes = [C.c_uint32, _p, _p, _p, _p, _p, _p, _p, C.c_float, C.c_float, C.c_int,
                                   _p, _p, _p, _p, _p, _p, _p, _p, _p]
        L.orc_collapse.restype = C.c_float
        L.orc_flatten_compact2.argtypes = [C.c_uint32, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p,
                                           C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_flatten_compact2.restype = C.c_int
        L.orc_trace.argtypes = [_p, _p, _p, _p, C.c_int64, C.c_int, _p, C.c_int]
        L.orc_atrbvh_schedule.argtypes = [C.c_int, C.c_int, _p, C.c_int]
        L.orc_atrbvh_schedule.restype = C.c_int
        L.orc_expand_bits.argtypes = [C.c_uint32]
        L.orc_expand_bits.restype = C.c_uint32
        L.orc_morton30_point.argtypes = [C.c_float] * 3
        L.orc_morton30_point.restype = C.c_uint32
        L.orc_morton63_point.argtypes = [C.c_float] * 3
        L.orc_morton63_point.restype = C.c_uint64
        L.orc_box_area.argtypes = [_p, _p]
        L.orc_box_area.restype = C.c_float
        L.orc_union_area.argtypes = [_p, _p, _p, _p]
        L.orc_union_area.restype = C.c_float
        L.orc_gen_ao_rays.argtypes = [_p, _p, _p, C.c_int64, C.c_int64, C.c_int, C.c_float, C.c_uint32, _p]
        L.orc_sort_rays.argtypes = [_p, C.c_int64, _p, _p]
        L.orc_gen_scene.argtypes = [C.c_int, C.c_uint32, C.c_uint64, _p]
        L.orc_gen_rays_pinhole.argtypes = [C.c_uint32, C.c_uint32, _p, C.c_float, _p]
        L.orc_gen_rays_random.argtypes = [C.c_uint64, C.c_uint64, _p, _p, _p]
        L.orc_gen_batch_sizes.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, _p]
        L.orc_gen_batch_scene.argtypes = [C.c_uint32, _p, C.c_uint64, _p]
        for f in (L.orc_gen_scene, L.orc_gen_rays_pinhole, L.orc_gen_rays_random, L.orc_gen_batch_sizes,
                  L.orc_gen_batch_scene):
            f.restype = C.c_int
        L.orc_build_lbvh_split.argtypes = [C.c_uint32, _p, _p, _p, _p, _p, C.c_int] + [_p] * 7 + [C.c_int]
        L.orc_build_lbvh_split.restype = C.c_int
        L.orc_split_triangles.argtypes = [_p, C.c_uint32, C.c_float, C.c_uint32, _p, _p, _p]
        L.orc_split_triangles.restype = C.c_int64
    return _lib


def _ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def max_threads() -> int:
    return lib().orc_max_threads()


@dataclass
class Tree:
    parent: np.ndarray
    left: np.ndarray
    right: np.ndarray
    data: np.ndarray
    bbox_min: np.ndarray
    bbox_max: np.ndarray
    area: np.ndarray

    @staticmethod
    def empty(n: int) -> "Tree":
        nn = 2 * n - 1
        return Tree(*(np.zeros(nn, np.int32) for _ in range(4)), np.zeros((nn, 4), np.float32),
                    np.zeros((nn, 4), np.float32), np.zeros(nn, np.float32))

    def copy(self) -> "Tree":
        return Tree(*(a.copy() for a in (self.parent, self.left, self.right, self.data, self.bbox_min,
                                          self.bbox_max, self.area)))

    @property
    def n(self) -> int:
        return (len(self.parent) + 1) // 2

    def ptrs(self):
        return [_ptr(a) for a in (self.parent, self.left, self.right, self.data, self.bbox_min, self.bbox_max,
                                  self.area)]


def scene_aabb(v: np.ndarray):
    mn = np.zeros(3, np.float32)
    mx = np.zeros(3, np.float32)
    v = np.ascontiguousarray(v, np.float32)
    lib().orc_scene_aabb(_ptr(v), v.shape[0], _ptr(mn), _ptr(mx))
    return mn, mx


def morton(v: np.ndarray, bbmin, bbmax, bits: int = 30, threads: int = 1) -> np.ndarray:
    v = np.ascontiguousarray(v, np.float32)
    mn = np.asarray(bbmin, np.float32)
    mx = np.asarray(bbmax, np.float32)
    n = v.shape[0]
    if bits == 30:
        k = np.empty(n, np.uint32)
        lib().orc_morton(_ptr(v), n, _ptr(mn), _ptr(mx), _ptr(k), None, threads)
    else:
        k = np.empty(n, np.uint64)
        lib().orc_morton(_ptr(v), n, _ptr(mn), _ptr(mx), None, _ptr(k), threads)
    return k


def sort_pairs(keys: np.ndarray, threads: int = 1):
    k = np.ascontiguousarray(keys).copy()
    idx = np.empty(len(k), np.uint32)
    if k.dtype == np.uint32:
        lib().orc_sort_pairs32(_ptr(k), _ptr(idx), len(k), threads)
    else:
        lib().orc_sort_pairs64(_ptr(k), _ptr(idx), len(k))
    return k, idx


def build_lbvh(v: np.ndarray, bbmin, bbmax, bits: int = 30, threads: int = 1):
    """Returns (Tree, sorted_keys uint64, sorted_idx uint32)."""
    v = np.ascontiguousarray(v, np.float32)
    n = v.shape[0]
    t = Tree.empty(n)
    sk = np.empty(n, np.uint64)
    si = np.empty(n, np.uint32)
    mn = np.asarray(bbmin, np.float32)
    mx = np.asarray(bbmax, np.float32)
    rc = lib().orc_build_lbvh(_ptr(v), n, _ptr(mn), _ptr(mx), bits, *t.ptrs(), _ptr(sk), _ptr(si), threads)
    if rc != 0:
        raise ValueError(f"orc_build_lbvh rc={rc}")
    return t, sk, si


def split_triangles(v: np.ndarray, split_ratio: float, max_prims: int | None = None):
    """The triangle-splitting pre-pass restated: (bmin float4[P], bmax float4[P],
    data uint32[P]) of the fragments, in triangle order."""
    v = np.ascontiguousarray(v, np.float32)
    n = v.shape[0]
    cap = max_prims if max_prims is not None else n * 8
    bmin = np.zeros((cap, 4), np.float32)
    bmax = np.zeros((cap, 4), np.float32)
    data = np.zeros(cap, np.uint32)
    cnt = lib().orc_split_triangles(_ptr(v), n, split_ratio, cap, _ptr(bmin), _ptr(bmax), _ptr(data))
    if cnt < 0:
        raise ValueError("orc_split_triangles: no room")
    return bmin[:cnt].copy(), bmax[:cnt].copy(), data[:cnt].copy()


def build_lbvh_split(bmin4: np.ndarray, bmax4: np.ndarray, data: np.ndarray, bbmin, bbmax, bits: int = 30,
                     threads: int = 1) -> "Tree":
    """The reference's primitive-box LBVH (LBVH.cu:99-161, 320-428, 572-669)
    restated: one leaf per primitive box."""
    bmin4 = np.ascontiguousarray(bmin4, np.float32)
    bmax4 = np.ascontiguousarray(bmax4, np.float32)
    data = np.ascontiguousarray(data, np.uint32)
    n = len(data)
    t = Tree.empty(n)
    mn = np.asarray(bbmin, np.float32)
    mx = np.asarray(bbmax, np.float32)
    rc = lib().orc_build_lbvh_split(n, _ptr(bmin4), _ptr(bmax4), _ptr(data), _ptr(mn), _ptr(mx), bits, *t.ptrs(),
                                    threads)
    if rc != 0:
        raise ValueError(f"orc_build_lbvh_split rc={rc}")
    return t


def atrbvh(t: Tree, treelet: int = 9, iterations: int = 2, ci: float = 1.2, ct: float = 1.0,
           threads: int = 1) -> Tree:
    out = t.copy()
    rc = lib().orc_atrbvh(out.n, *out.ptrs(), treelet, iterations, ci, ct, threads)
    if rc != 0:
        raise ValueError(f"orc_atrbvh rc={rc}")
    return out


def trbvh(t: Tree, treelet: int = 7, iterations: int = 3, ci: float = 1.2, ct: float = 1.0,
          threads: int = 1) -> Tree:
    out = t.copy()
    rc = lib().orc_trbvh(out.n, *out.ptrs(), treelet, iterations, ci, ct, threads)
    if rc != 0:
        raise ValueError(f"orc_trbvh rc={rc}")
    return out


def refit(t: Tree, v: np.ndarray, threads: int = 0) -> Tree:
    """Boxes and areas of t's topology recomputed from vertices v."""
    out = t.copy()
    v = np.ascontiguousarray(v, np.float32)
    lib().orc_refit(_ptr(v), out.n, *out.ptrs(), threads)
    return out


def sah(t: Tree, ci: float = 1.2, ct: float = 1.0) -> float:
    return float(lib().orc_sah(t.n, _ptr(t.area), 0, ci, ct))


@dataclass
class Collapsed:
    parent: np.ndarray
    left: np.ndarray
    right: np.ndarray
    data: np.ndarray
    triangle_count: np.ndarray
    bbox_min: np.ndarray
    bbox_max: np.ndarray
    triangle_indices: np.ndarray
    cost: np.ndarray
    sah: float


def collapse(t: Tree, ci: float = 1.2, ct: float = 1.0, max_leaf: int = 0) -> Collapsed:
    n = t.n
    nn = 2 * n - 1
    c = Collapsed(*(np.zeros(nn, np.int32) for _ in range(5)), np.zeros((nn, 4), np.float32),
                  np.zeros((nn, 4), np.float32), np.full(n, -1, np.int32), np.zeros(nn, np.float32), 0.0)
    s = lib().orc_collapse(n, _ptr(t.parent), _ptr(t.left), _ptr(t.right), _ptr(t.data), _ptr(t.bbox_min),
                           _ptr(t.bbox_max), _ptr(t.area), ci, ct, max_leaf, _ptr(c.parent), _ptr(c.left),
                           _ptr(c.right), _ptr(c.data), _ptr(c.triangle_count), _ptr(c.bbox_min),
                           _ptr(c.bbox_max), _ptr(c.triangle_indices), _ptr(c.cost))
    c.sah = float(s)
    return c


def leaf_lists(left, right, data, count, tri_indices, n: int) -> dict:
    """Map each leaf reachable from the root of a collapsed tree to its triangle list."""
    out = {}
    stack = [0]
    while stack:
        x = stack.pop()
        for ch in (int(left[x]), int(right[x])):
            if data[ch] >= 0:
                if count[ch] > 1:
                    off = int(data[ch])
                    out[ch] = tuple(int(i) for i in tri_indices[off:off + int(count[ch])])
                else:
                    out[ch] = (int(data[ch]),)
            else:
                stack.append(ch)
    return out


@dataclass
class Compact:
    nodes: np.ndarray  # (num_nodes, 16) int32
    woop: np.ndarray   # (num_woop, 4) float32
    tri_index: np.ndarray


def flatten(c: Collapsed, v: np.ndarray) -> Compact:
    n = len(c.triangle_indices)
    v = np.ascontiguousarray(v, np.float32)
    nodes = np.zeros((max(n - 1, 1), 16), np.int32)
    woop = np.zeros((4 * n, 4), np.float32)
    tri = np.zeros(4 * n, np.int32)
    nn = C.c_int64()
    nw = C.c_int64()
    rc = lib().orc_flatten_compact2(n, _ptr(c.left), _ptr(c.right), _ptr(c.data), _ptr(c.triangle_count),
                                    _ptr(c.bbox_min), _ptr(c.bbox_max), _ptr(c.triangle_indices), _ptr(v),
                                    _ptr(nodes), _ptr(woop), _ptr(tri), C.byref(nn), C.byref(nw))
    if rc != 0:
        raise ValueError("orc_flatten_compact2 failed")
    return Compact(nodes[:nn.value].copy(), woop[:nw.value].copy(), tri[:nw.value].copy())


def trace(cp: Compact, rays: np.ndarray, any_hit: bool = False, threads: int = 0) -> np.ndarray:
    rays = np.ascontiguousarray(rays, np.float32)
    nr = rays.shape[0]
    res = np.zeros((nr, 4), np.int32)
    lib().orc_trace(_ptr(cp.nodes), _ptr(cp.woop), _ptr(cp.tri_index), _ptr(rays), nr, 1 if any_hit else 0,
                    _ptr(res), threads)
    return res


def atrbvh_schedule(treelet: int, warp: int = 32) -> np.ndarray:
    out = np.zeros(4096, np.int32)
    k = lib().orc_atrbvh_schedule(treelet, warp, _ptr(out), len(out))
    return out[:k]


# ---- seeded workloads (the checker's own generators) --------------------------

SCENE_UNIFORM, SCENE_CLUSTERED = 0, 1


def _ok(rc: int, what: str) -> None:
    if rc != 0:
        raise ValueError(f"{what}: invalid arguments")


def gen_scene(kind: int, n: int, seed: int = 0) -> np.ndarray:
    """(n, 3, 4) float32 triangle soup of the unit-cube (0) or clustered (1) scene."""
    out = np.empty((n, 3, 4), np.float32)
    _ok(lib().orc_gen_scene(kind, n, seed, _ptr(out)), "gen_scene")
    return out


def gen_rays_pinhole(w: int, h: int, eye=(0.5, 0.5, -1.5), fov_deg: float = 60.0) -> np.ndarray:
    out = np.empty((w * h, 2, 4), np.float32)
    e = np.asarray(eye, np.float32)
    _ok(lib().orc_gen_rays_pinhole(w, h, _ptr(e), fov_deg, _ptr(out)), "gen_rays_pinhole")
    return out


def gen_rays_random(n: int, bbmin, bbmax, seed: int = 0) -> np.ndarray:
    out = np.empty((n, 2, 4), np.float32)
    mn = np.asarray(bbmin, np.float32)
    mx = np.asarray(bbmax, np.float32)
    _ok(lib().orc_gen_rays_random(n, seed, _ptr(mn), _ptr(mx), _ptr(out)), "gen_rays_random")
    return out


def gen_batch_sizes(count: int, lo: int, hi: int, seed: int = 0) -> np.ndarray:
    out = np.empty(count, np.uint32)
    _ok(lib().orc_gen_batch_sizes(count, lo, hi, seed, _ptr(out)), "gen_batch_sizes")
    return out


def gen_batch_scene(sizes: np.ndarray, seed: int = 0) -> np.ndarray:
    sizes = np.ascontiguousarray(sizes, np.uint32)
    out = np.empty((int(sizes.sum(dtype=np.uint64)), 3, 4), np.float32)
    _ok(lib().orc_gen_batch_scene(len(sizes), _ptr(sizes), seed, _ptr(out)), "gen_batch_scene")
    return out


# ---- the reference's own code on the host (oracle/_ref/libbvhrt_ref_host.so) ----

REF_HOST_LIB = HERE / "_ref" / "libbvhrt_ref_host.so"
_ref_host = None


def ref_host_available() -> bool:
    return REF_HOST_LIB.exists()


def ref_host_lib() -> C.CDLL:
    """The reference's BVHRT-Core sources compiled for the host execution
    model (oracle/ref_cpu/, built by oracle/build.py where the reference tree
    is present)."""
    global _ref_host
    if _ref_host is None:
        L = C.CDLL(str(REF_HOST_LIB))
        L.ref_host_run.restype = C.c_int
        L.ref_host_run.argtypes = [_p, C.c_uint, _p, _p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int] + \
            [_p] * 15 + [_p, _p]
        L.ref_host_morton.argtypes = [_p, C.c_uint, _p, _p, C.c_int, _p, _p, _p]
        L.ref_host_morton.restype = C.c_int
        L.ref_host_morton30_point.argtypes = [C.c_float] * 3
        L.ref_host_morton30_point.restype = C.c_uint32
        L.ref_host_morton63_point.argtypes = [C.c_float] * 3
        L.ref_host_morton63_point.restype = C.c_uint64
        L.ref_host_expand_bits.argtypes = [C.c_uint32]
        L.ref_host_expand_bits.restype = C.c_uint32
        for f in (L.ref_host_box_area3, L.ref_host_box_area4, L.ref_host_box_area_arr):
            f.argtypes = [_p, _p]
            f.restype = C.c_float
        for f in (L.ref_host_union_area3, L.ref_host_union_area4):
            f.argtypes = [_p, _p, _p, _p]
            f.restype = C.c_float
        L.ref_host_sah.argtypes = [C.c_uint, _p, C.c_float, C.c_float]
        L.ref_host_sah.restype = C.c_float
        L.ref_host_lbvh_ts.argtypes = [C.c_uint, _p, _p, _p, _p, _p, C.c_int] + [_p] * 7
        L.ref_host_lbvh_ts.restype = C.c_int
        _ref_host = L
    return _ref_host


def ref_host_run(v: np.ndarray, bbmin, bbmax, *, use64=False, optimizer=0, treelet=9, iterations=2,
                 collapse=False):
    """The reference's own pipeline (LBVHBuilder, optimiser, collapser) on the
    host; returns (Tree, Collapsed | None, times_ms)."""
    v = np.ascontiguousarray(v, np.float32)
    n = v.shape[0]
    t = Tree.empty(n)
    nn = 2 * n - 1
    c = None
    if collapse:
        c = Collapsed(*(np.zeros(nn, np.int32) for _ in range(5)), np.zeros((nn, 4), np.float32),
                      np.zeros((nn, 4), np.float32), np.zeros(n, np.int32), np.zeros(0, np.float32), 0.0)
    sah_out = np.zeros(1, np.float32)
    times = np.zeros(3, np.float64)
    mn = np.asarray(bbmin, np.float32)
    mx = np.asarray(bbmax, np.float32)
    cp = [None] * 8 if c is None else [_ptr(c.parent), _ptr(c.left), _ptr(c.right), _ptr(c.data),
                                      _ptr(c.triangle_count), _ptr(c.bbox_min), _ptr(c.bbox_max),
                                      _ptr(c.triangle_indices)]
    ref_host_lib().ref_host_run(_ptr(v), n, _ptr(mn), _ptr(mx), 1 if use64 else 0, optimizer, treelet, iterations,
                                1 if collapse else 0, 1, *t.ptrs(), *cp, _ptr(sah_out), _ptr(times))
    if c is not None:
        c.sah = float(sah_out[0])
    return t, c, times


def ref_host_lbvh_split(bmin4: np.ndarray, bmax4: np.ndarray, data: np.ndarray, bbmin, bbmax,
                        use64: bool = False) -> "Tree":
    """The reference's own primitive-box LBVH kernels on the host."""
    bmin4 = np.ascontiguousarray(bmin4, np.float32)
    bmax4 = np.ascontiguousarray(bmax4, np.float32)
    data = np.ascontiguousarray(data, np.uint32)
    n = len(data)
    t = Tree.empty(n)
    mn = np.asarray(bbmin, np.float32)
    mx = np.asarray(bbmax, np.float32)
    ref_host_lib().ref_host_lbvh_ts(n, _ptr(bmin4), _ptr(bmax4), _ptr(data), _ptr(mn), _ptr(mx),
                                    1 if use64 else 0, *t.ptrs())
    return t


def ref_host_morton(v: np.ndarray, bbmin, bbmax, bits: int = 30):
    """The reference's Morton kernel output (keys in triangle order, indices)."""
    v = np.ascontiguousarray(v, np.float32)
    n = v.shape[0]
    mn = np.asarray(bbmin, np.float32)
    mx = np.asarray(bbmax, np.float32)
    idx = np.zeros(n, np.uint32)
    if bits == 30:
        k = np.zeros(n, np.uint32)
        ref_host_lib().ref_host_morton(_ptr(v), n, _ptr(mn), _ptr(mx), 0, _ptr(k), None, _ptr(idx))
    else:
        k = np.zeros(n, np.uint64)
        ref_host_lib().ref_host_morton(_ptr(v), n, _ptr(mn), _ptr(mx), 1, None, _ptr(k), _ptr(idx))
    return k, idx


def gen_ao_rays(v: np.ndarray, rays: np.ndarray, results: np.ndarray, samples: int, max_dist: float, seed: int,
                first: int = 0, count: int | None = None) -> np.ndarray:
    """Ambient-occlusion rays (count * samples, 2, 4) from the hits of rays[first:first+count]."""
    v = np.ascontiguousarray(v, np.float32)
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    results = np.ascontiguousarray(results, np.int32).reshape(-1, 4)
    count = len(rays) - first if count is None else count
    out = np.empty((count * samples, 2, 4), np.float32)
    lib().orc_gen_ao_rays(_ptr(v), _ptr(rays), _ptr(results), first, count, samples, max_dist, seed, _ptr(out))
    return out


def sort_rays(rays: np.ndarray):
    """(perm, box): perm[j] = old slot of the ray at sorted position j."""
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    perm = np.empty(len(rays), np.uint32)
    box = np.empty(6, np.float32)
    lib().orc_sort_rays(_ptr(rays), len(rays), _ptr(perm), _ptr(box))
    return perm, box
