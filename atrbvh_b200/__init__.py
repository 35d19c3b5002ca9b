"""atrbvh_b200 -- ATRBVH build-and-traverse on NVIDIA B200 (sm_100a).

Python mirror of the reference's BVHRT-Core builder interface over the C ABI in
include/atrbvh.h (libatrbvh.so, built in-tree by ``python -m atrbvh_b200.build``).
Class and method names follow the reference:

    scene = SceneWrapper(ctx, vertices, bbmin, bbmax)     # BVHRT::SceneWrapper
    tree = LBVHBuilder(False).BuildTree(scene)            # BVHRT::LBVHBuilder
    AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)    # BVHRT::AgglomerativeTreeletOptimizer
    TRBVHOptimizer(7, 3).Optimize(tree)                   # BVHRT::TRBVHOptimizer
    collapsed, sah = BVHTreeCollapser().Collapse(tree)    # BVHRT::BVHTreeCollapser
    host = BVHTreeInstanceManager().DeviceToHostTree(tree)
    bvh = CudaBVH(collapsed, scene)                       # Compact2 + Woop layout
    bvh.trace(rays_ptr, num_rays, results_ptr)            # kepler_dynamic_fetch trace()

Errors raise AtrError (the reference exits the process instead).  There is no
CPU fallback: without the library or a B200 every call raises.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libatrbvh.so"

ATR_OK = 0
SCENE_UNIFORM = 0
SCENE_CLUSTERED = 1
TUNE_ATR_WARPS = 0
TUNE_ATR_GROUP_MIN = 1
TUNE_SORT_BITS = 2
TUNE_ATR_LEVELS = 3
TUNE_QUAD_MIN = 4
TUNE_WARP_MAX = 5


class AtrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"atrbvh status {status}: {msg}")
        self.status = status


_lib: C.CDLL | None = None

_p = C.c_void_p
_i32p = C.POINTER(C.c_int32)
_f32p = C.POINTER(C.c_float)


class TreeView(C.Structure):
    _fields_ = [("num_triangles", C.c_uint32), ("root", C.c_int32), ("parent", _p), ("left", _p),
                ("right", _p), ("data", _p), ("bbox_min", _p), ("bbox_max", _p), ("area", _p)]


class CollapsedView(C.Structure):
    _fields_ = [("num_triangles", C.c_uint32), ("root", C.c_int32), ("parent", _p), ("left", _p),
                ("right", _p), ("data", _p), ("triangle_count", _p), ("bbox_min", _p), ("bbox_max", _p),
                ("triangle_indices", _p)]


class CompactView(C.Structure):
    _fields_ = [("num_nodes", C.c_int64), ("num_woop", C.c_int64), ("nodes", _p), ("woop", _p),
                ("tri_index", _p), ("max_depth", C.c_int32)]


class ServerRequest(C.Structure):
    _fields_ = [("kind", C.c_int), ("mesh_id", C.c_uint64), ("vertices", _p), ("num_triangles", C.c_uint32),
                ("rays", _p), ("num_rays", C.c_uint32), ("results", _p), ("keep_resident", C.c_int)]


class ServerResult(C.Structure):
    _fields_ = [("status", C.c_int), ("sah", C.c_float), ("queue_ms", C.c_double), ("latency_ms", C.c_double),
                ("batch_requests", C.c_uint32), ("lane", C.c_uint32), ("error", C.c_char * 160)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("lanes", C.c_uint32), ("max_batch_requests", C.c_uint32),
                ("max_batch_triangles", C.c_uint64), ("treelet_size", C.c_int), ("iterations", C.c_int),
                ("max_leaf", C.c_int), ("class_treelet", _p), ("class_iters", _p)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("failed", C.c_uint64), ("builds", C.c_uint64), ("refits", C.c_uint64),
                ("evictions", C.c_uint64), ("triangles_built", C.c_uint64), ("triangles_refit", C.c_uint64),
                ("rays_traced", C.c_uint64), ("lane_batches", C.c_uint64), ("max_batch_requests_seen", C.c_uint32),
                ("max_lanes_busy", C.c_uint32), ("resident_meshes", C.c_uint32), ("resident_bytes", C.c_uint64),
                ("peak_bytes", C.c_uint64), ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("max_ms", C.c_double), ("overlap_fraction", C.c_double), ("busy_ms", C.c_double),
                ("host_copy_ms", C.c_double), ("lane_batch_ms", C.c_double)]


class PlanParams(C.Structure):
    _fields_ = [("morton_bits", C.c_int32), ("optimizer", C.c_int32), ("treelet_size", C.c_int32),
                ("iterations", C.c_int32), ("ci", C.c_float), ("ct", C.c_float), ("max_leaf", C.c_int32),
                ("flatten", C.c_int32)]


class CacheParams(C.Structure):
    _fields_ = [("morton_bits", C.c_int32), ("optimizer", C.c_int32), ("treelet_size", C.c_int32),
                ("iterations", C.c_int32), ("ci", C.c_float), ("ct", C.c_float), ("max_leaf", C.c_int32)]


class TuneEntry(C.Structure):
    _fields_ = [("treelet", C.c_uint8), ("iterations", C.c_uint8), ("atr_warps", C.c_uint8),
                ("sort_bits", C.c_uint8), ("build_ms", C.c_float), ("reference_ms", C.c_float),
                ("sah_ratio", C.c_float), ("sample_triangles", C.c_uint32), ("sample_meshes", C.c_uint32)]


class TuneTable(C.Structure):
    _fields_ = [("cls", TuneEntry * 32), ("tuned_mask", C.c_uint32)]

    def classes(self) -> dict:
        """{class: entry dict} of the tuned classes."""
        out = {}
        for c in range(32):
            if self.tuned_mask >> c & 1:
                e = self.cls[c]
                out[c] = {name: getattr(e, name) for name, _ in TuneEntry._fields_}
        return out

    def class_arrays(self) -> tuple[np.ndarray, np.ndarray]:
        """32-entry treelet / iteration arrays by class (nearest tuned class
        for the others), as the serving loop's configuration takes them."""
        ts = np.zeros(32, np.uint8)
        it = np.zeros(32, np.uint8)
        for c in range(32):
            e = TuneEntry()
            check(lib().atr_tune_lookup(C.byref(self), max(2, 1 << c), C.byref(e)))
            ts[c], it[c] = e.treelet, e.iterations
        return ts, it


class TuneOutcome(C.Structure):
    _fields_ = [("default_ms", C.c_float), ("tuned_ms", C.c_float), ("default_sah", C.c_double),
                ("tuned_sah", C.c_double), ("kept", C.c_int32)]


class AutotuneConfig(C.Structure):
    _fields_ = [("min_class", C.c_uint32), ("max_class", C.c_uint32), ("sample_triangles", C.c_uint64),
                ("sah_tolerance", C.c_float), ("reps", C.c_uint32), ("seed", C.c_uint64)]


# (name, restype, argtypes) for every exported entry point of include/atrbvh.h.
_SIGS = [
    ("atr_last_error", C.c_char_p, []),
    ("atr_version", C.c_char_p, []),
    ("atr_ctx_create", C.c_int, [C.c_int, _p, C.POINTER(_p)]),
    ("atr_ctx_destroy", C.c_int, [_p]),
    ("atr_ctx_synchronize", C.c_int, [_p]),
    ("atr_ctx_get_stream", C.c_int, [_p, C.POINTER(_p)]),
    ("atr_ctx_launch_count", C.c_int, [_p, C.POINTER(C.c_uint64)]),
    ("atr_ctx_set_timing", C.c_int, [_p, C.c_int]),
    ("atr_ctx_set_tuning", C.c_int, [_p, C.c_int, C.c_int]),
    ("atr_ctx_get_tuning", C.c_int, [_p, C.c_int, C.POINTER(C.c_int)]),
    ("atr_ctx_phase_times", C.c_int, [_p, _f32p, C.c_int, C.POINTER(C.c_int)]),
    ("atr_ctx_phase_names", C.c_char_p, [_p]),
    ("atr_scene_create", C.c_int, [_p, _p, C.c_uint32, _f32p, _f32p, C.c_int, C.POINTER(_p)]),
    ("atr_scene_destroy", C.c_int, [_p]),
    ("atr_scene_bounds", C.c_int, [_p, _p, _f32p, _f32p]),
    ("atr_scene_device_vertices", C.c_int, [_p, C.POINTER(_p), C.POINTER(C.c_uint32)]),
    ("atr_scene_set_vertices", C.c_int, [_p, _p, _p, C.c_int]),
    ("atr_build_lbvh", C.c_int, [_p, _p, C.c_int, C.POINTER(_p)]),
    ("atr_build_lbvh_split", C.c_int, [_p, C.c_uint32, _p, _p, _p, _f32p, _f32p, C.c_int, C.POINTER(_p)]),
    ("atr_split_triangles", C.c_int, [_p, _p, C.c_float, C.c_uint32, _p, _p, _p, C.POINTER(C.c_uint32)]),
    ("atr_tree_destroy", C.c_int, [_p]),
    ("atr_tree_view_get", C.c_int, [_p, C.POINTER(TreeView)]),
    ("atr_tree_download", C.c_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p]),
    ("atr_tree_sah", C.c_int, [_p, _p, C.c_float, C.c_float, _f32p]),
    ("atr_tree_sorted_keys", C.c_int, [_p, _p, _p, _p]),
    ("atr_device_morton", C.c_int, [_p, _p, C.c_uint32, _f32p, _f32p, C.c_int, _p]),
    ("atr_device_sort_pairs", C.c_int, [_p, _p, _p, C.c_uint32, C.c_int]),
    ("atr_optimize_atrbvh", C.c_int, [_p, _p, C.c_int, C.c_int, C.c_float, C.c_float]),
    ("atr_optimize_trbvh", C.c_int, [_p, _p, C.c_int, C.c_int, C.c_float, C.c_float]),
    ("atr_refit", C.c_int, [_p, _p, _p]),
    ("atr_refit_noalloc", C.c_int, [_p, C.c_uint32, _p, _p, _p, _p, _p, _p, _p, _p]),
    ("atr_collapse", C.c_int, [_p, _p, C.c_float, C.c_float, C.c_int, C.POINTER(_p), _f32p]),
    ("atr_collapsed_destroy", C.c_int, [_p]),
    ("atr_collapsed_view_get", C.c_int, [_p, C.POINTER(CollapsedView)]),
    ("atr_collapsed_download", C.c_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    ("atr_flatten_compact2", C.c_int, [_p, _p, _p, C.POINTER(_p)]),
    ("atr_compact_destroy", C.c_int, [_p]),
    ("atr_compact_view_get", C.c_int, [_p, C.POINTER(CompactView)]),
    ("atr_compact_download", C.c_int, [_p, _p, _p, _p, _p]),
    ("atr_plan_create", C.c_int, [_p, _p, C.POINTER(PlanParams), C.POINTER(_p)]),
    ("atr_plan_run", C.c_int, [_p, _p, C.c_int]),
    ("atr_plan_tree", C.c_int, [_p, C.POINTER(_p)]),
    ("atr_plan_collapsed", C.c_int, [_p, C.POINTER(_p)]),
    ("atr_plan_compact", C.c_int, [_p, _p, C.POINTER(_p)]),
    ("atr_plan_sah", C.c_int, [_p, _p, C.POINTER(C.c_float)]),
    ("atr_plan_times", C.c_int, [_p, _p, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    ("atr_plan_phase_times", C.c_int, [_p, _p, _p, C.c_int, C.POINTER(C.c_int)]),
    ("atr_plan_phase_names", C.c_char_p, [_p]),
    ("atr_plan_destroy", C.c_int, [_p]),
    ("atr_compact_serialize", C.c_int, [_p, _p, _p, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("atr_compact_deserialize", C.c_int, [_p, _p, C.c_uint64, C.POINTER(_p)]),
    ("atr_cache_key", C.c_int, [_p, C.c_uint32, C.POINTER(CacheParams), C.POINTER(C.c_uint64)]),
    ("atr_trace", C.c_int, [_p, _p, _p, C.c_int64, C.c_int, _p]),
    ("atr_batch_create", C.c_int, [_p, _p, _p, C.c_uint32, _p, C.c_int, C.POINTER(_p)]),
    ("atr_batch_destroy", C.c_int, [_p]),
    ("atr_batch_set_params", C.c_int, [_p, _p, _p, _p]),
    ("atr_batch_build", C.c_int, [_p, _p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int]),
    ("atr_batch_info", C.c_int, [_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    ("atr_batch_mesh_view", C.c_int, [_p, C.c_uint32, C.POINTER(TreeView)]),
    ("atr_batch_download_mesh", C.c_int, [_p, _p, C.c_uint32, _p, _p, _p, _p, _p, _p, _p]),
    ("atr_batch_sah", C.c_int, [_p, _p, C.c_float, C.c_float, _p]),
    ("atr_batch_collapse", C.c_int, [_p, _p, C.c_float, C.c_float, C.c_int, _p]),
    ("atr_batch_flatten", C.c_int, [_p, _p]),
    ("atr_batch_compact_view", C.c_int, [_p, C.c_uint32, C.POINTER(CompactView)]),
    ("atr_batch_compact_download", C.c_int, [_p, _p, C.c_uint32, _p, _p, _p]),
    ("atr_batch_trace", C.c_int, [_p, _p, _p, C.c_int64, _p, _p, C.c_uint32, C.c_int, _p]),
    ("atr_batch_refit_mesh", C.c_int, [_p, _p, C.c_uint32, _p, C.c_int]),
    ("atr_gen_bounce_rays", C.c_int, [_p, _p, _p, _p, C.c_int64, C.c_uint64, _p]),
    ("atr_gen_ao_rays", C.c_int, [_p, _p, _p, _p, C.c_int64, C.c_int64, C.c_int, C.c_float, C.c_uint32, _p]),
    ("atr_sort_rays", C.c_int, [_p, _p, _p, C.c_int64, _p, _p, _p]),
    ("atr_gen_scene", C.c_int, [C.c_int, C.c_uint32, C.c_uint64, _p]),
    ("atr_gen_batch_sizes", C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, _p]),
    ("atr_gen_batch_scene", C.c_int, [C.c_uint32, _p, C.c_uint64, _p]),
    ("atr_gen_rays_pinhole", C.c_int, [C.c_uint32, C.c_uint32, _f32p, C.c_float, _p]),
    ("atr_gen_rays_random", C.c_int, [C.c_uint64, C.c_uint64, _f32p, _f32p, _p]),
    ("atr_autotune", C.c_int, [_p, C.POINTER(AutotuneConfig), C.POINTER(TuneTable)]),
    ("atr_tune_lookup", C.c_int, [C.POINTER(TuneTable), C.c_uint32, C.POINTER(TuneEntry)]),
    ("atr_batch_apply_tuning", C.c_int, [_p, _p, C.POINTER(TuneTable)]),
    ("atr_batch_autotune", C.c_int, [_p, _p, C.POINTER(AutotuneConfig), C.POINTER(TuneTable),
                                     C.POINTER(TuneOutcome)]),
    ("atr_server_create", C.c_int, [C.c_int, C.POINTER(ServerConfig), C.POINTER(_p)]),
    ("atr_server_submit", C.c_int, [_p, C.POINTER(ServerRequest), C.POINTER(C.c_uint64)]),
    ("atr_server_wait", C.c_int, [_p, C.c_uint64, C.POINTER(ServerResult)]),
    ("atr_server_release", C.c_int, [_p, C.c_uint64]),
    ("atr_server_stats_get", C.c_int, [_p, C.POINTER(ServerStats)]),
    ("atr_server_destroy", C.c_int, [_p]),
]

EXPORTED = [name for name, _, _ in _SIGS]


def lib() -> C.CDLL:
    """Load libatrbvh.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise AtrError(-1, f"{LIB_PATH} is missing; run `python -m atrbvh_b200.build`")
        l = C.CDLL(str(LIB_PATH))
        for name, res, args in _SIGS:
            f = getattr(l, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def check(status: int) -> None:
    if status != ATR_OK:
        raise AtrError(status, lib().atr_last_error().decode(errors="replace"))


def _f3(v) -> C.Array:
    a = (C.c_float * 3)(*[float(x) for x in v])
    return a


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


# ---- synthetic workloads ------------------------------------------------------

def gen_scene(kind: int, n: int, seed: int = 0) -> np.ndarray:
    """Triangle soup (n, 3, 4) float32 of the given distribution."""
    out = np.empty((n, 3, 4), dtype=np.float32)
    check(lib().atr_gen_scene(kind, n, seed, _ptr(out)))
    return out


def gen_batch_sizes(count: int, lo: int, hi: int, seed: int = 0) -> np.ndarray:
    out = np.empty(count, dtype=np.uint32)
    check(lib().atr_gen_batch_sizes(count, lo, hi, seed, _ptr(out)))
    return out


def gen_batch_scene(sizes: np.ndarray, seed: int = 0) -> np.ndarray:
    sizes = np.ascontiguousarray(sizes, dtype=np.uint32)
    out = np.empty((int(sizes.sum()), 3, 4), dtype=np.float32)
    check(lib().atr_gen_batch_scene(len(sizes), _ptr(sizes), seed, _ptr(out)))
    return out


def gen_rays_pinhole(w: int, h: int, eye=(0.5, 0.5, -1.5), fov_deg: float = 60.0) -> np.ndarray:
    out = np.empty((w * h, 2, 4), dtype=np.float32)
    check(lib().atr_gen_rays_pinhole(w, h, _f3(eye), fov_deg, _ptr(out)))
    return out


def gen_rays_random(n: int, bbmin, bbmax, seed: int = 0) -> np.ndarray:
    out = np.empty((n, 2, 4), dtype=np.float32)
    check(lib().atr_gen_rays_random(n, seed, _f3(bbmin), _f3(bbmax), _ptr(out)))
    return out


# ---- runtime objects -----------------------------------------------------------

class Context:
    """One CUDA stream plus scratch pool (atr_ctx)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        h = C.c_void_p()
        check(lib().atr_ctx_create(device, C.c_void_p(stream) if stream else None, C.byref(h)))
        self.handle = h
        # Objects whose device memory came from this context's pool: they are
        # freed before the context (a destroy after it would touch freed state).
        self._deps = weakref.WeakSet()

    def _adopt(self, obj) -> None:
        self._deps.add(obj)

    def synchronize(self) -> None:
        check(lib().atr_ctx_synchronize(self.handle))

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().atr_ctx_get_stream(self.handle, C.byref(s)))
        return s.value or 0

    def launch_count(self) -> int:
        c = C.c_uint64()
        check(lib().atr_ctx_launch_count(self.handle, C.byref(c)))
        return c.value

    def set_tuning(self, knob: int, value: int) -> None:
        check(lib().atr_ctx_set_tuning(self.handle, knob, value))

    def get_tuning(self, knob: int) -> int:
        v = C.c_int()
        check(lib().atr_ctx_get_tuning(self.handle, knob, C.byref(v)))
        return v.value

    def set_timing(self, on: bool) -> None:
        check(lib().atr_ctx_set_timing(self.handle, 1 if on else 0))

    def phase_times(self) -> list[tuple[str, float]]:
        """(name, ms) of every timed phase since timing was enabled or last read."""
        cap = 4096
        buf = (C.c_float * cap)()
        n = C.c_int()
        check(lib().atr_ctx_phase_times(self.handle, buf, cap, C.byref(n)))
        names = lib().atr_ctx_phase_names(self.handle).decode().split(",")
        return [(names[i] if i < len(names) else "?", buf[i]) for i in range(min(n.value, cap))]

    def close(self) -> None:
        if getattr(self, "handle", None):
            for obj in list(getattr(self, "_deps", ())):
                obj.close()
            lib().atr_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pinned_like(a: np.ndarray) -> np.ndarray:
    """A page-locked host copy of a (through torch's pinned allocator), for
    request buffers that the server and the upload paths copy directly."""
    import torch
    t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
    out = t.numpy().view(a.dtype).reshape(a.shape)
    out[...] = a
    return out  # the view's base is the tensor, which keeps the pinned storage alive


def scene_bounds(vertices) -> tuple[np.ndarray, np.ndarray]:
    """Host-side scene box as the reference's SceneConverter computes it
    (gpu-ray-traversal/src/rt/SceneConverter.cpp:19-72): the minimum over all
    vertices, and the maximum seeded with FLT_MIN (the smallest positive
    normal float), for SceneWrapper's bbmin/bbmax."""
    v = np.asarray(vertices, dtype=np.float32).reshape(-1, 4)[:, :3]
    mn = v.min(axis=0)
    mx = np.maximum(v.max(axis=0), np.finfo(np.float32).tiny)
    return mn.astype(np.float32), mx.astype(np.float32)


class SceneWrapper:
    """BVHRT::SceneWrapper: device copy of the triangle soup and its box."""

    def __init__(self, ctx: Context, vertices, bbmin=None, bbmax=None, device_ptr: int | None = None,
                 num_triangles: int | None = None):
        self.ctx = ctx
        h = C.c_void_p()
        if device_ptr is not None:
            n = int(num_triangles)
            src, on_dev = C.c_void_p(device_ptr), 1
        else:
            v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3, 4)
            n = v.shape[0]
            src, on_dev = _ptr(v), 0
            self._host = v
        bmin = _f3(bbmin) if bbmin is not None else None
        bmax = _f3(bbmax) if bbmax is not None else None
        check(lib().atr_scene_create(ctx.handle, src, n, bmin, bmax, on_dev, C.byref(h)))
        self.handle = h
        self.n = n
        ctx._adopt(self)

    def bounds(self) -> tuple[np.ndarray, np.ndarray]:
        a = (C.c_float * 3)()
        b = (C.c_float * 3)()
        check(lib().atr_scene_bounds(self.ctx.handle, self.handle, a, b))
        return np.array(a[:], np.float32), np.array(b[:], np.float32)

    def set_vertices(self, vertices=None, device_ptr: int | None = None) -> None:
        if device_ptr is not None:
            check(lib().atr_scene_set_vertices(self.ctx.handle, self.handle, C.c_void_p(device_ptr), 1))
        else:
            v = np.ascontiguousarray(vertices, dtype=np.float32)
            check(lib().atr_scene_set_vertices(self.ctx.handle, self.handle, _ptr(v), 0))
            self.ctx.synchronize()

    def device_vertices(self) -> int:
        p = C.c_void_p()
        check(lib().atr_scene_device_vertices(self.handle, C.byref(p), None))
        return p.value

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().atr_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class HostTree:
    """Host mirror of a device tree (SoABVHTree after DeviceToHostTree)."""
    parent: np.ndarray
    left: np.ndarray
    right: np.ndarray
    data: np.ndarray
    bbox_min: np.ndarray  # (2N-1, 4)
    bbox_max: np.ndarray
    area: np.ndarray

    @property
    def num_triangles(self) -> int:
        return (len(self.parent) + 1) // 2

    def RootIndex(self) -> int:
        return 0

    def SAH(self, ci: float = 1.2, ct: float = 1.0) -> float:
        """SoABVHTree::SAH with the reference's sequential float32 sums."""
        a = self.area.astype(np.float32)
        n = self.num_triangles
        si = np.float32(a[0])
        for x in a[1:n - 1]:
            si = np.float32(si + x)
        sl = np.float32(0.0)
        for x in a[n - 1:]:
            sl = np.float32(sl + x)
        return float(np.float32(np.float32(np.float32(ci) * si) + np.float32(np.float32(ct) * sl)) / a[0])


class BVHTree:
    """Device tree handle (atr_tree); arrays in the reference's SoA layout."""

    def __init__(self, ctx: Context, handle: C.c_void_p, n: int):
        self.ctx = ctx
        self.handle = handle
        self.n = n
        ctx._adopt(self)

    def view(self) -> TreeView:
        v = TreeView()
        check(lib().atr_tree_view_get(self.handle, C.byref(v)))
        return v

    def NumberOfTriangles(self) -> int:
        return self.n

    def sah(self, ci: float = 1.2, ct: float = 1.0) -> float:
        s = C.c_float()
        check(lib().atr_tree_sah(self.ctx.handle, self.handle, ci, ct, C.byref(s)))
        return s.value

    def sorted_keys(self) -> tuple[np.ndarray, np.ndarray]:
        k = np.empty(self.n, np.uint64)
        i = np.empty(self.n, np.uint32)
        check(lib().atr_tree_sorted_keys(self.ctx.handle, self.handle, _ptr(k), _ptr(i)))
        return k, i

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().atr_tree_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LBVHBuilder:
    """BVHRT::LBVHBuilder(use64BitMortonCodes)."""

    def __init__(self, use64BitMortonCodes: bool = False):
        self.bits = 63 if use64BitMortonCodes else 30

    def BuildTree(self, scene: SceneWrapper) -> BVHTree:
        h = C.c_void_p()
        check(lib().atr_build_lbvh(scene.ctx.handle, scene.handle, self.bits, C.byref(h)))
        return BVHTree(scene.ctx, h, scene.n)


def split_triangles(scene: SceneWrapper, split_ratio: float = 0.3, max_primitives: int | None = None):
    """Triangle splitting (atr_split_triangles): up to split_ratio * n extra
    primitives for the triangles whose boxes waste the most surface.  Returns
    device tensors (bmin float32 [P, 4], bmax float32 [P, 4], data int32 [P])
    of the fragments, fragments of one triangle together in triangle order."""
    import torch
    cap = max_primitives if max_primitives is not None else scene.n + int(split_ratio * scene.n) + 1
    bmin = torch.empty((cap, 4), dtype=torch.float32, device="cuda")
    bmax = torch.empty((cap, 4), dtype=torch.float32, device="cuda")
    data = torch.empty(cap, dtype=torch.int32, device="cuda")
    cnt = C.c_uint32()
    check(lib().atr_split_triangles(scene.ctx.handle, scene.handle, split_ratio, cap, bmin.data_ptr(),
                                    bmax.data_ptr(), data.data_ptr(), C.byref(cnt)))
    n = cnt.value
    return bmin[:n], bmax[:n], data[:n]


def build_lbvh_split(ctx: Context, bmin, bmax, data, scene_bmin, scene_bmax, bits: int = 30) -> BVHTree:
    """The triangle-splitting LBVH (atr_build_lbvh_split) over primitive boxes
    (contiguous device tensors: float32 [P, 4] twice, int32 [P]) in the box
    scene_bmin..scene_bmax."""
    n = int(data.shape[0])
    h = C.c_void_p()
    check(lib().atr_build_lbvh_split(ctx.handle, n, bmin.data_ptr(), bmax.data_ptr(), data.data_ptr(),
                                     _f3(scene_bmin), _f3(scene_bmax), bits, C.byref(h)))
    return BVHTree(ctx, h, n)


class AgglomerativeTreeletOptimizer:
    """BVHRT::AgglomerativeTreeletOptimizer(treeletSize=9, iterations=2)."""

    def __init__(self, treeletSize: int = 9, iterations: int = 2, ci: float = 1.2, ct: float = 1.0):
        self.treelet, self.iterations, self.ci, self.ct = treeletSize, iterations, ci, ct

    def Optimize(self, tree: BVHTree) -> None:
        check(lib().atr_optimize_atrbvh(tree.ctx.handle, tree.handle, self.treelet, self.iterations,
                                        self.ci, self.ct))


class TRBVHOptimizer:
    """BVHRT::TRBVHOptimizer(treeletSize=7, iterations=3)."""

    def __init__(self, treeletSize: int = 7, iterations: int = 3, ci: float = 1.2, ct: float = 1.0):
        self.treelet, self.iterations, self.ci, self.ct = treeletSize, iterations, ci, ct

    def Optimize(self, tree: BVHTree) -> None:
        check(lib().atr_optimize_trbvh(tree.ctx.handle, tree.handle, self.treelet, self.iterations,
                                       self.ci, self.ct))


def Refit(tree: BVHTree, scene: SceneWrapper) -> None:
    """Bottom-up box refit of a resident tree from the scene's current vertices."""
    check(lib().atr_refit(tree.ctx.handle, tree.handle, scene.handle))


@dataclass
class HostCollapsedTree:
    parent: np.ndarray
    left: np.ndarray
    right: np.ndarray
    data: np.ndarray
    triangle_count: np.ndarray
    bbox_min: np.ndarray
    bbox_max: np.ndarray
    triangle_indices: np.ndarray


class BVHCollapsedTree:
    def __init__(self, ctx: Context, handle: C.c_void_p, n: int):
        self.ctx, self.handle, self.n = ctx, handle, n
        ctx._adopt(self)

    def view(self) -> CollapsedView:
        v = CollapsedView()
        check(lib().atr_collapsed_view_get(self.handle, C.byref(v)))
        return v

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().atr_collapsed_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BVHTreeCollapser:
    """BVHRT::BVHTreeCollapser::Collapse(tree, &sah, ci, ct); max_leaf=0 is the reference."""

    def Collapse(self, tree: BVHTree, ci: float = 1.2, ct: float = 1.0, max_leaf: int = 0, want_sah: bool = True):
        """Returns (collapsed tree, SAH); with want_sah=False the SAH is None
        and no host synchronisation happens."""
        h = C.c_void_p()
        s = C.c_float()
        check(lib().atr_collapse(tree.ctx.handle, tree.handle, ci, ct, max_leaf, C.byref(h),
                                 C.byref(s) if want_sah else None))
        return BVHCollapsedTree(tree.ctx, h, tree.n), (s.value if want_sah else None)


class BVHTreeInstanceManager:
    """Host copies of device trees (BVHRT::BVHTreeInstanceManager)."""

    def DeviceToHostTree(self, tree: BVHTree) -> HostTree:
        nn = 2 * tree.n - 1
        ht = HostTree(*(np.empty(nn, np.int32) for _ in range(4)), np.empty((nn, 4), np.float32),
                      np.empty((nn, 4), np.float32), np.empty(nn, np.float32))
        check(lib().atr_tree_download(tree.ctx.handle, tree.handle, _ptr(ht.parent), _ptr(ht.left),
                                      _ptr(ht.right), _ptr(ht.data), _ptr(ht.bbox_min), _ptr(ht.bbox_max),
                                      _ptr(ht.area)))
        return ht

    def DeviceToHostCollapsedTree(self, c: BVHCollapsedTree) -> HostCollapsedTree:
        nn = 2 * c.n - 1
        h = HostCollapsedTree(*(np.empty(nn, np.int32) for _ in range(5)), np.empty((nn, 4), np.float32),
                              np.empty((nn, 4), np.float32), np.empty(c.n, np.int32))
        check(lib().atr_collapsed_download(c.ctx.handle, c.handle, _ptr(h.parent), _ptr(h.left),
                                           _ptr(h.right), _ptr(h.data), _ptr(h.triangle_count),
                                           _ptr(h.bbox_min), _ptr(h.bbox_max), _ptr(h.triangle_indices)))
        return h

    def FreeDeviceTree(self, tree: BVHTree) -> None:
        tree.close()

    def FreeDeviceCollapsedTree(self, c: BVHCollapsedTree) -> None:
        c.close()


class Batch:
    """Segmented batch of meshes built together (atr_batch).

    vertices: (N, 3, 4) float32 soup of all meshes end to end (host array or
    device pointer with num_triangles); offsets: (M+1,) uint32 triangle offsets.
    """

    ATRBVH, TRBVH, NONE = 1, 2, 0

    def __init__(self, ctx: Context, vertices=None, offsets=None, device_ptr: int | None = None, bounds=None):
        self.ctx = ctx
        off = np.ascontiguousarray(offsets, dtype=np.uint32)
        self.offsets = off
        self.count = len(off) - 1
        h = C.c_void_p()
        b = None if bounds is None else np.ascontiguousarray(bounds, dtype=np.float32)
        if device_ptr is not None:
            src, on_dev = C.c_void_p(device_ptr), 1
        else:
            v = np.ascontiguousarray(vertices, dtype=np.float32)
            src, on_dev = _ptr(v), 0
        check(lib().atr_batch_create(ctx.handle, src, _ptr(off), self.count, None if b is None else _ptr(b), on_dev,
                                     C.byref(h)))
        self.handle = h
        ctx._adopt(self)

    def set_params(self, treelet_sizes=None, iterations=None) -> None:
        if treelet_sizes is None:
            check(lib().atr_batch_set_params(self.ctx.handle, self.handle, None, None))
            return
        ts = np.ascontiguousarray(treelet_sizes, dtype=np.uint8)
        it = np.ascontiguousarray(iterations, dtype=np.uint8)
        check(lib().atr_batch_set_params(self.ctx.handle, self.handle, _ptr(ts), _ptr(it)))

    def apply_tuning(self, table: "TuneTable") -> None:
        """Per-mesh treelet/iterations from an autotuner table, and the
        context's launch tuning from the class holding most triangles."""
        check(lib().atr_batch_apply_tuning(self.ctx.handle, self.handle, C.byref(table)))

    def build(self, optimizer: int = 1, treelet: int = 9, iterations: int = 2, ci: float = 1.2, ct: float = 1.0,
              graph: bool = False) -> None:
        check(lib().atr_batch_build(self.ctx.handle, self.handle, optimizer, treelet, iterations, ci, ct,
                                    1 if graph else 0))

    def mesh(self, m: int) -> HostTree:
        n = int(self.offsets[m + 1] - self.offsets[m])
        nn = 2 * n - 1
        ht = HostTree(*(np.empty(nn, np.int32) for _ in range(4)), np.empty((nn, 4), np.float32),
                      np.empty((nn, 4), np.float32), np.empty(nn, np.float32))
        check(lib().atr_batch_download_mesh(self.ctx.handle, self.handle, m, _ptr(ht.parent), _ptr(ht.left),
                                            _ptr(ht.right), _ptr(ht.data), _ptr(ht.bbox_min), _ptr(ht.bbox_max),
                                            _ptr(ht.area)))
        return ht

    def sah(self, ci: float = 1.2, ct: float = 1.0) -> np.ndarray:
        out = np.empty(self.count, np.float32)
        check(lib().atr_batch_sah(self.ctx.handle, self.handle, ci, ct, _ptr(out)))
        return out

    def collapse(self, ci: float = 1.2, ct: float = 1.0, max_leaf: int = 0, want_sah: bool = True):
        out = np.empty(self.count, np.float32) if want_sah else None
        check(lib().atr_batch_collapse(self.ctx.handle, self.handle, ci, ct, max_leaf,
                                       _ptr(out) if want_sah else None))
        return out

    def flatten(self) -> None:
        check(lib().atr_batch_flatten(self.ctx.handle, self.handle))

    def compact_view(self, m: int) -> CompactView:
        v = CompactView()
        check(lib().atr_batch_compact_view(self.handle, m, C.byref(v)))
        return v

    def compact(self, m: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Host copies of mesh m's Compact2 arrays (nodes, woop, tri_index)."""
        v = self.compact_view(m)
        nodes = np.empty((v.num_nodes, 16), np.int32)
        woop = np.empty((v.num_woop, 4), np.float32)
        tri = np.empty(v.num_woop, np.int32)
        check(lib().atr_batch_compact_download(self.ctx.handle, self.handle, m, _ptr(nodes), _ptr(woop), _ptr(tri)))
        return nodes, woop, tri

    def trace(self, rays_ptr: int, num_rays: int, ray_offsets, group_mesh, results_ptr: int,
              any_hit: bool = False) -> None:
        off = np.ascontiguousarray(ray_offsets, dtype=np.uint32)
        gm = np.ascontiguousarray(group_mesh, dtype=np.uint32)
        check(lib().atr_batch_trace(self.ctx.handle, self.handle, C.c_void_p(rays_ptr), num_rays, _ptr(off),
                                    _ptr(gm), len(gm), 1 if any_hit else 0, C.c_void_p(results_ptr)))

    def refit_mesh(self, m: int, vertices=None, device_ptr: int | None = None) -> None:
        if device_ptr is not None:
            check(lib().atr_batch_refit_mesh(self.ctx.handle, self.handle, m, C.c_void_p(device_ptr), 1))
        else:
            v = np.ascontiguousarray(vertices, dtype=np.float32)
            check(lib().atr_batch_refit_mesh(self.ctx.handle, self.handle, m, _ptr(v), 0))
            self.ctx.synchronize()

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().atr_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CudaBVH:
    """Compact2 layout + Woop triangles of a collapsed tree, and its traversal."""

    def __init__(self, collapsed: BVHCollapsedTree, scene: SceneWrapper):
        h = C.c_void_p()
        check(lib().atr_flatten_compact2(scene.ctx.handle, collapsed.handle, scene.handle, C.byref(h)))
        self.ctx = scene.ctx
        self.handle = h
        self.ctx._adopt(self)

    def view(self) -> CompactView:
        v = CompactView()
        check(lib().atr_compact_view_get(self.handle, C.byref(v)))
        return v

    def download(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Host copies (nodes (M,16) int32, woop (W,4) float32, tri_index (W,) int32)."""
        v = self.view()
        nodes = np.empty((v.num_nodes, 16), np.int32)
        woop = np.empty((v.num_woop, 4), np.float32)
        tri = np.empty(v.num_woop, np.int32)
        check(lib().atr_compact_download(self.ctx.handle, self.handle, _ptr(nodes), _ptr(woop), _ptr(tri)))
        return nodes, woop, tri

    @classmethod
    def from_image(cls, ctx: "Context", image: bytes) -> "CudaBVH":
        """A traversal layout loaded from a cache image (atr_compact_deserialize)."""
        buf = np.frombuffer(image, dtype=np.uint8)
        h = C.c_void_p()
        check(lib().atr_compact_deserialize(ctx.handle, _ptr(buf), len(buf), C.byref(h)))
        self = cls.__new__(cls)
        self.ctx = ctx
        self.handle = h
        ctx._adopt(self)
        return self

    def serialize(self) -> bytes:
        """The cache image in the reference's CudaBVH stream format."""
        size = C.c_uint64()
        check(lib().atr_compact_serialize(self.ctx.handle, self.handle, None, 0, C.byref(size)))
        out = np.empty(size.value, np.uint8)
        check(lib().atr_compact_serialize(self.ctx.handle, self.handle, _ptr(out), size.value, C.byref(size)))
        return out.tobytes()

    def trace(self, rays_ptr: int, num_rays: int, results_ptr: int, any_hit: bool = False) -> None:
        """rays: device float4 pairs; results: device int4 per ray."""
        check(lib().atr_trace(self.ctx.handle, self.handle, C.c_void_p(rays_ptr), num_rays,
                              1 if any_hit else 0, C.c_void_p(results_ptr)))

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().atr_compact_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Borrowed:
    """A plan-owned tree, collapsed tree or layout: usable like the objects the
    builders return, but freed with the plan (close() does nothing)."""

    def close(self) -> None:
        self.handle = None


class BuildPlan:
    """The steady-state build of one scene (atr_plan): LBVH -> optimiser ->
    collapse (-> Compact2) into plan-owned outputs; run(graph=True) replays it
    from a CUDA graph with one launch."""

    def __init__(self, scene: SceneWrapper, morton_bits: int = 30, optimizer: int = 1, treelet: int = 9,
                 iterations: int = 2, ci: float = 1.2, ct: float = 1.0, max_leaf: int = 0, flatten: bool = True):
        self.ctx = scene.ctx
        self.scene = scene
        self.n = scene.n
        p = PlanParams(morton_bits, optimizer, treelet, iterations, ci, ct, max_leaf, 1 if flatten else 0)
        h = C.c_void_p()
        check(lib().atr_plan_create(self.ctx.handle, scene.handle, C.byref(p), C.byref(h)))
        self.handle = h
        self.ctx._adopt(self)

    def run(self, graph: bool = True) -> None:
        check(lib().atr_plan_run(self.ctx.handle, self.handle, 1 if graph else 0))

    def tree(self) -> BVHTree:
        h = C.c_void_p()
        check(lib().atr_plan_tree(self.handle, C.byref(h)))
        t = BVHTree.__new__(BVHTree)
        t.ctx, t.handle, t.n = self.ctx, h, self.n
        t.close = _Borrowed.close.__get__(t)
        return t

    def collapsed(self) -> BVHCollapsedTree:
        h = C.c_void_p()
        check(lib().atr_plan_collapsed(self.handle, C.byref(h)))
        c = BVHCollapsedTree.__new__(BVHCollapsedTree)
        c.ctx, c.handle, c.n = self.ctx, h, self.n
        c.close = _Borrowed.close.__get__(c)
        return c

    def compact(self) -> "CudaBVH":
        h = C.c_void_p()
        check(lib().atr_plan_compact(self.ctx.handle, self.handle, C.byref(h)))
        b = CudaBVH.__new__(CudaBVH)
        b.ctx, b.handle = self.ctx, h
        b.close = _Borrowed.close.__get__(b)
        return b

    def sah(self) -> float:
        s = C.c_float()
        check(lib().atr_plan_sah(self.ctx.handle, self.handle, C.byref(s)))
        return s.value

    def phase_times(self) -> list[tuple[str, float]]:
        """(phase, device ms) of the last graph replay."""
        ms = (C.c_float * 64)()
        k = C.c_int()
        check(lib().atr_plan_phase_times(self.ctx.handle, self.handle, ms, 64, C.byref(k)))
        names = lib().atr_plan_phase_names(self.handle).decode().split(",")
        return list(zip(names, ms[:k.value]))

    def times(self) -> tuple[float, float]:
        """Device ms of the last run: (Morton through collapse, flatten)."""
        a, b = C.c_float(), C.c_float()
        check(lib().atr_plan_times(self.ctx.handle, self.handle, C.byref(a), C.byref(b)))
        return a.value, b.value

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().atr_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ray_batches(num_input_rays: int, num_samples: int, max_batch: int = 1 << 20):
    """Slices [lo, hi) of an input ray batch whose secondary rays fit in
    max_batch rays, as RayGen::batching cuts them
    (gpu-ray-traversal/src/rt/ray/RayGen.cpp:240-258; the benchmark's batches
    hold 2^20 rays)."""
    lo = 0
    step = max(1, max_batch // num_samples)
    while lo < num_input_rays:
        hi = min(num_input_rays, lo + step)
        yield lo, hi
        lo = hi


def gen_ao_rays(scene: SceneWrapper, rays_ptr: int, results_ptr: int, first: int, count: int, num_samples: int,
                max_dist: float, seed: int, out_ptr: int) -> None:
    """Ambient-occlusion rays for rays[first:first+count] (device arrays), see atr_gen_ao_rays."""
    check(lib().atr_gen_ao_rays(scene.ctx.handle, scene.handle, C.c_void_p(rays_ptr), C.c_void_p(results_ptr),
                                first, count, num_samples, max_dist, seed & 0xFFFFFFFF, C.c_void_p(out_ptr)))


def sort_rays(ctx: "Context", rays_ptr: int, num_rays: int, out_rays_ptr: int, slot_to_id_ptr: int | None = None,
              out_slot_to_id_ptr: int | None = None, out_id_to_slot_ptr: int | None = None) -> None:
    """Morton sort of a ray batch on the device (atr_sort_rays)."""
    p = lambda x: None if x is None else C.c_void_p(x)  # noqa: E731
    check(lib().atr_sort_rays(ctx.handle, C.c_void_p(rays_ptr), p(slot_to_id_ptr), num_rays, C.c_void_p(out_rays_ptr),
                              p(out_slot_to_id_ptr), p(out_id_to_slot_ptr)))


def cache_key(vertices, morton_bits: int = 30, optimizer: int = 1, treelet: int = 9, iterations: int = 2,
              ci: float = 1.2, ct: float = 1.0, max_leaf: int = 0) -> int:
    """64-bit cache key of a scene and the build parameters (atr_cache_key)."""
    v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3, 4)
    p = CacheParams(morton_bits, optimizer, treelet, iterations, ci, ct, max_leaf)
    k = C.c_uint64()
    check(lib().atr_cache_key(_ptr(v), v.shape[0], C.byref(p), C.byref(k)))
    return k.value


class BVHCache:
    """Directory of cache images named by cache key ("<key as 16 hex
    digits>.dat"), as Renderer::getCudaBVH names its files
    (gpu-ray-traversal/src/rt/cuda/Renderer.cpp:137-158): load() returns the
    stored layout or None, store() writes one atomically."""

    def __init__(self, directory):
        from pathlib import Path
        self.dir = Path(directory)
        self.dir.mkdir(parents=True, exist_ok=True)

    def path(self, key: int):
        return self.dir / f"{key:016x}.dat"

    def load(self, ctx: "Context", key: int) -> "CudaBVH | None":
        p = self.path(key)
        if not p.exists():
            return None
        return CudaBVH.from_image(ctx, p.read_bytes())

    def store(self, key: int, bvh: "CudaBVH") -> None:
        import os
        p = self.path(key)
        tmp = p.with_suffix(f".tmp{os.getpid()}")
        tmp.write_bytes(bvh.serialize())
        os.replace(tmp, p)


def autotune(ctx: Context, min_class: int = 8, max_class: int = 21, sample_triangles: int = 1 << 21,
             sah_tolerance: float = 0.0, reps: int = 3, seed: int = 0) -> TuneTable:
    """Per size class, the fastest ATRBVH treelet size / iterations at an SAH no
    worse than ATRBVH(9,2) (within sah_tolerance), then the fastest ATRBVH
    block size and sort digit width (atr_autotune)."""
    cfg = AutotuneConfig(min_class, max_class, sample_triangles, sah_tolerance, reps, seed)
    t = TuneTable()
    check(lib().atr_autotune(ctx.handle, C.byref(cfg), C.byref(t)))
    return t


def batch_autotune(ctx: Context, batch: "Batch", sample_triangles: int = 1 << 22, sah_tolerance: float = 0.0,
                   reps: int = 3, seed: int = 0) -> tuple[TuneTable, dict]:
    """Tune the batch's size classes, keep the table only if the batch itself
    builds faster with it (atr_batch_autotune); returns (table, outcome)."""
    cfg = AutotuneConfig(1, 29, sample_triangles, sah_tolerance, reps, seed)
    t = TuneTable()
    o = TuneOutcome()
    check(lib().atr_batch_autotune(ctx.handle, batch.handle, C.byref(cfg), C.byref(t), C.byref(o)))
    return t, {name: getattr(o, name) for name, _ in TuneOutcome._fields_}


# ---- serving loop ----------------------------------------------------------------

REQ_BUILD, REQ_REFIT = 0, 1
ERR_NOT_RESIDENT = 7


class Server:
    """Build/refit + trace request server (atr_server): admission by device
    memory, resident BVHs for refits, continuous batching over `lanes` streams.

    submit() returns a ticket; the arrays passed stay referenced until wait()
    returns that ticket's result (a dict).  results (N, 4) int32 is filled in
    place."""

    def __init__(self, device: int = 0, hbm_budget: int = 120 << 30, lanes: int = 2, max_batch_requests: int = 64,
                 max_batch_triangles: int = 1 << 26, treelet: int = 9, iterations: int = 2, max_leaf: int = 0,
                 class_treelet=None, class_iters=None):
        cfg = ServerConfig(hbm_budget, lanes, max_batch_requests, max_batch_triangles, treelet, iterations, max_leaf,
                           None, None)
        if class_treelet is not None:
            self._ct = np.ascontiguousarray(class_treelet, dtype=np.uint8)
            self._ci = np.ascontiguousarray(class_iters, dtype=np.uint8)
            assert self._ct.shape == (32,) and self._ci.shape == (32,)
            cfg.class_treelet, cfg.class_iters = self._ct.ctypes.data, self._ci.ctypes.data
        h = C.c_void_p()
        check(lib().atr_server_create(device, C.byref(cfg), C.byref(h)))
        self.handle = h
        self._keep: dict[int, tuple] = {}

    def submit(self, kind: int, mesh_id: int, vertices, rays=None, results=None, keep_resident: bool = True) -> int:
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3, 4)
        r = None if rays is None else np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        nr = 0 if r is None else r.shape[0]
        if nr:
            assert results is not None and results.dtype == np.int32 and results.flags.c_contiguous
            assert results.size >= 4 * nr
        req = ServerRequest(kind, mesh_id, v.ctypes.data, v.shape[0], None if r is None else r.ctypes.data, nr,
                            None if not nr else results.ctypes.data, 1 if keep_resident else 0)
        t = C.c_uint64()
        check(lib().atr_server_submit(self.handle, C.byref(req), C.byref(t)))
        self._keep[t.value] = (v, r, results)
        return t.value

    def wait(self, ticket: int) -> dict:
        res = ServerResult()
        check(lib().atr_server_wait(self.handle, ticket, C.byref(res)))
        self._keep.pop(ticket, None)
        return {"status": res.status, "sah": res.sah, "queue_ms": res.queue_ms, "latency_ms": res.latency_ms,
                "batch_requests": res.batch_requests, "lane": res.lane, "error": res.error.decode()}

    def release(self, mesh_id: int) -> None:
        check(lib().atr_server_release(self.handle, mesh_id))

    def stats(self) -> dict:
        st = ServerStats()
        check(lib().atr_server_stats_get(self.handle, C.byref(st)))
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().atr_server_destroy(self.handle)
            self.handle = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
