"""ORACLE -- test infrastructure only.

Builds the checkers:
  oracle/liboracle.so              CPU restatement (atr_oracle.cpp), g++ -O2
                                   -ffp-contract=off -fopenmp.
  oracle/_ref/libbvhrt_ref.so      the reference's own BVHRT-Core CUDA sources,
  oracle/_ref/libbvhrt_ref_fmad.so compiled in place from the reference tree for
                                   sm_100a (-fmad=false, and nvcc's default
                                   contraction), with oracle/ref_shims/.
The reference build runs only where the reference tree is present; the built
files travel with the repository to the GPU machine.
Run as ``python -m oracle.build``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_SRC = Path("/root/reference/BVHRT-Core/src")
REF_OUT = HERE / "_ref"

# Reference files on the build path (CubWrapper.cu is replaced by
# ref_shims/sort_shim.cu; DeviceSum in it has no callers).
REF_DEVICE = ["LBVH.cu", "AgglomerativeTreelet.cu", "TRBVH.cu", "TreeCollapser.cu"]
REF_HOST = ["LBVHBuilder.cpp", "AgglomerativeTreeletOptimizer.cpp", "AgglomerativeScheduler.cpp",
            "TRBVHOptimizer.cpp", "TRBVHScheduler.cpp", "BVHTreeCollapser.cpp",
            "BVHTreeInstanceManager.cpp", "SoABVHTree.cpp", "BVHCollapsedTree.cpp", "SceneWrapper.cpp",
            "CudaTimer.cpp"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_oracle() -> Path:
    out = HERE / "liboracle.so"
    src = HERE / "atr_oracle.cpp"
    if out.exists() and out.stat().st_mtime >= src.stat().st_mtime:
        return out
    _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
          "-shared", "-o", str(out), str(src)])
    return out


def build_reference(fmad: bool) -> Path | None:
    if not REF_SRC.is_dir():
        return None
    REF_OUT.mkdir(exist_ok=True)
    tag = "fmad" if fmad else "nofmad"
    lib = REF_OUT / ("libbvhrt_ref_fmad.so" if fmad else "libbvhrt_ref.so")
    shims = HERE / "ref_shims"
    srcs = [REF_SRC / f for f in REF_DEVICE + REF_HOST] + [shims / "sort_shim.cu", shims / "ref_capi.cu"]
    newest = max(p.stat().st_mtime for p in srcs + [shims / "legacy_warp.h", Path(__file__)])
    if lib.exists() and lib.stat().st_mtime >= newest:
        return lib
    objdir = REF_OUT / f"obj_{tag}"
    objdir.mkdir(exist_ok=True)
    base = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++14",
            f"-fmad={'true' if fmad else 'false'}", "-Xcompiler", "-fPIC", "-w",
            "-include", str(shims / "legacy_warp.h"), "-I", str(REF_SRC), "-I", str(shims)]
    jobs = []
    objs = []
    for s in srcs:
        o = objdir / (s.name + ".o")
        objs.append(o)
        lang = ["-x", "cu"] if s.suffix == ".cpp" else []
        cmd = base + lang + ["-c", str(s), "-o", str(o)]
        if s.parent == shims:  # own shim sources: no legacy-intrinsic macros
            cmd = [a for a in cmd if a not in ("-include", str(shims / "legacy_warp.h"))]
        jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        for f in [ex.submit(_run, j) for j in jobs]:
            f.result()
    _run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(lib), *map(str, objs)])
    return lib


def build_all() -> None:
    build_oracle()
    build_reference(False)
    build_reference(True)


if __name__ == "__main__":
    build_all()
    print("oracle built")
