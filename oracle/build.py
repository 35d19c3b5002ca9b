"""ORACLE -- test infrastructure only.

Builds the checkers:
  oracle/liboracle.so                CPU restatement (atr_oracle.cpp,
                                     raygen_oracle.cpp) and the seeded
                                     workload generators
                                     (workload_oracle.cpp), g++ -O2
                                     -ffp-contract=off -fopenmp.
  oracle/_ref/libbvhrt_ref_host.so   the reference's own BVHRT-Core sources
                                     (kernels and host classes), compiled in
                                     place by g++ for the host execution model
                                     of oracle/ref_cpu/ (every CUDA thread a
                                     fiber), where the reference tree is
                                     present.  It travels with the repository.

The reference's own sources are located through the ATRBVH_REFERENCE
environment variable (the root of the leonardo-domingues/atrbvh tree; default
/root/reference, a read-only checkout).  Nothing here runs the reference's CUDA
kernels.
Run as ``python -m oracle.build``.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_OUT = HERE / "_ref"


def reference_root() -> Path | None:
    """Root of the reference tree, or None where it is absent (the GPU box)."""
    root = Path(os.environ.get("ATRBVH_REFERENCE", "/root/reference"))
    return root if (root / "BVHRT-Core" / "src").is_dir() else None


def _run(cmd: list[str], **kw) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_oracle() -> Path:
    out = HERE / "liboracle.so"
    srcs = [HERE / "atr_oracle.cpp", HERE / "workload_oracle.cpp", HERE / "raygen_oracle.cpp"]
    if out.exists() and out.stat().st_mtime >= max(p.stat().st_mtime for p in srcs):
        return out
    _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
          "-shared", "-o", str(out), *map(str, srcs)])
    return out


# ---- the reference's BVHRT-Core sources under the host execution model --------

# Reference files compiled in place (paths under BVHRT-Core/src).  CubWrapper.cu
# is replaced by ref_cpu/sort_host.cpp (the sort it performs, into the *Out
# buffers); DeviceSum in it has no callers on this path.
REF_KERNELS = ["LBVH.cu", "AgglomerativeTreelet.cu", "TRBVH.cu", "TreeCollapser.cu"]
REF_HOST = ["LBVHBuilder.cpp", "AgglomerativeTreeletOptimizer.cpp", "AgglomerativeScheduler.cpp",
            "TRBVHOptimizer.cpp", "TRBVHScheduler.cpp", "BVHTreeCollapser.cpp", "BVHTreeInstanceManager.cpp",
            "SoABVHTree.cpp", "BVHCollapsedTree.cpp", "SceneWrapper.cpp", "CudaTimer.cpp"]
OWN = HERE / "ref_cpu"
HOST_LIB = REF_OUT / "libbvhrt_ref_host.so"

# Places where the reference relies on the pre-Volta lock-step warp: a lane
# reads what other lanes of its warp wrote with no collective in between.  The
# host model runs lanes one after another between collectives, so a warp sync
# makes that ordering explicit there (file, anchor regex, text inserted after
# the anchor).
#   * AgglomerativeTreelet.cu findMinimumDistance: every lane scans the
#     distance matrix that all lanes filled just before, in
#     calculateDistancesMatrix (its last stores follow its last shuffle) or in
#     updateDistancesMatrix (stores after its shuffles).
#   * AgglomerativeTreelet.cu updateTreelet: every lane evaluates
#     treeletLeavesAreas[1] < nodesSah[root] and lane 1 then stores the
#     root's new nodesSah; in lock-step all lanes compare before that store,
#     so the comparison is taken, then the warp syncs, then it branches.
#   * TRBVH.cu updateTreelet, the treelet rewrite's work stack: every lane
#     reads stackSize (the loop condition, then lastStackSize) before lane 0
#     clears it, and every lane pushes its left child (atomicAdd on
#     currentInternalNode and stackSize, in lane order) before any lane
#     pushes its right child.  Warp syncs go before the loop condition, after
#     the lastStackSize read and before the right-child block.
LOCKSTEP_SYNCS = [
    ("AgglomerativeTreelet.cu", r"void\s+findMinimumDistance\s*\([^)]*\)\s*\{", " SIMT_WARP_SYNC(1);"),
    ("TRBVH.cu", r"int\s+lastStackSize\s*=\s*stackSize\[globalWarpIndex\]\s*;", " SIMT_WARP_SYNC(4);"),
]
# (file, anchor regex, replacement) for the comparison above.
LOCKSTEP_REWRITES = [
    ("AgglomerativeTreelet.cu",
     r"if\s*\(\s*treeletLeavesAreas\[1\]\s*<\s*nodesSah\[treeletInternalNodes\[0\]\]\s*\)",
     "const bool simtAccept = treeletLeavesAreas[1] < nodesSah[treeletInternalNodes[0]]; SIMT_WARP_SYNC(2); "
     "if (simtAccept)"),
    ("TRBVH.cu", r"while\s*\(\s*stackSize\[globalWarpIndex\]\s*>\s*0\s*\)",
     "while ((SIMT_WARP_SYNC(3), stackSize[globalWarpIndex] > 0))"),
    ("TRBVH.cu", r"if\s*\(\s*__popc\(partitionComplement\)\s*>\s*1\s*\)",
     "SIMT_WARP_SYNC(5); if (__popc(partitionComplement) > 1)"),
]
# Translation units whose code must keep source order in its layout: the host
# model orders divergent collectives by code address (TRBVH.cu calls
# __shfl_down inside a branch that some lanes skip, in processSubsets).
SOURCE_ORDER = {"TRBVH.cu"}


def _matching(text: str, i: int, open_ch: str, close_ch: str) -> int:
    """Index just past the bracket that closes the one at text[i]."""
    depth = 0
    for j in range(i, len(text)):
        if text[j] == open_ch:
            depth += 1
        elif text[j] == close_ch:
            depth -= 1
            if depth == 0:
                return j + 1
    raise ValueError(f"unbalanced {open_ch}{close_ch} at {i}")


def cuda_source_for_host(text: str, name: str) -> str:
    """The reference's CUDA source with its two constructs that C++ lacks
    rewritten for the host model: kernel<<<cfg>>>(args) becomes
    ::simt::run(::simt::Launch(cfg), [=]() { kernel(args); }), and
    extern __shared__ T a[] becomes a pointer to the launch's dynamic shared
    buffer.  Line breaks are kept, so diagnostics keep the reference's lines."""
    import re
    # Some launches are written "<< <cfg >> >(".
    text = re.sub(r"<<\s+<", "<<<", text)
    text = re.sub(r">>\s+>\s*\(", ">>>(", text)
    text = re.sub(r"extern\s+__shared__\s+([\w:]+)\s+(\w+)\s*\[\s*\]\s*;",
                  r"\1* \2 = reinterpret_cast<\1*>(::simt::dynamic_shared());", text)
    out = []
    pos = 0
    while True:
        k = text.find("<<<", pos)
        if k < 0:
            break
        # kernel expression: identifier, optionally with template arguments
        e = k
        while text[e - 1].isspace():
            e -= 1
        b = e
        if text[b - 1] == ">":
            depth = 0
            while True:
                b -= 1
                if text[b] == ">":
                    depth += 1
                elif text[b] == "<":
                    depth -= 1
                    if depth == 0:
                        break
        while text[b - 1].isalnum() or text[b - 1] in "_:":
            b -= 1
        kernel = text[b:e]
        c_end = text.find(">>>", k)
        cfg = text[k + 3:c_end]
        a = c_end + 3
        while text[a].isspace():
            a += 1
        assert text[a] == "(", f"{name}: kernel launch without arguments at {a}"
        a_end = _matching(text, a, "(", ")")
        args = text[a:a_end]
        out.append(text[pos:b])
        out.append(f"::simt::run(::simt::Launch({cfg}), [=]() {{ {kernel}{args}; }})")
        pos = a_end
    out.append(text[pos:])
    text = "".join(out)
    for fname, anchor, insert in LOCKSTEP_SYNCS:
        if fname == name:
            text, count = re.subn(anchor, lambda m: m.group(0) + insert, text, count=1)
            assert count == 1, f"{name}: lock-step anchor not found"
    for fname, anchor, replacement in LOCKSTEP_REWRITES:
        if fname == name:
            text, count = re.subn(anchor, lambda m: replacement, text, count=1)
            assert count == 1, f"{name}: lock-step anchor not found"
    return text


def build_reference_host() -> Path | None:
    """Compile the reference's BVHRT-Core sources, in place, for the host
    execution model into oracle/_ref/libbvhrt_ref_host.so."""
    root = reference_root()
    if root is None:
        return None
    src = root / "BVHRT-Core" / "src"
    own = sorted(OWN.glob("*.cpp")) + sorted(OWN.glob("*.h")) + sorted((OWN / "include").glob("*.h"))
    inputs = [src / f for f in REF_KERNELS + REF_HOST] + own + [Path(__file__)]
    if HOST_LIB.exists() and HOST_LIB.stat().st_mtime >= max(p.stat().st_mtime for p in inputs):
        return HOST_LIB
    REF_OUT.mkdir(exist_ok=True)
    objdir = REF_OUT / "obj_host"
    objdir.mkdir(exist_ok=True)
    base = ["g++", "-std=c++17", "-O2", "-fno-omit-frame-pointer", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
            "-fpermissive", "-w", "-I", str(OWN / "include"), "-I", str(OWN), "-I", str(src)]
    jobs = []
    objs = []
    for f in REF_KERNELS:
        o = objdir / (f + ".o")
        objs.append(o)
        text = cuda_source_for_host((src / f).read_text(errors="replace"), f)
        text = f'#line 1 "{src / f}"\n' + text
        opt = ["-O0"] if f in SOURCE_ORDER else []
        jobs.append((base + opt + ["-D__CUDA_ARCH__=350", "-x", "c++", "-c", "-", "-o", str(o)], text))
    for f in REF_HOST:
        o = objdir / (f + ".o")
        objs.append(o)
        jobs.append((base + ["-x", "c++", "-c", str(src / f), "-o", str(o)], None))
    for p in sorted(OWN.glob("*.cpp")):
        o = objdir / (p.name + ".o")
        objs.append(o)
        jobs.append((base + ["-c", str(p), "-o", str(o)], None))
    import concurrent.futures as cf
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        futs = [ex.submit(_run, cmd, input=stdin) if stdin is not None else ex.submit(_run, cmd) for cmd, stdin in jobs]
        for f in futs:
            f.result()
    _run(["g++", "-shared", "-o", str(HOST_LIB), *map(str, objs)])
    return HOST_LIB


def build_all() -> None:
    build_oracle()
    build_reference_host()


if __name__ == "__main__":
    build_all()
    print("oracle built")
