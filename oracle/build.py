"""ORACLE -- test infrastructure only.

Builds the checker:
  oracle/liboracle.so   CPU restatement (atr_oracle.cpp) and the seeded
                        workload generators (workload_oracle.cpp), g++ -O2
                        -ffp-contract=off -fopenmp.

The reference's own sources are located through the ATRBVH_REFERENCE
environment variable (the root of the leonardo-domingues/atrbvh tree; default
/root/reference, where this build's container mounts it read-only).  Nothing
here runs the reference's CUDA kernels.
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
    srcs = [HERE / "atr_oracle.cpp", HERE / "workload_oracle.cpp"]
    if out.exists() and out.stat().st_mtime >= max(p.stat().st_mtime for p in srcs):
        return out
    _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
          "-shared", "-o", str(out), *map(str, srcs)])
    return out


def build_all() -> None:
    build_oracle()


if __name__ == "__main__":
    build_all()
    print("oracle built")
