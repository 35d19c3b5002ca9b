"""The reference's caller sequence compiled in C++ against include/bvhrt.hpp
gives the same SAH values as the oracle."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

import atrbvh_b200 as ab
import oracle as O

ROOT = Path(__file__).resolve().parent.parent
pytestmark = pytest.mark.gpu


def test_renderer_call_sequence(tmp_path):
    exe = tmp_path / "renderer_sequence"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "renderer_sequence.cpp"), "-L", str(ROOT / "atrbvh_b200"),
                    "-latrbvh", f"-Wl,-rpath,{ROOT / 'atrbvh_b200'}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), "4096"], check=True, capture_output=True, text=True).stdout.split()
    vals = dict(zip(out[0::2], out[1::2]))
    v = ab.gen_scene(ab.SCENE_CLUSTERED, 4096, 2)
    mn, mx = O.scene_aabb(v)
    t, _, _ = O.build_lbvh(v, mn, mx)
    a = O.atrbvh(t, 9, 2)
    c = O.collapse(a)
    assert np.float32(float(vals["tree_sah"])) == np.float32(O.sah(a))
    assert np.float32(float(vals["collapse_sah"])) == np.float32(c.sah)
    leaves = O.leaf_lists(c.left, c.right, c.data, c.triangle_count, c.triangle_indices, len(v))
    assert int(vals["leaves"]) == len(leaves)
