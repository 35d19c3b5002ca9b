"""Cache keys (atr_cache_key, host-only): stable for equal scenes and build
parameters, different when any vertex byte or build parameter changes."""
import numpy as np

import atrbvh_b200 as ab
from tests._util import scene_case


def test_cache_key_is_stable_and_sensitive():
    v = scene_case("u4097")
    k = ab.cache_key(v)
    assert k == ab.cache_key(v.copy())
    w = v.copy()
    w[2049, 1, 2] = np.nextafter(w[2049, 1, 2], np.float32(2))
    assert ab.cache_key(w) != k
    variants = [dict(morton_bits=63), dict(optimizer=2), dict(treelet=7), dict(iterations=3), dict(ci=1.0),
                dict(ct=2.0), dict(max_leaf=4)]
    keys = {ab.cache_key(v, **kw) for kw in variants}
    assert len(keys) == len(variants) and k not in keys
    assert ab.cache_key(v[:4096]) != k
    big = ab.gen_scene(ab.SCENE_CLUSTERED, 1 << 18, 1)
    assert ab.cache_key(big) == ab.cache_key(big.copy())
