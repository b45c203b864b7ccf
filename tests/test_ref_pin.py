"""The oracle against the reference's own sources compiled here, on fresh seeded inputs
(runs only where oracle/_ref was built, i.e. where the reference tree was available)."""
import numpy as np
import pytest

import pyoracle
import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

pytestmark = pytest.mark.skipif(not pyoracle.Reference.available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("seed,msaa", [(21, 2), (22, 16)])
def test_oracle_equals_reference_build(oracle, seed, msaa):
    ref = pyoracle.Reference()
    sc = scenes.make_scene(12, 150, seed)
    v, t, n = ref.generate_topology(sc)
    sc.verts, sc.tri_shade, sc.nodes = v, t, n
    w, h = 96, 80
    smp = scenes.barrel_samples(w, h)
    xf = scenes.camera_transform(eye=(1.0 + seed * 0.1, 1.8, 8.0), target=(0.0, 0.1, -1.0))
    vp = scenes.viewport_for(w, h)
    a = oracle.render(sc, smp, xf, vp, w, h, msaa, fp_mode=_abi.HVVR_FP_STRICT, threads=4)
    b = ref.render(sc, smp, xf, vp, w, h, msaa, fp_mode=_abi.HVVR_FP_STRICT, threads=4)
    for field in ("nodes", "block_sizes", "block_entries", "tile_counts", "tile_indices", "remap"):
        assert np.array_equal(getattr(a, field), getattr(b, field)), field
    n = len(smp)  # the reference leaves padding samples past the last valid one uninitialised
    for field in ("hit_ids", "gb_n", "gb_tri", "gb_mask", "colors"):
        assert np.array_equal(getattr(a, field)[:n], getattr(b, field)[:n]), field
    assert np.array_equal(a.depth.view(np.uint32)[:n], b.depth.view(np.uint32)[:n])
    assert np.array_equal(a.beams.view(np.uint32)[:n], b.beams.view(np.uint32)[:n])
