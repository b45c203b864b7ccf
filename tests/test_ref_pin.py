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


@pytest.mark.parametrize("msaa,lens", [(4, None), (8, (0.05, 6.0))])
def test_textured_shading_equals_reference_build(oracle, msaa, lens):
    """ShadeMSAA's texture coordinates and derivatives (RC/resolve.cu:230-270) and GGXShade's
    texture reads (RC/shading.h:84-161), pinhole and thin lens: with a sampler whose value depends
    on every bit of the query, the oracle's colours equal the reference's own shading code."""
    ref = pyoracle.Reference()
    sc = scenes.make_scene(12, 150, 23)
    v, t, n = ref.generate_topology(sc)
    sc.verts, sc.tri_shade, sc.nodes = v, t, n
    sc = scenes.with_textures(sc, 5, seed=3)
    w, h = 80, 64
    smp = scenes.barrel_samples(w, h)
    xf = scenes.camera_transform(eye=(1.2, 1.8, 8.0), target=(0.0, 0.1, -1.0))
    vp = scenes.viewport_for(w, h)
    kw = dict(fp_mode=_abi.HVVR_FP_STRICT, threads=4, lens=lens or (0.0, 1.0), textures=5, sampler=oracle.hash_sampler,
              want=("hits", "colors"))
    a = oracle.render(sc, smp, xf, vp, w, h, msaa, **kw)
    b = ref.render(sc, smp, xf, vp, w, h, msaa, **kw)
    n = len(smp)
    assert np.array_equal(a.hit_ids[:n], b.hit_ids[:n])
    assert np.array_equal(a.colors[:n], b.colors[:n])
    # the texture reads change the picture
    plain = oracle.render(sc, smp, xf, vp, w, h, msaa, **dict(kw, textures=0))
    assert (plain.colors[:n] != a.colors[:n]).mean() > 0.2
