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


def test_topology_builder_matches_reference_at_995k_triangles():
    """The product's BVH builder against the reference's GenerateTopology on the benchmarked
    995,072-triangle scene: nodes, triangle order and vertex order identical."""
    ref = pyoracle.Reference()
    a = scenes.scene_c2()
    v, t, n = ref.generate_topology(a)
    hv.generate_topology(a)
    assert len(a.tri_shade) == 995072
    assert np.array_equal(a.nodes.view(np.uint8), n.view(np.uint8))
    assert np.array_equal(a.tri_shade.view(np.uint8), t.view(np.uint8))
    assert np.array_equal(a.verts.view(np.uint8), v.view(np.uint8))


def test_oracle_equals_reference_build_on_benchmarked_eye(oracle):
    """The oracle against the reference build on the left eye of the benchmarked stereo frame
    (995,072 triangles, 1080x1200 barrel samples, 8x MSAA, STRICT): block stacks and per-tile
    lists over the whole frame, hits, depth, G-buffer pairs and colours over the valid samples."""
    from helpers import scene
    sc = scene("c2")
    w, h = 1080, 1200
    smp = scenes.barrel_samples(w, h)
    xf = scenes.stereo_eyes(0.064)[0]
    vp = scenes.viewport_for(w, h)
    want = ("lists", "hits", "colors", "blocks", "gbuffer")
    a = oracle.render(sc, smp, xf, vp, w, h, 8, fp_mode=_abi.HVVR_FP_STRICT, want=want)
    b = pyoracle.Reference().render(sc, smp, xf, vp, w, h, 8, fp_mode=_abi.HVVR_FP_STRICT, want=want)
    for field in ("block_sizes", "block_entries", "tile_counts", "tile_indices"):
        assert np.array_equal(getattr(a, field), getattr(b, field)), field
    n = len(smp)
    for field in ("hit_ids", "gb_n", "gb_tri", "gb_mask", "colors"):
        assert np.array_equal(getattr(a, field)[:n], getattr(b, field)[:n]), field
    assert np.array_equal(a.depth.view(np.uint32)[:n], b.depth.view(np.uint32)[:n])


def test_reference_session_frames_equal_single_renders():
    """The reference arm's per-frame path (scene and sample setup once, then frames with threaded
    traversal) gives the same colours and image as a whole single-frame render, frame after frame."""
    ref = pyoracle.Reference()
    sc = scenes.make_scene(12, 150, 24)
    v, t, n = ref.generate_topology(sc)
    sc.verts, sc.tri_shade, sc.nodes = v, t, n
    w, h = 96, 80
    smp = scenes.barrel_samples(w, h)
    vp = scenes.viewport_for(w, h)
    s = ref.session(sc, smp, vp, w, h, 4)
    for k in range(3):
        xf = scenes.camera_transform(eye=(0.5 * k, 1.8, 8.0), target=(0.0, 0.1, -1.0))
        img = s.frame(xf, threads=3).copy()
        one = ref.render(sc, smp, xf, vp, w, h, 4, fp_mode=_abi.HVVR_FP_STRICT, threads=2, want=("colors", "image"))
        assert np.array_equal(s.colors[:len(smp)], one.colors[:len(smp)])
        assert np.array_equal(img, one.image)
    s.close()
