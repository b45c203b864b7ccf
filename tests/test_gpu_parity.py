"""CUDA path vs the CPU oracle, through the C ABI, on seeded scenes.

Bit-exact: refit BVH, precomputed triangles, block cull stacks, per-tile triangle lists,
per-subsample hit triangle IDs, the compressed G-buffer pairs and depth (same operation
order in both). Colours: within 1 LSB per channel (powf and the truncating 8-bit
conversion may differ by one unit between the device and host math libraries).
"""
import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import scenes

from helpers import list_mismatch, render_gpu, render_oracle, scene

pytestmark = pytest.mark.gpu


def _compare(cam, rc, fo, msaa):
    nodes = rc.scene_nodes()
    assert np.array_equal(nodes.view(np.uint8), fo.nodes.view(np.uint8)), "refit BVH differs"
    assert np.array_equal(rc.scene_triangles().view(np.uint32), fo.tris.view(np.uint32)), "triangles differ"
    sizes, entries = cam.block_stacks()
    assert np.array_equal(sizes, fo.block_sizes)
    assert np.array_equal(entries, fo.block_entries)
    counts, idx = cam.tile_lists()
    assert list_mismatch(counts, idx, fo.tile_counts, fo.tile_indices) == 0
    ids, depth = cam.hits()
    assert np.array_equal(ids, fo.hit_ids), "hit IDs differ at %d subsamples" % int((ids != fo.hit_ids).sum())
    assert np.array_equal(depth.view(np.uint32), fo.depth.view(np.uint32)), "depth differs"
    n, tri, mask = cam.gbuffer()
    assert np.array_equal(n, fo.gb_n) and np.array_equal(tri, fo.gb_tri) and np.array_equal(mask, fo.gb_mask)
    col = cam.sample_colors()
    d = np.abs(col.view(np.uint8).astype(np.int32) - fo.colors.view(np.uint8).astype(np.int32))
    assert d.max() <= 1, "colour differs by %d LSB" % d.max()
    return d


@pytest.mark.parametrize("fp_mode", [hv.HVVR_FP_FMA, hv.HVVR_FP_STRICT])
def test_c1_grid_msaa1(oracle, fp_mode):
    sc = scene("c1")
    w, h = 640, 480
    smp = scenes.grid_samples(w, h)
    rc, cam = render_gpu(sc, smp, w, h, 1, fp_mode=fp_mode)
    fo = render_oracle(oracle, sc, smp, w, h, 1, fp_mode=fp_mode)
    _compare(cam, rc, fo, 1)
    img = cam.image
    diff = np.abs(img.view(np.uint8).astype(np.int32) - fo.image.view(np.uint8).astype(np.int32))
    assert diff.max() <= 1
    assert np.array_equal(cam.sample_remap(), fo.remap)
    assert np.array_equal(cam.beams().view(np.uint32), fo.beams.view(np.uint32))
    rc.close()


@pytest.mark.parametrize("msaa", [2, 4, 8, 16, 32])
def test_small_barrel_msaa(oracle, msaa):
    sc = scene("small")
    w, h = 160, 176
    smp = scenes.barrel_samples(w, h)
    rc, cam = render_gpu(sc, smp, w, h, msaa)
    fo = render_oracle(oracle, sc, smp, w, h, msaa)
    _compare(cam, rc, fo, msaa)
    rc.close()


def test_c1_barrel_msaa8_offaxis(oracle):
    sc = scene("c1")
    w, h = 320, 352
    smp = scenes.barrel_samples(w, h)
    xf = scenes.camera_transform(eye=(3.0, 1.2, 6.0), target=(-2.0, 0.3, -1.0))
    rc, cam = render_gpu(sc, smp, w, h, 8, cam_xf=xf)
    fo = render_oracle(oracle, sc, smp, w, h, 8, cam_xf=xf)
    _compare(cam, rc, fo, 8)
    rc.close()


def test_c1_frame_sequence_two_cameras(oracle):
    """Frames after the first schedule tiles by the previous frame's traversal cost and cull
    the slowest ones on a second stream; two cameras render concurrently. Every frame of a
    moving camera pair must still match the oracle exactly."""
    sc = scene("c1")
    w, h = 320, 288
    smp = scenes.barrel_samples(w, h)
    rc = hv.Raycaster()
    rc.create_model(sc)
    for l in sc.lights:
        rc.create_light(l)
    cams = []
    for _ in range(2):
        cam = rc.create_camera(scenes.viewport_for(w, h))
        cam.set_render_target(w, h)
        cam.set_samples(smp, 1)
        cam.set_msaa(4)
        cam.set_capture(hv.HVVR_CAPTURE_HITS)
        cams.append(cam)
    path = [((0.0, 2.0, 10.0), (0.0, 0.0, 0.0)), ((2.5, 1.0, 7.0), (-1.0, 0.5, 0.0)), ((-3.0, 3.0, 8.0), (1.0, 0.0, -2.0))]
    for frame, (eye, target) in enumerate(path):
        xfs = []
        for k, cam in enumerate(cams):
            xf = scenes.camera_transform(eye=(eye[0] + 0.3 * k, eye[1], eye[2]), target=target)
            cam.set_camera_to_world(xf)
            xfs.append(xf)
        rc.render()
        for cam, xf in zip(cams, xfs):
            fo = render_oracle(oracle, sc, smp, w, h, 4, cam_xf=xf)
            _compare(cam, rc, fo, 4)
    rc.close()


@pytest.mark.parametrize("msaa,fp_mode", [(1, hv.HVVR_FP_FMA), (4, hv.HVVR_FP_FMA), (8, hv.HVVR_FP_STRICT),
                                          (16, hv.HVVR_FP_FMA)])
def test_thin_lens_depth_of_field(oracle, msaa, fp_mode):
    """Thin-lens depth of field (the reference's IntersectTriangleThreadDoF path with its
    lens-position table indexed by the occupied-tile rank), two frames so the second one
    culls its slowest tiles first."""
    sc = scene("small")
    w, h = 160, 176
    smp = scenes.barrel_samples(w, h)
    xf = scenes.camera_transform(eye=(1.0, 2.2, 8.5), target=(0.0, 0.0, -1.0))
    lens = (0.08, 7.5)
    rc, cam = render_gpu(sc, smp, w, h, msaa, cam_xf=xf, fp_mode=fp_mode, lens=lens)
    fo = render_oracle(oracle, sc, smp, w, h, msaa, cam_xf=xf, fp_mode=fp_mode, lens=lens)
    _compare(cam, rc, fo, msaa)
    rc.render()
    _compare(cam, rc, fo, msaa)
    pin = render_oracle(oracle, sc, smp, w, h, msaa, cam_xf=xf, fp_mode=fp_mode)
    assert (fo.hit_ids != pin.hit_ids).any(), "the lens did not change the hits"
    rc.close()


@pytest.mark.skipif(not __import__("pyoracle").ReferenceGpu.available(), reason="oracle/_ref GPU library not built")
@pytest.mark.parametrize("name,w,h,msaa,kind", [("c1", 640, 480, 1, "grid"), ("c1", 640, 480, 4, "barrel"),
                                               ("c1", 640, 480, 8, "barrel"), ("c1", 320, 240, 16, "grid"),
                                               ("small", 256, 192, 32, "barrel")])
def test_against_reference_kernels(name, w, h, msaa, kind):
    """Hit IDs, coverage masks and colours against the reference's own IntersectKernel and
    ResolveKernel built for this GPU (oracle/refshim/ref_gpu_intersect.cu), fed the reference
    host code's beams, world tile frusta and tile lists: the compressed G-buffer (triangle, mask)
    pairs equal on every sample of every occupied tile but at most one, and colours within 1 LSB
    elsewhere. The reference's kernels are built with fast math (nvcc contracts their products
    into FMAs where it chooses); on three of these cases one subsample on an edge shared by two
    triangles resolves to the other triangle - C1 barrel MSAA 4 sample 217585 subsample 3, C1 barrel
    MSAA 8 sample 235826 subsample 0, the small scene MSAA 32 sample 41379 subsample 7 - in both of
    this library's FP modes."""
    import pyoracle
    from hvvr_b200 import scenes as sc_mod
    refg, refh = pyoracle.ReferenceGpu(), pyoracle.Reference()
    sc = scene(name)
    smp = sc_mod.grid_samples(w, h) if kind == "grid" else sc_mod.barrel_samples(w, h)
    xf = sc_mod.camera_transform()
    fr = refh.render(sc, smp, xf, sc_mod.viewport_for(w, h), w, h, msaa, fp_mode=hv.HVVR_FP_STRICT, threads=8,
                     want=("beams", "tile_frusta", "lists", "scene", "gbuffer", "colors"))
    r = refg.intersect_resolve(msaa, fr, sc, xf)
    n = len(smp)
    occupied = np.nonzero(np.repeat(fr.tile_counts > 0, 128)[:n])[0]
    for mode in (hv.HVVR_FP_FMA, hv.HVVR_FP_STRICT):
        rc, cam = render_gpu(sc, smp, w, h, msaa, cam_xf=xf, fp_mode=mode)
        gn, gt, gm = cam.gbuffer()
        col = cam.sample_colors()
        rc.close()
        bad = [s for s in occupied if not (np.array_equal(gt[s, :gn[s]], r["gb_tri"][s, :gn[s]]) and
                                            np.array_equal(gm[s, :gn[s]], r["gb_mask"][s, :gn[s]]))]
        assert len(bad) <= 1, (mode, bad[:8])
        keep = np.ones(n, bool)
        keep[bad] = False
        d = np.abs(col[:n].view(np.uint8).astype(np.int32) - r["colors"][:n].view(np.uint8).astype(np.int32))
        assert d.reshape(n, 4)[keep].max() <= 1, (mode, int(d.reshape(n, 4)[keep].max()))


def _split_samples(w, h, split, seed):
    """split copies of a jittered grid, each copy jittered again (one per colour channel)"""
    rng = np.random.default_rng(seed)
    base = scenes.grid_samples(w, h)
    base["position"] += rng.uniform(-0.4, 0.4, (len(base), 2)).astype(np.float32) / np.array([w, h], np.float32)
    smp = np.repeat(base, split)
    smp["position"] += rng.uniform(-0.1, 0.1, (len(smp), 2)).astype(np.float32) / np.array([w, h], np.float32)
    return smp


@pytest.mark.parametrize("split", [2, 3])
def test_split_color_images_match_oracle(oracle, split):
    """Split-colour sample sets (Camera::setSamples with splitColorSamples 2 or 3; the remap of
    RC/remap.cu:35-124 packs the channels of 2 (pentile) or 3 samples into one pixel): hits, colours
    and the remapped image against the oracle."""
    sc = scene("small")
    w, h = 200, 160
    smp = _split_samples(w, h, split, 40 + split)
    rc, cam = render_gpu(sc, smp, w, h, 4, split=split)
    fo = render_oracle(oracle, sc, smp, w, h, 4, split=split)
    _compare(cam, rc, fo, 4)
    assert np.array_equal(cam.sample_remap(split), fo.remap)
    img = cam.image
    d = np.abs(img.view(np.uint8).astype(np.int32) - fo.image.view(np.uint8).astype(np.int32))
    assert d.max() <= 1 and (img != 0).any()
    rc.close()


def test_five_models_under_root_fixup_nodes(oracle):
    """Five models in one raycaster, each with its own transform: Raycaster::buildScene merges them
    under two levels of root fix-up nodes (RC/scene_update.cpp:22-143); the merged BVH after refit,
    the triangles, the lists, hits and colours must equal the oracle's merge of the same models."""
    parts = [scenes.make_scene(10, 60, seed=30 + k) for k in range(5)]
    for p in parts:
        hv.generate_topology(p)
    xfs = []
    for k in range(5):
        a = 0.3 * k
        rot = (0.0, float(np.sin(a / 2)), 0.0, float(np.cos(a / 2)))
        xfs.append(_abi_transform(rot, (-8.0 + 4.0 * k, 0.2 * k, -2.0 * (k % 2)), 0.6 + 0.1 * k))
    rc = hv.Raycaster()
    for p, xf in zip(parts, xfs):
        m = rc.create_model(p)
        m.set_transform(xf)
    for l in parts[0].lights:
        rc.create_light(l)
    w, h = 320, 240
    smp = scenes.barrel_samples(w, h)
    cam_xf = scenes.camera_transform(eye=(0.0, 6.0, 14.0), target=(0.0, 0.0, 0.0))
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h)
    cam.set_samples(smp)
    cam.set_camera_to_world(cam_xf)
    cam.set_msaa(4)
    cam.set_capture(hv.HVVR_CAPTURE_HITS)
    rc.render()
    fo = oracle.render(parts, smp, cam_xf, scenes.viewport_for(w, h), w, h, 4, model_xf=xfs)
    assert len(rc.scene_nodes()) == sum(len(p.nodes) for p in parts) + 2
    _compare(cam, rc, fo, 4)
    ids, _ = cam.hits()
    tri_base = np.cumsum([0] + [len(p.tri_shade) for p in parts])
    hit_models = set(np.searchsorted(tri_base, ids[ids != 0xFFFFFFFF], side="right") - 1)
    assert len(hit_models) >= 3, hit_models
    rc.close()


def _empty_scene(like):
    """A model with no triangles, vertices or materials (empty MeshData), with the lights of `like`."""
    return scenes.Scene(like.verts[:0].copy(), like.tri_shade[:0].copy(), like.materials[:0].copy(), like.lights)


def test_empty_models(oracle):
    """Models without triangles: a raycaster whose only model is empty renders the background
    (every sample 0xFF000000, every subsample a miss, status OK), and an empty model among others
    takes no child slot of the root fix-up nodes, so the frame equals the oracle's merge of the
    non-empty models."""
    small = scene("small")
    w, h = 160, 176
    smp = scenes.barrel_samples(w, h)
    xf = scenes.camera_transform(eye=(1.0, 2.5, 9.0), target=(0.0, 0.0, 0.0))
    rc = hv.Raycaster()
    rc.create_model(_empty_scene(small))
    for l in small.lights:
        rc.create_light(l)
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h)
    cam.set_samples(smp)
    cam.set_camera_to_world(xf)
    cam.set_msaa(4)
    cam.set_capture(hv.HVVR_CAPTURE_HITS)
    rc.render()
    ids, depth = cam.hits()
    assert (ids == 0xFFFFFFFF).all() and np.isinf(depth).all()
    assert (cam.sample_colors() == 0xFF000000).all()
    mapped = cam.sample_remap() >= 0
    assert mapped.any() and (cam.image.reshape(-1)[mapped.reshape(-1)] == 0xFF000000).all()
    rc.close()
    parts = [scenes.make_scene(10, 60, seed=40 + k) for k in range(3)]
    for p in parts:
        hv.generate_topology(p)
    xfs = [_abi_transform((0.0, 0.0, 0.0, 1.0), (-5.0 + 5.0 * k, 0.0, 0.0), 0.7) for k in range(3)]
    rc = hv.Raycaster()
    for p, mxf in ((parts[0], xfs[0]), (_empty_scene(parts[0]), xfs[0]), (parts[1], xfs[1]),
                   (_empty_scene(parts[0]), xfs[0]), (parts[2], xfs[2])):
        rc.create_model(p).set_transform(mxf)
    for l in parts[0].lights:
        rc.create_light(l)
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h)
    cam.set_samples(smp)
    cam.set_camera_to_world(xf)
    cam.set_msaa(4)
    cam.set_capture(hv.HVVR_CAPTURE_HITS)
    rc.render()
    fo = oracle.render(parts, smp, xf, scenes.viewport_for(w, h), w, h, 4, model_xf=xfs)
    assert len(rc.scene_nodes()) == sum(len(p.nodes) for p in parts) + 1
    _compare(cam, rc, fo, 4)
    rc.close()


def _abi_transform(rot, trans, scale):
    from hvvr_b200 import _abi
    return _abi.transform(rot, trans, scale)


@pytest.mark.parametrize("msaa", [1, 4, 8, 16])
def test_rotated_grid_pattern_matches_oracle(oracle, msaa):
    """The rotated-grid (n-rooks) MSAA pattern, the library's named alternative to the reference's
    spiral: lists, hit IDs, depth and G-buffer pairs bit-exact vs the oracle with the same pattern,
    colours within 1 LSB; and the hits differ from the spiral's."""
    sc = scene("small")
    w, h = 160, 176
    smp = scenes.barrel_samples(w, h)
    rc = hv.Raycaster()
    rc.create_model(sc)
    for l in sc.lights:
        rc.create_light(l)
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h)
    cam.set_samples(smp)
    cam.set_camera_to_world(scenes.camera_transform())
    cam.set_msaa(msaa)
    cam.set_msaa_pattern(hv.HVVR_MSAA_ROTATED_GRID)
    cam.set_capture(hv.HVVR_CAPTURE_HITS)
    rc.render()
    fo = oracle.render(sc, smp, scenes.camera_transform(), scenes.viewport_for(w, h), w, h, msaa, msaa_pattern=1)
    _compare(cam, rc, fo, msaa)
    spiral = render_oracle(oracle, sc, smp, w, h, msaa)
    assert (spiral.hit_ids != fo.hit_ids).any()
    rc.close()
