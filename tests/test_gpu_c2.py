"""The benchmarked configuration itself against the oracle and the reference build.

Scene: the seeded 995,072-triangle scene (256x256-quad heightfield + 72,000 boxes). Views: a
stereo pair of 1080x1200 barrel-distorted sample sets (r' = r(1 + 0.22 r^2 + 0.24 r^4)), 64 mm
IPD, 8x MSAA, both eyes rendered as one frame by one raycaster, exactly as the benchmark renders
them. Two frames are compared: the first culls tiles in index order, the second in the previous
frame's cost order with the slowest eighth on a side stream.

Against the oracle (FMA mode, every sample of both eyes): block stacks, per-tile lists, hit
triangle IDs, depth and G-buffer pairs bit-exact; colours and images within 1 LSB per channel.
Against the reference's own sources compiled here (STRICT mode, left eye): the same, over valid
samples. FP32 depth against the oracle's FP64 ray-triangle solve: relative error below 1e-5.
"""
import os

import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import scenes

from helpers import list_mismatch, scene

pytestmark = pytest.mark.gpu

W, H, MSAA, IPD = 1080, 1200, 8, 0.064


def _stereo(sc, fp_mode):
    rc = hv.Raycaster(fp_mode=fp_mode, tri_index_capacity=128 << 20)
    rc.create_model(sc)
    for l in sc.lights:
        rc.create_light(l)
    smp = scenes.barrel_samples(W, H)
    cams = []
    for xf in scenes.stereo_eyes(IPD):
        cam = rc.create_camera(scenes.viewport_for(W, H))
        cam.set_render_target(W, H)
        cam.set_samples(smp)
        cam.set_camera_to_world(xf)
        cam.set_msaa(MSAA)
        cam.set_capture(hv.HVVR_CAPTURE_HITS)
        cams.append(cam)
    return rc, cams, smp


def _check(cam, fo, valid=None):
    n = valid if valid is not None else len(fo.hit_ids)
    sizes, entries = cam.block_stacks()
    assert np.array_equal(sizes, fo.block_sizes) and np.array_equal(entries, fo.block_entries), "block stacks differ"
    counts, idx = cam.tile_lists()
    bad = list_mismatch(counts, idx, fo.tile_counts, fo.tile_indices)
    assert bad == 0, "%d tile lists differ" % bad
    ids, depth = cam.hits()
    diff = int((ids[:n] != fo.hit_ids[:n]).sum())
    assert diff == 0, "hit IDs differ at %d subsamples" % diff
    assert np.array_equal(depth[:n].view(np.uint32), fo.depth[:n].view(np.uint32)), "depth differs"
    gn, gt, gm = cam.gbuffer()
    assert np.array_equal(gn[:n], fo.gb_n[:n]) and np.array_equal(gt[:n], fo.gb_tri[:n]) and \
        np.array_equal(gm[:n], fo.gb_mask[:n]), "G-buffer pairs differ"
    col = cam.sample_colors()
    d = np.abs(col[:n].view(np.uint8).astype(np.int32) - fo.colors[:n].view(np.uint8).astype(np.int32))
    assert d.max() <= 1, "colour differs by %d LSB" % d.max()
    return ids[:n], depth[:n]


def test_c2_stereo_frame_matches_oracle(oracle):
    sc = scene("c2")
    rc, cams, smp = _stereo(sc, hv.HVVR_FP_FMA)
    eyes = scenes.stereo_eyes(IPD)
    ref = [oracle.render(sc, smp, xf, scenes.viewport_for(W, H), W, H, MSAA, fp_mode=hv.HVVR_FP_FMA,
                         threads=os.cpu_count(), want=("lists", "hits", "colors", "image", "blocks", "gbuffer"))
           for xf in eyes]
    for frame in range(2):
        rc.render()
        for cam, fo in zip(cams, ref):
            ids, depth = _check(cam, fo)
            img = cam.image
            d = np.abs(img.view(np.uint8).astype(np.int32) - fo.image.view(np.uint8).astype(np.int32))
            assert d.max() <= 1, "image differs by %d LSB" % d.max()
    # FP32 depth against the FP64 solve of the same hits
    for fo in ref:
        hit = fo.hit_ids != 0xFFFFFFFF
        rel = np.abs(fo.depth[hit].astype(np.float64) - fo.depth64[hit]) / np.abs(fo.depth64[hit])
        assert hit.sum() > 10 ** 6 and rel.max() < 1e-5, rel.max()
    rc.close()


@pytest.mark.skipif(not __import__("pyoracle").Reference.available(), reason="oracle/_ref not built")
def test_c2_left_eye_strict_matches_reference_build():
    """STRICT mode against the reference's own traversal and intersect/shade code (oracle/_ref)
    on the left eye of the benchmarked frame, over the valid samples (the reference leaves the
    padding samples of the last block unwritten)."""
    import pyoracle
    sc = scene("c2")
    rc, cams, smp = _stereo(sc, hv.HVVR_FP_STRICT)
    rc.render()
    xf = scenes.stereo_eyes(IPD)[0]
    fr = pyoracle.Reference().render(sc, smp, xf, scenes.viewport_for(W, H), W, H, MSAA, fp_mode=hv.HVVR_FP_STRICT,
                                     threads=os.cpu_count(), want=("lists", "hits", "colors", "blocks", "gbuffer"))
    _check(cams[0], fr, valid=len(smp))
    rc.close()
