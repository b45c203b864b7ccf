"""Model transforms through the device scene update (vertex transform, triangle precompute, BVH
refit), against the reference's own scene update kernels (gpu_scene_state.cu, built for the GPU in
oracle/_ref) and against the oracle. In the fused mode (the default) positions, precomputed
triangles and refit bounds are bit-exact with the reference kernels, whose build contracts the
matrix product; in either mode renders of a transformed model match the oracle's."""
import math

import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

import pyoracle
from helpers import list_mismatch, scene

pytestmark = pytest.mark.gpu
needs_ref_gpu = pytest.mark.skipif(not pyoracle.ReferenceGpu.available(), reason="oracle/_ref GPU library not built")


def _rotation(angle_deg, axis):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    s = math.sin(math.radians(angle_deg) / 2)
    return (a[0] * s, a[1] * s, a[2] * s, math.cos(math.radians(angle_deg) / 2))


TRANSFORMS = {
    "identity": _abi.transform(),
    "translate": _abi.transform(translation=(0.37, -1.25, 2.5)),
    "rotate_scale": _abi.transform(rotation=_rotation(37.0, (0.3, 1.0, -0.2)), translation=(0.5, 0.1, -0.75),
                                   scale=1.3),
    "small_scale": _abi.transform(rotation=_rotation(-121.0, (1.0, 0.2, 0.4)), translation=(-2.0, 0.3, 1.0),
                                  scale=0.37),
}


def _first_diff(a, b):
    bad = np.flatnonzero(a != b)
    return "%d differ, first at %s" % (len(bad), bad[:4].tolist())


@needs_ref_gpu
@pytest.mark.parametrize("name", list(TRANSFORMS))
def test_scene_update_against_reference_kernels(name):
    sc = scene("small")
    rc = hv.Raycaster()
    model = rc.create_model(sc)
    xf = TRANSFORMS[name]
    model.set_transform(xf)
    cam = rc.create_camera(scenes.viewport_for(64, 48))
    cam.set_render_target(64, 48)
    cam.set_samples(scenes.grid_samples(64, 48))
    rc.render()
    rc.synchronize()
    nodes, tris = rc.scene_nodes(), rc.scene_triangles()
    rc.close()
    ref = pyoracle.ReferenceGpu()
    world, rtris, rnodes = ref.scene_update(nodes, sc.verts, np.zeros(len(sc.verts), np.uint32), [xf], sc.tri_shade)
    assert np.array_equal(tris.view(np.uint32), rtris.view(np.uint32)), "triangles: " + _first_diff(
        tris.view(np.uint32), rtris.view(np.uint32))
    assert np.array_equal(nodes.view(np.uint8), rnodes.view(np.uint8)), "nodes: " + _first_diff(
        nodes.view(np.uint32), rnodes.view(np.uint32))


@pytest.mark.parametrize("fp_mode", [hv.HVVR_FP_FMA, hv.HVVR_FP_STRICT], ids=["fma", "strict"])
@pytest.mark.parametrize("name", ["translate", "rotate_scale"])
def test_transformed_model_render_matches_oracle(oracle, name, fp_mode):
    sc = scene("small")
    w, h, msaa = 160, 120, 4
    xf = TRANSFORMS[name]
    cam_xf = scenes.camera_transform(eye=(0.4, 2.2, 9.5))
    rc = hv.Raycaster(fp_mode=fp_mode)
    model = rc.create_model(sc)
    for light in sc.lights:
        rc.create_light(light)
    model.set_transform(xf)
    smp = scenes.barrel_samples(w, h)
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h)
    cam.set_samples(smp)
    cam.set_camera_to_world(cam_xf)
    cam.set_msaa(msaa)
    cam.set_capture(hv.HVVR_CAPTURE_HITS)
    rc.render()
    rc.synchronize()
    fo = oracle.render(sc, smp, cam_xf, scenes.viewport_for(w, h), w, h, msaa, fp_mode=fp_mode, model_xf=xf)
    assert np.array_equal(rc.scene_nodes().view(np.uint8), fo.nodes.view(np.uint8)), "refit BVH differs"
    assert np.array_equal(rc.scene_triangles().view(np.uint32), fo.tris.view(np.uint32)), "triangles differ"
    counts, idx = cam.tile_lists()
    assert list_mismatch(counts, idx, fo.tile_counts, fo.tile_indices) == 0
    ids, depth = cam.hits()
    assert np.array_equal(ids, fo.hit_ids)
    assert np.array_equal(depth.view(np.uint32), fo.depth.view(np.uint32))
    img = cam.image.view(np.uint8).astype(np.int16)
    ref = fo.image.view(np.uint8).astype(np.int16)
    assert np.abs(img - ref).max() <= 1
    rc.close()
