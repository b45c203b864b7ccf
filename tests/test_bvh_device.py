"""The device BVH build (hvvr_generate_topology_device, spec.bvh_build = HVVR_BVH_DEVICE): a linear
BVH built on the GPU. It has no counterpart in the reference, so it is pinned two ways: the GPU
build equals its CPU restatement (oracle_lbvh_build) node for node and triangle for triangle, and
the restatement is a valid BVH of the mesh (every triangle in exactly one leaf, leaf slots before
internal slots, child offsets forward) whose render equals the SAH topology's image; a raycaster
that builds its models' topology on the device renders exactly what the oracle renders on that
topology."""
import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

from helpers import list_mismatch, render_oracle, scene


def _check_structure(tris_in, tris, nodes):
    a = tris.view(np.uint32).reshape(-1, 4)
    b = tris_in.view(np.uint32).reshape(-1, 4)
    assert sorted(map(tuple, a)) == sorted(map(tuple, b))
    covered = np.zeros(len(tris), np.int32)
    for i, nd in enumerate(nodes):
        mask, data = int(nd["leaf_mask"]), nd["data"]
        seen_internal = False
        for k in range(4):
            if mask >> k & 1:
                assert not seen_internal, "leaf slot after an internal slot"
                lo, hi = int(data[k]), int(data[k + 1])
                assert lo <= hi <= len(tris)
                covered[lo:hi] += 1
            else:
                seen_internal = True
                c = i + int(data[1 + k])
                assert i < c < len(nodes)
    assert (covered == 1).all()


@pytest.mark.parametrize("args", [(1, 0, 3), (3, 0, 2), (24, 300, 11), (128, 2048, 1)])
def test_oracle_lbvh_is_a_valid_bvh_with_the_same_image(oracle, args):
    sc = scenes.make_scene(*args)
    tris, nodes = oracle.lbvh_build(sc)
    _check_structure(sc.tri_shade, tris, nodes)
    sah = scenes.Scene(sc.verts.copy(), sc.tri_shade.copy(), sc.materials, sc.lights)
    hv.generate_topology(sah)
    lb = scenes.Scene(sc.verts.copy(), tris, sc.materials, sc.lights)
    lb.nodes = nodes
    w, h = 160, 120
    smp = scenes.barrel_samples(w, h)
    a = render_oracle(oracle, sah, smp, w, h, 4)
    b = render_oracle(oracle, lb, smp, w, h, 4)
    assert (a.colors == b.colors).mean() > 0.999


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small", "c1", "c2"])
def test_device_build_equals_oracle(oracle, name):
    base = {"small": lambda: scenes.make_scene(24, 300, seed=11), "c1": scenes.scene_c1, "c2": scenes.scene_c2}[name]()
    ref_tris, ref_nodes = oracle.lbvh_build(base)
    dev = scenes.Scene(base.verts.copy(), base.tri_shade.copy(), base.materials, base.lights)
    hv.generate_topology_device(dev)
    assert np.array_equal(dev.nodes.view(np.uint32), ref_nodes.view(np.uint32))
    assert np.array_equal(dev.tri_shade.view(np.uint32), ref_tris.view(np.uint32))
    assert np.array_equal(dev.verts.view(np.uint32), base.verts.view(np.uint32))


@pytest.mark.gpu
def test_device_built_scene_renders_like_the_oracle(oracle):
    """A raycaster with bvh_build = HVVR_BVH_DEVICE builds its model's topology on the GPU; its
    lists, hits and colours equal the oracle's render of the same (device) topology."""
    sc = scenes.scene_c1()
    spec = _abi.Spec()
    hv.lib().hvvr_spec_default(spec)
    spec.bvh_build = _abi.HVVR_BVH_DEVICE
    w, h = 320, 240
    smp = scenes.barrel_samples(w, h)
    xf = scenes.camera_transform(eye=(2.0, 2.5, 9.0), target=(0.0, 0.0, 0.0))
    raw = scenes.Scene(sc.verts.copy(), sc.tri_shade.copy(), sc.materials, sc.lights)  # no topology
    with hv.Raycaster(spec=spec) as rc:
        rc.create_model(raw)
        for l in sc.lights:
            rc.create_light(l)
        cam = rc.create_camera(scenes.viewport_for(w, h))
        cam.set_render_target(w, h)
        cam.set_samples(smp)
        cam.set_msaa(8)
        cam.set_camera_to_world(xf)
        cam.set_capture(hv.HVVR_CAPTURE_HITS)
        rc.render()
        counts, idx = cam.tile_lists()
        ids, depth = cam.hits()
        col = cam.sample_colors()
    tris, nodes = oracle.lbvh_build(sc)
    lb = scenes.Scene(sc.verts.copy(), tris, sc.materials, sc.lights)
    lb.nodes = nodes
    fo = render_oracle(oracle, lb, smp, w, h, 8, cam_xf=xf)
    assert list_mismatch(counts, idx, fo.tile_counts, fo.tile_indices) == 0
    assert np.array_equal(ids, fo.hit_ids)
    assert np.array_equal(depth.view(np.uint32), fo.depth.view(np.uint32))
    d = np.abs(col.view(np.uint8).astype(np.int32) - fo.colors.view(np.uint8).astype(np.int32))
    assert d.max() <= 1
