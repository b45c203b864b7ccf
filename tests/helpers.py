"""Shared setup for the parity tests: scenes, cameras and running both paths."""
import numpy as np

import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

_SCENE_CACHE = {}


def scene(name):
    """Seeded scenes with topology built by the product's host BVH builder (cached)."""
    if name not in _SCENE_CACHE:
        if name == "c1":
            sc = scenes.scene_c1()
        elif name == "small":
            sc = scenes.make_scene(24, 300, seed=11)
        elif name == "c2":
            sc = scenes.scene_c2()
        else:
            raise KeyError(name)
        hv.generate_topology(sc)
        _SCENE_CACHE[name] = sc
    return _SCENE_CACHE[name]


def render_gpu(sc, samples, width, height, msaa, cam_xf=None, fp_mode=hv.HVVR_FP_FMA, capture=True, split=1,
               viewport=None, lens=None):
    rc = hv.Raycaster(fp_mode=fp_mode)
    rc.create_model(sc)
    for l in sc.lights:
        rc.create_light(l)
    cam = rc.create_camera(viewport or scenes.viewport_for(width, height))
    cam.set_render_target(width, height)
    cam.set_samples(samples, split)
    cam.set_camera_to_world(cam_xf or scenes.camera_transform())
    cam.set_msaa(msaa)
    if lens is not None:
        cam.set_lens(*lens)
    if capture:
        cam.set_capture(hv.HVVR_CAPTURE_HITS)
    rc.render()
    return rc, cam


def render_oracle(oracle, sc, samples, width, height, msaa, cam_xf=None, fp_mode=hv.HVVR_FP_FMA, split=1,
                  viewport=None, lens=None):
    return oracle.render(sc, samples, cam_xf or scenes.camera_transform(), viewport or scenes.viewport_for(width, height),
                         width, height, msaa, fp_mode=fp_mode, split=split, lens=lens or (0.0, 1.0))


def list_mismatch(counts_a, idx_a, counts_b, idx_b):
    """Number of tiles whose ordered triangle lists differ."""
    oa = np.concatenate([[0], np.cumsum(counts_a, dtype=np.int64)])
    ob = np.concatenate([[0], np.cumsum(counts_b, dtype=np.int64)])
    bad = 0
    for t in range(len(counts_a)):
        if counts_a[t] != counts_b[t] or not np.array_equal(idx_a[oa[t]:oa[t + 1]], idx_b[ob[t]:ob[t + 1]]):
            bad += 1
    return bad
