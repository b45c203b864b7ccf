"""The oracle's scene update in the fused mode against the world-space positions the reference's
own SceneTransformVerticesKernel produced on a B200 for a rotated, translated and scaled model
(tests/golden/scene_update_rotate_scale.npz, written by tests/golden/make_scene_update_golden.py):
the precomputed triangles built from those positions are bit-exact with the oracle's. The strict
mode (the matrix product without contraction) differs, so the fixture tells the two apart."""
import os

import numpy as np

import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

from golden_io import GOLDEN_DIR
from helpers import scene


def _triangles_from(world, tri_shade):
    i = tri_shade["indices"]
    v0, v1, v2 = world[i[:, 0]], world[i[:, 1]], world[i[:, 2]]
    return np.concatenate([v0, v1 - v0, v2 - v0], axis=1).astype(np.float32)


def test_oracle_transform_matches_reference_kernel(oracle):
    g = np.load(os.path.join(GOLDEN_DIR, "scene_update_rotate_scale.npz"))
    sc = scene(str(g["scene"]))
    xf = _abi.Transform.from_buffer_copy(g["transform"].tobytes())
    expected = _triangles_from(g["world_pos"], sc.tri_shade)
    w, h = 32, 24
    got = {}
    for mode in (hv.HVVR_FP_FMA, hv.HVVR_FP_STRICT):
        fo = oracle.render(sc, scenes.grid_samples(w, h), scenes.camera_transform(), scenes.viewport_for(w, h), w, h,
                           1, fp_mode=mode, model_xf=xf, want=("scene",))
        got[mode] = fo.tris.view(np.uint32)
    assert np.array_equal(got[hv.HVVR_FP_FMA], expected.view(np.uint32))
    assert not np.array_equal(got[hv.HVVR_FP_STRICT], expected.view(np.uint32))
