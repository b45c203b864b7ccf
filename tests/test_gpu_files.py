"""A scene written to and read back from the reference's binary scene format (with its prebuilt
topology), and a sample set through a sample file, render the same lists, hit IDs and image as
the original arrays."""
import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import scenes

from helpers import scene

pytestmark = pytest.mark.gpu


def _render(sc, lights, smp, w, h):
    rc = hv.Raycaster()
    rc.create_model(sc)
    for l in lights:
        rc.create_light(l)
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h)
    cam.set_samples(smp)
    cam.set_msaa(4)
    cam.set_capture(hv.HVVR_CAPTURE_HITS)
    cam.set_camera_to_world(scenes.camera_transform(eye=(0.5, 2.0, 9.0)))
    rc.render()
    rc.synchronize()
    out = (cam.tile_lists(), cam.hits()[0], cam.image.copy())
    rc.close()
    return out


def test_scene_and_sample_files_render_the_same(tmp_path):
    sc = scene("c1")
    w, h = 256, 192
    smp = scenes.barrel_samples(w, h)
    hv.save_scene_file(str(tmp_path / "c1.bin"), [sc], sc.lights)
    hv.save_samples(str(tmp_path / "c1.samples"), smp)
    f = hv.load_scene_file(str(tmp_path / "c1.bin"))
    (a_counts, a_idx), a_ids, a_img = _render(sc, sc.lights, smp, w, h)
    (b_counts, b_idx), b_ids, b_img = _render(f["meshes"][0], f["lights"], hv.load_samples(str(tmp_path / "c1.samples")),
                                              w, h)
    assert np.array_equal(a_counts, b_counts) and np.array_equal(a_idx, b_idx)
    assert np.array_equal(a_ids, b_ids) and np.array_equal(a_img, b_img)
