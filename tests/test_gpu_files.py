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


def test_textured_scene_file_through_create_objects(tmp_path):
    """A textured scene saved with its textures and loaded through create_objects (textures first,
    so material texture ids keep naming the file's textures) renders the same image as the
    scene built directly."""
    sc = scenes.with_textures(scene("small"), 3, seed=9)
    tex = [{"format": hv.HVVR_TEXTURE_RGBA8_UNORM_SRGB if i % 2 == 0 else hv.HVVR_TEXTURE_RGBA8_UNORM,
            "width": w, "height": h, "texels": scenes.texture_rgba8(w, h, seed=50 + i)}
           for i, (w, h) in enumerate([(64, 32), (16, 16), (33, 65)])]
    path = str(tmp_path / "tex.bin")
    hv.save_scene_file(path, [sc], sc.lights, textures=tex)
    w, h = 192, 128
    smp = scenes.barrel_samples(w, h)

    def render(build):
        rc = hv.Raycaster()
        build(rc)
        cam = rc.create_camera(scenes.viewport_for(w, h))
        cam.set_render_target(w, h)
        cam.set_samples(smp)
        cam.set_msaa(4)
        cam.set_camera_to_world(scenes.camera_transform(eye=(0.5, 2.0, 9.0)))
        rc.render()
        rc.synchronize()
        img = cam.image.copy()
        rc.close()
        return img

    def direct(rc):
        for t in tex:
            rc.create_texture(t["texels"], t["format"])
        rc.create_model(sc)
        for light in sc.lights:
            rc.create_light(light)

    a = render(direct)
    b = render(lambda rc: hv.create_objects(rc, hv.load_scene_file(path)))
    assert np.array_equal(a, b)
    plain = render(lambda rc: (rc.create_model(sc), [rc.create_light(x) for x in sc.lights]))
    assert (plain != a).mean() > 0.1
