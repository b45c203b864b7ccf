"""The sample hierarchy built on the device (clustering, tile and block frusta, beams, image
remap) against the host build of the same sample set: beams and remap bit-exact, and renders
through either setup give the same block stacks, tile lists, hit IDs and colours. Sets with two
samples at one position take the host build (std::sort decides their order)."""
import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import scenes

from helpers import list_mismatch, scene

pytestmark = pytest.mark.gpu


def _render(sc, smp, w, h, msaa, setup, split=1, lens=None):
    rc = hv.Raycaster(sample_setup=setup)
    rc.create_model(sc)
    for light in sc.lights:
        rc.create_light(light)
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h)
    cam.set_samples(smp, split)
    cam.set_camera_to_world(scenes.camera_transform(eye=(0.4, 2.2, 9.5)))
    cam.set_msaa(msaa)
    if lens is not None:
        cam.set_lens(*lens)
    cam.set_capture(hv.HVVR_CAPTURE_HITS)
    on_host = cam.prepare()
    rc.render()
    rc.synchronize()
    out = {"on_host": on_host, "beams": cam.beams(), "remap": cam.sample_remap(split), "stacks": cam.block_stacks(),
           "lists": cam.tile_lists(), "hits": cam.hits()[0], "colors": cam.sample_colors(), "image": cam.image.copy()}
    rc.close()
    return out


def _jittered(w, h, seed):
    rng = np.random.default_rng(seed)
    s = scenes.grid_samples(w, h)
    s["position"] += rng.uniform(-0.4, 0.4, (len(s), 2)).astype(np.float32) / np.array([w, h], np.float32)
    return s


@pytest.mark.parametrize("case", ["grid", "barrel", "jittered", "foveated", "split3", "lens"])
def test_device_setup_equals_host(case):
    sc = scene("small")
    w, h, split, lens, msaa = 320, 240, 1, None, 4
    if case == "grid":
        smp = scenes.grid_samples(w, h)
    elif case == "barrel":
        w, h = 540, 600
        smp = scenes.barrel_samples(w, h)
    elif case == "jittered":
        smp = _jittered(w, h, 5)
    elif case == "foveated":
        w, h = 360, 400
        smp = scenes.foveated_samples(60000, out_w=w, out_h=h)
    elif case == "split3":
        base = _jittered(w, h, 6)
        smp = np.repeat(base, 3)
        rng = np.random.default_rng(7)
        smp["position"] += rng.uniform(-0.1, 0.1, (len(smp), 2)).astype(np.float32) / np.array([w, h], np.float32)
        split = 3
    else:
        smp = scenes.barrel_samples(w, h)
        lens = (0.05, 6.0)
    a = _render(sc, smp, w, h, msaa, hv.HVVR_SETUP_DEVICE, split, lens)
    b = _render(sc, smp, w, h, msaa, hv.HVVR_SETUP_HOST, split, lens)
    assert not a["on_host"] and b["on_host"]
    assert np.array_equal(a["beams"].view(np.uint32), b["beams"].view(np.uint32))
    assert np.array_equal(a["remap"], b["remap"])
    assert np.array_equal(a["stacks"][0], b["stacks"][0]) and np.array_equal(a["stacks"][1], b["stacks"][1])
    ca, ia = a["lists"]
    cb, ib = b["lists"]
    assert list_mismatch(ca, ia, cb, ib) == 0
    for k in ("hits", "colors", "image"):
        assert np.array_equal(a[k], b[k]), k


def test_duplicate_positions_take_the_host_build():
    sc = scene("small")
    w, h = 160, 120
    smp = scenes.grid_samples(w, h)
    smp["position"][1000] = smp["position"][1001]  # two samples at one position
    a = _render(sc, smp, w, h, 4, hv.HVVR_SETUP_DEVICE)
    b = _render(sc, smp, w, h, 4, hv.HVVR_SETUP_HOST)
    assert a["on_host"] and b["on_host"]
    assert np.array_equal(a["remap"], b["remap"]) and np.array_equal(a["hits"], b["hits"])


def test_prepare_errors_and_reuse():
    """prepare() without samples is an error; a second prepare() reuses the setup; new samples
    rebuild it; the spherical mapping takes the host build."""
    rc = hv.Raycaster()
    cam = rc.create_camera(scenes.viewport_for(64, 48))
    cam.set_render_target(64, 48)
    with pytest.raises(hv.HvvrError):
        cam.prepare()
    cam.set_samples(scenes.grid_samples(64, 48))
    assert cam.prepare() is False
    b0 = cam.beams()
    assert cam.prepare() is False
    assert np.array_equal(cam.beams(), b0)
    cam.set_samples(scenes.barrel_samples(64, 48))
    assert cam.prepare() is False
    assert not np.array_equal(cam.beams(), b0)
    _check = hv._check
    _check(hv._lib.hvvr_camera_set_spherical_warp(cam.handle, hv.C.c_float(90.0), hv.C.c_float(70.0)))
    assert cam.prepare() is True
    rc.close()
