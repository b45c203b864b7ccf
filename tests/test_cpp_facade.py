"""The C++ facade (include/hvvr.hpp): a C++ program written like the reference's sample viewer
(Raycaster / Camera / Model / Light with the reference's names) is compiled against the header and
the library and run. On the CPU it must report the missing device as an hvvr::Error (no crash, no
exit from inside the library); on the GPU its image must equal the Python binding's render of the
same scene, pose and samples bit for bit."""
import os
import subprocess

import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

from conftest import ROOT, have_gpu

SRC = os.path.join(ROOT, "tests", "cpp", "facade_render.cpp")
LIBDIR = os.path.join(ROOT, "hvvr_b200", "_lib")


def _build(tmp_path):
    exe = str(tmp_path / "facade_render")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"), SRC,
           "-L" + LIBDIR, "-lhvvr_b200", "-Wl,-rpath," + LIBDIR, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def _case(tmp_path, w=160, h=120, msaa=4):
    sc = scenes.make_scene(12, 80, seed=17)
    smp = scenes.grid_samples(w, h)
    model_xf = _abi.transform((0.0, 0.2588190, 0.0, 0.9659258), (0.5, -0.2, 0.0), 0.9)
    cam_xf = scenes.camera_transform(eye=(1.0, 2.5, 9.0), target=(0.0, 0.0, 0.0))
    path = tmp_path / "scene.in"
    with open(path, "wb") as f:
        f.write(np.array([len(sc.verts), len(sc.tri_shade), len(sc.materials), len(sc.lights), len(smp), w, h, msaa],
                         np.uint32).tobytes())
        for a in (sc.verts, sc.tri_shade, sc.materials):
            f.write(np.ascontiguousarray(a).tobytes())
        for l in sc.lights:
            f.write(bytes(l))
        f.write(np.ascontiguousarray(smp).tobytes())
        f.write(bytes(model_xf))
        f.write(bytes(cam_xf))
    return sc, smp, model_xf, cam_xf, str(path)


@pytest.mark.skipif(have_gpu(), reason="checks the no-device error path")
def test_facade_compiles_and_reports_missing_device(tmp_path):
    exe = _build(tmp_path)
    _, _, _, _, inp = _case(tmp_path)
    r = subprocess.run([exe, inp, str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 3, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.startswith("hvvr::Error %d:" % _abi.HVVR_ERR_CUDA), r.stdout


@pytest.mark.gpu
def test_facade_image_equals_python_binding(tmp_path):
    exe = _build(tmp_path)
    w, h, msaa = 160, 120, 4
    sc, smp, model_xf, cam_xf, inp = _case(tmp_path, w, h, msaa)
    out = tmp_path / "out.bin"
    r = subprocess.run([exe, inp, str(out)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    img_cpp = np.fromfile(out, dtype=np.uint32).reshape(h, w)
    # the same scene through the Python binding: topology from the library's builder in both
    hv.generate_topology(sc)
    with hv.Raycaster() as rc:
        m = rc.create_model(sc)
        m.set_transform(model_xf)
        for l in sc.lights:
            rc.create_light(l)
        cam = rc.create_camera(scenes.viewport_for(w, h))
        cam.set_render_target(w, h)
        cam.set_samples(smp)
        cam.set_msaa(msaa)
        cam.set_camera_to_world(cam_xf)
        rc.render()
        rc.render()
        img_py = cam.image.copy()
    assert (img_py != 0).any()
    assert np.array_equal(img_cpp, img_py)
