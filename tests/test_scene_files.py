"""Scene and sample files in the reference's binary formats: the library's writer and reader
against the reference's own model_import::saveBin / loadBin and saveSamples / loadSamples
(compiled in oracle/_ref), in both directions, byte for byte; malformed files are errors."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import pyoracle  # noqa: E402

from helpers import scene  # noqa: E402

needs_ref = pytest.mark.skipif(not pyoracle.Reference.available(), reason="oracle/_ref not built")


def _meshes():
    a = scene("small")
    b = scene("c1")
    b.transform = _abi.transform(rotation=(0.0, 0.38268343, 0.0, 0.92387953), translation=(1.0, -2.0, 3.5), scale=0.5)
    a.transform = _abi.transform()
    return [a, b], list(a.lights)


def _mesh_bytes(sc):
    nodes = sc.nodes if sc.nodes is not None else np.zeros(0, _abi.TOPO_DTYPE)
    return (bytes(sc.transform) + sc.verts.tobytes() + sc.tri_shade.tobytes() + nodes.tobytes() +
            sc.materials.tobytes())


def _ref():
    lib = pyoracle.Reference().lib
    lib.ref_bin_save.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                 C.c_uint32, C.c_uint32]
    lib.ref_bin_load.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p]
    lib.ref_samples_save.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32]
    lib.ref_samples_load.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32, C.c_void_p]
    return lib


@needs_ref
def test_library_scene_file_loads_in_reference(tmp_path):
    meshes, lights = _meshes()
    path = str(tmp_path / "lib.bin")
    hv.save_scene_file(path, meshes, lights)
    lib = _ref()
    counts = np.zeros(4, np.uint64)
    assert lib.ref_bin_load(path.encode(), counts.ctypes.data, None) == 0
    assert counts[:3].tolist() == [0, len(lights), len(meshes)]
    out = np.zeros(int(counts[3]), np.uint8)
    assert lib.ref_bin_load(path.encode(), counts.ctypes.data, out.ctypes.data) == 0
    want = b"".join(bytes(l) for l in lights) + b"".join(_mesh_bytes(m) for m in meshes)
    assert out.tobytes() == want


@needs_ref
def test_library_scene_file_with_textures_loads_in_reference(tmp_path):
    meshes, lights = _meshes()
    tex = [{"format": 1, "width": 7, "height": 5, "texels": scenes.texture_rgba8(7, 5, seed=2)},
           {"format": 4, "width": 3, "height": 2, "stride": 4,
            "texels": np.arange(4 * 2 * 4, dtype=np.float32)}]
    path = str(tmp_path / "lib_tex.bin")
    hv.save_scene_file(path, meshes, lights, textures=tex)
    lib = _ref()
    counts = np.zeros(4, np.uint64)
    assert lib.ref_bin_load(path.encode(), counts.ctypes.data, None) == 0
    assert counts[:3].tolist() == [2, len(lights), len(meshes)]
    out = np.zeros(int(counts[3]), np.uint8)
    assert lib.ref_bin_load(path.encode(), counts.ctypes.data, out.ctypes.data) == 0
    want = b""
    for t in tex:
        want += np.array([t["format"], t["width"], t["height"], t.get("stride", t["width"])], np.uint32).tobytes()
        want += np.ascontiguousarray(t["texels"]).tobytes()
    want += b"".join(bytes(l) for l in lights) + b"".join(_mesh_bytes(m) for m in meshes)
    assert out.tobytes() == want
    f = hv.load_scene_file(path)
    assert [(t["format"], t["width"], t["height"], t["stride"]) for t in f["textures"]] == [(1, 7, 5, 7), (4, 3, 2, 4)]
    assert f["textures"][1]["texels"].tobytes() == tex[1]["texels"].tobytes()


@needs_ref
def test_reference_scene_file_loads_in_library(tmp_path):
    meshes, lights = _meshes()
    path = str(tmp_path / "ref.bin")
    mds = (_abi.MeshData * len(meshes))()
    xfs = (_abi.Transform * len(meshes))()
    for i, m in enumerate(meshes):
        mds[i] = _abi.MeshData(_abi.ptr(m.verts), len(m.verts), _abi.ptr(m.tri_shade), len(m.tri_shade),
                               _abi.ptr(m.nodes), len(m.nodes), _abi.ptr(m.materials), len(m.materials))
        xfs[i] = m.transform
    ls = (_abi.LightUnion * len(lights))(*lights)
    texels = np.arange(5 * 3 * 4, dtype=np.uint8)
    assert _ref().ref_bin_save(path.encode(), mds, xfs, len(meshes), ls, len(lights), texels.ctypes.data, 5, 3) == 0
    f = hv.load_scene_file(path)
    assert len(f["meshes"]) == 2 and len(f["lights"]) == len(lights)
    assert [bytes(l) for l in f["lights"]] == [bytes(l) for l in lights]
    for got, want in zip(f["meshes"], meshes):
        assert _mesh_bytes(got) == _mesh_bytes(want)
    (t,) = f["textures"]
    assert (t["format"], t["width"], t["height"], t["stride"]) == (2, 5, 3, 5)
    assert np.array_equal(t["texels"], texels)


@needs_ref
def test_sample_files_both_ways(tmp_path):
    smp = scenes.barrel_samples(64, 48)
    lib = _ref()
    p1, p2 = str(tmp_path / "lib.samples"), str(tmp_path / "ref.samples")
    hv.save_samples(p1, smp)
    out = np.zeros(len(smp), _abi.SAMPLE_DTYPE)
    n = C.c_uint32(0)
    assert lib.ref_samples_load(p1.encode(), out.ctypes.data, len(out), C.byref(n)) == 0
    assert n.value == len(smp) and out.tobytes() == smp.tobytes()
    assert lib.ref_samples_save(p2.encode(), smp.ctypes.data, len(smp)) == 0
    assert hv.load_samples(p2).tobytes() == smp.tobytes()


def test_scene_file_round_trip_and_errors(tmp_path):
    meshes, lights = _meshes()
    path = str(tmp_path / "s.bin")
    hv.save_scene_file(path, meshes, lights)
    f = hv.load_scene_file(path)
    assert [_mesh_bytes(m) for m in f["meshes"]] == [_mesh_bytes(m) for m in meshes]
    raw = open(path, "rb").read()
    bad = tmp_path / "bad.bin"
    bad.write_bytes(raw[: len(raw) - 7])  # truncated
    with pytest.raises(hv.HvvrError, match="truncated"):
        hv.load_scene_file(str(bad))
    bad.write_bytes(b"\x02\x00\x00\x00" + raw[4:])  # version 2
    with pytest.raises(hv.HvvrError, match="version"):
        hv.load_scene_file(str(bad))
    with pytest.raises(hv.HvvrError, match="cannot open"):
        hv.load_scene_file(str(tmp_path / "missing.bin"))
    bad.write_bytes(b"\x00\x00\x00\x00" * 4)  # not a sample file
    with pytest.raises(hv.HvvrError, match="not a sample file"):
        hv.load_samples(str(bad))
