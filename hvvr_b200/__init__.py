"""hvvr_b200 - B200-native primary-visibility-and-shading path with HVVR's interface.

Python mirror of the reference's Raycaster / Camera / Model / Light API over the C ABI in
include/hvvr_c.h (libhvvr_b200.so, built in-tree by ``make -C hvvr_b200/csrc``). There is
no CPU fallback: every entry point runs the CUDA library, and importing this package when
the library has not been built raises immediately.
"""
import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import (HVVR_CAPTURE_HITS, HVVR_FP_FMA, HVVR_FP_STRICT, HVVR_MEMORY_CPU, HVVR_MEMORY_CUDA,  # noqa: F401
                   HVVR_OK, HVVR_SETUP_DEVICE, HVVR_SETUP_HOST, HVVR_TEXTURE_R32_FLOAT, HVVR_TEXTURE_RGBA8_UNORM, HVVR_TEXTURE_RGBA8_UNORM_SRGB,
                   HVVR_TEXTURE_RGBA16_FLOAT, HVVR_TEXTURE_RGBA16_UNORM, HVVR_TEXTURE_RGBA32_FLOAT,
                   HVVR_TEXTURE_R11G11B10_FLOAT, HVVR_MSAA_SPIRAL, HVVR_MSAA_ROTATED_GRID, HVVR_BVH_HOST,
                   HVVR_BVH_DEVICE)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("HVVR_B200_LIB") or os.path.join(_HERE, "_lib", "libhvvr_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError("hvvr_b200: %s is not built; run `make -C hvvr_b200/csrc` (or __graft_entry__.build())" % LIB_PATH)

_lib = C.CDLL(LIB_PATH)
_vp = C.c_void_p
_u32 = C.c_uint32
_p = C.POINTER


def _sig(name, *args):
    f = getattr(_lib, name)
    f.argtypes = list(args)
    f.restype = C.c_int
    return f


_lib.hvvr_last_error.restype = C.c_char_p
_lib.hvvr_last_error.argtypes = []
_lib.hvvr_spec_default.argtypes = [_p(_abi.Spec)]
_lib.hvvr_spec_default.restype = None
_sig("hvvr_version")
_sig("hvvr_raycaster_create", _p(_abi.Spec), _p(_vp))
_sig("hvvr_raycaster_destroy", _vp)
_sig("hvvr_raycaster_set_scene_dirty", _vp)
_sig("hvvr_raycaster_render", _vp, C.c_double, _vp)
_sig("hvvr_raycaster_synchronize", _vp)
_sig("hvvr_model_create", _vp, _p(_abi.MeshData), _p(_vp))
_sig("hvvr_model_destroy", _vp, _vp)
_sig("hvvr_model_set_transform", _vp, _p(_abi.Transform))
_sig("hvvr_model_update_vertices", _vp, _vp, _u32)
_sig("hvvr_light_create", _vp, _p(_abi.LightUnion), _p(_vp))
_sig("hvvr_light_destroy", _vp, _vp)
_sig("hvvr_texture_create", _vp, _p(_abi.TextureData), _p(_vp))
_sig("hvvr_texture_destroy", _vp, _vp)
_sig("hvvr_texture_get_id", _vp, _p(_u32))
_sig("hvvr_texture_read_level", _vp, _u32, _vp, C.c_uint64, _p(_u32), _p(_u32))
_sig("hvvr_texture_sample", _vp, _u32, _vp, _vp)
_sig("hvvr_camera_create", _vp, _p(_abi.FloatRect), C.c_float, _p(_vp))
_sig("hvvr_camera_destroy", _vp, _vp)
_sig("hvvr_camera_set_enabled", _vp, C.c_int)
_sig("hvvr_camera_set_viewport", _vp, _p(_abi.FloatRect))
_sig("hvvr_camera_set_lens", _vp, _p(_abi.ThinLens))
_sig("hvvr_camera_set_aperture", _vp, C.c_float)
_sig("hvvr_camera_set_focal_depth", _vp, C.c_float)
_sig("hvvr_camera_set_eye_dir", _vp, _p(_abi.Vec3))
_sig("hvvr_camera_set_spherical_warp", _vp, C.c_float, C.c_float)
_sig("hvvr_camera_set_render_target", _vp, _p(_abi.ImageDesc))
_sig("hvvr_camera_set_samples", _vp, _vp, _u32, _u32)
_sig("hvvr_camera_set_camera_to_world", _vp, _p(_abi.Transform))
_sig("hvvr_camera_prepare", _vp, _p(_u32))
_sig("hvvr_camera_set_msaa", _vp, _u32)
_sig("hvvr_camera_set_msaa_pattern", _vp, _u32)
_sig("hvvr_camera_get_sample_count", _vp, _p(_u32))
_sig("hvvr_camera_set_capture", _vp, _u32)
_sig("hvvr_camera_get_layout", _vp, _p(_u32), _p(_u32), _p(_u32), _p(_u32))
_sig("hvvr_camera_read_tile_lists", _vp, _vp, _vp, C.c_uint64, _p(C.c_uint64))
_sig("hvvr_camera_read_block_stacks", _vp, _vp, _vp)
_sig("hvvr_camera_read_hits", _vp, _vp, _vp)
_sig("hvvr_camera_read_gbuffer", _vp, _vp, _vp, _vp)
_sig("hvvr_camera_read_sample_colors", _vp, _vp)
_sig("hvvr_camera_read_sample_remap", _vp, _vp, C.c_uint64)
_sig("hvvr_camera_read_beams", _vp, _vp)
_sig("hvvr_camera_read_timings", _vp, _vp)
_sig("hvvr_camera_read_list_total", _vp, _p(C.c_uint64))
_sig("hvvr_scene_get_counts", _vp, _p(_u32), _p(_u32), _p(_u32))
_sig("hvvr_scene_read_nodes", _vp, _vp)
_sig("hvvr_scene_read_triangles", _vp, _vp)
_sig("hvvr_generate_topology", _vp, _u32, _vp, _u32, _vp, _u32, _p(_u32))
_sig("hvvr_generate_topology_device", _vp, _u32, _vp, _u32, _vp, _u32, _p(_u32), _vp)
_sig("hvvr_grid_samples", _u32, _u32, _vp)
_sig("hvvr_scene_file_load", C.c_char_p, _p(_vp))
_sig("hvvr_scene_file_counts", _vp, _p(_u32), _p(_u32), _p(_u32))
_sig("hvvr_scene_file_mesh", _vp, _u32, _p(_abi.MeshData), _p(_abi.Transform))
_sig("hvvr_scene_file_light", _vp, _u32, _p(_abi.LightUnion))
_sig("hvvr_scene_file_texture", _vp, _u32, _p(_u32), _p(_u32), _p(_u32), _p(_u32), _p(_vp), _p(C.c_uint64))
_lib.hvvr_scene_file_close.argtypes = [_vp]
_lib.hvvr_scene_file_close.restype = None
_sig("hvvr_scene_file_save", C.c_char_p, _vp, _u32, _vp, _vp, _u32, _vp, _u32)
_sig("hvvr_samples_load", C.c_char_p, _vp, _u32, _p(_u32))
_sig("hvvr_samples_save", C.c_char_p, _vp, _u32)
_sig("hvvr_polar_foveated_layout", _vp, _p(_u32), _p(_u32), _p(_u32), _p(_u32))
_sig("hvvr_polar_foveated_samples", _vp, _vp, _vp, _vp, _vp)
_sig("hvvr_tile_cull_static", _vp, _vp, _vp, C.c_uint64, _p(C.c_uint64), _vp)
_lib.hvvr_batch_config_default.argtypes = [_p(_abi.BatchConfig)]
_lib.hvvr_batch_config_default.restype = None
_sig("hvvr_batch_create", _p(_vp), _u32, _p(_abi.BatchConfig), _p(_vp))
_sig("hvvr_batch_create_views", _p(_vp), _u32, _p(_abi.BatchConfig), _p(_vp))
_sig("hvvr_batch_destroy", _vp)
_sig("hvvr_model_update_vertices_device", _vp, _u32, _u32, _vp, _vp)
_sig("hvvr_batch_render", _vp, C.c_double, _vp)
_sig("hvvr_batch_synchronize", _vp)
_sig("hvvr_batch_get_config", _vp, _p(_abi.BatchConfig))
_sig("hvvr_batch_set_config", _vp, _p(_abi.BatchConfig))
_sig("hvvr_batch_autotune", _vp, _u32, _p(_abi.BatchConfig))
_sig("hvvr_batch_read_timings", _vp, _vp)
_sig("hvvr_batch_read_kernel_times", _vp, _vp)
_sig("hvvr_batch_read_stats", _vp, _vp)
_sig("hvvr_batch_read_counters", _vp, _vp, _u32)
_sig("hvvr_raycaster_read_counters", _vp, _vp, _u32)
_lib.hvvr_server_config_default.argtypes = [_p(_abi.ServerConfig)]
_lib.hvvr_server_config_default.restype = None
_sig("hvvr_server_create", _p(_vp), _u32, _p(_abi.ServerConfig), _p(_vp))
_sig("hvvr_server_destroy", _vp)
_sig("hvvr_server_add_view", _vp, _u32, _p(_abi.FloatRect), _vp, _u32, _u32, _u32, _u32, _p(_u32))
_sig("hvvr_server_submit", _vp, _p(_abi.Request), _p(C.c_uint64))
_sig("hvvr_server_submit_group", _vp, _p(_abi.Request), _u32, _p(C.c_uint64))
_sig("hvvr_server_prewarm", _vp, _u32, _u32)
_sig("hvvr_server_poll", _vp, _p(_abi.Completion), _u32, _p(_u32), C.c_double)
_sig("hvvr_server_update_vertices", _vp, _vp, _u32, _u32, _vp)
_sig("hvvr_server_get_stats", _vp, _p(_abi.ServerStats))
_sig("hvvr_raycaster_read_kernel_times", _vp, _vp)
_sig("hvvr_raycaster_get_batch_config", _vp, _p(_abi.BatchConfig))
_sig("hvvr_raycaster_set_batch_config", _vp, _p(_abi.BatchConfig))
_sig("hvvr_raycaster_read_part_times", _vp, _vp)
_sig("hvvr_batch_read_part_times", _vp, _vp)
_sig("hvvr_camera_read_tile_costs", _vp, _vp)
_sig("hvvr_camera_read_foveated_frame", _vp, _vp, _vp, _vp)
_sig("hvvr_camera_read_foveated_resolve", _vp, _vp, _vp, _vp, _vp)
_sig("hvvr_camera_read_polar_textures", _vp, _vp, _vp, _vp)
_sig("hvvr_foveated_frame_matrices", _p(_abi.Transform), _p(_abi.Vec3), _p(_abi.FloatRect), _p(_abi.FloatRect),
     _vp, _vp, _vp, _vp, _vp, _vp)

EXPORTED = [
    "hvvr_last_error", "hvvr_version", "hvvr_spec_default", "hvvr_raycaster_create", "hvvr_raycaster_destroy",
    "hvvr_raycaster_set_scene_dirty", "hvvr_raycaster_render", "hvvr_raycaster_synchronize", "hvvr_model_create",
    "hvvr_model_destroy", "hvvr_model_set_transform", "hvvr_model_update_vertices", "hvvr_light_create",
    "hvvr_light_destroy", "hvvr_texture_create", "hvvr_texture_destroy", "hvvr_texture_get_id",
    "hvvr_texture_read_level", "hvvr_texture_sample", "hvvr_camera_create", "hvvr_camera_destroy", "hvvr_camera_set_enabled",
    "hvvr_camera_set_viewport", "hvvr_camera_set_lens", "hvvr_camera_set_aperture", "hvvr_camera_set_focal_depth",
    "hvvr_camera_set_eye_dir", "hvvr_camera_set_spherical_warp", "hvvr_camera_set_render_target",
    "hvvr_camera_set_samples", "hvvr_camera_set_camera_to_world", "hvvr_camera_prepare", "hvvr_camera_set_msaa",
    "hvvr_camera_get_sample_count", "hvvr_camera_set_capture", "hvvr_camera_get_layout", "hvvr_camera_set_msaa_pattern",
    "hvvr_camera_read_tile_lists", "hvvr_camera_read_block_stacks", "hvvr_camera_read_hits",
    "hvvr_camera_read_gbuffer", "hvvr_camera_read_sample_colors", "hvvr_camera_read_sample_remap",
    "hvvr_camera_read_beams", "hvvr_camera_read_timings", "hvvr_camera_read_list_total", "hvvr_scene_get_counts",
    "hvvr_scene_read_nodes", "hvvr_scene_read_triangles", "hvvr_generate_topology", "hvvr_generate_topology_device",
    "hvvr_grid_samples",
    "hvvr_polar_foveated_layout", "hvvr_polar_foveated_samples", "hvvr_scene_file_load", "hvvr_scene_file_counts",
    "hvvr_scene_file_mesh", "hvvr_scene_file_light", "hvvr_scene_file_texture", "hvvr_scene_file_close",
    "hvvr_scene_file_save", "hvvr_samples_load", "hvvr_samples_save",
    "hvvr_tile_cull_static", "hvvr_batch_config_default", "hvvr_batch_create", "hvvr_batch_create_views",
    "hvvr_batch_destroy", "hvvr_model_update_vertices_device",
    "hvvr_batch_render", "hvvr_batch_synchronize", "hvvr_batch_get_config", "hvvr_batch_set_config",
    "hvvr_batch_autotune", "hvvr_batch_read_timings", "hvvr_batch_read_kernel_times",
    "hvvr_raycaster_read_kernel_times", "hvvr_camera_read_tile_costs", "hvvr_batch_read_stats",
    "hvvr_raycaster_read_part_times", "hvvr_batch_read_part_times", "hvvr_batch_read_counters",
    "hvvr_raycaster_read_counters", "hvvr_raycaster_get_batch_config", "hvvr_raycaster_set_batch_config",
    "hvvr_camera_read_foveated_frame", "hvvr_camera_read_foveated_resolve", "hvvr_foveated_frame_matrices",
    "hvvr_camera_read_polar_textures",
    "hvvr_server_config_default", "hvvr_server_create", "hvvr_server_destroy", "hvvr_server_add_view",
    "hvvr_server_submit", "hvvr_server_submit_group", "hvvr_server_prewarm", "hvvr_server_poll", "hvvr_server_update_vertices", "hvvr_server_get_stats",
]


class HvvrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("hvvr error %d: %s" % (code, msg))
        self.code = code


def _check(rc):
    if rc != HVVR_OK:
        raise HvvrError(rc, _lib.hvvr_last_error().decode())


def lib():
    """The loaded ctypes library (for callers that bind the C ABI directly)."""
    return _lib


def generate_topology(scene):
    """GenerateTopology: builds scene.nodes and reorders scene.verts / scene.tri_shade in place."""
    nodes = np.zeros(len(scene.tri_shade) + 4, dtype=_abi.TOPO_DTYPE)
    cnt = _u32(0)
    _check(_lib.hvvr_generate_topology(scene.verts.ctypes.data, len(scene.verts), scene.tri_shade.ctypes.data,
                                       len(scene.tri_shade), nodes.ctypes.data, len(nodes), C.byref(cnt)))
    scene.nodes = nodes[: cnt.value].copy()
    return scene


def generate_topology_device(scene, stream=None):
    """The device BVH build (hvvr_generate_topology_device): builds scene.nodes on the GPU and
    reorders scene.tri_shade in place (vertices keep their order)."""
    nodes = np.zeros(len(scene.tri_shade) + 4, dtype=_abi.TOPO_DTYPE)
    cnt = _u32(0)
    _check(_lib.hvvr_generate_topology_device(scene.verts.ctypes.data, len(scene.verts), scene.tri_shade.ctypes.data,
                                              len(scene.tri_shade), nodes.ctypes.data, len(nodes), C.byref(cnt),
                                              stream))
    scene.nodes = nodes[: cnt.value].copy()
    return scene


def foveated_spec(degree_tracking_error=0.5, max_fov_degrees=110.0, mar_slope=0.022, foveal_mar_degrees=1.0 / 60.0,
                  **kw):
    """hvvr_spec with the foveated sample-pattern parameters (RayCasterSpecification::FoveatedSamplePattern)."""
    spec = _abi.Spec()
    _lib.hvvr_spec_default(C.byref(spec))
    spec.foveated_degree_tracking_error = degree_tracking_error
    spec.foveated_max_fov_degrees = max_fov_degrees
    spec.foveated_mar_slope = mar_slope
    spec.foveated_foveal_mar_degrees = foveal_mar_degrees
    for k, v in kw.items():
        setattr(spec, k, v)
    return spec


def polar_foveated_samples(spec=None):
    """The polar foveated sample set the library builds for spec (see hvvr_polar_foveated_samples)."""
    spr, rings, valid, padded = _u32(0), _u32(0), _u32(0), _u32(0)
    sp = C.byref(spec) if spec is not None else None
    _check(_lib.hvvr_polar_foveated_layout(sp, C.byref(spr), C.byref(rings), C.byref(valid), C.byref(padded)))
    out = {"samples_per_ring": spr.value, "ring_count": rings.value, "valid": valid.value, "padded": padded.value,
           "beams": np.zeros((valid.value, 9), np.float32), "remap": np.zeros((padded.value, 2), np.uint32),
           "tile_rays": np.zeros((padded.value // 128, 24), np.float32),
           "block_rays": np.zeros((padded.value // 8192, 24), np.float32)}
    _check(_lib.hvvr_polar_foveated_samples(sp, out["beams"].ctypes.data, out["remap"].ctypes.data,
                                            out["tile_rays"].ctypes.data, out["block_rays"].ctypes.data))
    return out


def foveated_frame_matrices(xf, eye_dir, sample_bounds, viewport, history=None):
    """A foveated camera's per-frame matrices on the host (hvvr_foveated_frame_matrices).
    history: (world_to_eye_prev [16], eye_prev_to_sample_prev [9]) or None for a new camera;
    returns a dict with eye_to_world, cull_planes, sample_to_eye, eye_to_sample_prev and the
    next frame's history."""
    if history is None:
        w2ep, ep2sp = np.zeros(16, np.float32), np.eye(3, dtype=np.float32).reshape(9)
    else:
        w2ep, ep2sp = (np.array(h, np.float32).reshape(n).copy() for h, n in zip(history, (16, 9)))
    out = {"eye_to_world": np.zeros(16, np.float32), "cull_planes": np.zeros((4, 4), np.float32),
           "sample_to_eye": np.zeros(9, np.float32), "eye_to_sample_prev": np.zeros(16, np.float32)}
    ed = _abi.Vec3(*eye_dir)
    _check(_lib.hvvr_foveated_frame_matrices(C.byref(xf), C.byref(ed), C.byref(sample_bounds), C.byref(viewport),
                                             w2ep.ctypes.data, ep2sp.ctypes.data, out["eye_to_world"].ctypes.data,
                                             out["cull_planes"].ctypes.data, out["sample_to_eye"].ctypes.data,
                                             out["eye_to_sample_prev"].ctypes.data))
    out["history"] = (w2ep, ep2sp)
    return out


def load_scene_file(path):
    """A scene file in the reference's binary format (model_import::loadBin): dict with "meshes"
    (a scenes.Scene per mesh, its topology in .nodes and model transform in .transform), "lights"
    (LightUnion list) and "textures" (dicts of format, width, height, stride, texels)."""
    from . import scenes
    h = _vp()
    _check(_lib.hvvr_scene_file_load(os.fsencode(path), C.byref(h)))
    try:
        nt, nl, nm = _u32(0), _u32(0), _u32(0)
        _check(_lib.hvvr_scene_file_counts(h, C.byref(nt), C.byref(nl), C.byref(nm)))
        lights = []
        for i in range(nl.value):
            l = _abi.LightUnion()
            _check(_lib.hvvr_scene_file_light(h, i, C.byref(l)))
            lights.append(l)
        meshes = []
        for i in range(nm.value):
            md, xf = _abi.MeshData(), _abi.Transform()
            _check(_lib.hvvr_scene_file_mesh(h, i, C.byref(md), C.byref(xf)))

            def arr(ptr, n, dt):
                if not n:
                    return np.zeros(0, dt)
                return np.frombuffer(C.string_at(ptr, n * dt.itemsize), dt).copy()
            sc = scenes.Scene(arr(md.verts, md.vert_count, _abi.VERTEX_DTYPE),
                              arr(md.tri_shade, md.tri_count, _abi.TRISHADE_DTYPE),
                              arr(md.materials, md.material_count, _abi.MATERIAL_DTYPE), lights)
            sc.nodes = arr(md.nodes, md.node_count, _abi.TOPO_DTYPE) if md.node_count else None
            sc.transform = xf
            meshes.append(sc)
        textures = []
        for i in range(nt.value):
            fmt, w, hh, st, ptr, nb = _u32(0), _u32(0), _u32(0), _u32(0), _vp(), C.c_uint64(0)
            _check(_lib.hvvr_scene_file_texture(h, i, C.byref(fmt), C.byref(w), C.byref(hh), C.byref(st), C.byref(ptr),
                                                C.byref(nb)))
            textures.append({"format": fmt.value, "width": w.value, "height": hh.value, "stride": st.value,
                             "texels": np.frombuffer(C.string_at(ptr, nb.value), np.uint8).copy()})
        return {"meshes": meshes, "lights": lights, "textures": textures}
    finally:
        _lib.hvvr_scene_file_close(h)


def create_objects(rc, loaded):
    """model_import::createObjects (libraries/hvvr/samples_shared/model_import.cpp:41-63): the
    textures of a load_scene_file result first (so their ids are the file's texture indices), then
    its lights, then one model per mesh with the mesh's transform. Returns (textures, lights, models)."""
    texs = [rc.create_texture(t["texels"], t["format"], t["width"], t["height"], t["stride"])
            for t in loaded["textures"]]
    lights = [rc.create_light(l) for l in loaded["lights"]]
    models = []
    for sc in loaded["meshes"]:
        m = rc.create_model(sc)
        m.set_transform(sc.transform)
        models.append(m)
    return texs, lights, models


def save_scene_file(path, meshes, lights=(), textures=()):
    """Writes textures (dicts as load_scene_file returns them), lights and scenes.Scene meshes
    (topology from .nodes when set, transform from .transform or identity) in the reference's
    binary scene format."""
    tds = (_abi.TextureData * max(1, len(textures)))()
    tkeep = []
    for i, t in enumerate(textures):
        b = np.ascontiguousarray(t["texels"]).view(np.uint8)
        tkeep.append(b)
        tds[i] = _abi.TextureData(b.ctypes.data, t["format"], t["width"], t["height"], t.get("stride", t["width"]))
    mds = (_abi.MeshData * max(1, len(meshes)))()
    xfs = (_abi.Transform * max(1, len(meshes)))()
    keep = []
    for i, sc in enumerate(meshes):
        nodes = sc.nodes if sc.nodes is not None else np.zeros(0, _abi.TOPO_DTYPE)
        arrays = [np.ascontiguousarray(a) for a in (sc.verts, sc.tri_shade, nodes, sc.materials)]
        keep.append(arrays)
        mds[i] = _abi.MeshData(_abi.ptr(arrays[0]), len(arrays[0]), _abi.ptr(arrays[1]), len(arrays[1]),
                               _abi.ptr(arrays[2]) if len(arrays[2]) else None, len(arrays[2]),
                               _abi.ptr(arrays[3]), len(arrays[3]))
        xfs[i] = getattr(sc, "transform", None) or _abi.transform()
    ls = (_abi.LightUnion * max(1, len(lights)))(*lights)
    _check(_lib.hvvr_scene_file_save(os.fsencode(path), tds, len(textures), mds, xfs, len(meshes), ls, len(lights)))


def load_samples(path):
    """A sample file in the reference's format (loadSamples): SAMPLE_DTYPE array."""
    n = _u32(0)
    _check(_lib.hvvr_samples_load(os.fsencode(path), None, 0, C.byref(n)))
    out = np.zeros(n.value, dtype=_abi.SAMPLE_DTYPE)
    _check(_lib.hvvr_samples_load(os.fsencode(path), out.ctypes.data, n.value, C.byref(n)))
    return out


def save_samples(path, samples):
    samples = np.ascontiguousarray(samples, dtype=_abi.SAMPLE_DTYPE)
    _check(_lib.hvvr_samples_save(os.fsencode(path), samples.ctypes.data, len(samples)))


def grid_samples(width, height):
    s = np.zeros(width * height, dtype=_abi.SAMPLE_DTYPE)
    _check(_lib.hvvr_grid_samples(width, height, s.ctypes.data))
    return s


class Model:
    def __init__(self, rc, handle, scene):
        self._rc, self.handle, self.scene = rc, handle, scene

    def set_transform(self, xf):
        _check(_lib.hvvr_model_set_transform(self.handle, C.byref(xf)))

    def update_vertices(self, verts):
        verts = np.ascontiguousarray(verts, dtype=_abi.VERTEX_DTYPE)
        _check(_lib.hvvr_model_update_vertices(self.handle, verts.ctypes.data, len(verts)))

    def update_vertices_device(self, first, count, device_ptr, stream=None):
        """copy count vertices (32 B each) from device memory over vertices [first, first+count)"""
        _check(_lib.hvvr_model_update_vertices_device(self.handle, first, count, _vp(device_ptr), stream))


_TEXEL_DTYPE = {HVVR_TEXTURE_RGBA8_UNORM_SRGB: (np.uint8, 4), HVVR_TEXTURE_RGBA8_UNORM: (np.uint8, 4),
                HVVR_TEXTURE_RGBA16_UNORM: (np.uint16, 4), HVVR_TEXTURE_RGBA32_FLOAT: (np.float32, 4),
                HVVR_TEXTURE_RGBA16_FLOAT: (np.float16, 4), HVVR_TEXTURE_R32_FLOAT: (np.float32, 1)}


class Texture:
    """A material texture (Raycaster::createTexture); materials name it by .id."""

    def __init__(self, rc, handle, fmt, width, height):
        self.rc, self.handle, self.format, self.width, self.height = rc, handle, fmt, width, height
        i = _u32(0)
        _check(_lib.hvvr_texture_get_id(handle, C.byref(i)))
        self.id = i.value

    def read_level(self, level):
        """Mip level `level` as [h, w, channels] of the format's texel type."""
        w, h = _u32(0), _u32(0)
        _check(_lib.hvvr_texture_read_level(self.handle, level, None, 0, C.byref(w), C.byref(h)))
        dt, ch = _TEXEL_DTYPE[self.format]
        out = np.zeros((h.value, w.value, ch), dt)
        _check(_lib.hvvr_texture_read_level(self.handle, level, out.ctypes.data_as(_vp), out.nbytes, C.byref(w),
                                            C.byref(h)))
        return out

    def sample(self, q):
        """ReadTexture at queries q [n, 6] = (u, v, ddx.x, ddx.y, ddy.x, ddy.y): [n, 4] float32."""
        q = np.ascontiguousarray(q, dtype=np.float32).reshape(-1, 6)
        out = np.zeros((len(q), 4), np.float32)
        _check(_lib.hvvr_texture_sample(self.handle, len(q), q.ctypes.data_as(_vp), out.ctypes.data_as(_vp)))
        return out


class Camera:
    def __init__(self, rc, handle):
        self._rc, self.handle = rc, handle
        self._target = None
        self.width = self.height = 0

    def set_render_target(self, width, height, device_ptr=None, stride=0):
        """CPU_MEMORY target (a numpy image owned by the camera) or CUDA_MEMORY (device_ptr)."""
        d = _abi.ImageDesc()
        d.pixel_format = 0
        d.width, d.height, d.stride = width, height, stride
        self._size = (width, height)
        # the previous image stays alive until the library has released (unregistered) it
        new = None
        if device_ptr is None:
            new = np.zeros((height, stride or width), dtype=np.uint32)
            d.memory_type = HVVR_MEMORY_CPU
            d.data = new.ctypes.data
        else:
            d.memory_type = HVVR_MEMORY_CUDA
            d.data = device_ptr
        _check(_lib.hvvr_camera_set_render_target(self.handle, C.byref(d)))
        self._target = new
        self.width, self.height = width, height

    @property
    def image(self):
        return self._target

    def set_samples(self, samples, split=1):
        samples = np.ascontiguousarray(samples, dtype=_abi.SAMPLE_DTYPE)
        self._samples = samples
        _check(_lib.hvvr_camera_set_samples(self.handle, samples.ctypes.data, len(samples), split))

    def set_camera_to_world(self, xf):
        _check(_lib.hvvr_camera_set_camera_to_world(self.handle, C.byref(xf)))

    def set_viewport(self, vp):
        _check(_lib.hvvr_camera_set_viewport(self.handle, C.byref(vp)))

    def prepare(self):
        """Builds the sample setup now; returns True when it was built on the host."""
        on_host = _u32(0)
        _check(_lib.hvvr_camera_prepare(self.handle, C.byref(on_host)))
        return bool(on_host.value)

    def set_msaa_pattern(self, pattern):
        """HVVR_MSAA_SPIRAL (the reference's, default) or HVVR_MSAA_ROTATED_GRID"""
        _check(_lib.hvvr_camera_set_msaa_pattern(self.handle, pattern))

    def set_msaa(self, rate):
        _check(_lib.hvvr_camera_set_msaa(self.handle, rate))

    def set_enabled(self, enabled):
        _check(_lib.hvvr_camera_set_enabled(self.handle, 1 if enabled else 0))

    def set_capture(self, flags):
        _check(_lib.hvvr_camera_set_capture(self.handle, flags))

    def set_eye_dir(self, d):
        """gaze direction in camera space (Camera::setEyeDir); used by the foveated polar mode"""
        _check(_lib.hvvr_camera_set_eye_dir(self.handle, C.byref(_abi.Vec3(*[float(x) for x in d]))))

    def set_lens(self, radius, focal_distance):
        _check(_lib.hvvr_camera_set_lens(self.handle, C.byref(_abi.ThinLens(radius, focal_distance))))

    def sample_count(self):
        n = _u32(0)
        _check(_lib.hvvr_camera_get_sample_count(self.handle, C.byref(n)))
        return n.value

    def layout(self):
        b, t, p, m = _u32(0), _u32(0), _u32(0), _u32(0)
        _check(_lib.hvvr_camera_get_layout(self.handle, C.byref(b), C.byref(t), C.byref(p), C.byref(m)))
        return b.value, t.value, p.value, m.value

    def tile_lists(self):
        blocks, tiles, padded, msaa = self.layout()
        counts = np.zeros(tiles, dtype=np.uint32)
        total = C.c_uint64(0)
        _check(_lib.hvvr_camera_read_tile_lists(self.handle, counts.ctypes.data, None, 0, C.byref(total)))
        idx = np.zeros(max(total.value, 1), dtype=np.uint32)
        _check(_lib.hvvr_camera_read_tile_lists(self.handle, counts.ctypes.data, idx.ctypes.data, len(idx),
                                                C.byref(total)))
        return counts, idx[: total.value]

    def block_stacks(self):
        blocks, tiles, padded, msaa = self.layout()
        sizes = np.zeros(blocks, dtype=np.uint32)
        entries = np.zeros((blocks, 64, 3), dtype=np.uint32)
        _check(_lib.hvvr_camera_read_block_stacks(self.handle, sizes.ctypes.data, entries.ctypes.data))
        return sizes, entries

    def hits(self):
        blocks, tiles, padded, msaa = self.layout()
        ids = np.zeros((padded, msaa), dtype=np.uint32)
        depth = np.zeros((padded, msaa), dtype=np.float32)
        _check(_lib.hvvr_camera_read_hits(self.handle, ids.ctypes.data, depth.ctypes.data))
        return ids, depth

    def gbuffer(self):
        blocks, tiles, padded, msaa = self.layout()
        n = np.zeros(padded, dtype=np.uint32)
        tri = np.zeros((padded, msaa), dtype=np.uint32)
        mask = np.zeros((padded, msaa), dtype=np.uint32)
        _check(_lib.hvvr_camera_read_gbuffer(self.handle, n.ctypes.data, tri.ctypes.data, mask.ctypes.data))
        return n, tri, mask

    def sample_colors(self):
        blocks, tiles, padded, msaa = self.layout()
        c = np.zeros(padded, dtype=np.uint32)
        _check(_lib.hvvr_camera_read_sample_colors(self.handle, c.ctypes.data))
        return c

    def beams(self):
        blocks, tiles, padded, msaa = self.layout()
        b = np.zeros((padded, 9), dtype=np.float32)
        _check(_lib.hvvr_camera_read_beams(self.handle, b.ctypes.data))
        return b

    def sample_remap(self, split=1):
        r = np.zeros(self.width * self.height * split, dtype=np.int32)
        _check(_lib.hvvr_camera_read_sample_remap(self.handle, r.ctypes.data, len(r)))
        return r

    def timings(self):
        t = np.zeros(6, dtype=np.float32)
        _check(_lib.hvvr_camera_read_timings(self.handle, t.ctypes.data))
        return t

    def foveated_frame(self):
        """foveated polar mode: (eye_to_world [16], cull planes [4, 4], view depth [padded])"""
        m = np.zeros(16, np.float32)
        p = np.zeros((4, 4), np.float32)
        d = np.zeros(self.layout()[2], np.float32)
        _check(_lib.hvvr_camera_read_foveated_frame(self.handle, m.ctypes.data, p.ctypes.data, d.ctypes.data))
        return m, p, d

    def foveated_resolve(self):
        """foveated polar mode: the last frame's resolve - (sample_to_eye [9], eye_to_sample_prev
        [16], the temporally filtered image it wrote [h, w], the previous result it read [h, w])"""
        w, h = self._size
        s2e, e2p = np.zeros(9, np.float32), np.zeros(16, np.float32)
        res, hist = np.zeros((h, w), np.uint32), np.zeros((h, w), np.uint32)
        _check(_lib.hvvr_camera_read_foveated_resolve(self.handle, s2e.ctypes.data, e2p.ctypes.data,
                                                      res.ctypes.data, hist.ctypes.data))
        return s2e, e2p, res, hist

    def polar_textures(self, samples_per_ring, ring_count):
        """foveated polar mode: the last frame's polar colour [rings, spr], view depth [rings, spr]
        and moments [rings, spr, 2, 4] (uint16)"""
        col = np.zeros((ring_count, samples_per_ring), np.uint32)
        dep = np.zeros((ring_count, samples_per_ring), np.float32)
        mom = np.zeros((ring_count, samples_per_ring, 2, 4), np.uint16)
        _check(_lib.hvvr_camera_read_polar_textures(self.handle, col.ctypes.data, dep.ctypes.data, mom.ctypes.data))
        return col, dep, mom

    def tile_costs(self):
        """BVH nodes visited per tile by the last frame's tile cull"""
        n = self.layout()[1]
        v = np.zeros(n, dtype=np.uint32)
        _check(_lib.hvvr_camera_read_tile_costs(self.handle, v.ctypes.data))
        return v

    def list_total(self):
        total = C.c_uint64(0)
        _check(_lib.hvvr_camera_read_list_total(self.handle, C.byref(total)))
        return total.value


class Raycaster:
    """Raycaster(const RayCasterSpecification&) (libraries/hvvr/raycaster/raycaster.h:44)."""

    def __init__(self, fp_mode=HVVR_FP_FMA, tri_index_capacity=0, device=0, spec=None, sample_setup=HVVR_SETUP_DEVICE):
        """spec: a full hvvr_spec (e.g. foveated_spec(...)); otherwise the defaults with these fields"""
        if spec is None:
            spec = _abi.Spec()
            _lib.hvvr_spec_default(C.byref(spec))
            spec.fp_mode = fp_mode
            spec.tri_index_capacity = tri_index_capacity
            spec.device = device
            spec.sample_setup = sample_setup
        h = _vp()
        _check(_lib.hvvr_raycaster_create(C.byref(spec), C.byref(h)))
        self.handle = h
        self.cameras, self.models, self.lights, self.textures = [], [], [], []
        self.batches = []

    def close(self):
        if self.handle:
            for b in list(self.batches):
                b.close()
            _check(_lib.hvvr_raycaster_destroy(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def create_model(self, scene):
        md = _abi.MeshData(_abi.ptr(scene.verts), len(scene.verts), _abi.ptr(scene.tri_shade), len(scene.tri_shade),
                           _abi.ptr(scene.nodes) if scene.nodes is not None else None,
                           len(scene.nodes) if scene.nodes is not None else 0,
                           _abi.ptr(scene.materials), len(scene.materials))
        h = _vp()
        _check(_lib.hvvr_model_create(self.handle, C.byref(md), C.byref(h)))
        m = Model(self, h, scene)
        self.models.append(m)
        return m

    def create_light(self, light):
        h = _vp()
        _check(_lib.hvvr_light_create(self.handle, C.byref(light), C.byref(h)))
        self.lights.append(h)
        return h

    def create_texture(self, texels, fmt=HVVR_TEXTURE_RGBA8_UNORM_SRGB, width=None, height=None, stride=None):
        """createTexture(TextureData): texels as [h, w, channels] of the format's texel type, or raw
        bytes with width, height and stride (in texels) given."""
        a = np.ascontiguousarray(texels)
        if width is None:
            height, width = a.shape[0], a.shape[1]
        stride = stride if stride is not None else width
        td = _abi.TextureData(a.ctypes.data, fmt, width, height, stride)
        h = _vp()
        _check(_lib.hvvr_texture_create(self.handle, C.byref(td), C.byref(h)))
        t = Texture(self, h, fmt, width, height)
        self.textures.append(t)
        return t

    def destroy_texture(self, tex):
        _check(_lib.hvvr_texture_destroy(self.handle, tex.handle))
        self.textures.remove(tex)

    def create_camera(self, viewport, aperture=0.0):
        h = _vp()
        _check(_lib.hvvr_camera_create(self.handle, C.byref(viewport), C.c_float(aperture), C.byref(h)))
        c = Camera(self, h)
        self.cameras.append(c)
        return c

    def destroy_camera(self, cam):
        _check(_lib.hvvr_camera_destroy(self.handle, cam.handle))
        self.cameras.remove(cam)

    def destroy_model(self, model):
        _check(_lib.hvvr_model_destroy(self.handle, model.handle))
        self.models.remove(model)

    def set_scene_dirty(self):
        _check(_lib.hvvr_raycaster_set_scene_dirty(self.handle))

    def render(self, elapsed=0.0, stream=None):
        _check(_lib.hvvr_raycaster_render(self.handle, C.c_double(elapsed), stream))

    def synchronize(self):
        _check(_lib.hvvr_raycaster_synchronize(self.handle))

    def kernel_times(self):
        """device ms of the last frame's launches: tile cull, intersect/shade, block cull, remap"""
        t = np.zeros(4, dtype=np.float32)
        _check(_lib.hvvr_raycaster_read_kernel_times(self.handle, t.ctypes.data))
        return t

    def batch_config(self):
        """the configuration of the batch behind render()"""
        cfg = _abi.BatchConfig()
        _check(_lib.hvvr_raycaster_get_batch_config(self.handle, C.byref(cfg)))
        return cfg

    def set_batch_config(self, cfg=None, **kw):
        """set the configuration of the batch behind render(): cfg, or the current one with the
        keyword fields changed (e.g. timing=1 for per-stage, kernel and part times)"""
        cfg = cfg if cfg is not None else self.batch_config()
        for k, v in kw.items():
            setattr(cfg, k, v)
        _check(_lib.hvvr_raycaster_set_batch_config(self.handle, C.byref(cfg)))

    def counters(self):
        """the last frame's counters: list pool entries, retried tiles, status, views, list entries
        that passed the intersect's per-tile tests, (warp, entry) pairs whose subsample tests ran"""
        t = np.zeros(6, dtype=np.uint64)
        _check(_lib.hvvr_raycaster_read_counters(self.handle, t.ctypes.data, 6))
        return t

    def part_times(self):
        """the last frame's timeline per launch part [36, 3]: tile cull start, tile cull end,
        intersect end (ms from the frame start, -1 where the part did not run); part 2r holds
        rate class r's slowest tiles, 2r+1 the rest"""
        t = np.zeros((36, 3), dtype=np.float32)
        _check(_lib.hvvr_raycaster_read_part_times(self.handle, t.ctypes.data))
        return t

    def scene_counts(self):
        n, t, v = _u32(0), _u32(0), _u32(0)
        _check(_lib.hvvr_scene_get_counts(self.handle, C.byref(n), C.byref(t), C.byref(v)))
        return n.value, t.value, v.value

    def scene_nodes(self):
        n, t, v = self.scene_counts()
        a = np.zeros(n, dtype=_abi.NODE_DTYPE)
        _check(_lib.hvvr_scene_read_nodes(self.handle, a.ctypes.data))
        return a

    def scene_triangles(self):
        n, t, v = self.scene_counts()
        a = np.zeros((t, 9), dtype=np.float32)
        _check(_lib.hvvr_scene_read_triangles(self.handle, a.ctypes.data))
        return a


def batch_config(**kw):
    """hvvr_batch_config with the library defaults, overridden by keyword."""
    cfg = _abi.BatchConfig()
    _lib.hvvr_batch_config_default(C.byref(cfg))
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


class Batch:
    """The enabled cameras of several raycasters (one scene each, one device) rendered as one
    frame: one launch per stage over all views, replayed from a CUDA graph once stable."""

    def __init__(self, raycasters=None, config=None, cameras=None):
        """Every enabled camera of `raycasters`, or exactly `cameras` (of any raycasters)."""
        h = _vp()
        cfg = C.byref(config) if config is not None else None
        if cameras is not None:
            arr = (_vp * len(cameras))(*[c.handle for c in cameras])
            _check(_lib.hvvr_batch_create_views(arr, len(cameras), cfg, C.byref(h)))
            raycasters = []
            for c in cameras:
                if c._rc not in raycasters:
                    raycasters.append(c._rc)
        else:
            arr = (_vp * len(raycasters))(*[r.handle for r in raycasters])
            _check(_lib.hvvr_batch_create(arr, len(raycasters), cfg, C.byref(h)))
        self.handle = h
        self.raycasters = list(raycasters)
        for r in self.raycasters:
            r.batches.append(self)

    def close(self):
        if self.handle:
            _check(_lib.hvvr_batch_destroy(self.handle))
            self.handle = None
            for r in self.raycasters:
                if self in r.batches:
                    r.batches.remove(self)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, elapsed=0.0, stream=None):
        _check(_lib.hvvr_batch_render(self.handle, C.c_double(elapsed), stream))

    def synchronize(self):
        _check(_lib.hvvr_batch_synchronize(self.handle))

    @property
    def config(self):
        cfg = _abi.BatchConfig()
        _check(_lib.hvvr_batch_get_config(self.handle, C.byref(cfg)))
        return cfg

    @config.setter
    def config(self, cfg):
        _check(_lib.hvvr_batch_set_config(self.handle, C.byref(cfg)))

    def autotune(self, frames=5):
        cfg = _abi.BatchConfig()
        _check(_lib.hvvr_batch_autotune(self.handle, frames, C.byref(cfg)))
        return cfg

    def kernel_times(self):
        """device ms of the last frame's launches: tile cull, intersect/shade, block cull, remap"""
        t = np.zeros(4, dtype=np.float32)
        _check(_lib.hvvr_batch_read_kernel_times(self.handle, t.ctypes.data))
        return t

    def part_times(self):
        """the last frame's timeline per launch part [36, 3] (see Raycaster.part_times)"""
        t = np.zeros((36, 3), dtype=np.float32)
        _check(_lib.hvvr_batch_read_part_times(self.handle, t.ctypes.data))
        return t

    def stats(self):
        """last frame: list-pool entries taken, tiles re-culled with the large stack, status, views"""
        t = np.zeros(4, dtype=np.uint64)
        _check(_lib.hvvr_batch_read_stats(self.handle, t.ctypes.data))
        return {"pool_entries": int(t[0]), "retried_tiles": int(t[1]), "status": int(t[2]), "views": int(t[3])}

    def timings(self):
        """device ms of the last frame: total, block cull, first tile cull, rest of cull +
        intersect/shade, remap + copies (stages 0 unless config.timing is 1)"""
        t = np.zeros(5, dtype=np.float32)
        _check(_lib.hvvr_batch_read_timings(self.handle, t.ctypes.data))
        return t


def server_config(**kw):
    """hvvr_server_config with the library defaults, overridden by keyword."""
    cfg = _abi.ServerConfig()
    _lib.hvvr_server_config_default(C.byref(cfg))
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


class Server:
    """Render-request server over resident scenes (raycasters): admission against an HBM
    budget, continuous batching into frame batches, completions with timestamps."""

    def __init__(self, raycasters, config=None):
        arr = (_vp * len(raycasters))(*[r.handle for r in raycasters])
        h = _vp()
        _check(_lib.hvvr_server_create(arr, len(raycasters), C.byref(config) if config is not None else None,
                                       C.byref(h)))
        self.handle = h
        self.raycasters = list(raycasters)
        self.views = []
        # CPU output arrays of requests in flight: the server writes a request's image into its
        # array when the request completes, so the array is held here until poll() returns its
        # completion (or the server is closed)
        self._outputs = {}
        for r in self.raycasters:
            r.batches.append(self)  # closed before its raycasters

    def close(self):
        if self.handle:
            _check(_lib.hvvr_server_destroy(self.handle))
            self.handle = None
            self._outputs.clear()
            for r in self.raycasters:
                if self in r.batches:
                    r.batches.remove(self)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_view(self, scene_index, viewport, samples, width, height, split=1):
        samples = np.ascontiguousarray(samples, dtype=_abi.SAMPLE_DTYPE)
        vid = _u32(0)
        _check(_lib.hvvr_server_add_view(self.handle, scene_index, C.byref(viewport), samples.ctypes.data,
                                         len(samples), split, width, height, C.byref(vid)))
        self.views.append((width, height, len(samples)))
        return vid.value

    def prewarm(self, view, count):
        _check(_lib.hvvr_server_prewarm(self.handle, view, count))

    def submit(self, view, msaa, camera_to_world, output=None, device_ptr=None, tag=0, priority=0):
        """output: a (height, width) uint32 numpy array (CPU), or device_ptr for CUDA memory;
        priority 1: the latency class (rendered at once on a latency slot)"""
        r = _abi.Request()
        r.view, r.msaa, r.camera_to_world, r.tag, r.priority = view, msaa, camera_to_world, tag, priority
        if device_ptr is not None:
            r.memory_type, r.output = HVVR_MEMORY_CUDA, device_ptr
        else:
            assert output.flags["C_CONTIGUOUS"] and output.dtype == np.uint32
            r.memory_type, r.output = HVVR_MEMORY_CPU, output.ctypes.data
        rid = C.c_uint64(0)
        _check(_lib.hvvr_server_submit(self.handle, C.byref(r), C.byref(rid)))
        if device_ptr is None:
            self._outputs[rid.value] = output
        return rid.value

    def submit_group(self, items, priority=0):
        """Submits several requests at once (e.g. the two eyes of a stereo frame), so that they can
        render in one batch. items: (view, msaa, camera_to_world, output or None, device_ptr or None,
        tag) tuples. Returns their request ids."""
        reqs = (_abi.Request * len(items))()
        keep = []
        for r, (view, msaa, xf, output, device_ptr, tag) in zip(reqs, items):
            r.view, r.msaa, r.camera_to_world, r.tag, r.priority = view, msaa, xf, tag, priority
            if device_ptr is not None:
                r.memory_type, r.output = HVVR_MEMORY_CUDA, device_ptr
                keep.append(None)
            else:
                assert output.flags["C_CONTIGUOUS"] and output.dtype == np.uint32
                r.memory_type, r.output = HVVR_MEMORY_CPU, output.ctypes.data
                keep.append(output)
        ids = (C.c_uint64 * len(items))()
        _check(_lib.hvvr_server_submit_group(self.handle, reqs, len(items), ids))
        for i, out in zip(ids, keep):
            if out is not None:
                self._outputs[i] = out
        return list(ids)

    def poll(self, capacity=256, wait_ms=0.0):
        out = (_abi.Completion * capacity)()
        n = _u32(0)
        _check(_lib.hvvr_server_poll(self.handle, out, capacity, C.byref(n), C.c_double(wait_ms)))
        done = [out[i] for i in range(n.value)]
        for c in done:
            self._outputs.pop(c.id, None)
        return done

    def update_vertices(self, model, first, count, device_ptr):
        _check(_lib.hvvr_server_update_vertices(self.handle, model.handle, first, count, _vp(device_ptr)))

    def stats(self):
        st = _abi.ServerStats()
        _check(_lib.hvvr_server_get_stats(self.handle, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}
