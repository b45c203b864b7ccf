"""Python bindings of the CPU oracle and of the reference build (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs import
this module. ``Oracle`` wraps oracle/libhvvr_oracle.so (the scalar restatement);
``Reference`` wraps oracle/_ref/libhvvr_ref.so (the reference's own sources compiled here),
which exists only where the reference tree was available at build time.
"""
import ctypes as C
import os

import numpy as np

from hvvr_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libhvvr_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhvvr_ref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libhvvr_ref_gpu.so")


class FrameIn(C.Structure):
    _fields_ = [("model_count", C.c_uint32), ("models", C.POINTER(_abi.MeshData)),
                ("model_xf", C.POINTER(_abi.Transform)), ("lights", C.POINTER(_abi.LightUnion)),
                ("light_count", C.c_uint32), ("viewport", _abi.FloatRect), ("lens", _abi.ThinLens),
                ("cam_xf", _abi.Transform), ("samples", C.c_void_p), ("sample_count", C.c_uint32),
                ("split_color_samples", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32),
                ("msaa", C.c_uint32), ("fp_mode", C.c_uint32), ("threads", C.c_uint32),
                ("texture_count", C.c_uint32), ("texture_sample", C.c_void_p), ("texture_ctx", C.c_void_p),
                ("msaa_pattern", C.c_uint32)]


class FrameOut(C.Structure):
    _fields_ = [("block_sizes", C.c_void_p), ("block_entries", C.c_void_p), ("tile_counts", C.c_void_p),
                ("tile_indices", C.c_void_p), ("tile_capacity", C.c_uint64), ("tile_total", C.c_uint64),
                ("hit_ids", C.c_void_p), ("depth", C.c_void_p), ("depth64", C.c_void_p), ("gb_n", C.c_void_p),
                ("gb_tri", C.c_void_p), ("gb_mask", C.c_void_p), ("colors", C.c_void_p), ("image", C.c_void_p),
                ("remap", C.c_void_p), ("beams", C.c_void_p), ("nodes", C.c_void_p), ("tris", C.c_void_p),
                ("tile_rays", C.c_void_p), ("status", C.c_uint32), ("tmax", C.c_void_p), ("tile_frusta", C.c_void_p)]


class FovIn(C.Structure):
    _fields_ = [("degree_tracking_error", C.c_float), ("max_fov_degrees", C.c_float), ("mar_slope", C.c_float),
                ("foveal_mar_degrees", C.c_float), ("samples_per_ring", C.c_uint32), ("ring_count", C.c_uint32),
                ("valid", C.c_uint32), ("colors", C.c_void_p), ("tmax", C.c_void_p), ("remap", C.c_void_p),
                ("width", C.c_uint32), ("height", C.c_uint32), ("sample_to_eye", C.c_float * 9),
                ("eye_to_sample_prev", C.c_float * 16), ("history", C.c_void_p), ("threads", C.c_uint32)]


class FovOut(C.Structure):
    _fields_ = [("polar_color", C.c_void_p), ("moments", C.c_void_p), ("result", C.c_void_p),
                ("filtered", C.c_void_p), ("image", C.c_void_p)]


class BeamsIn(C.Structure):
    _fields_ = [("beams", C.c_void_p), ("tile_rays", C.c_void_p), ("block_rays", C.c_void_p), ("blocks", C.c_uint32),
                ("batch_to_world", C.c_void_p), ("cull_planes", C.c_void_p)]


def layout(sample_count):
    blocks = (sample_count + 8191) // 8192
    return blocks, blocks * 64, blocks * 8192


class Frame:
    """Outputs of one rendered frame, as numpy arrays."""


def _run(fn, scene, samples, cam_xf, viewport, width, height, msaa, fp_mode=_abi.HVVR_FP_FMA, lens=(0.0, 1.0),
         threads=None, split=1, want=("lists", "hits", "colors", "image", "blocks", "gbuffer", "scene", "beams"),
         model_xf=None, tile_capacity=None, beams_in=None, textures=0, sampler=None, msaa_pattern=0):
    # one scene, or a list of scenes (models of one raycaster, merged under root fix-up nodes as
    # Raycaster::buildScene does) with a list of model transforms; the lights are the first scene's
    models = list(scene) if isinstance(scene, (list, tuple)) else [scene]
    if any(m.nodes is None for m in models):
        raise ValueError("scene has no topology")
    if isinstance(model_xf, (list, tuple)):
        model_xfs = list(model_xf)
    else:
        model_xfs = [model_xf if model_xf is not None else _abi.transform()] * len(models)
    n = len(samples) if beams_in is None else len(beams_in["beams"])
    blocks, tiles, padded = layout(n)
    mds = (_abi.MeshData * len(models))(*[
        _abi.MeshData(_abi.ptr(m.verts), len(m.verts), _abi.ptr(m.tri_shade), len(m.tri_shade), _abi.ptr(m.nodes),
                      len(m.nodes), _abi.ptr(m.materials), len(m.materials)) for m in models])
    xfs = (_abi.Transform * len(models))(*model_xfs)
    lights = (_abi.LightUnion * len(models[0].lights))(*models[0].lights)
    node_total = sum(len(m.nodes) for m in models) + ((len(models) + 1) // 3 if len(models) > 1 else 0)
    tri_total = sum(len(m.tri_shade) for m in models)
    scene = models[0]
    fin = FrameIn()
    fin.model_count = len(models)
    fin.models = mds
    fin.model_xf = xfs
    fin.lights = lights
    fin.light_count = len(scene.lights)
    fin.viewport = viewport
    fin.lens = _abi.ThinLens(*lens)
    fin.cam_xf = cam_xf
    fin.samples = _abi.ptr(samples) if samples is not None else None
    fin.sample_count = n
    fin.split_color_samples = split
    fin.width, fin.height = width, height
    fin.msaa = msaa
    fin.fp_mode = fp_mode
    fin.threads = threads if threads is not None else (os.cpu_count() or 1)
    # material textures: ids below `textures` are live and read through `sampler` (the address
    # of a C sampler such as Oracle.hash_sampler / Oracle.table_sampler)
    fin.texture_count = textures
    fin.texture_sample = sampler
    fin.msaa_pattern = msaa_pattern
    f = Frame()
    out = FrameOut()
    keep = []

    def alloc(name, shape, dtype, field):
        a = np.zeros(shape, dtype=dtype)
        setattr(f, name, a)
        setattr(out, field, a.ctypes.data)
        keep.append(a)

    if "blocks" in want:
        alloc("block_sizes", blocks, np.uint32, "block_sizes")
        alloc("block_entries", (blocks, 64, 3), np.uint32, "block_entries")
    if "lists" in want:
        alloc("tile_counts", tiles, np.uint32, "tile_counts")
        cap = tile_capacity if tile_capacity is not None else 64 << 20
        alloc("tile_indices", cap, np.uint32, "tile_indices")
        out.tile_capacity = cap
    if "hits" in want:
        alloc("hit_ids", (padded, msaa), np.uint32, "hit_ids")
        alloc("depth", (padded, msaa), np.float32, "depth")
        alloc("depth64", (padded, msaa), np.float64, "depth64")
    if "gbuffer" in want:
        alloc("gb_n", padded, np.uint32, "gb_n")
        alloc("gb_tri", (padded, msaa), np.uint32, "gb_tri")
        alloc("gb_mask", (padded, msaa), np.uint32, "gb_mask")
    if "colors" in want:
        alloc("colors", padded, np.uint32, "colors")
    if "image" in want:
        alloc("image", (height, width), np.uint32, "image")
        alloc("remap", height * width * split, np.int32, "remap")
    if "beams" in want:
        alloc("beams", (padded, 9), np.float32, "beams")
    if "tile_rays" in want:
        alloc("tile_rays", (tiles, 24), np.float32, "tile_rays")
    if "scene" in want:
        alloc("nodes", node_total, _abi.NODE_DTYPE, "nodes")
        alloc("tris", (tri_total, 9), np.float32, "tris")
    if "tmax" in want:
        alloc("tmax", padded, np.float32, "tmax")
    if "tile_frusta" in want:
        alloc("tile_frusta", (tiles, 24), np.float32, "tile_frusta")
    if beams_in is None:
        rc = fn(C.byref(fin), C.byref(out))
    else:
        arrs = {k: np.ascontiguousarray(beams_in[k], dtype=np.float32)
                for k in ("beams", "tile_rays", "block_rays", "batch_to_world")}
        planes = beams_in.get("cull_planes")
        if planes is not None:
            arrs["cull_planes"] = np.ascontiguousarray(planes, dtype=np.float32)
        keep.extend(arrs.values())
        bi = BeamsIn(arrs["beams"].ctypes.data, arrs["tile_rays"].ctypes.data, arrs["block_rays"].ctypes.data, blocks,
                     arrs["batch_to_world"].ctypes.data,
                     arrs["cull_planes"].ctypes.data if planes is not None else None)
        rc = fn(C.byref(fin), C.byref(bi), C.byref(out))
    if rc != 0:
        raise RuntimeError("render failed: %d" % rc)
    f.status = out.status
    f.tile_total = out.tile_total
    if "lists" in want:
        f.tile_indices = f.tile_indices[: min(out.tile_total, len(f.tile_indices))]
        f.tile_offsets = np.concatenate([[0], np.cumsum(f.tile_counts, dtype=np.uint64)])
    f.blocks, f.tiles, f.padded = blocks, tiles, padded
    return f


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError("oracle library not built: %s" % path)
        self.lib = C.CDLL(path)
        self.lib.oracle_render.argtypes = [C.POINTER(FrameIn), C.POINTER(FrameOut)]
        self.lib.oracle_render.restype = C.c_int
        self.lib.oracle_msaa_offsets.argtypes = [C.c_uint32, C.c_void_p]

    def render(self, *a, **k):
        return _run(self.lib.oracle_render, *a, **k)

    # texture samplers (addresses for render(..., sampler=)) and the table sampler's state
    @property
    def hash_sampler(self):
        return C.cast(self.lib.oracle_texture_hash, C.c_void_p).value

    @property
    def table_sampler(self):
        return C.cast(self.lib.oracle_texture_table, C.c_void_p).value

    def table_record(self):
        self.lib.oracle_texture_table_reset(1)

    def table_queries(self):
        """The recorded texture queries: ids [n] uint32 and q [n, 6] float32 (u, v, ddx, ddy)."""
        f = self.lib.oracle_texture_table_queries
        f.restype = C.c_uint32
        n = f(None, None, 0)
        ids = np.zeros(n, np.uint32)
        q = np.zeros((n, 6), np.float32)
        f(ids.ctypes.data_as(C.c_void_p), q.ctypes.data_as(C.c_void_p), n)
        return ids, q

    def table_set(self, ids, q, rgba):
        ids = np.ascontiguousarray(ids, np.uint32)
        q = np.ascontiguousarray(q, np.float32)
        rgba = np.ascontiguousarray(rgba, np.float32)
        self.lib.oracle_texture_table_set(C.c_uint32(len(ids)), ids.ctypes.data_as(C.c_void_p),
                                          q.ctypes.data_as(C.c_void_p), rgba.ctypes.data_as(C.c_void_p))

    def table_missing(self):
        self.lib.oracle_texture_table_missing.restype = C.c_uint32
        return int(self.lib.oracle_texture_table_missing())

    def render_beams(self, scene, beams_in, msaa, fp_mode=_abi.HVVR_FP_FMA, threads=None,
                     want=("lists", "hits", "colors", "scene", "tmax")):
        """The foveated frame on given batch-space beams [padded, 9], tile/block frusta, the
        batch-to-world matrix (16 floats, column-major) and optional world cull planes (16 floats)."""
        f = self.lib.oracle_render_beams
        f.argtypes = [C.POINTER(FrameIn), C.POINTER(BeamsIn), C.POINTER(FrameOut)]
        f.restype = C.c_int
        return _run(f, scene, None, _abi.transform(), _abi.FloatRect(), 0, 0, msaa, fp_mode=fp_mode, threads=threads,
                    want=want, beams_in=beams_in)

    def foveated_resolve(self, pattern, polar, colors, tmax, width, height, sample_to_eye, eye_to_sample_prev,
                         history, threads=None):
        """One frame of the foveated resolve. pattern: (degree tracking error, max FOV, MAR slope,
        foveal MAR); polar: the sample set dict (samples_per_ring, ring_count, valid, remap);
        colors / tmax: per sample [>= valid]; history: the previous result [height, width].
        Returns a dict of polar_color, moments [rings, spr, 2, 4], result, filtered, image."""
        f = self.lib.oracle_foveated_resolve
        f.argtypes = [C.POINTER(FovIn), C.POINTER(FovOut)]
        f.restype = C.c_int
        spr, rings, valid = polar["samples_per_ring"], polar["ring_count"], polar["valid"]
        colors = np.ascontiguousarray(colors[:valid], np.uint32)
        tmax = np.ascontiguousarray(tmax[:valid], np.float32)
        remap = np.ascontiguousarray(polar["remap"][:valid], np.uint32)
        history = np.ascontiguousarray(history, np.uint32)
        fi = FovIn(*(float(v) for v in pattern), spr, rings, valid, colors.ctypes.data, tmax.ctypes.data,
                   remap.ctypes.data, width, height)
        fi.sample_to_eye[:] = [float(v) for v in np.asarray(sample_to_eye, np.float32).ravel()]
        fi.eye_to_sample_prev[:] = [float(v) for v in np.asarray(eye_to_sample_prev, np.float32).ravel()]
        fi.history = history.ctypes.data
        fi.threads = threads or min(32, os.cpu_count() or 1)
        out = {"polar_color": np.zeros((rings, spr), np.uint32), "moments": np.zeros((rings, spr, 2, 4), np.uint16),
               "result": np.zeros((height, width), np.uint32), "filtered": np.zeros((height, width), np.uint32),
               "image": np.zeros((height, width), np.uint32)}
        fo = FovOut(*(out[k].ctypes.data for k in ("polar_color", "moments", "result", "filtered", "image")))
        if f(C.byref(fi), C.byref(fo)) != 0:
            raise RuntimeError("oracle_foveated_resolve failed")
        return out

    def lbvh_build(self, scene):
        """The device BVH build restated (oracle_lbvh_build): (tri_shade in leaf order, nodes)."""
        f = self.lib.oracle_lbvh_build
        f.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                      C.POINTER(C.c_uint32)]
        f.restype = C.c_int
        n = len(scene.tri_shade)
        tris = np.zeros_like(scene.tri_shade)
        nodes = np.zeros(n + 4, dtype=_abi.TOPO_DTYPE)
        cnt = C.c_uint32(0)
        rc = f(scene.verts.ctypes.data, len(scene.verts), scene.tri_shade.ctypes.data, n, tris.ctypes.data,
               nodes.ctypes.data, len(nodes), C.byref(cnt))
        if rc != 0:
            raise RuntimeError("oracle_lbvh_build failed: %d" % rc)
        return tris, nodes[: cnt.value].copy()

    def msaa_offsets(self, n):
        o = np.zeros((n, 2), dtype=np.float32)
        self.lib.oracle_msaa_offsets(n, o.ctypes.data)
        return o


class Reference:
    """The reference's own sources compiled here (oracle/_ref)."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError("reference build not present: %s" % path)
        self.lib = C.CDLL(path)
        self.lib.ref_render.argtypes = [C.POINTER(FrameIn), C.POINTER(FrameOut)]
        self.lib.ref_render.restype = C.c_int
        self.lib.ref_generate_topology.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                                   C.c_uint32, C.POINTER(C.c_uint32)]
        self.lib.ref_generate_topology.restype = C.c_int

    @staticmethod
    def available():
        return os.path.exists(REF_SO)

    def render(self, *a, **k):
        return _run(self.lib.ref_render, *a, **k)

    def polar_foveated(self, degree_tracking_error=0.5, max_fov_degrees=110.0, mar_slope=0.022,
                       foveal_mar_degrees=1.0 / 60.0):
        """The reference's polar foveated sample set: dict of samples_per_ring, ring_count, valid,
        padded, beams [valid, 9], remap [valid, 2], tile_rays / block_rays [n, 24]."""
        f = self.lib.ref_polar_foveated
        f.argtypes = [C.c_float] * 4 + [C.c_void_p] * 5
        f.restype = C.c_int
        args = [C.c_float(degree_tracking_error), C.c_float(max_fov_degrees), C.c_float(mar_slope),
                C.c_float(foveal_mar_degrees)]
        counts = np.zeros(4, dtype=np.uint32)
        f(*args, counts.ctypes.data, None, None, None, None)
        spr, rings, valid, padded = (int(v) for v in counts)
        out = {"samples_per_ring": spr, "ring_count": rings, "valid": valid, "padded": padded,
               "beams": np.zeros((valid, 9), np.float32), "remap": np.zeros((valid, 2), np.uint32),
               "tile_rays": np.zeros((padded // 128, 24), np.float32),
               "block_rays": np.zeros((padded // 8192, 24), np.float32)}
        f(*args, counts.ctypes.data, out["beams"].ctypes.data, out["remap"].ctypes.data,
          out["tile_rays"].ctypes.data, out["block_rays"].ctypes.data)
        return out

    def foveated_frame_matrices(self, xf, eye_dir, sample_bounds, viewport, history=None):
        """The reference's per-frame foveated matrices (same dict as hvvr_b200.foveated_frame_matrices)."""
        f = self.lib.ref_foveated_frame_matrices
        f.argtypes = [C.POINTER(_abi.Transform)] + [C.c_void_p] * 9
        f.restype = C.c_int
        if history is None:
            w2ep, ep2sp = np.zeros(16, np.float32), np.eye(3, dtype=np.float32).reshape(9)
        else:
            w2ep, ep2sp = (np.array(h, np.float32).reshape(n).copy() for h, n in zip(history, (16, 9)))
        ed = np.array(eye_dir, np.float32)
        sb = np.array([sample_bounds.lower.x, sample_bounds.lower.y, sample_bounds.upper.x, sample_bounds.upper.y],
                      np.float32)
        vp = np.array([viewport.lower.x, viewport.lower.y, viewport.upper.x, viewport.upper.y], np.float32)
        out = {"eye_to_world": np.zeros(16, np.float32), "cull_planes": np.zeros((4, 4), np.float32),
               "sample_to_eye": np.zeros(9, np.float32), "eye_to_sample_prev": np.zeros(16, np.float32)}
        f(C.byref(xf), ed.ctypes.data, sb.ctypes.data, vp.ctypes.data, w2ep.ctypes.data, ep2sp.ctypes.data,
          out["eye_to_world"].ctypes.data, out["cull_planes"].ctypes.data, out["sample_to_eye"].ctypes.data,
          out["eye_to_sample_prev"].ctypes.data)
        out["history"] = (w2ep, ep2sp)
        return out

    def session(self, scene, samples, viewport, width, height, msaa, lens=(0.0, 1.0)):
        """A camera kept across frames: scene upload, refit and sample setup once, then
        ``frame(cam_xf, threads)`` per frame (see RefSession)."""
        return RefSession(self.lib, scene, samples, viewport, width, height, msaa, lens)

    def generate_topology(self, scene):
        """GenerateTopology on copies of the scene arrays; returns (verts, tri_shade, nodes)."""
        verts = scene.verts.copy()
        tris = scene.tri_shade.copy()
        cap = len(tris) + 4
        nodes = np.zeros(cap, dtype=_abi.TOPO_DTYPE)
        cnt = C.c_uint32(0)
        rc = self.lib.ref_generate_topology(verts.ctypes.data, len(verts), tris.ctypes.data, len(tris),
                                            nodes.ctypes.data, cap, C.byref(cnt))
        if rc != 0:
            raise RuntimeError("GenerateTopology failed: %d" % rc)
        return verts, tris, nodes[: cnt.value].copy()


class RefSession:
    """The reference's per-frame path for one camera over a scene, as its Raycaster runs it frame
    after frame: ref_session_create uploads and refits the scene and builds the camera's SampleData
    once; each frame() transforms the frusta to world space, traverses the blocks and tiles on
    ``threads`` threads (cullThread), runs the intersect/shade code per tile on the same threads and
    remaps the colours into the image."""

    def __init__(self, lib, scene, samples, viewport, width, height, msaa, lens):
        if scene.nodes is None:
            raise ValueError("scene has no topology")
        lib.ref_session_create.argtypes = [C.POINTER(FrameIn), C.POINTER(C.c_void_p)]
        lib.ref_session_create.restype = C.c_int
        lib.ref_session_frame.argtypes = [C.c_void_p, C.POINTER(_abi.Transform), C.c_uint32, C.c_void_p, C.c_void_p]
        lib.ref_session_frame.restype = C.c_int
        lib.ref_session_destroy.argtypes = [C.c_void_p]
        lib.ref_session_destroy.restype = None
        self.lib = lib
        self._keep = (scene, samples)
        md = _abi.MeshData(_abi.ptr(scene.verts), len(scene.verts), _abi.ptr(scene.tri_shade), len(scene.tri_shade),
                           _abi.ptr(scene.nodes), len(scene.nodes), _abi.ptr(scene.materials), len(scene.materials))
        self._mds = (_abi.MeshData * 1)(md)
        self._xfs = (_abi.Transform * 1)(_abi.transform())
        self._lights = (_abi.LightUnion * len(scene.lights))(*scene.lights)
        fin = FrameIn()
        fin.model_count = 1
        fin.models = self._mds
        fin.model_xf = self._xfs
        fin.lights = self._lights
        fin.light_count = len(scene.lights)
        fin.viewport = viewport
        fin.lens = _abi.ThinLens(*lens)
        fin.samples = _abi.ptr(samples)
        fin.sample_count = len(samples)
        fin.split_color_samples = 1
        fin.width, fin.height = width, height
        fin.msaa = msaa
        fin.fp_mode = _abi.HVVR_FP_STRICT
        self.handle = C.c_void_p()
        rc = lib.ref_session_create(C.byref(fin), C.byref(self.handle))
        if rc != 0:
            raise RuntimeError("ref_session_create failed: %d" % rc)
        _, _, self.padded = layout(len(samples))
        self.colors = np.zeros(self.padded, np.uint32)
        self.image = np.zeros((height, width), np.uint32)

    def frame(self, cam_xf, threads):
        rc = self.lib.ref_session_frame(self.handle, C.byref(cam_xf), threads, self.colors.ctypes.data,
                                        self.image.ctypes.data)
        if rc != 0:
            raise RuntimeError("ref_session_frame failed: %d" % rc)
        return self.image

    def close(self):
        if self.handle:
            self.lib.ref_session_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        self.close()


class ReferenceGpu:
    """The reference's own texture creation (CreateTexture with its mip generator), texture reads
    (ReadTexture) and foveated resolve kernels built for the GPU (oracle/_ref/libhvvr_ref_gpu.so);
    needs a GPU."""

    def __init__(self, path=REF_GPU_SO):
        if not os.path.exists(path):
            raise FileNotFoundError("reference GPU library not built: %s" % path)
        self.lib = C.CDLL(path)
        self.lib.ref_gpu_texture_create.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        self.lib.ref_gpu_texture_create.restype = C.c_int
        self.lib.ref_gpu_texture_read_level.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64,
                                                        C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        self.lib.ref_gpu_texture_read_level.restype = C.c_int
        self.lib.ref_gpu_texture_sample.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        self.lib.ref_gpu_texture_sample.restype = C.c_int

    @staticmethod
    def available():
        return os.path.exists(REF_GPU_SO)

    def create_texture(self, texels, fmt):
        """RGBA8 texels [h, w, 4] (the reference's mip generator writes 8-bit texels); returns the
        reference's atlas id"""
        a = np.ascontiguousarray(texels, np.uint8)
        h, w = a.shape[0], a.shape[1]
        return self.lib.ref_gpu_texture_create(a.ctypes.data_as(C.c_void_p), fmt, w, h, w)

    def read_level(self, tex_id, level):
        w, h = C.c_uint32(0), C.c_uint32(0)
        rc = self.lib.ref_gpu_texture_read_level(tex_id, level, None, 0, C.byref(w), C.byref(h))
        if rc != 0:
            raise RuntimeError("read_level: %d" % rc)
        out = np.zeros((h.value, w.value, 4), np.uint8)
        rc = self.lib.ref_gpu_texture_read_level(tex_id, level, out.ctypes.data_as(C.c_void_p), out.nbytes,
                                                 C.byref(w), C.byref(h))
        if rc != 0:
            raise RuntimeError("read_level: %d" % rc)
        return out

    def foveated_resolve(self, pattern, samples_per_ring, ring_count, polar_color, polar_depth, width, height,
                         sample_to_eye, eye_to_sample_prev, history):
        """The reference's own resolve kernels (ComputeMoments, FoveatedPolarToScreenSpaceKernel, the two
        SeparableFilterUsingEccentricity passes, FinishConstrastEnhancement) on the given polar textures
        and matrices: dict of moments [rings, spr, 2, 4], result, filtered, image [h, w]."""
        f = self.lib.ref_gpu_foveated_resolve
        f.restype = C.c_int
        out = {"moments": np.zeros((ring_count, samples_per_ring, 2, 4), np.uint16),
               "result": np.zeros((height, width), np.uint32), "filtered": np.zeros((height, width), np.uint32),
               "image": np.zeros((height, width), np.uint32)}
        ins = [np.ascontiguousarray(polar_color, np.uint32), np.ascontiguousarray(polar_depth, np.float32),
               np.ascontiguousarray(sample_to_eye, np.float32), np.ascontiguousarray(eye_to_sample_prev, np.float32),
               np.ascontiguousarray(history, np.uint32)]
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        rc = f(*[C.c_float(x) for x in pattern], C.c_uint32(samples_per_ring), C.c_uint32(ring_count), p(ins[0]),
               p(ins[1]), C.c_uint32(width), C.c_uint32(height), p(ins[2]), p(ins[3]), p(ins[4]),
               p(out["moments"]), p(out["result"]), p(out["filtered"]), p(out["image"]))
        if rc != 0:
            raise RuntimeError("foveated_resolve: %d" % rc)
        return out

    def intersect_resolve(self, msaa, frame, scene, cam_xf):
        """The reference's IntersectKernel + ResolveKernel on a reference-harness frame's beams, world
        tile frusta, tile lists and triangles (render(..., want=("beams", "tile_frusta", "lists",
        "scene"))) and the scene's shading arrays: dict of gb_tri, gb_mask [padded, msaa], colors,
        tmax [padded]."""
        f = self.lib.ref_gpu_intersect_resolve
        f.restype = C.c_int
        padded, tiles = frame.padded, frame.tiles
        out = {"gb_tri": np.full((padded, msaa), 0xFFFFFFFF, np.uint32), "gb_mask": np.zeros((padded, msaa), np.uint32),
               "colors": np.zeros(padded, np.uint32), "tmax": np.zeros(padded, np.float32)}
        keep = [np.ascontiguousarray(frame.beams, np.float32), np.ascontiguousarray(frame.tile_frusta, np.float32),
                np.ascontiguousarray(frame.tile_counts, np.uint32), np.ascontiguousarray(frame.tile_indices, np.uint32),
                np.ascontiguousarray(frame.tris, np.float32), np.ascontiguousarray(scene.tri_shade),
                np.ascontiguousarray(scene.verts), np.ascontiguousarray(scene.materials)]
        lights = (_abi.LightUnion * max(1, len(scene.lights)))(*scene.lights)
        xf = _abi.Transform()
        C.memmove(C.byref(xf), C.byref(cam_xf), C.sizeof(xf))
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        rc = f(C.c_uint32(msaa), p(keep[0]), C.c_uint32(padded), p(keep[1]), C.c_uint32(tiles), p(keep[2]), p(keep[3]),
               p(keep[4]), p(keep[5]), C.c_uint32(len(keep[5])), p(keep[6]), C.c_uint32(len(keep[6])), p(keep[7]),
               C.c_uint32(len(keep[7])), C.cast(lights, C.c_void_p), C.c_uint32(len(scene.lights)),
               C.cast(C.byref(xf), C.c_void_p), p(out["gb_tri"]), p(out["gb_mask"]), p(out["colors"]), p(out["tmax"]))
        if rc != 0:
            raise RuntimeError("intersect_resolve: %d" % rc)
        return out

    def foveated_scatter(self, samples_per_ring, ring_count, colors, tmax, remap):
        """The reference's RemapPolarFoveatedKernel: sample colours and view depths [valid] scattered
        by remap [valid, 2] into the polar textures; returns (colour [rings, spr], depth [rings, spr])."""
        f = self.lib.ref_gpu_foveated_scatter
        f.restype = C.c_int
        c = np.ascontiguousarray(colors, np.uint32)
        t = np.ascontiguousarray(tmax, np.float32)
        r = np.ascontiguousarray(remap, np.uint32)
        col = np.zeros((ring_count, samples_per_ring), np.uint32)
        dep = np.zeros((ring_count, samples_per_ring), np.float32)
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        rc = f(C.c_uint32(samples_per_ring), C.c_uint32(ring_count), C.c_uint32(len(c)), p(c), p(t), p(r), p(col), p(dep))
        if rc != 0:
            raise RuntimeError("foveated_scatter: %d" % rc)
        return col, dep

    def scene_update(self, nodes, verts, vert_model, transforms, tri_shade):
        """The reference's scene update kernels (SceneTransformVerticesKernel, SceneRefitPreKernel,
        ScenePrecomputeTrianglesKernel, SceneRefitIntFixupKernel, SceneRefitNodeMultiPassKernel) on a
        BVH (its child and leaf data), the untransformed vertices, each vertex's model and the model
        transforms: returns (world vertices, precomputed triangles [t, 9], refit nodes)."""
        f = self.lib.ref_gpu_scene_update
        f.restype = C.c_int
        n = np.ascontiguousarray(nodes, _abi.NODE_DTYPE)
        v = np.ascontiguousarray(verts, _abi.VERTEX_DTYPE)
        vm = np.ascontiguousarray(vert_model, np.uint32)
        xf = (_abi.Transform * len(transforms))(*transforms)
        ts = np.ascontiguousarray(tri_shade)
        world = np.zeros_like(v)
        tris = np.zeros((len(ts), 9), np.float32)
        out = np.zeros_like(n)
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        rc = f(p(n), C.c_uint32(len(n)), p(v), C.c_uint32(len(v)), p(vm), C.cast(xf, C.c_void_p),
               C.c_uint32(len(transforms)), p(ts), C.c_uint32(len(ts)), p(world), p(tris), p(out))
        if rc != 0:
            raise RuntimeError("scene_update: %d" % rc)
        return world, tris, out

    def sample(self, ids, q):
        """ReadTexture through the reference's atlas: ids [n], q [n, 6] -> [n, 4] float32"""
        ids = np.ascontiguousarray(ids, np.uint32)
        q = np.ascontiguousarray(q, np.float32).reshape(-1, 6)
        out = np.zeros((len(q), 4), np.float32)
        rc = self.lib.ref_gpu_texture_sample(len(q), ids.ctypes.data_as(C.c_void_p), q.ctypes.data_as(C.c_void_p),
                                             out.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise RuntimeError("sample: %d" % rc)
        return out
