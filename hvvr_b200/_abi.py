"""ctypes mirrors of the structs declared in include/hvvr_c.h.

The layouts are byte-compatible with the reference's public types (Sample, ShadingVertex,
PrecomputedTriangleShade, TopologyNode, SimpleMaterial, LightUnion, transform); numpy
structured dtypes with the same layout are provided for bulk arrays.
"""
import ctypes as C

import numpy as np

HVVR_OK = 0
HVVR_ERR_INVALID = 1
HVVR_ERR_NOT_FOUND = 2
HVVR_ERR_CUDA = 3
HVVR_ERR_OOM = 4
HVVR_ERR_OVERFLOW = 5
HVVR_ERR_TIMEOUT = 6
HVVR_ERR_STATE = 7

HVVR_LIGHT_NONE, HVVR_LIGHT_DIRECTIONAL, HVVR_LIGHT_POINT, HVVR_LIGHT_SPOT = 0, 1, 2, 3
HVVR_MEMORY_CPU, HVVR_MEMORY_CUDA = 0, 1
HVVR_MODE_DEFERRED_MSAA_RESOLVE, HVVR_MODE_FOVEATED_POLAR = 0, 1
HVVR_FP_FMA, HVVR_FP_STRICT = 0, 1
HVVR_SETUP_DEVICE, HVVR_SETUP_HOST = 0, 1
HVVR_BVH_HOST, HVVR_BVH_DEVICE = 0, 1
HVVR_MSAA_SPIRAL, HVVR_MSAA_ROTATED_GRID = 0, 1
HVVR_CAPTURE_HITS = 1


class Vec2(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float)]


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class Vec4(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("w", C.c_float)]


class FloatRect(C.Structure):
    _fields_ = [("lower", Vec2), ("upper", Vec2)]


class ThinLens(C.Structure):
    _fields_ = [("radius", C.c_float), ("focal_distance", C.c_float)]


class Transform(C.Structure):
    _fields_ = [("rotation", Vec4), ("translation", Vec3), ("scale", C.c_float)]


class LightDirectional(C.Structure):
    _fields_ = [("direction", Vec3), ("power", Vec3)]


class LightPoint(C.Structure):
    _fields_ = [("position", Vec3), ("falloff_end", C.c_float), ("color", Vec3), ("falloff_scale", C.c_float)]


class LightSpot(C.Structure):
    _fields_ = [("position", Vec3), ("falloff_end", C.c_float), ("direction", Vec3), ("falloff_scale", C.c_float),
                ("color", Vec3), ("cos_outer_angle", C.c_float), ("cos_angle_scale", C.c_float)]


class _LightU(C.Union):
    _fields_ = [("directional", LightDirectional), ("point", LightPoint), ("spot", LightSpot)]


class LightUnion(C.Structure):
    _fields_ = [("type", C.c_uint32), ("u", _LightU)]


class MeshData(C.Structure):
    _fields_ = [("verts", C.c_void_p), ("vert_count", C.c_uint32),
                ("tri_shade", C.c_void_p), ("tri_count", C.c_uint32),
                ("nodes", C.c_void_p), ("node_count", C.c_uint32),
                ("materials", C.c_void_p), ("material_count", C.c_uint32)]


# TextureFormat (libraries/hvvr/raycaster/texture.h:16-27) and its texel sizes (getTextureSize)
(HVVR_TEXTURE_NONE, HVVR_TEXTURE_RGBA8_UNORM_SRGB, HVVR_TEXTURE_RGBA8_UNORM, HVVR_TEXTURE_RGBA16_UNORM,
 HVVR_TEXTURE_RGBA32_FLOAT, HVVR_TEXTURE_RGBA16_FLOAT, HVVR_TEXTURE_R11G11B10_FLOAT, HVVR_TEXTURE_R32_FLOAT) = range(8)
TEXTURE_ELEMENT_SIZE = {1: 4, 2: 4, 3: 8, 4: 16, 5: 8, 6: 4, 7: 4}


class TextureData(C.Structure):
    _fields_ = [("data", C.c_void_p), ("format", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32),
                ("stride_elements", C.c_uint32)]


class ImageDesc(C.Structure):
    _fields_ = [("pixel_format", C.c_uint32), ("memory_type", C.c_uint32), ("data", C.c_void_p),
                ("width", C.c_uint32), ("height", C.c_uint32), ("stride", C.c_uint64)]


class Spec(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("thread_count", C.c_uint32),
                ("foveated_degree_tracking_error", C.c_float), ("foveated_max_fov_degrees", C.c_float),
                ("foveated_mar_slope", C.c_float), ("foveated_foveal_mar_degrees", C.c_float),
                ("output_format", C.c_uint32), ("output_to_3d_api", C.c_uint32),
                ("fp_mode", C.c_uint32), ("tri_index_capacity", C.c_uint64), ("device", C.c_int),
                ("sample_setup", C.c_uint32), ("bvh_build", C.c_uint32)]


class TileCullArgs(C.Structure):
    """hvvr_tile_cull_args: device inputs of hvvr_tile_cull_static."""
    _fields_ = [("nodes", C.c_void_p), ("node_count", C.c_uint32), ("tile_rays", C.c_void_p),
                ("tile_count", C.c_uint32), ("block_stacks", C.c_void_p), ("block_sizes", C.c_void_p),
                ("camera_to_world", Transform), ("tile_stack_entries", C.c_uint32)]


class BatchConfig(C.Structure):
    """hvvr_batch_config: knobs of a frame batch (set by hand or by hvvr_batch_autotune)."""
    _fields_ = [("tile_cull_warps", C.c_uint32), ("heavy_divisor", C.c_uint32), ("tri_index_capacity", C.c_uint64),
                ("use_graph", C.c_uint32), ("frame_ms", C.c_float), ("tile_stack_entries", C.c_uint32),
                ("timing", C.c_uint32), ("pipeline", C.c_uint32), ("tile_cull_ctas_per_sm", C.c_uint32),
                ("tile_cull_persistent", C.c_uint32), ("stream_tiles", C.c_uint32)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("slots", C.c_uint32), ("max_batch_views", C.c_uint32),
                ("slot_list_capacity", C.c_uint64), ("tile_cull_warps", C.c_uint32), ("heavy_divisor", C.c_uint32),
                ("min_batch_views", C.c_uint32), ("max_wait_ms", C.c_float), ("latency_slots", C.c_uint32),
                ("tile_cull_ctas_per_sm", C.c_uint32), ("latency_isolation", C.c_uint32)]


class Request(C.Structure):
    _fields_ = [("view", C.c_uint32), ("msaa", C.c_uint32), ("camera_to_world", Transform),
                ("memory_type", C.c_uint32), ("output", C.c_void_p), ("tag", C.c_uint64), ("priority", C.c_uint32)]


class Completion(C.Structure):
    _fields_ = [("id", C.c_uint64), ("tag", C.c_uint64), ("status", C.c_int), ("batch_views", C.c_uint32),
                ("submit_ms", C.c_double), ("dispatch_ms", C.c_double), ("done_ms", C.c_double),
                ("priority", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("batches", C.c_uint64), ("queued", C.c_uint64), ("in_flight", C.c_uint64),
                ("instances", C.c_uint64), ("hbm_used", C.c_uint64), ("hbm_peak", C.c_uint64),
                ("mean_batch_views", C.c_double), ("evicted", C.c_uint64), ("batch_gpu_ms", C.c_double),
                ("dispatch_host_ms", C.c_double)]


# numpy layouts of the bulk arrays
SAMPLE_DTYPE = np.dtype([("pixel", "<u4", 2), ("position", "<f4", 2), ("minor", "<f4", 2), ("major", "<f4")])
VERTEX_DTYPE = np.dtype([("pos", "<f4", 3), ("normal", "<u2", 4), ("uv", "<f4", 2), ("pad", "<u4")])
TRISHADE_DTYPE = np.dtype([("indices", "<u4", 3), ("material", "<u4")])
TOPO_DTYPE = np.dtype([("leaf_mask", "<u4"), ("data", "<u4", 7)])
MATERIAL_DTYPE = np.dtype([("emissive", "<f4", 4), ("diffuse", "<f4", 4), ("specular", "<f4", 4),
                           ("glossiness", "<f4"), ("opacity", "<f4"), ("code", "<u8")])
NODE_DTYPE = np.dtype([("bounds", "<f4", (6, 4)), ("leaf_mask", "<u4"), ("tri", "<u4", 5), ("pad", "<u4", 2)])

assert SAMPLE_DTYPE.itemsize == 28
assert VERTEX_DTYPE.itemsize == 32
assert TRISHADE_DTYPE.itemsize == 16
assert TOPO_DTYPE.itemsize == 32
assert MATERIAL_DTYPE.itemsize == 64
assert NODE_DTYPE.itemsize == 128
assert C.sizeof(LightUnion) == 56
assert C.sizeof(Transform) == 32


def ptr(a):
    """ctypes void pointer to a C-contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


def transform(rotation=(0.0, 0.0, 0.0, 1.0), translation=(0.0, 0.0, 0.0), scale=1.0):
    t = Transform()
    t.rotation = Vec4(*[float(v) for v in rotation])
    t.translation = Vec3(*[float(v) for v in translation])
    t.scale = float(scale)
    return t
