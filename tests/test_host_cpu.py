"""Host-side pieces that need no GPU: the C-ABI library's exports, struct layouts, the BVH
builder against the reference's GenerateTopology, and refusal without a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

from conftest import ROOT, have_gpu
from golden_io import load, names


def header_functions():
    src = open(os.path.join(ROOT, "include", "hvvr_c.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hvvr_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    declared = header_functions()
    assert len(declared) >= 40
    for name in declared:
        assert hasattr(hv.lib(), name), name
    assert sorted(hv.EXPORTED) == declared


def test_struct_sizes_match_reference_layouts():
    assert _abi.SAMPLE_DTYPE.itemsize == 28         # Sample
    assert _abi.VERTEX_DTYPE.itemsize == 32         # ShadingVertex
    assert _abi.TRISHADE_DTYPE.itemsize == 16       # PrecomputedTriangleShade
    assert _abi.TOPO_DTYPE.itemsize == 32           # TopologyNode
    assert _abi.MATERIAL_DTYPE.itemsize == 64       # SimpleMaterial
    assert _abi.NODE_DTYPE.itemsize == 128          # BVHNode
    assert C.sizeof(_abi.LightUnion) == 56          # LightUnion
    assert C.sizeof(_abi.Transform) == 32           # transform


@pytest.mark.parametrize("name", names())
def test_topology_builder_matches_reference(name):
    g, *_ = load(name)
    sc = scenes.Scene(g["in_verts"].copy(), g["in_tris"].copy(), None, [])
    hv.generate_topology(sc)
    assert np.array_equal(sc.nodes, g["topo_nodes"])
    assert np.array_equal(sc.tri_shade, g["topo_tris"])
    assert np.array_equal(sc.verts, g["topo_verts"])


def test_grid_samples_match_generator():
    a = hv.grid_samples(37, 23)
    b = scenes.grid_samples(37, 23)
    assert a.tobytes() == b.tobytes()


def test_bad_arguments_are_reported_not_fatal():
    sc = scenes.make_scene(4, 2, 1)
    nodes = np.zeros(4, dtype=_abi.TOPO_DTYPE)
    cnt = C.c_uint32(0)
    bad = sc.tri_shade.copy()
    bad["indices"][0, 0] = 10 ** 6
    rc = hv.lib().hvvr_generate_topology(sc.verts.ctypes.data, len(sc.verts), bad.ctypes.data, len(bad),
                                         nodes.ctypes.data, len(nodes), C.byref(cnt))
    assert rc == _abi.HVVR_ERR_INVALID


@pytest.mark.skipif(have_gpu(), reason="checks the no-device path")
def test_no_device_is_an_error_not_a_fallback():
    with pytest.raises(hv.HvvrError) as e:
        hv.Raycaster()
    assert e.value.code == _abi.HVVR_ERR_CUDA


def test_batch_config_defaults():
    """hvvr_batch_config_default: the configuration the stereo frame was tuned on (one-warp
    persistent tile-cull CTAs, the slowest eighth of the tiles as the heavy part, the cull ->
    shade pipeline, CUDA graph replay)."""
    cfg = hv.batch_config()
    assert (cfg.tile_cull_warps, cfg.heavy_divisor, cfg.pipeline, cfg.tile_cull_persistent) == (1, 8, 1, 1)
    assert (cfg.use_graph, cfg.timing, cfg.tile_stack_entries, cfg.tile_cull_ctas_per_sm) == (1, 0, 0, 0)
    assert cfg.stream_tiles == 400
    assert C.sizeof(_abi.BatchConfig) == 48

