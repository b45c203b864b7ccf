"""hvvr_tile_cull_static: the tile cull for callers that may not allocate device memory.

A render thread with a frame deadline, or a plugin whose host application owns every device
allocation, cannot let the library call cudaMalloc. hvvr_tile_cull_static takes the caller's
device inputs and outputs and keeps its working lists in a fixed area compiled into the
library. This file checks, through the C ABI, that two calls in a row return exactly the
per-tile triangle lists that the regular render path produced for the same frame (integer
output, so the tolerance is zero), and that work beyond the fixed limit is refused.
It is collected last so that a run stopping at the first failure has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

from helpers import render_gpu, scene

pytestmark = pytest.mark.gpu


def _call(args, counts_ptr, idx_ptr, cap, total):
    return hv.lib().hvvr_tile_cull_static(C.c_void_p(C.addressof(args)), counts_ptr, idx_ptr, cap, C.byref(total),
                                          None)


def test_static_cull_matches_render_path(oracle):
    import torch
    sc = scene("c1")
    w, h = 640, 480
    smp = scenes.grid_samples(w, h)
    xf = scenes.camera_transform(eye=(1.0, 1.5, 8.0), target=(0.0, 0.2, 0.0))
    rc, cam = render_gpu(sc, smp, w, h, 1, cam_xf=xf, capture=False)
    counts_ref, idx_ref = cam.tile_lists()
    nodes = rc.scene_nodes()
    sizes, entries = cam.block_stacks()
    rays = oracle.render(sc, smp, xf, scenes.viewport_for(w, h), w, h, 1, want=("tile_rays",)).tile_rays
    dev = torch.device("cuda")
    d_nodes = torch.from_numpy(nodes.view(np.uint8).copy()).to(dev)
    d_rays = torch.from_numpy(rays.copy()).to(dev)
    d_stacks = torch.from_numpy(entries.view(np.int32).copy()).to(dev)
    d_sizes = torch.from_numpy(sizes.view(np.int32).copy()).to(dev)
    tiles = len(counts_ref)
    cap = len(idx_ref) + 4096
    d_counts = torch.empty(tiles, dtype=torch.int32, device=dev)
    d_idx = torch.empty(cap, dtype=torch.int32, device=dev)
    args = _abi.TileCullArgs(d_nodes.data_ptr(), len(nodes), d_rays.data_ptr(), tiles, d_stacks.data_ptr(),
                             d_sizes.data_ptr(), xf)
    for _ in range(2):
        d_counts.fill_(-1)
        d_idx.fill_(-1)
        torch.cuda.synchronize()
        total = C.c_uint64(0)
        rc_ = _call(args, C.c_void_p(d_counts.data_ptr()), C.c_void_p(d_idx.data_ptr()), cap, total)
        assert rc_ == hv.HVVR_OK, hv.lib().hvvr_last_error().decode()
        counts = d_counts.cpu().numpy().view(np.uint32)
        idx = d_idx.cpu().numpy().view(np.uint32)
        assert total.value == len(idx_ref)
        assert np.array_equal(counts, counts_ref)
        assert np.array_equal(idx[: total.value], idx_ref)
        assert (idx[total.value:] == 0xFFFFFFFF).all()
    # an output buffer smaller than the lists is reported, with the total, and counts still written
    total = C.c_uint64(0)
    rc_ = _call(args, C.c_void_p(d_counts.data_ptr()), C.c_void_p(d_idx.data_ptr()), 16, total)
    assert rc_ == _abi.HVVR_ERR_OVERFLOW and total.value == len(idx_ref)
    # work beyond the fixed limit is refused before anything runs
    big = _abi.TileCullArgs(d_nodes.data_ptr(), len(nodes), d_rays.data_ptr(), 65536 + 64, d_stacks.data_ptr(),
                            d_sizes.data_ptr(), xf)
    rc_ = _call(big, C.c_void_p(d_counts.data_ptr()), C.c_void_p(d_idx.data_ptr()), cap, total)
    assert rc_ == _abi.HVVR_ERR_INVALID and b"65536" in hv.lib().hvvr_last_error()
    rc.close()
