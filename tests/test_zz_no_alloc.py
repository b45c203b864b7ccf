"""hvvr_tile_cull_static: the tile cull for callers that may not allocate device memory.

A render thread with a frame deadline, or a plugin whose host application owns every device
allocation, cannot let the library call cudaMalloc. hvvr_tile_cull_static takes the caller's
device inputs and outputs and keeps its working lists in a fixed area compiled into the
library. This file checks, through the C ABI, that two calls in a row return exactly the
per-tile triangle lists that the regular render path produced for the same frame (integer
output, so the tolerance is zero), that the second call leaves the device's free memory
unchanged (cudaMemGetInfo), that malformed inputs and work beyond the fixed limits are refused,
that the retry pass (tiles whose traversal stack outgrows the main pass's) gives the same lists
from the fixed area, and that lists longer than the fixed area are reported rather than cut.
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
    for k in range(2):
        d_counts.fill_(-1)
        d_idx.fill_(-1)
        torch.cuda.synchronize()
        total = C.c_uint64(0)
        free_before, _ = torch.cuda.mem_get_info()  # cudaMemGetInfo
        rc_ = _call(args, C.c_void_p(d_counts.data_ptr()), C.c_void_p(d_idx.data_ptr()), cap, total)
        free_after, _ = torch.cuda.mem_get_info()
        assert rc_ == hv.HVVR_OK, hv.lib().hvvr_last_error().decode()
        if k == 1:  # the first call may load the library's kernels; the second allocates nothing at all
            assert free_after == free_before, (free_before, free_after)
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
    # malformed inputs (built on the CPU) are checked on the device before the cull runs: a block
    # stack longer than 64 entries, a stack entry naming a node past node_count, a child offset
    # pointing outside the node array
    bad_sizes = sizes.copy()
    bad_sizes[int(np.argmax(sizes))] = 65
    bad_entries = entries.copy()
    b0 = int(np.argmax(sizes))
    bad_entries[b0, 0, 2] = len(nodes) + 5
    for name, e_arr, s_arr in (("size", entries, bad_sizes), ("entry", bad_entries, sizes), ("child", entries, sizes)):
        if name == "child":
            raw = nodes.view(np.uint32).reshape(len(nodes), 32).copy()
            first_internal = int(np.nonzero((raw[:, 24] & 1) == 0)[0][0])
            raw[first_internal, 26] = 0x40000000  # child offset of slot 0 far past the array
            n_dev = torch.from_numpy(raw.view(np.uint8).reshape(-1).copy()).to(dev)
        else:
            n_dev = d_nodes
        e_dev = torch.from_numpy(e_arr.view(np.int32).copy()).to(dev)
        s_dev = torch.from_numpy(s_arr.view(np.int32).copy()).to(dev)
        a = _abi.TileCullArgs(n_dev.data_ptr(), len(nodes), d_rays.data_ptr(), tiles, e_dev.data_ptr(),
                              s_dev.data_ptr(), xf)
        rc_ = _call(a, C.c_void_p(d_counts.data_ptr()), C.c_void_p(d_idx.data_ptr()), cap, total)
        assert rc_ == _abi.HVVR_ERR_INVALID and b"malformed" in hv.lib().hvvr_last_error(), name
    # the well-formed inputs still cull after the rejected calls
    rc_ = _call(args, C.c_void_p(d_counts.data_ptr()), C.c_void_p(d_idx.data_ptr()), cap, total)
    assert rc_ == hv.HVVR_OK and total.value == len(idx_ref)
    # a 16-entry main-pass stack sends most tiles through the retry pass (4096-entry stacks in the
    # same fixed area): the lists are unchanged; a stack size outside [8, 256] is refused
    small = _abi.TileCullArgs(d_nodes.data_ptr(), len(nodes), d_rays.data_ptr(), tiles, d_stacks.data_ptr(),
                              d_sizes.data_ptr(), xf, 16)
    d_counts.fill_(-1)
    d_idx.fill_(-1)
    rc_ = _call(small, C.c_void_p(d_counts.data_ptr()), C.c_void_p(d_idx.data_ptr()), cap, total)
    assert rc_ == hv.HVVR_OK, hv.lib().hvvr_last_error().decode()
    assert total.value == len(idx_ref)
    assert np.array_equal(d_counts.cpu().numpy().view(np.uint32), counts_ref)
    assert np.array_equal(d_idx.cpu().numpy().view(np.uint32)[: total.value], idx_ref)
    small.tile_stack_entries = 5
    rc_ = _call(small, C.c_void_p(d_counts.data_ptr()), C.c_void_p(d_idx.data_ptr()), cap, total)
    assert rc_ == _abi.HVVR_ERR_INVALID and b"tile_stack_entries" in hv.lib().hvvr_last_error()
    rc.close()


def test_static_cull_reports_list_overflow():
    """Lists longer than the fixed area (7,864,320 entries) are reported as HVVR_ERR_OVERFLOW, not
    truncated silently: one eye of the 995,072-triangle stereo benchmark frame has about 8.6M
    list entries."""
    import torch
    sc = scene("c2")
    w, h = 1080, 1200
    smp = scenes.barrel_samples(w, h)
    xf = scenes.stereo_eyes(0.064)[0]
    rc, cam = render_gpu(sc, smp, w, h, 8, cam_xf=xf, capture=False)
    counts_ref, idx_ref = cam.tile_lists()
    assert len(idx_ref) > 7864320
    nodes = rc.scene_nodes()
    sizes, entries = cam.block_stacks()
    import pyoracle
    rays = pyoracle.Oracle().render(sc, smp, xf, scenes.viewport_for(w, h), w, h, 8, want=("tile_rays",)).tile_rays
    dev = torch.device("cuda")
    d_nodes = torch.from_numpy(nodes.view(np.uint8).copy()).to(dev)
    d_rays = torch.from_numpy(rays.copy()).to(dev)
    d_stacks = torch.from_numpy(entries.view(np.int32).copy()).to(dev)
    d_sizes = torch.from_numpy(sizes.view(np.int32).copy()).to(dev)
    tiles = len(counts_ref)
    d_counts = torch.empty(tiles, dtype=torch.int32, device=dev)
    args = _abi.TileCullArgs(d_nodes.data_ptr(), len(nodes), d_rays.data_ptr(), tiles, d_stacks.data_ptr(),
                             d_sizes.data_ptr(), xf)
    total = C.c_uint64(0)
    rc_ = _call(args, C.c_void_p(d_counts.data_ptr()), None, 0, total)
    assert rc_ == _abi.HVVR_ERR_OVERFLOW and b"7,864,320" in hv.lib().hvvr_last_error()
    rc.close()
