"""Batched frames: the cameras of several raycasters (different scenes, sizes and MSAA rates)
rendered as one frame, over several frames so that the later ones replay a CUDA graph and
cull the slowest tiles on their own streams. Every view must match the oracle exactly, as the
same camera rendered on its own does (same lists, hit IDs, depth, G-buffer; colour <= 1 LSB).
"""
import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

from helpers import list_mismatch, render_oracle, scene

pytestmark = pytest.mark.gpu


def _check_view(oracle, sc, cam, smp, w, h, msaa, xf):
    fo = render_oracle(oracle, sc, smp, w, h, msaa, cam_xf=xf)
    counts, idx = cam.tile_lists()
    assert list_mismatch(counts, idx, fo.tile_counts, fo.tile_indices) == 0
    ids, depth = cam.hits()
    assert np.array_equal(ids, fo.hit_ids), "hit IDs differ at %d subsamples" % int((ids != fo.hit_ids).sum())
    assert np.array_equal(depth.view(np.uint32), fo.depth.view(np.uint32)), "depth differs"
    col = cam.sample_colors()
    d = np.abs(col.view(np.uint8).astype(np.int32) - fo.colors.view(np.uint8).astype(np.int32))
    assert d.max() <= 1
    img = cam.image
    di = np.abs(img.view(np.uint8).astype(np.int32) - fo.image.view(np.uint8).astype(np.int32))
    assert di.max() <= 1


def _make_rc(sc):
    rc = hv.Raycaster()
    rc.create_model(sc)
    for l in sc.lights:
        rc.create_light(l)
    return rc


def _add_cam(rc, w, h, kind, msaa):
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h)
    smp = scenes.grid_samples(w, h) if kind == "grid" else scenes.barrel_samples(w, h)
    cam.set_samples(smp, 1)
    cam.set_msaa(msaa)
    cam.set_capture(hv.HVVR_CAPTURE_HITS)
    return cam, smp


@pytest.mark.parametrize("use_graph", [1, 0])
def test_batch_two_scenes_mixed_rates(oracle, use_graph):
    sc_a, sc_b = scene("c1"), scene("small")
    rc_a, rc_b = _make_rc(sc_a), _make_rc(sc_b)
    views = []  # (raycaster scene, camera, samples, w, h, msaa)
    for (rc, sc, w, h, kind, msaa) in [(rc_a, sc_a, 320, 288, "barrel", 4), (rc_a, sc_a, 256, 192, "grid", 1),
                                       (rc_b, sc_b, 160, 176, "barrel", 8), (rc_b, sc_b, 200, 120, "grid", 4)]:
        cam, smp = _add_cam(rc, w, h, kind, msaa)
        views.append((sc, cam, smp, w, h, msaa))
    batch = hv.Batch([rc_a, rc_b], hv.batch_config(use_graph=use_graph, tri_index_capacity=1 << 22))
    path = [((0.0, 2.0, 10.0), (0.0, 0.0, 0.0)), ((2.5, 1.0, 7.0), (-1.0, 0.5, 0.0)),
            ((-3.0, 3.0, 8.0), (1.0, 0.0, -2.0)), ((1.0, 1.5, 9.0), (0.0, 0.2, 0.0))]
    for eye, target in path:
        xfs = []
        for k, (sc, cam, smp, w, h, msaa) in enumerate(views):
            xf = scenes.camera_transform(eye=(eye[0] + 0.25 * k, eye[1], eye[2]), target=target)
            cam.set_camera_to_world(xf)
            xfs.append(xf)
        batch.render()
        t = batch.timings()
        assert t[0] > 0
        for (sc, cam, smp, w, h, msaa), xf in zip(views, xfs):
            _check_view(oracle, sc, cam, smp, w, h, msaa, xf)
    batch.close()
    rc_a.close()
    rc_b.close()


def test_batch_matches_single_view_and_autotune():
    """A camera in a batch gives the same bits as the camera rendered by its own raycaster,
    before and after the autotuner has changed the batch configuration."""
    sc = scene("small")
    w, h = 160, 176
    rc = _make_rc(sc)
    cam, smp = _add_cam(rc, w, h, "barrel", 8)
    other, _ = _add_cam(rc, 96, 64, "grid", 2)
    xf = scenes.camera_transform(eye=(1.0, 2.5, 8.0), target=(0.0, 0.0, 0.0))
    cam.set_camera_to_world(xf)
    other.set_camera_to_world(xf)
    rc.render()
    ref_ids, ref_depth = cam.hits()
    ref_img = cam.image.copy()
    batch = hv.Batch([rc])
    cfg = batch.autotune(frames=2)
    assert cfg.tile_cull_warps in (1, 2, 4, 8) and cfg.frame_ms > 0
    assert cfg.tri_index_capacity >= 1 << 20
    for _ in range(3):
        batch.render()
        ids, depth = cam.hits()
        assert np.array_equal(ids, ref_ids)
        assert np.array_equal(depth.view(np.uint32), ref_depth.view(np.uint32))
        assert np.array_equal(cam.image, ref_img)
    batch.close()
    rc.close()


def test_animated_refit_matches_oracle(oracle):
    """Device-side vertex animation (10% of the vertices, one contiguous range) followed by the
    GPU refit: refit BVH, lists and hits match the oracle run on the animated mesh, over frames."""
    import copy
    import torch
    from hvvr_b200 import workloads
    sc = scene("small")
    w, h = 160, 176
    rc = _make_rc(sc)
    model = rc.models[0]
    cam, smp = _add_cam(rc, w, h, "barrel", 4)
    xf = scenes.camera_transform(eye=(0.5, 2.0, 9.0), target=(0.0, 0.0, 0.0))
    cam.set_camera_to_world(xf)
    rc.render()
    anim = workloads.Animator(torch, model, sc)
    for t in (0.3, 1.7, 2.9):
        anim.step(t)
        rc.render()
        moved = copy.copy(sc)
        moved.verts = anim.host_vertices(sc)
        fo = render_oracle(oracle, moved, smp, w, h, 4, cam_xf=xf)
        assert np.array_equal(rc.scene_nodes().view(np.uint8), fo.nodes.view(np.uint8)), "refit BVH differs"
        counts, idx = cam.tile_lists()
        assert list_mismatch(counts, idx, fo.tile_counts, fo.tile_indices) == 0
        ids, depth = cam.hits()
        assert np.array_equal(ids, fo.hit_ids)
        assert np.array_equal(depth.view(np.uint32), fo.depth.view(np.uint32))
    rc.close()


@pytest.mark.parametrize("pipeline", [1, 0, 2])
def test_stack_retry_pass_matches_oracle(oracle, pipeline):
    """A 16-entry main-pass stack sends every tile whose sorted stack grows deeper to the retry
    pass (4096 entries); the lists, hits and colours must not change. With the cull -> shade
    pipeline the retried tiles are skipped by the pipelined shade and shaded by the retry list's
    own launch; a streamed tile (every tile streams in the third run) may already be in its shade's
    hands when its stack overflows, and the retry launches cull and shade it again after that."""
    sc = scene("c1")
    w, h = 320, 288
    rc = _make_rc(sc)
    cam, smp = _add_cam(rc, w, h, "barrel", 4)
    xf = scenes.camera_transform(eye=(3.0, 1.2, 6.0), target=(-2.0, 0.3, -1.0))
    cam.set_camera_to_world(xf)
    extra = {"stream_tiles": 1 << 20} if pipeline == 2 else {}
    batch = hv.Batch(cameras=[cam], config=hv.batch_config(tile_stack_entries=16, tri_index_capacity=1 << 22,
                                                           pipeline=min(pipeline, 1), **extra))
    for _ in range(3):
        batch.render()
        st = batch.stats()
        assert st["retried_tiles"] > 0 and st["status"] == 0
        _check_view(oracle, sc, cam, smp, w, h, 4, xf)
    batch.close()
    rc.close()


@pytest.mark.parametrize("use_graph", [1, 0])
def test_pipelined_and_split_frames_agree(oracle, use_graph):
    """The cull -> shade pipeline (default) against the split path (heavy part on its own stream,
    cull before shade), against the pipeline with a non-persistent tile cull (a warp per tile,
    as a served throughput batch runs) and against the pipeline with every tile streaming its list
    chunk by chunk to its shade, on a frame batch with three MSAA rates over two scenes, over
    three frames (the second and later ones cull in the previous frame's cost order): identical
    lists, hits and colours, and equal to the oracle."""
    sa, sb = scene("c1"), scene("small")
    rc_a, rc_b = _make_rc(sa), _make_rc(sb)
    views = [(rc_a, sa, 256, 224, "barrel", 8), (rc_a, sa, 192, 160, "grid", 1), (rc_b, sb, 160, 176, "barrel", 4)]
    cams = []
    for k, (rc, sc, w, h, kind, msaa) in enumerate(views):
        cam, smp = _add_cam(rc, w, h, kind, msaa)
        xf = scenes.camera_transform(eye=(0.4 * k, 2.0, 10.0), target=(0.0, 0.2 * k, 0.0))
        cam.set_camera_to_world(xf)
        cams.append((cam, sc, smp, w, h, msaa, xf))
    results = {}
    modes = (("pipelined", 1, 1, 0), ("split", 0, 1, 0), ("one tile per warp", 1, 0, 0), ("streamed", 1, 1, 1 << 20))
    for mode, pipeline, persistent, stream in modes:
        batch = hv.Batch([rc_a, rc_b], hv.batch_config(use_graph=use_graph, tri_index_capacity=1 << 22,
                                                       pipeline=pipeline, timing=1, tile_cull_warps=1 + pipeline,
                                                       tile_cull_persistent=persistent, stream_tiles=stream))
        for frame in range(3):
            batch.render()
            assert batch.stats()["status"] == 0
        parts = batch.part_times()
        assert parts is not None
        out = []
        for cam, sc, smp, w, h, msaa, xf in cams:
            counts, idx = cam.tile_lists()
            ids, depth = cam.hits()
            out.append((counts, idx, ids, depth, cam.sample_colors()))
            if mode == "pipelined":  # read while the batch that holds the lists is open
                _check_view(oracle, sc, cam, smp, w, h, msaa, xf)
        results[mode] = out
        batch.close()
    # streaming starts at a list's second chunk: some tiles here have more than one
    assert max(int(o[0].max()) for o in results["streamed"]) > 128
    for other in ("split", "one tile per warp", "streamed"):
        for a, b in zip(results["pipelined"], results[other]):
            for x, y in zip(a, b):
                assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), other
    rc_a.close()
    rc_b.close()


def test_batch_mixes_thin_lens_and_pinhole_views(oracle):
    """Thin-lens and pinhole views of the same rate in one batch run as separate kernels
    (rate classes); both match the oracle, over frames (graph replay)."""
    sc_a, sc_b = scene("c1"), scene("small")
    rc_a, rc_b = _make_rc(sc_a), _make_rc(sc_b)
    views = []
    for (rc, sc, w, h, kind, msaa, lens) in [(rc_a, sc_a, 192, 160, "barrel", 4, (0.06, 9.0)),
                                             (rc_a, sc_a, 128, 96, "grid", 4, None),
                                             (rc_b, sc_b, 160, 176, "barrel", 8, (0.1, 6.0)),
                                             (rc_b, sc_b, 96, 96, "grid", 1, (0.03, 10.0))]:
        cam, smp = _add_cam(rc, w, h, kind, msaa)
        if lens:
            cam.set_lens(*lens)
        views.append((sc, cam, smp, w, h, msaa, lens))
    batch = hv.Batch([rc_a, rc_b], hv.batch_config(tri_index_capacity=1 << 22))
    for eye in ((0.0, 2.0, 10.0), (2.0, 1.5, 8.0), (-1.0, 2.5, 9.0)):
        xfs = []
        for k, (sc, cam, smp, w, h, msaa, lens) in enumerate(views):
            xf = scenes.camera_transform(eye=(eye[0] + 0.2 * k, eye[1], eye[2]), target=(0.0, 0.0, 0.0))
            cam.set_camera_to_world(xf)
            xfs.append(xf)
        batch.render()
        for (sc, cam, smp, w, h, msaa, lens), xf in zip(views, xfs):
            fo = render_oracle(oracle, sc, smp, w, h, msaa, cam_xf=xf, lens=lens)
            counts, idx = cam.tile_lists()
            assert list_mismatch(counts, idx, fo.tile_counts, fo.tile_indices) == 0
            ids, depth = cam.hits()
            assert np.array_equal(ids, fo.hit_ids)
            assert np.array_equal(depth.view(np.uint32), fo.depth.view(np.uint32))
            d = np.abs(cam.image.view(np.uint8).astype(np.int32) - fo.image.view(np.uint8).astype(np.int32))
            assert d.max() <= 1
    batch.close()
    rc_a.close()
    rc_b.close()


@pytest.mark.parametrize("stream", [0, 1 << 20])
def test_list_pool_overflow_is_reported(oracle, stream):
    """Tile lists that outgrow the triangle-index pool are reported (HVVR_ERR_OVERFLOW) instead of
    being returned cut, with the cull -> shade pipeline and with every tile streaming its list (a
    streamed list ends after its last stored chunk, and its shade ends there with it); a batch with
    a pool large enough then renders the same view exactly."""
    sc = scene("c1")
    rc = _make_rc(sc)
    w, h = 256, 224
    cam, smp = _add_cam(rc, w, h, "barrel", 8)
    xf = scenes.camera_transform(eye=(0.0, 2.0, 10.0), target=(0.0, 0.0, 0.0))
    cam.set_camera_to_world(xf)
    small = hv.Batch(cameras=[cam], config=hv.batch_config(tri_index_capacity=4096, stream_tiles=stream))
    with pytest.raises(hv.HvvrError) as err:
        small.render()
        small.synchronize()
    assert err.value.code == _abi.HVVR_ERR_OVERFLOW
    small.close()
    big = hv.Batch(cameras=[cam], config=hv.batch_config(tri_index_capacity=1 << 22, stream_tiles=stream))
    for _ in range(2):
        big.render()
    big.synchronize()
    _check_view(oracle, sc, cam, smp, w, h, 8, xf)
    big.close()
    rc.close()
