"""Foveated polar mode: the raycaster's polar sample set (pinned against the reference by
test_foveated_setup.py) rendered in eye space with the per-frame eye transform and tile cull
planes. Lists, hit IDs and depth must equal the oracle run on the same beams, frusta, matrix
and planes; colours within 1 LSB; the per-sample view depth (TMaxBuffer) bit-exact."""
import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

from helpers import list_mismatch, scene

pytestmark = pytest.mark.gpu

PATTERN = (1.0, 35.0, 0.03, 0.06)  # degree tracking error, max FOV, MAR slope, foveal MAR


def _foveated_rc(sc, fp_mode=hv.HVVR_FP_FMA):
    spec = hv.foveated_spec(*PATTERN, mode=_abi.HVVR_MODE_FOVEATED_POLAR, fp_mode=fp_mode)
    rc = hv.Raycaster(spec=spec)
    rc.create_model(sc)
    for l in sc.lights:
        rc.create_light(l)
    return rc


@pytest.mark.parametrize("msaa,fp_mode", [(4, hv.HVVR_FP_FMA), (8, hv.HVVR_FP_STRICT), (1, hv.HVVR_FP_FMA)])
def test_foveated_eye_space_render_matches_oracle(oracle, msaa, fp_mode):
    sc = scene("c1")
    rc = _foveated_rc(sc, fp_mode)
    w, h = 320, 288
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h)
    cam.set_samples(scenes.grid_samples(w, h))
    cam.set_msaa(msaa)
    cam.set_capture(hv.HVVR_CAPTURE_HITS)
    polar = hv.polar_foveated_samples(hv.foveated_spec(*PATTERN))
    beams = np.zeros((polar["padded"], 9), np.float32)
    beams[: polar["valid"]] = polar["beams"]
    for eye, target, gaze in [((0.0, 2.0, 10.0), (0.0, 0.0, 0.0), (0.0, 0.0, -1.0)),
                              ((2.0, 1.5, 8.0), (-1.0, 0.3, 0.0), (0.2, -0.1, -0.97))]:
        cam.set_camera_to_world(scenes.camera_transform(eye=eye, target=target))
        cam.set_eye_dir(gaze)
        rc.render()
        m, planes, depth = cam.foveated_frame()
        assert np.isfinite(planes).all()
        fo = oracle.render_beams(sc, {"beams": beams, "tile_rays": polar["tile_rays"],
                                      "block_rays": polar["block_rays"], "batch_to_world": m, "cull_planes": planes},
                                 msaa, fp_mode=fp_mode)
        counts, idx = cam.tile_lists()
        assert list_mismatch(counts, idx, fo.tile_counts, fo.tile_indices) == 0
        assert (counts == 0).sum() > 0, "expected some tiles culled by the screen bounds"
        ids, d = cam.hits()
        assert np.array_equal(ids, fo.hit_ids)
        assert np.array_equal(d.view(np.uint32), fo.depth.view(np.uint32))
        assert np.array_equal(depth.view(np.uint32), fo.tmax.view(np.uint32))
        col = cam.sample_colors()
        dc = np.abs(col.view(np.uint8).astype(np.int32) - fo.colors.view(np.uint8).astype(np.int32))
        assert dc.max() <= 1
    rc.close()


def test_foveated_resolve_matches_oracle(oracle):
    """The resolve (polar textures, moments, temporal reprojection, eccentricity filters,
    contrast enhancement) over frames with camera and gaze motion, against the oracle run on the
    GPU's own sample colours and view depths with the GPU's previous result as the history. The
    GPU resolves through the texture unit with fast math, as the reference does (bit-exact against
    the reference's kernels, test below); the oracle restates it with a software texture unit and
    IEEE math, so the comparison is held to the bounds the texture unit's rounding allows: polar
    colour within 1 LSB, moments within 1/64 of full scale, the temporally filtered result within
    a few LSB, and the contrast-enhanced image (which scales the result's differences up to 9x)
    on average within 1.5 LSB. The per-frame matrices the GPU used must equal the host entry's
    (pinned against the reference by the CPU tests)."""
    sc = scene("c1")
    rc = _foveated_rc(sc)
    w, h = 320, 288
    vp = scenes.viewport_for(w, h)
    cam = rc.create_camera(vp)
    cam.set_render_target(w, h)
    samples = scenes.grid_samples(w, h)
    cam.set_samples(samples)
    cam.set_msaa(4)
    polar = hv.polar_foveated_samples(hv.foveated_spec(*PATTERN))
    valid = polar["valid"]
    sb = _abi.FloatRect()
    sb.lower.x, sb.lower.y = float(samples["position"][:, 0].min()), float(samples["position"][:, 1].min())
    sb.upper.x, sb.upper.y = float(samples["position"][:, 0].max()), float(samples["position"][:, 1].max())
    hist = np.zeros((h, w), np.uint32)
    history = None
    poses = [((0.0, 2.0, 10.0), (0.0, 0.0, -1.0)), ((0.15, 2.05, 9.9), (0.02, 0.01, -1.0)),
             ((0.3, 2.1, 9.8), (0.05, -0.02, -1.0)), ((0.3, 2.1, 9.8), (0.05, -0.02, -1.0))]
    for eye, gaze in poses:
        xf = scenes.camera_transform(eye=eye, target=(0.0, 0.0, 0.0))
        cam.set_camera_to_world(xf)
        cam.set_eye_dir(gaze)
        rc.render()
        m = hv.foveated_frame_matrices(xf, gaze, sb, vp, history)
        history = m["history"]
        s2e, e2p, res, hist_gpu = cam.foveated_resolve()
        assert np.array_equal(s2e.view(np.uint32), m["sample_to_eye"].view(np.uint32))
        assert np.array_equal(e2p.view(np.uint32), m["eye_to_sample_prev"].view(np.uint32))
        assert np.array_equal(hist_gpu, hist), "the frame did not read the previous frame's result"
        _, _, depth = cam.foveated_frame()
        colors = cam.sample_colors()
        fo = oracle.foveated_resolve(PATTERN, polar, colors[:valid], depth[:valid], w, h, s2e, e2p, hist)
        img = cam.image
        pcol, _, pmom = cam.polar_textures(polar["samples_per_ring"], polar["ring_count"])
        def diff(a, b):
            if a.dtype == np.uint16:
                return np.abs(a.astype(np.int32) - b.astype(np.int32))
            return np.abs(a.view(np.uint8).astype(np.int32) - b.view(np.uint8).astype(np.int32))
        dc, dm, dr, di = (diff(pcol, fo["polar_color"]), diff(pmom, fo["moments"]), diff(res, fo["result"]),
                          diff(img, fo["image"]))
        assert dc.max() <= 1, ("polar colour", int(dc.max()))
        assert dm.max() <= 1024, ("moments", int(dm.max()))
        assert dr.max() <= 8 and (dr > 1).mean() <= 0.005, ("result", int(dr.max()), float((dr > 1).mean()))
        assert di.mean() <= 1.5 and (di > 1).mean() <= 0.2, ("image", float(di.mean()), float((di > 1).mean()))
        hist = res
    assert (img >> 24).min() >= 254 and (img & 0xFFFFFF).any()
    rc.close()


@pytest.mark.skipif(not __import__("pyoracle").ReferenceGpu.available(), reason="oracle/_ref GPU library not built")
def test_foveated_resolve_against_reference_kernels():
    """The resolve against the reference's own kernels (gpu_foveated.cu built for this GPU by
    oracle/refshim/ref_gpu_foveated.cu) on the GPU's polar textures, matrices and history, over
    frames with camera and gaze motion: the polar textures (RemapPolarFoveatedKernel on the frame's
    sample colours and view depths), moments, temporally filtered result and final image
    bit-exact."""
    import pyoracle
    ref = pyoracle.ReferenceGpu()
    sc = scene("c1")
    rc = _foveated_rc(sc)
    w, h = 320, 288
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h)
    cam.set_samples(scenes.grid_samples(w, h))
    cam.set_msaa(4)
    polar = hv.polar_foveated_samples(hv.foveated_spec(*PATTERN))
    spr, rings = polar["samples_per_ring"], polar["ring_count"]
    stats = []
    for eye, gaze in [((0.0, 2.0, 10.0), (0.0, 0.0, -1.0)), ((0.15, 2.05, 9.9), (0.02, 0.01, -1.0)),
                      ((0.3, 2.1, 9.8), (0.05, -0.02, -1.0))]:
        cam.set_camera_to_world(scenes.camera_transform(eye=eye, target=(0.0, 0.0, 0.0)))
        cam.set_eye_dir(gaze)
        rc.render()
        s2e, e2p, res, hist = cam.foveated_resolve()
        pcol, pdep, pmom = cam.polar_textures(spr, rings)
        if polar["valid"] == spr * rings:
            # the scatter: RemapPolarFoveatedKernel on the frame's sample colours and view depths
            _, _, depth = cam.foveated_frame()
            rcol, rdep = ref.foveated_scatter(spr, rings, cam.sample_colors()[:polar["valid"]],
                                              depth[:polar["valid"]], polar["remap"][:polar["valid"]])
            assert np.array_equal(pcol, rcol)
            assert np.array_equal(pdep.view(np.uint32), rdep.view(np.uint32))
        r = ref.foveated_resolve(PATTERN, spr, rings, pcol, pdep, w, h, s2e, e2p, hist)
        dm = np.abs(pmom.astype(np.int32) - r["moments"].astype(np.int32))
        dr = np.abs(res.view(np.uint8).astype(np.int32) - r["result"].view(np.uint8).astype(np.int32))
        di = np.abs(cam.image.view(np.uint8).astype(np.int32) - r["image"].view(np.uint8).astype(np.int32))
        stats.append((dm.max(), dr.max(), (dr > 1).mean(), di.mean(), (di > 1).mean()))
    rc.close()
    for dm_max, dr_max, dr_gt1, di_mean, di_gt1 in stats:
        assert dm_max == 0 and dr_max == 0 and di_mean == 0, stats
