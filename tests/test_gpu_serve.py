"""Serving: requests submitted together are batched (continuous batching over resident scenes)
and each result must be the same image as the request rendered alone, and as the oracle.
Admission under a tight HBM budget must still complete every request (instances are reused
and evicted), and scene animation through the server must match the oracle's refit."""
import copy

import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import scenes

from helpers import render_oracle, scene

pytestmark = pytest.mark.gpu


def _rc(sc):
    rc = hv.Raycaster()
    rc.create_model(sc)
    for l in sc.lights:
        rc.create_light(l)
    return rc


def _templates():
    # (scene index, kind, width, height)
    return [(0, "barrel", 160, 176), (1, "grid", 128, 96), (0, "foveated", 144, 160), (1, "barrel", 96, 112)]


def _samples(kind, w, h):
    if kind == "grid":
        return scenes.grid_samples(w, h), scenes.viewport_for(w, h)
    if kind == "barrel":
        return scenes.barrel_samples(w, h), scenes.viewport_for(w, h)
    return scenes.foveated_samples(w * h // 2, w, h, 100.0, (4.0, -2.0)), scenes.viewport_fov(w, h, 100.0)


def _drain(srv, want, timeout_ms=60000):
    done = {}
    waited = 0.0
    while len(done) < want:
        got = srv.poll(wait_ms=50.0)
        for c in got:
            done[c.id] = c
        waited += 50.0
        assert waited < timeout_ms, "server did not complete %d requests" % want
    return done


def test_results_same_alone_and_in_mix(oracle):
    scs = [scene("c1"), scene("small")]
    rcs = [_rc(s) for s in scs]
    srv = hv.Server(rcs, hv.server_config(slots=2, max_batch_views=8, slot_list_capacity=1 << 22))
    tmpl = []
    for si, kind, w, h in _templates():
        smp, vp = _samples(kind, w, h)
        tmpl.append((srv.add_view(si, vp, smp, w, h), si, w, h, smp, vp))
    rng = np.random.default_rng(7)
    reqs = []
    for i in range(24):
        vid, si, w, h, smp, vp = tmpl[int(rng.integers(len(tmpl)))]
        ang = rng.uniform(0, 2 * np.pi)
        eye = (8.0 * np.sin(ang), rng.uniform(1.5, 4.0), 8.0 * np.cos(ang))
        xf = scenes.camera_transform(eye=eye, target=(0.0, 0.0, 0.0))
        reqs.append((vid, int([1, 4, 8, 16][int(rng.integers(4))]), xf, si, w, h, smp, vp))
    # the mix: everything submitted at once
    mix = []
    for k, (vid, msaa, xf, si, w, h, smp, vp) in enumerate(reqs):
        out = np.zeros((h, w), dtype=np.uint32)
        rid = srv.submit(vid, msaa, xf, output=out, tag=k)
        mix.append((rid, out))
    done = _drain(srv, len(mix))
    assert all(c.status == 0 for c in done.values())
    assert max(c.batch_views for c in done.values()) > 1, "requests were not batched"
    # alone: one request at a time
    for k, (vid, msaa, xf, si, w, h, smp, vp) in enumerate(reqs):
        out = np.zeros((h, w), dtype=np.uint32)
        rid = srv.submit(vid, msaa, xf, output=out)
        c = _drain(srv, 1)[rid]
        assert c.status == 0 and c.batch_views == 1
        assert np.array_equal(out, mix[k][1]), "request %d differs alone and in the mix" % k
        if k < 4:  # and the oracle agrees
            fo = render_oracle(oracle, scs[si], smp, w, h, msaa, cam_xf=xf, viewport=vp)
            d = np.abs(out.view(np.uint8).astype(np.int32) - fo.image.view(np.uint8).astype(np.int32))
            assert d.max() <= 1
    st = srv.stats()
    assert st["completed"] == 48 and st["failed"] == 0 and st["batches"] >= 2
    srv.close()
    for rc in rcs:
        rc.close()


def test_tight_budget_evicts_and_completes():
    scs = [scene("c1"), scene("small")]
    rcs = [_rc(s) for s in scs]
    cap = 1 << 20
    pools = 2 * cap * 4 * 129 // 128
    budget = pools + (3 << 20)  # room for two of these small views at a time, not all four
    srv = hv.Server(rcs, hv.server_config(slots=2, max_batch_views=4, slot_list_capacity=cap,
                                          hbm_budget_bytes=budget, latency_slots=0))
    ids = []
    for si, kind, w, h in _templates():
        smp, vp = _samples(kind, w, h)
        ids.append((srv.add_view(si, vp, smp, w, h), w, h))
    outs = []
    for k in range(16):
        vid, w, h = ids[k % len(ids)]
        out = np.zeros((h, w), dtype=np.uint32)
        srv.submit(vid, 4, scenes.camera_transform(eye=(1.0 + 0.1 * k, 2.0, 9.0)), output=out)
        outs.append(out)
    done = _drain(srv, 16)
    assert all(c.status == 0 for c in done.values())
    st = srv.stats()
    assert st["hbm_peak"] <= budget and st["evicted"] > 0
    srv.close()
    for rc in rcs:
        rc.close()


def test_served_animation_matches_oracle(oracle):
    import torch
    from hvvr_b200 import workloads
    sc = scene("small")
    rc = _rc(sc)
    model = rc.models[0]
    srv = hv.Server([rc], hv.server_config(slot_list_capacity=1 << 22))
    w, h = 160, 176
    smp, vp = _samples("barrel", w, h)
    vid = srv.add_view(0, vp, smp, w, h)
    xf = scenes.camera_transform(eye=(0.5, 2.0, 9.0))
    first, count = workloads.anim_range(sc)
    base = torch.from_numpy(np.ascontiguousarray(sc.verts[first:first + count]).view(np.float32).reshape(count, 8)
                            .copy()).cuda()
    for t in (0.4, 2.2):
        moved_dev = base.clone()
        moved_dev[:, 1] += 0.1 * torch.sin(torch.arange(count, device="cuda", dtype=torch.float32) + t)
        torch.cuda.synchronize()
        srv.update_vertices(model, first, count, moved_dev.data_ptr())
        out = np.zeros((h, w), dtype=np.uint32)
        rid = srv.submit(vid, 8, xf, output=out)
        assert _drain(srv, 1)[rid].status == 0
        moved = copy.copy(sc)
        v = sc.verts.copy()
        v.view(np.float32).reshape(len(v), 8)[first:first + count] = moved_dev.cpu().numpy()
        moved.verts = v
        fo = render_oracle(oracle, moved, smp, w, h, 8, cam_xf=xf, viewport=vp)
        d = np.abs(out.view(np.uint8).astype(np.int32) - fo.image.view(np.uint8).astype(np.int32))
        assert d.max() <= 1
    srv.close()
    rc.close()


def test_polar_foveated_requests_same_alone_in_mix_and_direct():
    """Polar foveated templates: every request is one first frame (no temporal history), so its
    resolved image must be the same alone, in a mix, and rendered directly by a camera of the
    same raycaster."""
    from hvvr_b200 import _abi
    sc = scene("small")
    spec = hv.foveated_spec(1.0, 35.0, 0.03, 0.06, mode=_abi.HVVR_MODE_FOVEATED_POLAR)
    rc = hv.Raycaster(spec=spec)
    rc.create_model(sc)
    for l in sc.lights:
        rc.create_light(l)
    srv = hv.Server([rc], hv.server_config(slots=2, max_batch_views=4, slot_list_capacity=1 << 22))
    sizes = [(160, 144), (128, 112)]
    vids = []
    for w, h in sizes:
        vids.append(srv.add_view(0, scenes.viewport_for(w, h), scenes.grid_samples(w, h), w, h))
    rng = np.random.default_rng(11)
    reqs = []
    for k in range(8):
        t = k % 2
        ang = rng.uniform(-0.5, 0.5)
        xf = scenes.camera_transform(eye=(8.0 * np.sin(ang), 2.5, 8.0 * np.cos(ang)), target=(0.0, 0.0, 0.0))
        reqs.append((t, int([4, 8][k % 2]), xf))
    mix = []
    for t, msaa, xf in reqs:
        w, h = sizes[t]
        out = np.zeros((h, w), np.uint32)
        mix.append((srv.submit(vids[t], msaa, xf, output=out), out))
    done = _drain(srv, len(mix))
    assert all(c.status == 0 for c in done.values())
    for k, (t, msaa, xf) in enumerate(reqs):
        w, h = sizes[t]
        out = np.zeros((h, w), np.uint32)
        rid = srv.submit(vids[t], msaa, xf, output=out)
        assert _drain(srv, 1)[rid].status == 0
        assert np.array_equal(out, mix[k][1]), "request %d differs alone and in the mix" % k
        assert (out & 0xFFFFFF).any()
    srv.close()  # the raycaster may be rendered directly only once its server is gone
    for k in range(2):
        t, msaa, xf = reqs[k]
        w, h = sizes[t]
        cam = rc.create_camera(scenes.viewport_for(w, h))
        cam.set_render_target(w, h)
        cam.set_samples(scenes.grid_samples(w, h))
        cam.set_msaa(msaa)
        cam.set_camera_to_world(xf)
        rc.render()
        assert np.array_equal(cam.image, mix[k][1]), "request %d differs from a direct render" % k
        cam.set_enabled(False)
    rc.close()


def test_latency_class_jumps_a_busy_mix(oracle):
    """A stereo pair submitted as one group of the latency class (priority 1) behind a queue of
    throughput requests is dispatched at once on the latency slot, both eyes in one batch, while
    throughput requests are still waiting; each eye's image equals the oracle's (and its completion
    says which class it was). A group with one refused request queues none of them."""
    scs = [scene("c1"), scene("small")]
    rcs = [_rc(s) for s in scs]
    srv = hv.Server(rcs, hv.server_config(slots=2, max_batch_views=4, slot_list_capacity=1 << 22, latency_slots=1,
                                          tile_cull_ctas_per_sm=3))
    tmpl = []
    for si, kind, w, h in _templates():
        smp, vp = _samples(kind, w, h)
        tmpl.append((srv.add_view(si, vp, smp, w, h), w, h))
    sw, sh = 320, 352
    ssmp = scenes.barrel_samples(sw, sh)
    stereo = srv.add_view(0, scenes.viewport_for(sw, sh), ssmp, sw, sh)
    rng = np.random.default_rng(9)
    busy = []  # the throughput requests' outputs, alive until their completions arrive
    poses = []
    for k in range(32):
        vid, w, h = tmpl[k % len(tmpl)]
        xf = scenes.camera_transform(eye=(float(rng.uniform(-4, 4)), 2.0, 9.0))
        busy.append(np.zeros((h, w), dtype=np.uint32))
        poses.append(xf)
        srv.submit(vid, 16, xf, output=busy[-1], tag=k)
    eyes = scenes.stereo_eyes(0.064)
    outs = [np.zeros((sh, sw), dtype=np.uint32) for _ in eyes]
    # both eyes as one group: they reach the worker together and render in one latency batch
    rids = srv.submit_group([(stereo, 8, xf, out, None, 1000 + e) for e, (xf, out) in enumerate(zip(eyes, outs))],
                            priority=1)
    outs = list(zip(rids, outs, eyes))
    done = _drain(srv, 34)
    assert all(c.status == 0 for c in done.values())
    thr = [c for c in done.values() if c.priority == 0]
    lat = [done[rid] for rid, _, _ in outs]
    assert all(c.priority == 1 for c in lat) and len(thr) == 32
    assert all(c.batch_views == 2 for c in lat) and lat[0].dispatch_ms == lat[1].dispatch_ms
    # dispatched ahead of throughput requests submitted before them
    assert max(c.dispatch_ms for c in lat) < max(c.dispatch_ms for c in thr)
    for rid, out, xf in outs:
        fo = render_oracle(oracle, scs[0], ssmp, sw, sh, 8, cam_xf=xf)
        d = np.abs(out.view(np.uint8).astype(np.int32) - fo.image.view(np.uint8).astype(np.int32))
        assert d.max() <= 1
    # throughput requests that ran beside the latency frame: their tiles may have been left by
    # yielding CTAs and done by the drain launches; the images are the oracle's all the same
    for k in (0, 1, 2, 3, 5, 6):
        si, kind, w, h = _templates()[k % len(tmpl)]
        smp, vp = _samples(kind, w, h)
        fo = render_oracle(oracle, scs[si], smp, w, h, 16, cam_xf=poses[k], viewport=vp)
        d = np.abs(busy[k].view(np.uint8).astype(np.int32) - fo.image.view(np.uint8).astype(np.int32))
        assert d.max() <= 1, k
    # a bad class is refused, alone and inside a group (which then queues nothing)
    with pytest.raises(hv.HvvrError):
        srv.submit(stereo, 8, eyes[0], output=np.zeros((sh, sw), dtype=np.uint32), priority=2)
    before = srv.stats()["submitted"]
    bad = np.zeros((sh, sw), dtype=np.uint32)
    with pytest.raises(hv.HvvrError):
        srv.submit_group([(stereo, 8, eyes[0], bad, None, 0), (stereo, 3, eyes[1], bad, None, 0)], priority=1)
    assert srv.stats()["submitted"] == before
    srv.close()
    for rc in rcs:
        rc.close()
