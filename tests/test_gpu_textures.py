"""Material textures on the GPU: createTexture (libraries/hvvr/raycaster/texture.cu:201-272),
ReadTexture (shading.h:45-47) and GGXShade's texture reads with ShadeMSAA's derivatives
(resolve.cu:230-270; shading.h:84-161), through the C ABI.

Texture filtering is the GPU's texture unit, configured as the reference configures it, so
parity is pinned against the reference's own texture code built for the GPU
(oracle/_ref/libhvvr_ref_gpu.so): mip chains and texture reads bit-exact. Textured renders
are checked against the oracle, whose texture reads are served by the reference's code at the
oracle's own texture coordinates and derivatives: hit IDs exact, colour within 1 LSB.
"""
import numpy as np
import pytest

import pyoracle
import hvvr_b200 as hv
from hvvr_b200 import scenes

from helpers import scene

pytestmark = pytest.mark.gpu
needs_ref_gpu = pytest.mark.skipif(not pyoracle.ReferenceGpu.available(), reason="oracle/_ref GPU library not built")

RGBA8 = [hv.HVVR_TEXTURE_RGBA8_UNORM_SRGB, hv.HVVR_TEXTURE_RGBA8_UNORM]


@pytest.fixture(scope="module")
def refgpu():
    return pyoracle.ReferenceGpu()


def _queries(n, seed):
    """Texture reads over wrapped coordinates with derivatives from texel-sized to whole-texture,
    isotropic to 16:1 anisotropic, including zero derivatives."""
    rng = np.random.default_rng(seed)
    uv = rng.uniform(-1.5, 2.5, (n, 2))
    mag = 10.0 ** rng.uniform(-4.0, 0.0, n)
    ratio = 10.0 ** rng.uniform(0.0, 1.2, n)
    ang = rng.uniform(0.0, 2.0 * np.pi, n)
    dx = np.stack([np.cos(ang), np.sin(ang)], 1) * mag[:, None]
    dy = np.stack([-np.sin(ang), np.cos(ang)], 1) * (mag / ratio)[:, None]
    dx[: n // 16] = 0.0
    dy[: n // 16] = 0.0
    return np.concatenate([uv, dx, dy], 1).astype(np.float32)


@needs_ref_gpu
@pytest.mark.parametrize("fmt", RGBA8)
def test_mip_chain_equals_reference(refgpu, fmt):
    rc = hv.Raycaster()
    try:
        for i, (w, h) in enumerate([(64, 48), (37, 19), (1, 5), (128, 128), (300, 7)]):
            texels = scenes.texture_rgba8(w, h, seed=100 + i)
            t = rc.create_texture(texels, fmt)
            rid = refgpu.create_texture(texels, fmt)
            assert np.array_equal(t.read_level(0), texels)
            for level in range(max(w, h).bit_length()):
                a, b = t.read_level(level), refgpu.read_level(rid, level)
                assert a.shape == b.shape
                assert np.array_equal(a, b), "level %d of %dx%d differs at %d texels" % (
                    level, w, h, int((a != b).any(-1).sum()))
    finally:
        rc.close()


@needs_ref_gpu
@pytest.mark.parametrize("fmt", RGBA8)
def test_texture_reads_equal_reference(refgpu, fmt):
    rc = hv.Raycaster()
    try:
        for i, (w, h) in enumerate([(64, 48), (37, 19), (256, 128)]):
            texels = scenes.texture_rgba8(w, h, seed=200 + i)
            t = rc.create_texture(texels, fmt)
            rid = refgpu.create_texture(texels, fmt)
            q = _queries(8192, seed=300 + i)
            a = t.sample(q)
            b = refgpu.sample(np.full(len(q), rid, np.uint32), q)
            assert np.isfinite(a).all()
            bad = (a.view(np.uint32) != b.view(np.uint32)).any(1)
            assert not bad.any(), "%d of %d reads differ" % (int(bad.sum()), len(q))
    finally:
        rc.close()


def _textured_scene(count):
    sc = scenes.with_textures(scene("small"), count, seed=5)
    sizes = [(64, 64), (32, 16), (128, 64), (17, 9)]
    texels = [scenes.texture_rgba8(w, h, seed=400 + i) for i, (w, h) in enumerate(sizes[:count])]
    fmts = [RGBA8[i % 2] for i in range(count)]
    return sc, texels, fmts


def _render_textured(sc, texels, fmts, smp, w, h, msaa, fp_mode, lens, destroy_last=False):
    rc = hv.Raycaster(fp_mode=fp_mode)
    rc.create_model(sc)
    for light in sc.lights:
        rc.create_light(light)
    texs = [rc.create_texture(t, f) for t, f in zip(texels, fmts)]
    assert [t.id for t in texs] == list(range(len(texs)))
    if destroy_last:
        rc.destroy_texture(texs[-1])
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h)
    cam.set_samples(smp)
    cam.set_camera_to_world(scenes.camera_transform(eye=(0.8, 1.6, 7.5), target=(0.0, 0.0, -1.0)))
    cam.set_msaa(msaa)
    if lens is not None:
        cam.set_lens(*lens)
    cam.set_capture(hv.HVVR_CAPTURE_HITS)
    rc.render()
    ids, _ = cam.hits()
    col = cam.sample_colors()
    rc.close()
    return ids, col


def _oracle_textured(oracle, refgpu, sc, texels, fmts, smp, w, h, msaa, fp_mode, lens, live):
    """The oracle's render with each texture read answered by the reference's GPU texture code."""
    ref_ids = np.array([refgpu.create_texture(t, f) for t, f in zip(texels, fmts)], np.uint32)
    kw = dict(fp_mode=fp_mode, lens=lens or (0.0, 1.0), textures=live, sampler=oracle.table_sampler,
              want=("hits", "colors"))
    xf = scenes.camera_transform(eye=(0.8, 1.6, 7.5), target=(0.0, 0.0, -1.0))
    vp = scenes.viewport_for(w, h)
    oracle.table_record()
    oracle.render(sc, smp, xf, vp, w, h, msaa, **kw)
    qid, q = oracle.table_queries()
    assert len(qid) > 0
    oracle.table_set(qid, q, refgpu.sample(ref_ids[qid], q))
    fo = oracle.render(sc, smp, xf, vp, w, h, msaa, **kw)
    assert oracle.table_missing() == 0
    return fo


@needs_ref_gpu
@pytest.mark.parametrize("msaa,fp_mode,lens", [(4, hv.HVVR_FP_FMA, None), (8, hv.HVVR_FP_STRICT, None),
                                               (1, hv.HVVR_FP_FMA, None), (4, hv.HVVR_FP_FMA, (0.04, 5.0))])
def test_textured_render_matches_oracle(oracle, refgpu, msaa, fp_mode, lens):
    sc, texels, fmts = _textured_scene(4)
    w, h = 160, 120
    smp = scenes.barrel_samples(w, h)
    ids, col = _render_textured(sc, texels, fmts, smp, w, h, msaa, fp_mode, lens)
    fo = _oracle_textured(oracle, refgpu, sc, texels, fmts, smp, w, h, msaa, fp_mode, lens, live=4)
    assert np.array_equal(ids, fo.hit_ids)
    d = np.abs(col.view(np.uint8).astype(np.int32) - fo.colors.view(np.uint8).astype(np.int32))
    assert d.max() <= 1, "colour differs by %d LSB at %d samples" % (d.max(), int((d > 1).any(-1).sum()))
    # the textures change the picture
    plain = oracle.render(sc, smp, scenes.camera_transform(eye=(0.8, 1.6, 7.5), target=(0.0, 0.0, -1.0)),
                          scenes.viewport_for(w, h), w, h, msaa, fp_mode=fp_mode, lens=lens or (0.0, 1.0),
                          want=("colors",))
    assert (plain.colors != fo.colors).mean() > 0.1


@needs_ref_gpu
def test_destroyed_texture_reads_as_none(oracle, refgpu):
    sc, texels, fmts = _textured_scene(4)
    w, h = 96, 72
    smp = scenes.grid_samples(w, h)
    ids, col = _render_textured(sc, texels, fmts, smp, w, h, 4, hv.HVVR_FP_FMA, None, destroy_last=True)
    fo = _oracle_textured(oracle, refgpu, sc, texels, fmts, smp, w, h, 4, hv.HVVR_FP_FMA, None, live=3)
    assert np.array_equal(ids, fo.hit_ids)
    d = np.abs(col.view(np.uint8).astype(np.int32) - fo.colors.view(np.uint8).astype(np.int32))
    assert d.max() <= 1


def test_wide_formats_level0_and_reads():
    """Formats beyond RGBA8: level 0 holds the texels given; a read at a texel centre with zero
    derivatives returns that texel; level 1 is the mean of the reference generator's four taps."""
    rng = np.random.default_rng(7)
    rc = hv.Raycaster()
    try:
        w, h = 16, 8
        cases = [(hv.HVVR_TEXTURE_RGBA32_FLOAT, rng.uniform(-2, 2, (h, w, 4)).astype(np.float32)),
                 (hv.HVVR_TEXTURE_RGBA16_FLOAT, rng.uniform(0, 4, (h, w, 4)).astype(np.float16)),
                 (hv.HVVR_TEXTURE_R32_FLOAT, rng.uniform(0, 1, (h, w, 1)).astype(np.float32)),
                 (hv.HVVR_TEXTURE_RGBA16_UNORM, rng.integers(0, 65536, (h, w, 4)).astype(np.uint16))]
        for fmt, texels in cases:
            t = rc.create_texture(texels, fmt)
            assert np.array_equal(t.read_level(0).view(np.uint8), texels.view(np.uint8))
            y, x = np.mgrid[0:h, 0:w]
            q = np.zeros((h * w, 6), np.float32)
            q[:, 0] = (x.ravel() + 0.5) / w
            q[:, 1] = (y.ravel() + 0.5) / h
            got = t.sample(q)
            want = texels.reshape(h * w, -1).astype(np.float64)
            if fmt == hv.HVVR_TEXTURE_RGBA16_UNORM:
                want = want / 65535.0
            assert np.allclose(got[:, :want.shape[1]], want, rtol=1e-6, atol=1e-6)
            # level 1: texel (i, j) averages level-0 texels 2i-1 .. 2i+2 per axis (clamped)
            src = texels.astype(np.float64) / (65535.0 if fmt == hv.HVVR_TEXTURE_RGBA16_UNORM else 1.0)
            ii = np.clip(np.arange(-1, w + 1), 0, w - 1)
            jj = np.clip(np.arange(-1, h + 1), 0, h - 1)
            pad = src[jj][:, ii]
            l1 = 0.25 * (pad[0:-2:2] + pad[1:-1:2] + pad[2::2] + pad[3::2])
            l1 = 0.25 * (l1[:, 0:-2:2] + l1[:, 1:-1:2] + l1[:, 2::2] + l1[:, 3::2])
            got1 = t.read_level(1).astype(np.float64)
            if fmt == hv.HVVR_TEXTURE_RGBA16_UNORM:
                assert np.abs(got1 - np.floor(np.minimum(l1 * 65535.0, 65535.0))).max() <= 1
            else:
                tol = 2e-3 if fmt == hv.HVVR_TEXTURE_RGBA16_FLOAT else 1e-5
                assert np.allclose(got1, l1, rtol=tol, atol=tol)
        with pytest.raises(hv.HvvrError):
            rc.create_texture(np.zeros((4, 4, 1), np.uint32), hv.HVVR_TEXTURE_R11G11B10_FLOAT)
        with pytest.raises(hv.HvvrError):
            rc.create_texture(np.zeros((4, 4, 4), np.uint8), 99)
    finally:
        rc.close()


def test_textured_and_untextured_scenes_in_one_batch():
    """A frame batch over two raycasters, one with textures: each view reads its own scene's
    texture table, so every camera's image equals its raycaster rendering alone."""
    sc, texels, fmts = _textured_scene(4)
    plain = scene("c1")
    w, h = 128, 96
    smp = scenes.barrel_samples(w, h)

    def build(s, textured):
        rc = hv.Raycaster()
        rc.create_model(s)
        for light in s.lights:
            rc.create_light(light)
        if textured:
            for t, f in zip(texels, fmts):
                rc.create_texture(t, f)
        cam = rc.create_camera(scenes.viewport_for(w, h))
        cam.set_render_target(w, h)
        cam.set_samples(smp)
        cam.set_camera_to_world(scenes.camera_transform(eye=(0.8, 1.6, 7.5), target=(0.0, 0.0, -1.0)))
        cam.set_msaa(4)
        return rc, cam

    alone = []
    for s, textured in ((sc, True), (plain, False)):
        rc, cam = build(s, textured)
        rc.render()
        rc.synchronize()
        alone.append(cam.image.copy())
        rc.close()
    rcs = [build(sc, True), build(plain, False)]
    batch = hv.Batch([r for r, _ in rcs])
    batch.render()
    batch.synchronize()
    for (rc, cam), want in zip(rcs, alone):
        assert np.array_equal(cam.image, want)
    batch.close()
    for rc, _ in rcs:
        rc.close()
