"""Foveated resolve on the host: the per-frame matrices (eye transform, tile cull planes,
sample-to-eye, eye-to-previous-sample-space and the temporal history update) must equal the
reference's own vector algebra compiled here, bit for bit, over several frames; the oracle's
software texture fetch at a pixel centre must select exactly that texel (the GPU reads the
texel directly there); and the oracle's first frame must read no history."""
import os
import sys

import numpy as np
import pytest

import hvvr_b200 as hv
from hvvr_b200 import _abi, scenes

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import pyoracle  # noqa: E402

PATTERN = (1.0, 35.0, 0.03, 0.06)


def _bounds(rng):
    sb = _abi.FloatRect()
    sb.lower.x, sb.lower.y = (float(v) for v in rng.uniform(0.0, 0.01, 2))
    sb.upper.x, sb.upper.y = (float(v) for v in 1.0 - rng.uniform(0.0, 0.01, 2))
    return sb


@pytest.mark.skipif(not pyoracle.Reference.available(), reason="oracle/_ref not built")
def test_frame_matrices_match_reference_build():
    ref = pyoracle.Reference()
    rng = np.random.default_rng(3)
    for trial in range(60):
        xf = scenes.camera_transform(eye=tuple(rng.uniform(-10, 10, 3)), target=tuple(rng.uniform(-2, 2, 3)))
        w, h = (int(v) for v in rng.integers(64, 2000, 2))
        vp = scenes.viewport_for(w, h) if trial % 2 else scenes.viewport_fov(w, h, float(rng.uniform(40, 120)))
        sb = _bounds(rng)
        ha = hb = None
        for _ in range(3):
            g = rng.normal(size=3)
            g[2] = -abs(g[2]) - 2.0
            g /= np.linalg.norm(g)
            a = hv.foveated_frame_matrices(xf, tuple(g), sb, vp, ha)
            b = ref.foveated_frame_matrices(xf, tuple(g), sb, vp, hb)
            for k in ("eye_to_world", "cull_planes", "sample_to_eye", "eye_to_sample_prev"):
                assert np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)), k
            for x, y in zip(a["history"], b["history"]):
                assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
            ha, hb = a["history"], b["history"]


def test_texel_centre_fetch_selects_the_texel():
    # u = (i + 0.5) / n, x = u * n - 0.5: the filter fraction rounds to 0 or 1 (in 256ths) and
    # the weighted texel is i, for every i of every width up to 8192 (float32 arithmetic)
    for n in list(range(1, 2049)) + list(range(2049, 8193, 37)) + [8192]:
        i = np.arange(n, dtype=np.float32)
        u = (i + np.float32(0.5)) / np.float32(n)
        x = u * np.float32(n) - np.float32(0.5)
        x = np.maximum(np.minimum(x, np.float32(n)), np.float32(-1.0))
        fl = np.floor(x)
        a8 = np.rint((x - fl) * np.float32(256.0)).astype(np.int64)
        sel = fl.astype(np.int64) + (a8 == 256)
        assert np.all((a8 == 0) | (a8 == 256)), n
        assert np.array_equal(sel, np.arange(n)), n


def test_oracle_first_frame_reads_no_history(oracle):
    polar = hv.polar_foveated_samples(hv.foveated_spec(*PATTERN))
    rng = np.random.default_rng(0)
    w, h = 96, 80
    cols = rng.integers(0, 1 << 24, polar["valid"], dtype=np.uint32) | np.uint32(0xFF000000)
    tm = rng.uniform(1.0, 20.0, polar["valid"]).astype(np.float32)
    xf = scenes.camera_transform(eye=(0.0, 2.0, 10.0), target=(0.0, 0.0, 0.0))
    m = hv.foveated_frame_matrices(xf, (0.0, 0.0, -1.0), _bounds(rng), scenes.viewport_for(w, h))
    assert not m["eye_to_sample_prev"].any()  # zero history matrix: every reprojection is NaN
    a = oracle.foveated_resolve(PATTERN, polar, cols, tm, w, h, m["sample_to_eye"], m["eye_to_sample_prev"],
                                np.zeros((h, w), np.uint32))
    b = oracle.foveated_resolve(PATTERN, polar, cols, tm, w, h, m["sample_to_eye"], m["eye_to_sample_prev"],
                                rng.integers(0, 1 << 32, (h, w), dtype=np.uint32))
    assert np.array_equal(a["image"], b["image"]) and np.array_equal(a["result"], b["result"])
    # the polar colour texture holds every sample once (the remap is a bijection)
    assert len(np.unique(polar["remap"][: polar["valid"]].view(np.uint64))) == polar["valid"]
    assert polar["valid"] == polar["samples_per_ring"] * polar["ring_count"]
