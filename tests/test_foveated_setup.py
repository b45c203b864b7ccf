"""The polar foveated sample set (host): the library's restatement of the reference's
getEyeSpacePolarFoveatedSamples, generateRemapForFoveatedSamples and ComputeEyeSpaceFrusta
must reproduce the reference's beams, polar remap and eye-space frusta bit for bit - they
define the foveated tiles and therefore the lists. Tiles past the last sample have no
frustum in the reference (its fit reads an uninitialised rotation); the library makes them
degenerate, so they are compared over the tiles that hold samples."""
import os
import sys

import numpy as np
import pytest

import hvvr_b200 as hv

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import pyoracle  # noqa: E402


def _check(p, beams, remap, tile_rays, block_rays, valid):
    assert np.array_equal(p["beams"].view(np.uint32), beams)
    assert np.array_equal(p["remap"][:valid], remap)
    assert (p["remap"][valid:] == 0xFFFFFFFF).all()
    used = (valid + 127) // 128
    assert np.array_equal(p["tile_rays"].view(np.uint32)[:used], tile_rays[:used])
    assert np.isinf(p["tile_rays"][used:, 0]).all()  # degenerate: origin at infinity
    assert np.array_equal(p["block_rays"].view(np.uint32), block_rays)


def test_polar_set_matches_reference_golden():
    g = dict(np.load(os.path.join(HERE, "golden", "polar_setup_small.npz")))
    dte, fov, slope, mar = (float(v) for v in g["params"])
    p = hv.polar_foveated_samples(hv.foveated_spec(dte, fov, slope, mar))
    spr, rings, valid, padded = (int(v) for v in g["counts"])
    assert (p["samples_per_ring"], p["ring_count"], p["valid"], p["padded"]) == (spr, rings, valid, padded)
    _check(p, g["beams_bits"], g["remap"], g["tile_rays_bits"], g["block_rays_bits"], valid)


@pytest.mark.skipif(not pyoracle.Reference.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("params", [(0.5, 110.0, 0.022, 1.0 / 60.0), (2.0, 50.0, 0.03, 0.05)])
def test_polar_set_matches_reference_build(params):
    ref = pyoracle.Reference().polar_foveated(*params)
    p = hv.polar_foveated_samples(hv.foveated_spec(*params))
    assert (p["samples_per_ring"], p["ring_count"], p["valid"]) == (ref["samples_per_ring"], ref["ring_count"],
                                                                     ref["valid"])
    _check(p, ref["beams"].view(np.uint32), ref["remap"], ref["tile_rays"].view(np.uint32),
           ref["block_rays"].view(np.uint32), ref["valid"])
