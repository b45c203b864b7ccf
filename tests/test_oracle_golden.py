"""The CPU oracle against golden vectors produced by the reference's own code (oracle/_ref).

Bit-exact in HVVR_FP_STRICT mode (the arithmetic the reference source has without FMA
contraction): refit BVH, precomputed triangles, beams, remap, block stacks, per-tile lists,
hit IDs, depth, G-buffer pairs, colours and the image. Per-sample outputs are compared over
the valid samples: the reference leaves the padding samples that fill the last block
uninitialised (BeamBatch2D stops writing at the last valid sample), while this build defines
them as zero samples. HVVR_FP_FMA mode moves the FMA-marked
edge-test terms, so hit IDs may differ only at exact triangle edges; the count is enumerated.
The `_dof` fixture renders through a thin lens (radius 0.08, focal distance 7.5): the
reference's IntersectTriangleThreadDoF path with its lens-position table.
"""
import numpy as np
import pytest

from hvvr_b200 import _abi, scenes

from golden_io import lens, load, names


@pytest.mark.parametrize("name", names())
def test_oracle_matches_reference_golden(oracle, name):
    g, sc, smp, xf, vp, w, h, msaa = load(name)
    f = oracle.render(sc, smp, xf, vp, w, h, msaa, fp_mode=_abi.HVVR_FP_STRICT, threads=2, lens=lens(g))
    assert f.status == 0
    assert np.array_equal(f.nodes, g["nodes"])
    assert np.array_equal(f.tris.view(np.uint32), g["tris_bits"])
    n = len(smp)
    assert np.array_equal(f.beams.view(np.uint32)[:n], g["beams_bits"][:n])
    assert np.array_equal(f.remap, g["remap"])
    assert np.array_equal(f.block_sizes, g["block_sizes"])
    assert np.array_equal(f.block_entries, g["block_entries"])
    assert np.array_equal(f.tile_counts, g["tile_counts"])
    assert np.array_equal(f.tile_indices, g["tile_indices"])
    assert np.array_equal(f.hit_ids[:n], g["hit_ids"][:n])
    assert np.array_equal(f.depth.view(np.uint32)[:n], g["depth_bits"][:n])
    assert np.array_equal(f.gb_n[:n], g["gb_n"][:n]) and np.array_equal(f.gb_tri[:n], g["gb_tri"][:n])
    assert np.array_equal(f.gb_mask[:n], g["gb_mask"][:n])
    assert np.array_equal(f.colors[:n], g["colors"][:n])
    assert np.array_equal(f.image, g["image"])


@pytest.mark.parametrize("name", names())
def test_oracle_fma_mode_edge_mismatches(oracle, name):
    g, sc, smp, xf, vp, w, h, msaa = load(name)
    f = oracle.render(sc, smp, xf, vp, w, h, msaa, fp_mode=_abi.HVVR_FP_FMA, threads=2, lens=lens(g))
    assert np.array_equal(f.tile_indices, g["tile_indices"])  # traversal does not depend on the mode
    n = len(smp)
    ids, gids = f.hit_ids[:n], g["hit_ids"][:n]
    mism = int((ids != gids).sum())
    assert mism <= max(2, gids.size // 10000), "FMA mode changed %d hit IDs" % mism
    same = (gids != 0xFFFFFFFF) & (ids == gids)
    d = f.depth[:n][same].astype(np.float64)
    dz = np.abs(d - g["depth_bits"][:n].view(np.float32)[same].astype(np.float64))
    assert (dz <= 1e-5 * np.abs(d)).all()


def test_depth_against_fp64(oracle):
    """FP32 depth against an FP64 ray-triangle solve of the same hits (relative error)."""
    g, sc, smp, xf, vp, w, h, msaa = load(names()[0])
    f = oracle.render(sc, smp, xf, vp, w, h, msaa, threads=2)
    hit = f.hit_ids != 0xFFFFFFFF
    rel = np.abs(f.depth[hit] - f.depth64[hit]) / np.abs(f.depth64[hit])
    assert rel.max() < 1e-4, rel.max()


def test_generator_is_stable():
    """The seeded generator still produces the fixtures' inputs (numpy PCG64 streams are fixed)."""
    g, *_ = load("grid_msaa1")
    sc = scenes.make_scene(8, 40, 3)
    assert np.array_equal(sc.verts, g["in_verts"]) and np.array_equal(sc.tri_shade, g["in_tris"])


def test_rotated_grid_offsets_are_n_rooks():
    """The rotated-grid pattern: one subsample per column and per row of the n x n grid, inside the
    unit disk the spiral fills, the sample's centre at rate 1."""
    import ctypes as C
    import pyoracle
    lib = pyoracle.Oracle().lib
    lib.oracle_msaa_offsets_rotated_grid.argtypes = [C.c_uint32, C.c_void_p]
    lib.oracle_msaa_offsets_rotated_grid.restype = None
    for n in (1, 2, 4, 8, 16, 32):
        o = np.zeros(2 * n, np.float32)
        lib.oracle_msaa_offsets_rotated_grid(n, o.ctypes.data)
        xy = o.reshape(n, 2) / np.float32(0.70710677)
        cols = np.rint((xy[:, 0] + 1) * n / 2 - 0.5).astype(int)
        rows = np.rint((xy[:, 1] + 1) * n / 2 - 0.5).astype(int)
        assert sorted(cols) == list(range(n)) and sorted(rows) == list(range(n))
        assert (np.hypot(o[0::2], o[1::2]) <= 1.0).all()
    o = np.zeros(2, np.float32)
    lib.oracle_msaa_offsets_rotated_grid(1, o.ctypes.data)
    assert (o == 0).all()
