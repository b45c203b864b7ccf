"""Regenerates tests/golden/*.npz from the reference's own sources compiled into oracle/_ref.

The reference ships no tests or golden vectors for this path, so the fixtures are produced
by running its code (GenerateTopology, SampleData, the AVX traversal driven like cullThread,
and the kernels' intersect/shade math compiled for the host; see oracle/refshim) on small
seeded inputs. Run from the repository root where the reference tree is available:

    make -C oracle && python tests/golden/make_golden.py

Each fixture stores its inputs (so the tests do not depend on the generator) and the
reference outputs. Floating-point outputs are stored as raw bits.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from hvvr_b200 import _abi, scenes  # noqa: E402
import pyoracle  # noqa: E402

CASES = {
    # name: (grid quads, boxes, seed, sample kind, width, height, msaa, eye, target[, thin lens (radius, focal distance)])
    "grid_msaa1": (8, 40, 3, "grid", 64, 48, 1, (0.0, 2.0, 10.0), (0.0, 0.0, 0.0)),
    "barrel_msaa4": (10, 60, 4, "barrel", 48, 56, 4, (2.0, 1.5, 7.0), (-1.0, 0.2, 0.0)),
    "grid_msaa8_low": (6, 30, 5, "grid", 40, 40, 8, (0.5, 0.6, 9.0), (0.0, 0.3, 0.0)),
    "barrel_msaa4_dof": (10, 60, 6, "barrel", 56, 48, 4, (1.0, 1.8, 8.0), (0.0, 0.0, -1.0), (0.08, 7.5)),
}


def make(name, ref):
    quads, boxes, seed, kind, w, h, msaa, eye, target = CASES[name][:9]
    lens = CASES[name][9] if len(CASES[name]) > 9 else (0.0, 1.0)
    sc = scenes.make_scene(quads, boxes, seed)
    in_verts, in_tris = sc.verts.copy(), sc.tri_shade.copy()
    verts, tris, nodes = ref.generate_topology(sc)
    sc.verts, sc.tri_shade, sc.nodes = verts, tris, nodes
    smp = scenes.grid_samples(w, h) if kind == "grid" else scenes.barrel_samples(w, h)
    xf = scenes.camera_transform(eye, target)
    vp = scenes.viewport_for(w, h)
    f = ref.render(sc, smp, xf, vp, w, h, msaa, fp_mode=_abi.HVVR_FP_STRICT, threads=4, tile_capacity=1 << 20,
                   lens=lens)
    assert f.status == 0
    lights = np.frombuffer(b"".join(bytes(l) for l in sc.lights), dtype=np.uint8)
    xf_arr = np.frombuffer(bytes(xf), dtype=np.uint8)
    vp_arr = np.frombuffer(bytes(vp), dtype=np.uint8)
    np.savez_compressed(
        os.path.join(ROOT, "tests", "golden", name + ".npz"),
        in_verts=in_verts, in_tris=in_tris, materials=sc.materials, lights=lights, samples=smp,
        cam_xf=xf_arr, viewport=vp_arr, dims=np.array([w, h, msaa], dtype=np.uint32),
        lens=np.array(lens, dtype=np.float32),
        topo_verts=verts, topo_tris=tris, topo_nodes=nodes,
        nodes=f.nodes, tris_bits=f.tris.view(np.uint32), beams_bits=f.beams.view(np.uint32), remap=f.remap,
        block_sizes=f.block_sizes, block_entries=f.block_entries, tile_counts=f.tile_counts,
        tile_indices=f.tile_indices, hit_ids=f.hit_ids, depth_bits=f.depth.view(np.uint32), gb_n=f.gb_n,
        gb_tri=f.gb_tri, gb_mask=f.gb_mask, colors=f.colors, image=f.image)
    print(name, "tris", len(tris), "nodes", len(nodes), "list entries", len(f.tile_indices),
          "hit subsamples", int((f.hit_ids != 0xFFFFFFFF).sum()))


POLAR_CASES = {
    # name: (degree tracking error, max FOV degrees, MAR slope, foveal MAR degrees)
    "polar_setup_small": (1.0, 12.0, 0.03, 0.06),
}


def make_polar(name, ref):
    """The reference's polar foveated sample set (getEyeSpacePolarFoveatedSamples,
    generateRemapForFoveatedSamples, ComputeEyeSpaceFrusta) for one parameter set."""
    dte, fov, slope, mar = POLAR_CASES[name]
    r = ref.polar_foveated(dte, fov, slope, mar)
    np.savez_compressed(
        os.path.join(ROOT, "tests", "golden", name + ".npz"),
        params=np.array([dte, fov, slope, mar], dtype=np.float32),
        counts=np.array([r["samples_per_ring"], r["ring_count"], r["valid"], r["padded"]], dtype=np.uint32),
        beams_bits=r["beams"].view(np.uint32), remap=r["remap"], tile_rays_bits=r["tile_rays"].view(np.uint32),
        block_rays_bits=r["block_rays"].view(np.uint32))
    print(name, "samples", r["valid"], "rings", r["ring_count"], "per ring", r["samples_per_ring"])


if __name__ == "__main__":
    # optional case names on the command line regenerate only those fixtures
    ref = pyoracle.Reference()
    for n in (sys.argv[1:] or list(CASES) + list(POLAR_CASES)):
        if n in POLAR_CASES:
            make_polar(n, ref)
        else:
            make(n, ref)
