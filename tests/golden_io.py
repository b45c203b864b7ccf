"""Loads tests/golden/*.npz fixtures into scenes and camera parameters."""
import ctypes as C
import glob
import os

import numpy as np

from hvvr_b200 import _abi, scenes

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    """The render fixtures (the polar_* fixtures hold sample sets only, the scene_update_* ones
    world-space vertex positions)."""
    return sorted(n for n in (os.path.splitext(os.path.basename(p))[0]
                              for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))
                  if not n.startswith(("polar_", "scene_update_")))


def load(name):
    g = dict(np.load(os.path.join(GOLDEN_DIR, name + ".npz")))
    lights = []
    raw = g["lights"].tobytes()
    for i in range(len(raw) // C.sizeof(_abi.LightUnion)):
        lights.append(_abi.LightUnion.from_buffer_copy(raw[i * C.sizeof(_abi.LightUnion):(i + 1) * C.sizeof(_abi.LightUnion)]))
    sc = scenes.Scene(g["topo_verts"].copy(), g["topo_tris"].copy(), g["materials"].copy(), lights)
    sc.nodes = g["topo_nodes"].copy()
    xf = _abi.Transform.from_buffer_copy(g["cam_xf"].tobytes())
    vp = _abi.FloatRect.from_buffer_copy(g["viewport"].tobytes())
    w, h, msaa = (int(v) for v in g["dims"])
    return g, sc, g["samples"], xf, vp, w, h, msaa


def lens(g):
    """(radius, focal distance) of the fixture's thin lens ((0, 1): pinhole)."""
    return tuple(float(v) for v in g["lens"]) if "lens" in g else (0.0, 1.0)
