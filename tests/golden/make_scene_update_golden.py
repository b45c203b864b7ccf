"""Writes scene_update_rotate_scale.npz: the world-space vertex positions the reference's own
scene update kernels (gpu_scene_state.cu SceneTransformVerticesKernel, built for the GPU in
oracle/_ref/libhvvr_ref_gpu.so) produce for the seeded "small" test scene under one rotated,
translated and scaled model transform. Needs a GPU and the built reference GPU library; run from
the repository root with the output directory as the argument."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests"), ROOT]

import numpy as np  # noqa: E402

import hvvr_b200 as hv  # noqa: E402
import pyoracle  # noqa: E402
from hvvr_b200 import scenes  # noqa: E402
from helpers import scene  # noqa: E402
from test_gpu_scene_update import TRANSFORMS  # noqa: E402


def main(out_dir):
    sc = scene("small")
    xf = TRANSFORMS["rotate_scale"]
    # the 128-byte BVH nodes of the scene (the kernels read only their child and leaf data)
    rc = hv.Raycaster()
    rc.create_model(sc)
    cam = rc.create_camera(scenes.viewport_for(64, 48))
    cam.set_render_target(64, 48)
    cam.set_samples(scenes.grid_samples(64, 48))
    rc.render()
    rc.synchronize()
    nodes = rc.scene_nodes()
    rc.close()
    world, _, _ = pyoracle.ReferenceGpu().scene_update(nodes, sc.verts, np.zeros(len(sc.verts), np.uint32), [xf],
                                                      sc.tri_shade)
    np.savez_compressed(os.path.join(out_dir, "scene_update_rotate_scale.npz"), scene=np.array("small"),
                        transform=np.frombuffer(bytes(xf), np.uint8), world_pos=world["pos"].astype(np.float32))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
