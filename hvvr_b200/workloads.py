"""Multi-view workloads built on the public API: the batched form (many views of uneven size
over several resident scenes, animated and refit every frame) and its plain counterpart.

Sizes follow the batched configuration: 4 scenes of about 100k, 500k, 1M and 2M triangles
from the procedural generator; views whose sample sets are drawn from {256x256 grid,
640x480 grid, 1080x1200 barrel-distorted, foveated 300k-1.2M samples}, with MSAA rates from
{1, 4, 8, 16}; 10% of every scene's vertices (one contiguous range in BVH order, i.e. one
region of the scene) move by a sinusoid of amplitude 0.1 each frame, followed by the GPU
refit. Everything is drawn from a seeded PCG64 generator.

The plain form renders the same views one view per launch: one single-view batch per view,
rendered in sequence on one stream. The batched form renders all views as one batch whose
frame is replayed from a CUDA graph. Both run the same kernels on the same data, so their
per-view results are bit-identical; only the launch structure differs.
"""
import math

import numpy as np

from . import scenes

SCENE_TRIS = (100_000, 500_000, 1_000_000, 2_000_000)
KINDS = ("grid256", "grid640x480", "barrel1080x1200", "foveated")
RATES = (1, 4, 8, 16)
ANIM_FRACTION, ANIM_AMPLITUDE = 0.10, 0.1


class ViewSpec:
    def __init__(self, scene, kind, width, height, msaa, eye, target, samples, viewport):
        self.scene, self.kind, self.width, self.height, self.msaa = scene, kind, width, height, msaa
        self.eye, self.target, self.samples, self.viewport = eye, target, samples, viewport

    @property
    def sample_count(self):
        return len(self.samples)


def make_views(count=64, seed=4, kinds=KINDS, rates=RATES, scene_count=len(SCENE_TRIS)):
    """`count` seeded view specs (scene index, sample set, MSAA rate, pose)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        kind = kinds[int(rng.integers(len(kinds)))]
        msaa = int(rates[int(rng.integers(len(rates)))])
        sc = int(rng.integers(scene_count))
        ang = rng.uniform(0.0, 2.0 * math.pi)
        rad = rng.uniform(7.0, 13.0)
        eye = (rad * math.sin(ang), rng.uniform(1.5, 5.0), rad * math.cos(ang))
        target = (rng.uniform(-3.0, 3.0), 0.0, rng.uniform(-3.0, 3.0))
        if kind == "grid256":
            w, h = 256, 256
            smp, vp = scenes.grid_samples(w, h), scenes.viewport_for(w, h)
        elif kind == "grid640x480":
            w, h = 640, 480
            smp, vp = scenes.grid_samples(w, h), scenes.viewport_for(w, h)
        elif kind == "barrel1080x1200":
            w, h = 1080, 1200
            smp, vp = scenes.barrel_samples(w, h), scenes.viewport_for(w, h)
        else:
            w, h = 1440, 1600
            n = int(rng.integers(300_000, 1_200_001))
            gaze = (rng.uniform(-10.0, 10.0), rng.uniform(-10.0, 10.0))
            smp = scenes.foveated_samples(n, w, h, 100.0, gaze)
            vp = scenes.viewport_fov(w, h, 100.0)
        out.append(ViewSpec(sc, kind, w, h, msaa, eye, target, smp, vp))
    return out


def make_scenes(tris=SCENE_TRIS, seed=10):
    """The resident scenes with topology (reorders their vertices and triangles)."""
    from . import generate_topology
    out = []
    for i, t in enumerate(tris):
        sc = scenes.scene_sized(t, seed=seed + i)
        generate_topology(sc)
        out.append(sc)
    return out


def anim_range(scene):
    """The animated vertex range [first, first + count) of a scene."""
    n = len(scene.verts)
    count = max(1, int(n * ANIM_FRACTION))
    first = (n - count) // 2
    return first, count


class Animator:
    """Device-side vertex animation of one model: y += amplitude * sin(t + phase_v) over the
    animated range, written to a device buffer and copied into the model on a stream."""

    def __init__(self, torch, model, scene, device="cuda"):
        self.torch, self.model = torch, model
        self.first, self.count = anim_range(scene)
        base = np.ascontiguousarray(scene.verts[self.first:self.first + self.count]).view(np.float32)
        base = base.reshape(self.count, 8)
        self.base = torch.from_numpy(base.copy()).to(device)
        rng = np.random.default_rng(1234 + self.count)
        self.phase = torch.from_numpy(rng.uniform(0.0, 2.0 * math.pi, self.count).astype(np.float32)).to(device)
        self.buf = self.base.clone()

    def step(self, t, stream_handle=None):
        torch = self.torch
        self.buf.copy_(self.base)
        self.buf[:, 1] += ANIM_AMPLITUDE * torch.sin(self.phase + float(t))
        self.model.update_vertices_device(self.first, self.count, self.buf.data_ptr(), stream_handle)

    def host_vertices(self, scene):
        """The whole scene's vertex array as last written by step() (for oracle checks)."""
        v = scene.verts.copy()
        f = v.view(np.float32).reshape(len(v), 8)
        f[self.first:self.first + self.count] = self.buf.cpu().numpy()
        return v
