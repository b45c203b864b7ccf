"""Seeded synthetic scenes, sample sets and cameras for the benchmark configurations.

The reference's scene assets are not available, so procedural scenes with the shapes,
sizes and value distributions of the benchmark configurations stand in for them:

* a heightfield of ``n x n`` quads over xz in [-10, 10]^2 whose height is a sum of four
  sinusoids (amplitude 0.5, wavelengths U[2, 8], random direction and phase);
* ``box_count`` boxes (12 triangles each) with centres uniform over the region resting on
  the terrain, edge lengths log-uniform in [0.05, 1.0] and a random yaw;
* one material per triangle: albedo U[0,1]^3, GGX roughness U[0.1, 0.9] (glossiness
  1 - roughness), F0 = 0.04, phong shading model, no textures (``with_textures`` adds them);
* one directional light plus four point lights.

Triangles are wound so their geometric normal e0 x e1 faces outward / up, since the
intersection test culls back faces (denom = -dir . (e0 x e1) must be positive).
Everything is generated with numpy's PCG64 from an explicit seed, so the arrays are
identical on every machine.
"""
import math

import numpy as np

from . import _abi

BAD_TEXTURE = 0xFFFF
PHONG = 1
SHADING_CODE = PHONG | (BAD_TEXTURE << 16) | (BAD_TEXTURE << 32) | (BAD_TEXTURE << 48)


class Scene:
    """Vertex/triangle/material arrays in the reference MeshData layout (no topology yet)."""

    def __init__(self, verts, tri_shade, materials, lights, heightfield=None):
        self.verts = verts
        self.tri_shade = tri_shade
        self.materials = materials
        self.lights = lights
        self.nodes = None
        self.heightfield = heightfield

    @property
    def tri_count(self):
        return len(self.tri_shade)


def _height_params(rng):
    ang = rng.uniform(0.0, 2.0 * math.pi, 4)
    lam = rng.uniform(2.0, 8.0, 4)
    phase = rng.uniform(0.0, 2.0 * math.pi, 4)
    return ang, lam, phase


def _height(params, x, z):
    ang, lam, phase = params
    h = np.zeros(np.broadcast(x, z).shape, dtype=np.float64)
    for k in range(4):
        d = np.cos(ang[k]) * x + np.sin(ang[k]) * z
        h += 0.5 * np.sin(2.0 * math.pi * d / lam[k] + phase[k])
    return h


def _height_grad(params, x, z):
    ang, lam, phase = params
    gx = np.zeros(np.broadcast(x, z).shape)
    gz = np.zeros_like(gx)
    for k in range(4):
        w = 2.0 * math.pi / lam[k]
        d = np.cos(ang[k]) * x + np.sin(ang[k]) * z
        c = 0.5 * w * np.cos(w * d + phase[k])
        gx += c * np.cos(ang[k])
        gz += c * np.sin(ang[k])
    return gx, gz


def _half(v):
    return np.asarray(v, dtype=np.float32).astype(np.float16).view(np.uint16)


def make_scene(grid_quads, box_count, seed=1):
    """Heightfield of grid_quads^2 quads (2 tris each) plus box_count boxes (12 tris each)."""
    rng = np.random.default_rng(seed)
    params = _height_params(rng)
    n = grid_quads
    xs = np.linspace(-10.0, 10.0, n + 1)
    X, Z = np.meshgrid(xs, xs, indexing="ij")  # X varies along i, Z along j
    H = _height(params, X, Z)
    gx, gz = _height_grad(params, X, Z)
    hn = np.stack([-gx, np.ones_like(gx), -gz], axis=-1)
    hn /= np.linalg.norm(hn, axis=-1, keepdims=True)
    hpos = np.stack([X, H, Z], axis=-1).reshape(-1, 3)
    hnorm = hn.reshape(-1, 3)
    huv = np.stack([(X + 10.0) / 20.0, (Z + 10.0) / 20.0], axis=-1).reshape(-1, 2)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    a = (i * (n + 1) + j).ravel()
    b = ((i + 1) * (n + 1) + j).ravel()
    c = (i * (n + 1) + j + 1).ravel()
    d = ((i + 1) * (n + 1) + j + 1).ravel()
    # (a, c, b) and (b, c, d) give +y geometric normals
    htris = np.empty((2 * len(a), 3), dtype=np.int64)
    htris[0::2] = np.stack([a, c, b], axis=1)
    htris[1::2] = np.stack([b, c, d], axis=1)

    # boxes: 6 faces x 4 verts, 2 tris per face, outward winding
    cx = rng.uniform(-10.0, 10.0, box_count)
    cz = rng.uniform(-10.0, 10.0, box_count)
    size = np.exp(rng.uniform(math.log(0.05), math.log(1.0), (box_count, 3)))
    yaw = rng.uniform(0.0, 2.0 * math.pi, box_count)
    base = _height(params, cx, cz)
    cy = base + 0.5 * size[:, 1] - 0.05 * size[:, 1]
    # unit cube face corners (counter-clockwise seen from outside) and normals
    faces = np.array([
        [[1, -1, -1], [1, 1, -1], [1, 1, 1], [1, -1, 1]],      # +x
        [[-1, -1, 1], [-1, 1, 1], [-1, 1, -1], [-1, -1, -1]],  # -x
        [[-1, 1, -1], [-1, 1, 1], [1, 1, 1], [1, 1, -1]],      # +y
        [[-1, -1, 1], [-1, -1, -1], [1, -1, -1], [1, -1, 1]],  # -y
        [[-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]],      # +z
        [[1, -1, -1], [-1, -1, -1], [-1, 1, -1], [1, 1, -1]],  # -z
    ], dtype=np.float64)
    fnorm = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], dtype=np.float64)
    corners = faces.reshape(24, 3) * 0.5
    cn = np.repeat(fnorm, 4, axis=0)
    cyaw, syaw = np.cos(yaw), np.sin(yaw)
    loc = corners[None, :, :] * size[:, None, :]
    bx = cyaw[:, None] * loc[..., 0] + syaw[:, None] * loc[..., 2] + cx[:, None]
    bz = -syaw[:, None] * loc[..., 0] + cyaw[:, None] * loc[..., 2] + cz[:, None]
    by = loc[..., 1] + cy[:, None]
    bpos = np.stack([bx, by, bz], axis=-1).reshape(-1, 3)
    nx = cyaw[:, None] * cn[None, :, 0] + syaw[:, None] * cn[None, :, 2]
    nz = -syaw[:, None] * cn[None, :, 0] + cyaw[:, None] * cn[None, :, 2]
    ny = np.broadcast_to(cn[None, :, 1], nx.shape)
    bnorm = np.stack([nx, ny, nz], axis=-1).reshape(-1, 3)
    buv = np.tile(np.array([[0, 0], [1, 0], [1, 1], [0, 1]] * 6, dtype=np.float64), (box_count, 1))
    # face quad (p0,p1,p2,p3) ccw from outside: tris (p0,p1,p2),(p0,p2,p3) have outward e0 x e1
    fq = np.arange(6)[:, None, None] * 4 + np.array([[0, 1, 2], [0, 2, 3]])[None, :, :]
    fq = fq.reshape(12, 3)
    boff = (np.arange(box_count) * 24 + len(hpos))[:, None, None]
    btris = (fq[None, :, :] + boff).reshape(-1, 3)

    pos = np.concatenate([hpos, bpos]).astype(np.float32)
    nrm = np.concatenate([hnorm, bnorm]).astype(np.float32)
    uv = np.concatenate([huv, buv]).astype(np.float32)
    tris = np.concatenate([htris, btris])

    verts = np.zeros(len(pos), dtype=_abi.VERTEX_DTYPE)
    verts["pos"] = pos
    verts["normal"][:, :3] = _half(nrm)
    verts["normal"][:, 3] = 0
    verts["uv"] = uv
    tri_count = len(tris)
    tri_shade = np.zeros(tri_count, dtype=_abi.TRISHADE_DTYPE)
    tri_shade["indices"] = tris.astype(np.uint32)
    tri_shade["material"] = np.arange(tri_count, dtype=np.uint32)

    materials = np.zeros(tri_count, dtype=_abi.MATERIAL_DTYPE)
    albedo = rng.uniform(0.0, 1.0, (tri_count, 3)).astype(np.float32)
    rough = rng.uniform(0.1, 0.9, tri_count).astype(np.float32)
    materials["diffuse"][:, :3] = albedo
    materials["diffuse"][:, 3] = 1.0
    materials["specular"][:, :3] = 0.04
    materials["glossiness"] = (1.0 - rough).astype(np.float32)
    materials["opacity"] = 1.0
    materials["code"] = SHADING_CODE

    lights = make_lights(rng)
    return Scene(verts, tri_shade, materials, lights, heightfield=params)


EMISSIVE = 2


def shading_code(model=PHONG, diffuse=BAD_TEXTURE, specular=BAD_TEXTURE, glossiness=BAD_TEXTURE):
    """SimpleMaterial::buildShadingCode (material.h:32-38): model in bits 0-15, then the glossiness,
    specular and diffuse/emissive texture ids."""
    return int(model) | (int(glossiness) << 16) | (int(specular) << 32) | (int(diffuse) << 48)


def texture_rgba8(width, height, seed=1, cells=8):
    """Seeded RGBA8 texels (rows of `width`): a checkerboard of random cell colours with
    per-texel noise, as a uint8 array [height, width, 4]."""
    rng = np.random.default_rng(seed)
    cw, ch = max(1, width // cells), max(1, height // cells)
    pal = rng.integers(0, 256, (cells + 1, cells + 1, 4))
    y, x = np.mgrid[0:height, 0:width]
    base = pal[np.minimum(y // ch, cells), np.minimum(x // cw, cells)]
    tex = np.clip(base + rng.integers(-24, 25, (height, width, 4)), 0, 255).astype(np.uint8)
    return tex


def with_textures(sc, texture_count, seed=1):
    """The scene with per-material texture use drawn from a seeded mix: untextured; a diffuse
    texture; diffuse, specular and glossiness textures; glossiness only; the emissive model with
    and without an emissive texture. Texture ids are below texture_count."""
    rng = np.random.default_rng(seed)
    m = sc.materials.copy()
    n = len(m)
    kind = rng.integers(0, 6, n)
    ids = rng.integers(0, texture_count, (n, 3))
    codes = np.empty(n, np.uint64)
    for i in range(n):
        k = kind[i]
        if k == 0:
            c = shading_code()
        elif k == 1:
            c = shading_code(diffuse=ids[i, 0])
        elif k == 2:
            c = shading_code(diffuse=ids[i, 0], specular=ids[i, 1], glossiness=ids[i, 2])
        elif k == 3:
            c = shading_code(glossiness=ids[i, 2])
        elif k == 4:
            c = shading_code(EMISSIVE, diffuse=ids[i, 0])
        else:
            c = shading_code(EMISSIVE)
        codes[i] = c
    m["code"] = codes
    em = rng.uniform(0.0, 0.6, (n, 3)).astype(np.float32)
    m["emissive"][:, :3] = np.where((kind >= 4)[:, None], em, 0.0)
    out = Scene(sc.verts, sc.tri_shade, m, sc.lights, heightfield=sc.heightfield)
    out.nodes = sc.nodes
    return out


def make_lights(rng):
    """One directional light (the reference viewer's default) plus four seeded point lights."""
    lights = []
    d = _abi.LightUnion()
    d.type = _abi.HVVR_LIGHT_DIRECTIONAL
    v = np.array([-0.25, 1.0, 0.1])
    v = v / np.linalg.norm(v)
    d.u.directional.direction = _abi.Vec3(*[float(np.float32(t)) for t in v])
    d.u.directional.power = _abi.Vec3(0.4, 0.35, 0.35)
    lights.append(d)
    for _ in range(4):
        p = _abi.LightUnion()
        p.type = _abi.HVVR_LIGHT_POINT
        p.u.point.position = _abi.Vec3(float(np.float32(rng.uniform(-8, 8))), float(np.float32(rng.uniform(1.0, 3.0))),
                                       float(np.float32(rng.uniform(-8, 8))))
        p.u.point.falloff_end = 8.0
        p.u.point.color = _abi.Vec3(*[float(np.float32(t)) for t in rng.uniform(1.0, 3.0, 3)])
        p.u.point.falloff_scale = float(np.float32(1.0 / 6.0))
        lights.append(p)
    return lights


# ---------------------------------------------------------------- the benchmark configurations (C1-C5)
def scene_c1(seed=1):
    """128x128-quad heightfield (32,768 tris) + 2,048 boxes (24,576 tris): 57,344 triangles."""
    return make_scene(128, 2048, seed)


def scene_c2(seed=1):
    """256x256-quad heightfield (131,072 tris) + 72,000 boxes (864,000 tris): 995,072 triangles."""
    return make_scene(256, 72000, seed)


def scene_sized(tri_target, seed=1):
    """Same generator at roughly tri_target triangles (heightfield about 13%, boxes the rest)."""
    quads = max(8, int(math.sqrt(tri_target * 0.13 / 2.0)))
    boxes = max(1, int((tri_target - 2 * quads * quads) / 12))
    return make_scene(quads, boxes, seed)


# ---------------------------------------------------------------- samples
def grid_samples(width, height):
    """getGridSamples (libraries/hvvr/raycaster/samples.cpp:21-42), float32 arithmetic."""
    inv_w = np.float32(1.0) / np.float32(width)
    inv_h = np.float32(1.0) / np.float32(height)
    y, x = np.meshgrid(np.arange(height, dtype=np.uint32), np.arange(width, dtype=np.uint32), indexing="ij")
    s = np.zeros(width * height, dtype=_abi.SAMPLE_DTYPE)
    s["pixel"][:, 0] = x.ravel()
    s["pixel"][:, 1] = y.ravel()
    s["position"][:, 0] = (x.ravel().astype(np.float32) + np.float32(0.5)) * inv_w
    s["position"][:, 1] = (y.ravel().astype(np.float32) + np.float32(0.5)) * inv_h
    if width > height:
        s["minor"][:, 0] = inv_w
        s["minor"][:, 1] = 0.0
        s["major"] = inv_h
    else:
        s["minor"][:, 0] = 0.0
        s["minor"][:, 1] = inv_h
        s["major"] = inv_w
    return s


def barrel_samples(width, height, k1=0.22, k2=0.24):
    """Grid samples warped by radial barrel distortion r' = r (1 + k1 r^2 + k2 r^4).

    r is measured in normalised [-1, 1]^2 sample space about the centre. The ellipse extents
    are scaled by the local radial derivative 1 + 3 k1 r^2 + 5 k2 r^4.
    """
    s = grid_samples(width, height)
    p = s["position"].astype(np.float64)
    q = 2.0 * p - 1.0
    r2 = (q * q).sum(axis=1)
    scale = 1.0 + k1 * r2 + k2 * r2 * r2
    deriv = 1.0 + 3.0 * k1 * r2 + 5.0 * k2 * r2 * r2
    q2 = q * scale[:, None]
    s["position"] = ((q2 + 1.0) * 0.5).astype(np.float32)
    s["minor"] = (s["minor"].astype(np.float64) * deriv[:, None]).astype(np.float32)
    s["major"] = (s["major"].astype(np.float64) * deriv).astype(np.float32)
    return s


def foveated_samples(count, out_w=1440, out_h=1600, fov_deg=100.0, gaze_deg=(0.0, 0.0), e0_deg=5.0,
                     jitter_seed=None):
    """About `count` samples over a fov_deg (vertical) field whose density per unit angle falls
    as 1 / (1 + (e / e0)^2) with the eccentricity e from the gaze direction.

    Placement: a Vogel (golden-angle) spiral about the gaze point with radius from the inverse
    of the radial CDF  N(E) ~ ln(1 + (E / e0)^2), clipped to the view rectangle; angles use
    the small-angle image-plane approximation e ~ |p - gaze| * fov / height. With jitter_seed,
    each sample moves by U[-0.5, 0.5] of its local spacing (per-frame temporal jitter).
    Each sample's ellipse is isotropic with the local spacing; its pixel is the output pixel
    under it. Use viewport_fov(out_w, out_h, fov_deg) for the matching camera viewport.
    """
    deg_per_px = fov_deg / out_h
    gx = out_w * 0.5 + gaze_deg[0] / deg_per_px
    gy = out_h * 0.5 + gaze_deg[1] / deg_per_px
    # farthest corner from the gaze, in degrees
    corners = np.array([[0, 0], [out_w, 0], [0, out_h], [out_w, out_h]], dtype=np.float64)
    emax = np.sqrt(((corners - [gx, gy]) ** 2).sum(axis=1)).max() * deg_per_px
    total_log = np.log1p((emax / e0_deg) ** 2)
    n = int(count)
    kept = None
    for _ in range(8):  # grow the spiral until `count` samples fall inside the rectangle
        i = np.arange(n, dtype=np.float64)
        u = (i + 0.5) / n
        e = e0_deg * np.sqrt(np.expm1(u * total_log))
        theta = i * (math.pi * (3.0 - math.sqrt(5.0)))
        r_px = e / deg_per_px
        x = gx + r_px * np.cos(theta)
        y = gy + r_px * np.sin(theta)
        inside = (x >= 0) & (x < out_w) & (y >= 0) & (y < out_h)
        kept = (x[inside], y[inside], e[inside], n)
        if inside.sum() >= count:
            break
        n = int(n * count / max(1, inside.sum()) * 1.02) + 1
    x, y, e, n = kept
    x, y, e = x[:count], y[:count], e[:count]
    # local density (samples per square degree) dN/dA = n / (pi e0^2 total_log) / (1 + (e/e0)^2)
    dens = n / (math.pi * e0_deg ** 2 * total_log) / (1.0 + (e / e0_deg) ** 2)
    spacing_px = 1.0 / np.sqrt(dens) / deg_per_px
    if jitter_seed is not None:
        rng = np.random.default_rng(jitter_seed)
        x = np.clip(x + rng.uniform(-0.5, 0.5, len(x)) * spacing_px, 0.0, out_w - 1e-3)
        y = np.clip(y + rng.uniform(-0.5, 0.5, len(y)) * spacing_px, 0.0, out_h - 1e-3)
    out = np.zeros(len(x), dtype=_abi.SAMPLE_DTYPE)
    out["pixel"][:, 0] = np.minimum(x.astype(np.int64), out_w - 1)
    out["pixel"][:, 1] = np.minimum(y.astype(np.int64), out_h - 1)
    out["position"][:, 0] = (x / out_w).astype(np.float32)
    out["position"][:, 1] = (y / out_h).astype(np.float32)
    out["minor"][:, 0] = (spacing_px / out_w).astype(np.float32)
    out["major"] = (spacing_px / out_h).astype(np.float32)
    return out


def viewport_fov(width, height, fov_deg):
    """Viewport with the given vertical field of view and the image's aspect ratio."""
    t = math.tan(math.radians(fov_deg) * 0.5)
    a = t * width / height
    return _abi.FloatRect(_abi.Vec2(-a, -t), _abi.Vec2(a, t))


# ---------------------------------------------------------------- cameras
def look_at_quaternion(eye, target, up=(0.0, 1.0, 0.0)):
    """Rotation (x, y, z, w) whose -z axis looks from eye to target with +y up."""
    eye = np.asarray(eye, dtype=np.float64)
    target = np.asarray(target, dtype=np.float64)
    look = target - eye
    z = -look / np.linalg.norm(look)
    upv = np.asarray(up, dtype=np.float64)
    y = upv - np.dot(upv, z) * z
    y /= np.linalg.norm(y)
    x = np.cross(y, z)
    m = np.stack([x, y, z], axis=1)  # columns
    tr = m[0, 0] + m[1, 1] + m[2, 2]
    if tr > 0:
        s = math.sqrt(tr + 1.0) * 2.0
        w = 0.25 * s
        qx = (m[2, 1] - m[1, 2]) / s
        qy = (m[0, 2] - m[2, 0]) / s
        qz = (m[1, 0] - m[0, 1]) / s
    elif m[0, 0] > m[1, 1] and m[0, 0] > m[2, 2]:
        s = math.sqrt(1.0 + m[0, 0] - m[1, 1] - m[2, 2]) * 2.0
        w = (m[2, 1] - m[1, 2]) / s
        qx = 0.25 * s
        qy = (m[0, 1] + m[1, 0]) / s
        qz = (m[0, 2] + m[2, 0]) / s
    elif m[1, 1] > m[2, 2]:
        s = math.sqrt(1.0 + m[1, 1] - m[0, 0] - m[2, 2]) * 2.0
        w = (m[0, 2] - m[2, 0]) / s
        qx = (m[0, 1] + m[1, 0]) / s
        qy = 0.25 * s
        qz = (m[1, 2] + m[2, 1]) / s
    else:
        s = math.sqrt(1.0 + m[2, 2] - m[0, 0] - m[1, 1]) * 2.0
        w = (m[1, 0] - m[0, 1]) / s
        qx = (m[0, 2] + m[2, 0]) / s
        qy = (m[1, 2] + m[2, 1]) / s
        qz = 0.25 * s
    return tuple(float(np.float32(v)) for v in (qx, qy, qz, w))


def camera_transform(eye=(0.0, 2.0, 10.0), target=(0.0, 0.0, 0.0)):
    return _abi.transform(look_at_quaternion(eye, target), tuple(float(np.float32(v)) for v in eye), 1.0)


def viewport_for(width, height):
    """90-degree vertical field of view, the viewer's {(-w/h,-1),(w/h,1)} convention."""
    a = float(np.float32(width) / np.float32(height))
    return _abi.FloatRect(_abi.Vec2(-a, -1.0), _abi.Vec2(a, 1.0))


def stereo_eyes(ipd=0.064, eye=(0.0, 2.0, 10.0), target=(0.0, 0.0, 0.0)):
    """Left/right camera transforms offset by +-ipd/2 along the view's x axis."""
    e = np.asarray(eye, dtype=np.float64)
    t = np.asarray(target, dtype=np.float64)
    z = -(t - e) / np.linalg.norm(t - e)
    x = np.cross((0.0, 1.0, 0.0), z)
    x /= np.linalg.norm(x)
    out = []
    for sgn in (-1.0, 1.0):
        pe = e + sgn * 0.5 * ipd * x
        out.append(camera_transform(tuple(pe), tuple(t + sgn * 0.5 * ipd * x)))
    return out
