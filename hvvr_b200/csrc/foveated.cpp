// foveated.cpp - the polar foveated sample set of the reference (host, once per camera) and the
// per-frame eye-space transform and cull planes of its foveated render path.
//
// Restates, in the reference's operation order so that the samples, their clustering and the
// frusta (hence the tile lists) are the same:
//   EccentricityMap                      libraries/hvvr/raycaster/foveated.h:32-113
//   getEyeSpacePolarFoveatedSamples      libraries/hvvr/raycaster/samples.cpp:44-142
//   generateRemapForFoveatedSamples      libraries/hvvr/raycaster/foveated.cpp:19-45
//   ComputeEyeSpaceFrusta                libraries/hvvr/raycaster/frusta.cu:26-118 (host code)
//   renderFoveatedPolarSpaceCudaReconstruct / cullRectToCullPlanes and the resolve matrices
//                                        libraries/hvvr/raycaster/render.cpp:396-492
// with the vector algebra of libraries/hvvr/shared/vector_math.h (quaternion rotation, 3x3 and
// 4x4 inverses, Plane transform of graphics_types.h:195-200).
#include "foveated.h"

#include <math.h>

#include "host_setup.h"

#include <algorithm>

namespace hvb {

namespace {

constexpr float kPi = 3.141592653589f;          // Pi (libraries/hvvr/shared/constants_math.h:15)
constexpr float kRadPerDeg = kPi / 180.0f;      // RadiansPerDegree

struct V2 { float x, y; };
struct V3 { float x, y, z; };
struct V4 { float x, y, z, w; };
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
inline V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 divs(V3 a, float s) { const float inv = 1.0f / s; return v3(a.x * inv, a.y * inv, a.z * inv); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline V3 normalize(V3 v) { return divs(v, sqrtf(dot(v, v))); }
inline float fmin2(float a, float b) { return a < b ? a : b; }
inline float fmax2(float a, float b) { return a > b ? a : b; }

// column-major 3x3 and 4x4
struct M3 { V3 m0, m1, m2; };
struct M4 { V4 m0, m1, m2, m3; };
inline V3 mul(const M3& m, V3 v) {
    return v3(m.m0.x * v.x + m.m1.x * v.y + m.m2.x * v.z, m.m0.y * v.x + m.m1.y * v.y + m.m2.y * v.z,
              m.m0.z * v.x + m.m1.z * v.y + m.m2.z * v.z);
}
inline M3 mul(const M3& a, const M3& b) { return M3{mul(a, b.m0), mul(a, b.m1), mul(a, b.m2)}; }
inline M3 add(const M3& a, const M3& b) { return M3{a.m0 + b.m0, a.m1 + b.m1, a.m2 + b.m2}; }
inline M3 scale(const M3& a, float s) { return M3{a.m0 * s, a.m1 * s, a.m2 * s}; }
inline V4 mul(const M4& m, V4 v) {
    return V4{m.m0.x * v.x + m.m1.x * v.y + m.m2.x * v.z + m.m3.x * v.w,
              m.m0.y * v.x + m.m1.y * v.y + m.m2.y * v.z + m.m3.y * v.w,
              m.m0.z * v.x + m.m1.z * v.y + m.m2.z * v.z + m.m3.z * v.w,
              m.m0.w * v.x + m.m1.w * v.y + m.m2.w * v.z + m.m3.w * v.w};
}
inline M4 mul(const M4& a, const M4& b) { return M4{mul(a, b.m0), mul(a, b.m1), mul(a, b.m2), mul(a, b.m3)}; }

M3 invert3(const M3& m) {
    const V3& x = m.m0; const V3& y = m.m1; const V3& z = m.m2;
    const float det = x.x * (y.y * z.z - z.y * y.z) - x.y * (y.x * z.z - y.z * z.x) + x.z * (y.x * z.y - y.y * z.x);
    const M3 r{v3(y.y * z.z - z.y * y.z, x.z * z.y - x.y * z.z, x.y * y.z - x.z * y.y),
               v3(y.z * z.x - y.x * z.z, x.x * z.z - x.z * z.x, y.x * x.z - x.x * y.z),
               v3(y.x * z.y - z.x * y.y, z.x * x.y - x.x * z.y, x.x * y.y - y.x * x.y)};
    const float inv = 1.0f / det;
    return scale(r, inv);
}

M4 invert4(const M4& m) {
    const V4& x = m.m0; const V4& y = m.m1; const V4& z = m.m2; const V4& w = m.m3;
    float s0 = x.x * y.y - y.x * x.y, s1 = x.x * y.z - y.x * x.z, s2 = x.x * y.w - y.x * x.w;
    float s3 = x.y * y.z - y.y * x.z, s4 = x.y * y.w - y.y * x.w, s5 = x.z * y.w - y.z * x.w;
    float c5 = z.z * w.w - w.z * z.w, c4 = z.y * w.w - w.y * z.w, m3 = z.y * w.z - w.y * z.z;
    float m2 = z.x * w.w - w.x * z.w, m1 = z.x * w.z - w.x * z.z, m0 = z.x * w.y - w.x * z.y;
    const float det = s0 * c5 - s1 * c4 + s2 * m3 + s3 * m2 - s4 * m1 + s5 * m0;
    const float idet = 1.0f / det;
    s0 *= idet; s1 *= idet; s2 *= idet; s3 *= idet; s4 *= idet; s5 *= idet;
    m0 *= idet; m1 *= idet; m2 *= idet; m3 *= idet; c4 *= idet; c5 *= idet;
    return M4{V4{y.y * c5 - y.z * c4 + y.w * m3, x.z * c4 - x.y * c5 - x.w * m3, w.y * s5 - w.z * s4 + w.w * s3,
                 z.z * s4 - z.y * s5 - z.w * s3},
              V4{y.z * m2 - y.x * c5 - y.w * m1, x.x * c5 - x.z * m2 + x.w * m1, w.z * s2 - w.x * s5 - w.w * s1,
                 z.x * s5 - z.z * s2 + z.w * s1},
              V4{y.x * c4 - y.y * m2 + y.w * m0, x.y * m2 - x.x * c4 - x.w * m0, w.x * s4 - w.y * s2 + w.w * s0,
                 z.y * s2 - z.x * s4 - z.w * s0},
              V4{y.y * m1 - y.x * m3 - y.z * m0, x.x * m3 - x.y * m1 + x.z * m0, w.y * s1 - w.x * s3 - w.z * s0,
                 z.x * s3 - z.y * s1 + z.z * s0}};
}
inline M4 transpose4(const M4& m) {
    return M4{V4{m.m0.x, m.m1.x, m.m2.x, m.m3.x}, V4{m.m0.y, m.m1.y, m.m2.y, m.m3.y},
              V4{m.m0.z, m.m1.z, m.m2.z, m.m3.z}, V4{m.m0.w, m.m1.w, m.m2.w, m.m3.w}};
}

// matrix3x3::rotationFromZAxis
M3 rotationFromZAxis(V3 z) {
    V3 y = (fabsf(z.y) > 0.85f) ? v3(-1.0f, 0.0f, 0.0f) : v3(0.0f, 1.0f, 0.0f);
    const V3 x = normalize(cross(y, z));
    y = normalize(cross(z, x));
    return M3{x, y, z};
}
// matrix3x3::axisAngle: identity + k sin + k^2 (1 - cos), k = crossProductMatrix(axis)
M3 axisAngle(V3 a, float radians) {
    const float c = cosf(radians), s = sinf(radians);
    const M3 k{v3(0.0f, a.z, -a.y), v3(-a.z, 0, a.x), v3(a.y, -a.x, 0.0f)};
    const M3 id{v3(1.0f, 0.0f, 0.0f), v3(0.0f, 1.0f, 0.0f), v3(0.0f, 0.0f, 1.0f)};
    return add(add(id, scale(k, s)), scale(mul(k, k), 1.0f - c));
}

// quaternion::fromAxisAngle(axis, r) * v = q * (v, 0) * conjugate(q)
struct Q { float x, y, z, w; };
inline Q qmul(Q a, Q b) {
    return Q{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
             a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - (a.x * b.x + a.y * b.y + a.z * b.z)};
}
inline V3 rotate(V3 axis, float radians, V3 v) {
    const float c = cosf(radians * 0.5f), s = sinf(radians * 0.5f);
    const Q q{axis.x * s, axis.y * s, axis.z * s, c};
    const Q r = qmul(qmul(q, Q{v.x, v.y, v.z, 0.0f}), Q{-q.x, -q.y, -q.z, q.w});
    return v3(r.x, r.y, r.z);
}

struct EccMap {
    float m, w0, S, invLogA, invW0, invM;
    // EccentricityMap(marSlope, maxMARDegrees, maxResolutionDegrees)
    EccMap(float marSlope, float maxMARDegrees, float maxResolutionDegrees) {
        m = marSlope;
        w0 = maxMARDegrees * kRadPerDeg;
        S = maxResolutionDegrees * kRadPerDeg;
        invLogA = float(1.0 / log(1.0 + double(m)));
        invW0 = float(1.0 / w0);
        invM = float(1.0 / m);
    }
    float apply(float i) const {
        const float e0 = i * w0;
        const float x = (e0 - S) * invW0;
        const float g = (w0 * (powf(1.0f + m, x) - 1.0f)) * invM;
        const float e1 = g + S;
        return (e0 < S) ? e0 : e1;
    }
};

struct Sorted {
    float px, py; // (azimuth, eccentricity)
    uint32_t index;
};

// one frustum of ComputeEyeSpaceFrusta: the 63-orientation search for the smallest uv box
Rays4 fitFrustum(const std::vector<PolarBeam>& beams, size_t sBegin, size_t sEnd) {
    Rays4 f;
    if (sBegin >= sEnd) {
        // no samples: a degenerate frustum (origin at infinity), culled like the reference's
        // cull-plane rejects
        for (int i = 0; i < 4; i++)
            for (int a = 0; a < 3; a++) {
                f.o[i][a] = INFINITY;
                f.d[i][a] = 0.0f;
            }
        return f;
    }
    V3 dd = v3(0.0f, 0.0f, 0.0f);
    for (size_t s = sBegin; s < sEnd; s++) dd = dd + v3(beams[s].c[0], beams[s].c[1], beams[s].c[2]);
    dd = normalize(dd);
    const M3 rot = rotationFromZAxis(dd);
    float bestArea = INFINITY;
    M3 bestRot = rot;
    V2 bestMin{INFINITY, INFINITY}, bestMax{-INFINITY, -INFINITY};
    const int orientations = 63;
    const float slop = 2.0f;
    for (int o = 0; o < orientations; ++o) {
        const float range = (kPi / 2.0f) * 0.8f;
        const M3 cur = mul(axisAngle(v3(0, 0, 1), (range * o / float(orientations)) - (range / 2.0f)), rot);
        const M3 inv = invert3(cur);
        V2 mn{INFINITY, INFINITY}, mx{-INFINITY, -INFINITY};
        for (size_t s = sBegin; s < sEnd; s++) {
            const V3 c = v3(beams[s].c[0], beams[s].c[1], beams[s].c[2]);
            const V3 du = v3(beams[s].du[0], beams[s].du[1], beams[s].du[2]);
            const V3 dv = v3(beams[s].dv[0], beams[s].dv[1], beams[s].dv[2]);
            V3 v = mul(inv, c);
            const V2 uv{v.x / v.z, v.y / v.z};
            v = mul(inv, du + c);
            V2 d{uv.x - v.x / v.z, uv.y - v.y / v.z};
            float r = sqrtf(d.x * d.x + d.y * d.y);
            v = mul(inv, dv + c);
            d = V2{uv.x - v.x / v.z, uv.y - v.y / v.z};
            r = fmax2(r, sqrtf(d.x * d.x + d.y * d.y));
            r *= slop;
            mn = V2{fmin2(mn.x, uv.x - r), fmin2(mn.y, uv.y - r)};
            mx = V2{fmax2(mx.x, uv.x + r), fmax2(mx.y, uv.y + r)};
        }
        const float area = (mx.x - mn.x) * (mx.y - mn.y);
        if (area < bestArea) {
            bestRot = cur;
            bestArea = area;
            bestMin = mn;
            bestMax = mx;
        }
    }
    auto toDir = [&](float u, float v) { return mul(bestRot, normalize(v3(u, v, 1.0f))); };
    const V3 dirs[4] = {toDir(bestMin.x, bestMax.y), toDir(bestMax.x, bestMax.y), toDir(bestMax.x, bestMin.y),
                        toDir(bestMin.x, bestMin.y)};
    for (int i = 0; i < 4; i++) {
        f.o[i][0] = f.o[i][1] = f.o[i][2] = 0.0f;
        f.d[i][0] = dirs[i].x; f.d[i][1] = dirs[i].y; f.d[i][2] = dirs[i].z;
    }
    return f;
}

} // namespace

void buildPolarFoveatedSetup(float degreeTrackingError, float maxFOVDegrees, float marSlope, float fovealMARDegrees,
                             PolarSetup& out) {
    FtzDazScope ftz;
    const EccMap emap(marSlope, fovealMARDegrees, degreeTrackingError);
    out.eccM = emap.m;
    out.eccW0 = emap.w0;
    out.eccS = emap.S;
    out.eccInvW0 = emap.invW0;
    out.eccInvLogA = emap.invLogA;
    out.eccInvM = emap.invM;
    out.maxEccentricity = maxFOVDegrees * kRadPerDeg;
    // ring count and samples per ring (getEyeSpacePolarFoveatedSamples, first pass)
    size_t samplesPerRing = 0, ringCount = 0;
    {
        float E = 0.0f;
        while (E <= maxFOVDegrees * kRadPerDeg) {
            const float w = emap.apply(ringCount + 1.0f) - E;
            const float ringRadius = sinf(E);
            const float around = 2.0f * kPi * ringRadius;
            const size_t onAnnulus = size_t(std::ceil(around / w));
            samplesPerRing = std::max(samplesPerRing, onAnnulus);
            ++ringCount;
            E = emap.apply(float(ringCount));
        }
    }
    std::vector<PolarBeam> unsorted(ringCount * samplesPerRing);
    float E = 0.0f;
    for (size_t r = 0; r < ringCount; ++r) {
        const float eNext = emap.apply(r + 1.0f);
        const float ringRadius = sinf(E);
        const float around = 2.0f * kPi * ringRadius;
        const V3 base = normalize(rotate(v3(0, 1, 0), E, v3(0, 0, -1)));
        const V3 zenBase = normalize(rotate(v3(0, 1, 0), eNext, v3(0, 0, -1)));
        for (size_t i = 0; i < samplesPerRing; ++i) {
            const float rad = (i + 0.5f) / float(samplesPerRing) * 2.0f * kPi;
            const V3 p = normalize(rotate(v3(0, 0, -1), rad, base));
            const V3 zdir = normalize(rotate(v3(0, 0, -1), rad, zenBase));
            const V3 onTangent = zdir * (1.0f / dot(zdir, p));
            const V3 zenithDiff = onTangent - p;
            const V3 azUnit = cross(p, normalize(zenithDiff));
            const V3 azimuthalDiff = divs(azUnit * around, float(samplesPerRing));
            PolarBeam& b = unsorted[samplesPerRing * r + i];
            b.c[0] = p.x; b.c[1] = p.y; b.c[2] = p.z;
            b.du[0] = zenithDiff.x; b.du[1] = zenithDiff.y; b.du[2] = zenithDiff.z;
            b.dv[0] = azimuthalDiff.x; b.dv[1] = azimuthalDiff.y; b.dv[2] = azimuthalDiff.z;
        }
        E = eNext;
    }
    // cluster in (azimuth, eccentricity)
    const size_t n = unsorted.size();
    std::vector<Sorted> toSort(n);
    for (size_t i = 0; i < n; ++i) {
        const V3 v = v3(unsorted[i].c[0], unsorted[i].c[1], unsorted[i].c[2]);
        toSort[i].py = acosf(-v.z);
        const V3 dir = normalize(v3(v.x, v.y, 0.0f));
        toSort[i].px = atan2f(dir.y, dir.x);
        toSort[i].index = uint32_t(i);
    }
    const size_t blocks = (n + kBlockSize - 1) / kBlockSize;
    // naiveXYCluster on (azimuth, eccentricity)
    naiveCluster(toSort, blocks, [](const Sorted& a) { return a.px; }, [](const Sorted& a) { return a.py; });
    out.samplesPerRing = uint32_t(samplesPerRing);
    out.ringCount = uint32_t(ringCount);
    out.valid = uint32_t(n);
    out.blocks = uint32_t(blocks);
    out.tiles = uint32_t(blocks * kTilesPerBlock);
    out.padded = uint32_t(blocks * kBlockSize);
    out.beams.assign(n, PolarBeam{});
    out.remap.assign(size_t(out.padded) * 2, 0xffffffffu);
    for (size_t s = 0; s < n; ++s) {
        const uint32_t i = toSort[s].index;
        out.beams[s] = unsorted[i];
        out.remap[2 * s + 0] = uint32_t(i % samplesPerRing);
        out.remap[2 * s + 1] = uint32_t(i / samplesPerRing);
    }
    out.tileRays.resize(out.tiles);
    out.blockRays.resize(out.blocks);
    for (size_t t = 0; t < out.tiles; t++)
        out.tileRays[t] = fitFrustum(out.beams, std::min(t * kTileSize, n), std::min((t + 1) * kTileSize, n));
    for (size_t b = 0; b < out.blocks; b++)
        out.blockRays[b] = fitFrustum(out.beams, std::min(b * kBlockSize, n), std::min((b + 1) * kBlockSize, n));
}

void foveatedFrame(const float cameraToWorld[16], const hvvr_vec3& eyeDir, const hvvr_float_rect& sampleBounds,
                   const hvvr_float_rect& viewport, float eyeToWorld[16], float planes[4][4]) {
    FtzDazScope ftz;
    auto col = [&](const float* m, int c) { return V4{m[4 * c + 0], m[4 * c + 1], m[4 * c + 2], m[4 * c + 3]}; };
    const M4 c2w{col(cameraToWorld, 0), col(cameraToWorld, 1), col(cameraToWorld, 2), col(cameraToWorld, 3)};
    // eyeToCamera = rotationFromZAxis(-eyeDirection); eyeToWorld = cameraToWorld * matrix4x4(eyeToCamera)
    const M3 e2c = rotationFromZAxis(-v3(eyeDir.x, eyeDir.y, eyeDir.z));
    const M4 e2c4{V4{e2c.m0.x, e2c.m0.y, e2c.m0.z, 0.0f}, V4{e2c.m1.x, e2c.m1.y, e2c.m1.z, 0.0f},
                  V4{e2c.m2.x, e2c.m2.y, e2c.m2.z, 0.0f}, V4{0.0f, 0.0f, 0.0f, 1.0f}};
    const M4 e2w = mul(c2w, e2c4);
    const V4* cols = &e2w.m0;
    for (int c = 0; c < 4; c++) {
        eyeToWorld[4 * c + 0] = cols[c].x; eyeToWorld[4 * c + 1] = cols[c].y;
        eyeToWorld[4 * c + 2] = cols[c].z; eyeToWorld[4 * c + 3] = cols[c].w;
    }
    // cullRectToCullPlanes(sampleBounds, planes, sampleToCamera, invert(eyeToCamera), eyeToWorld)
    const M3 s2c{v3(viewport.upper.x - viewport.lower.x, 0, 0), v3(0, viewport.lower.y - viewport.upper.y, 0),
                 v3(viewport.lower.x, viewport.upper.y, -1)};
    const M3 c2e = invert3(e2c);
    const V2 U{sampleBounds.upper.x, sampleBounds.upper.y}, L{sampleBounds.lower.x, sampleBounds.lower.y};
    const V2 dirs[4] = {{U.x, U.y}, {L.x, U.y}, {L.x, L.y}, {U.x, L.y}};
    const M4 nT = transpose4(invert4(e2w));
    for (int i = 0; i < 4; ++i) {
        const V3 d0 = mul(s2c, v3(dirs[i].x, dirs[i].y, 1.0f));
        const V3 d1 = mul(s2c, v3(dirs[(i + 1) % 4].x, dirs[(i + 1) % 4].y, 1.0f));
        const V3 n = mul(c2e, normalize(cross(d1, d0)));
        const float dist = -0.01f;
        // Plane operator*(matrix4x4, Plane)
        const V3 pn = n * dist;
        const V4 O = mul(e2w, V4{pn.x, pn.y, pn.z, 1.0f});
        const V4 N4 = mul(nT, V4{n.x, n.y, n.z, 0});
        const V3 N = v3(N4.x, N4.y, N4.z);
        planes[i][0] = N.x;
        planes[i][1] = N.y;
        planes[i][2] = N.z;
        planes[i][3] = dot(v3(O.x, O.y, O.z), N);
    }
}

void foveatedResolveFrame(const float eyeToWorld[16], const hvvr_vec3& eyeDir, const hvvr_float_rect& viewport,
                          float worldToEyePrev[16], float eyePrevToSamplePrev[9], float sampleToEye[9],
                          float eyeToSamplePrev[16]) {
    FtzDazScope ftz;
    auto col4 = [&](const float* m, int c) { return V4{m[4 * c + 0], m[4 * c + 1], m[4 * c + 2], m[4 * c + 3]}; };
    auto col3 = [&](const float* m, int c) { return v3(m[3 * c + 0], m[3 * c + 1], m[3 * c + 2]); };
    const M4 e2w{col4(eyeToWorld, 0), col4(eyeToWorld, 1), col4(eyeToWorld, 2), col4(eyeToWorld, 3)};
    const M4 w2ep{col4(worldToEyePrev, 0), col4(worldToEyePrev, 1), col4(worldToEyePrev, 2), col4(worldToEyePrev, 3)};
    const M3 ep2sp{col3(eyePrevToSamplePrev, 0), col3(eyePrevToSamplePrev, 1), col3(eyePrevToSamplePrev, 2)};
    // sampleToEye = invert(eyeToCamera) * getSampleToCamera()
    const M3 e2c = rotationFromZAxis(-v3(eyeDir.x, eyeDir.y, eyeDir.z));
    const M3 s2c{v3(viewport.upper.x - viewport.lower.x, 0, 0), v3(0, viewport.lower.y - viewport.upper.y, 0),
                 v3(viewport.lower.x, viewport.upper.y, -1)};
    const M3 s2e = mul(invert3(e2c), s2c);
    // eyeToSamplePrevious = matrix4x4(eyePreviousToSamplePrevious) * (worldToEyePrevious * eyeToWorld)
    const M4 e2ep = mul(w2ep, e2w);
    const M4 ep2sp4{V4{ep2sp.m0.x, ep2sp.m0.y, ep2sp.m0.z, 0.0f}, V4{ep2sp.m1.x, ep2sp.m1.y, ep2sp.m1.z, 0.0f},
                    V4{ep2sp.m2.x, ep2sp.m2.y, ep2sp.m2.z, 0.0f}, V4{0.0f, 0.0f, 0.0f, 1.0f}};
    const M4 e2sp = mul(ep2sp4, e2ep);
    const V3* c3 = &s2e.m0;
    for (int c = 0; c < 3; c++) {
        sampleToEye[3 * c + 0] = c3[c].x; sampleToEye[3 * c + 1] = c3[c].y; sampleToEye[3 * c + 2] = c3[c].z;
    }
    const V4* c4 = &e2sp.m0;
    for (int c = 0; c < 4; c++) {
        eyeToSamplePrev[4 * c + 0] = c4[c].x; eyeToSamplePrev[4 * c + 1] = c4[c].y;
        eyeToSamplePrev[4 * c + 2] = c4[c].z; eyeToSamplePrev[4 * c + 3] = c4[c].w;
    }
    // the camera's history for the next frame
    const M4 w2e = invert4(e2w);
    const V4* h4 = &w2e.m0;
    for (int c = 0; c < 4; c++) {
        worldToEyePrev[4 * c + 0] = h4[c].x; worldToEyePrev[4 * c + 1] = h4[c].y;
        worldToEyePrev[4 * c + 2] = h4[c].z; worldToEyePrev[4 * c + 3] = h4[c].w;
    }
    const M3 e2s = invert3(s2e);
    const V3* h3 = &e2s.m0;
    for (int c = 0; c < 3; c++) {
        eyePrevToSamplePrev[3 * c + 0] = h3[c].x; eyePrevToSamplePrev[3 * c + 1] = h3[c].y;
        eyePrevToSamplePrev[3 * c + 2] = h3[c].z;
    }
}

} // namespace hvb
