// host_setup.cpp - camera matrices, MSAA offsets and the sample hierarchy (host).
#include "host_setup.h"

#include <immintrin.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <random>

namespace hvb {

FtzDazScope::FtzDazScope() {
    saved = _mm_getcsr();
    _mm_setcsr(saved | 0x8040u);
}
FtzDazScope::~FtzDazScope() { _mm_setcsr(saved); }

namespace {

struct V3 {
    float x, y, z;
};
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 scale(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 normalize(V3 v) {
    float inv = 1.0f / sqrtf(dot(v, v));
    return scale(v, inv);
}
inline float fmin2(float a, float b) { return a < b ? a : b; }
inline float fmax2(float a, float b) { return a > b ? a : b; }

// column-major 3x3 (matrix3x3 {m0,m1,m2})
struct M3 {
    V3 c0, c1, c2;
};
inline V3 mul(const M3& m, V3 v) {
    return v3(m.c0.x * v.x + m.c1.x * v.y + m.c2.x * v.z, m.c0.y * v.x + m.c1.y * v.y + m.c2.y * v.z,
              m.c0.z * v.x + m.c1.z * v.y + m.c2.z * v.z);
}

const int kTau[] = {1,  1,  1,  2,  3,  2,  5,  2,  3,  2,  3,  3,  5,  5,  3,  4,  7,  5,  5,  7,
                    9,  8,  5,  5,  7,  7,  7,  8,  5,  8,  11, 12, 7,  10, 13, 8,  11, 8,  7,  14};

struct Sorted {
    hvvr_sample s;
    uint32_t channel;
};

// naiveXYCluster (libraries/hvvr/raycaster/sample_clustering.h:17-49): y-then-x sort, then
// x-then-y within rows of blocks, y-then-x within blocks, x-then-y within runs of 8 tiles
void clusterXY(std::vector<Sorted>& v, size_t k) {
    naiveCluster(v, k, [](const Sorted& a) { return a.s.position.x; }, [](const Sorted& a) { return a.s.position.y; });
}

// sphericalUVToDirection (libraries/hvvr/raycaster/sample_hierarchy.cpp:27-35)
V3 sphericalDir(float u, float v, float fovX, float fovY) {
    const float rad = 3.141592653589f / 180.0f;
    const float yaw = (u - .5f) * (fovX * rad);
    const float pitch = -(v - .5f) * (fovY * rad);
    return normalize(v3(sinf(yaw) * cosf(pitch), sinf(pitch), -cosf(yaw) * cosf(pitch)));
}

// get3DFrustumFrom2D (libraries/hvvr/raycaster/sample_hierarchy.cpp:46-123). f = {xMin, -xMax, yMin, -yMax}.
Rays4 frustumFrom2D(const float f[4], const M3& S, const hvvr_thin_lens& lens, bool spherical, float fovX,
                    float fovY) {
    const float farPlane = -100.0f;
    const float xMin = f[0], xMax = -f[1], yMin = f[2], yMax = -f[3];
    const V3 nearP[4] = {v3(-lens.radius, -lens.radius, 0), v3(+lens.radius, -lens.radius, 0),
                         v3(+lens.radius, +lens.radius, 0), v3(-lens.radius, +lens.radius, 0)};
    V3 rd[4] = {mul(S, v3(xMin, yMax, 1)), mul(S, v3(xMax, yMax, 1)), mul(S, v3(xMax, yMin, 1)),
                mul(S, v3(xMin, yMin, 1))};
    Rays4 r;
    if (spherical) {
        const float uv[4][2] = {{xMin, yMax}, {xMax, yMax}, {xMax, yMin}, {xMin, yMin}};
        for (int i = 0; i < 4; i++) {
            rd[i] = sphericalDir(uv[i][0], uv[i][1], fovX, fovY);
            r.o[i][0] = nearP[i].x; r.o[i][1] = nearP[i].y; r.o[i][2] = nearP[i].z;
            r.d[i][0] = rd[i].x; r.d[i][1] = rd[i].y; r.d[i][2] = rd[i].z;
        }
        return r;
    }
    V3 focus[4];
    for (int i = 0; i < 4; i++) focus[i] = scale(rd[i], lens.focal_distance / -rd[i].z);
    float fxMax = -INFINITY, fxMin = INFINITY, fyMax = -INFINITY, fyMin = INFINITY;
    for (int i = 0; i < 4; ++i) {
        for (int j = 0; j < 4; ++j) {
            const V3 pos = nearP[i];
            const V3 dir = normalize(sub(focus[j], pos));
            const V3 p = add(pos, scale(dir, farPlane / dir.z));
            fxMax = fmax2(fxMax, p.x);
            fxMin = fmin2(fxMin, p.x);
            fyMax = fmax2(fyMax, p.y);
            fyMin = fmin2(fyMin, p.y);
        }
    }
    const V3 farP[4] = {v3(fxMin, fyMin, farPlane), v3(fxMax, fyMin, farPlane), v3(fxMax, fyMax, farPlane),
                        v3(fxMin, fyMax, farPlane)};
    for (int i = 0; i < 4; i++) {
        const V3 d = normalize(sub(farP[i], nearP[i]));
        r.o[i][0] = nearP[i].x; r.o[i][1] = nearP[i].y; r.o[i][2] = nearP[i].z;
        r.d[i][0] = d.x; r.d[i][1] = d.y; r.d[i][2] = d.z;
    }
    return r;
}

} // namespace

Mat4 transformToMatrix(const hvvr_transform& t) {
    const float qx = t.rotation.x, qy = t.rotation.y, qz = t.rotation.z, qw = t.rotation.w;
    const float x2 = qx + qx, y2 = qy + qy, z2 = qz + qz;
    const float xx = qx * x2, yy = qy * y2, zz = qz * z2;
    const float xy = qx * y2, yz = qy * z2, xz = qz * x2;
    const float wx = qw * x2, wy = qw * y2, wz = qw * z2;
    const float s = t.scale;
    Mat4 m;
    const float c0[3] = {1.0f - (yy + zz), xy + wz, xz - wy};
    const float c1[3] = {xy - wz, 1.0f - (xx + zz), yz + wx};
    const float c2[3] = {xz + wy, yz - wx, 1.0f - (xx + yy)};
    for (int r = 0; r < 3; r++) {
        m.m[0][r] = c0[r] * s;
        m.m[1][r] = c1[r] * s;
        m.m[2][r] = c2[r] * s;
    }
    m.m[0][3] = m.m[1][3] = m.m[2][3] = 0.0f;
    m.m[3][0] = t.translation.x;
    m.m[3][1] = t.translation.y;
    m.m[3][2] = t.translation.z;
    m.m[3][3] = 1.0f;
    return m;
}

void msaaOffsets(uint32_t n, float* out) {
    const int turns = kTau[n];
    for (uint32_t i = 0; i < n; i++) {
        const float alpha = float(int(i) + 0.5f) * (1.0f / float(n));
        const float angle = alpha * (float(turns) * 6.28f) + 0.0f;
        const float radius = sqrtf(alpha);
        out[2 * i + 0] = cosf(angle) * radius;
        out[2 * i + 1] = sinf(angle) * radius;
    }
}

// The alternative pattern (no counterpart in the reference): an n-rooks lattice, subsample i in
// column i and row (k i) mod n of an n x n grid over [-1, 1]^2 (k = 1, 3, 5, 9, 19 for
// n = 2, 4, 8, 16, 32: one subsample per row and column, the rows spread), scaled by 1/sqrt(2) into
// the unit disk the spiral fills; rate 1 is the sample's centre.
void msaaOffsetsRotatedGrid(uint32_t n, float* out) {
    const uint32_t k = n == 2 ? 1u : n == 4 ? 3u : n == 8 ? 5u : n == 16 ? 9u : n == 32 ? 19u : 0u;
    for (uint32_t i = 0; i < n; i++) {
        const float x = float(2 * i + 1) / float(n) - 1.0f;
        const float y = float(2 * ((k * i) % n) + 1) / float(n) - 1.0f;
        out[2 * i + 0] = x * 0.70710677f;
        out[2 * i + 1] = y * 0.70710677f;
    }
}

// GPUCamera::initLookupTables (libraries/hvvr/raycaster/gpu_camera.cu:59-88): for each of the 4
// table tiles and 128 samples one random rotation (std::mt19937, default seed, drawn through
// uniform_real_distribution<float> and scaled by Tau), and subsample i of that sample takes the
// rotated spiral position (7 i + 7) mod n. Layout [tile][subsample][sample], 2 floats each.
void lensTable(uint32_t n, float* out) {
    std::uniform_real_distribution<float> dist(0.0f, 1.0f);
    std::mt19937 gen;
    const float tauF = 6.283185307180f; // Tau (libraries/hvvr/shared/constants_math.h:16)
    const int turns = kTau[n];
    for (uint32_t tile = 0; tile < 4; tile++)
        for (uint32_t s = 0; s < kTileSize; s++) {
            const float rotation = dist(gen) * tauF;
            for (uint32_t i = 0; i < n; i++) {
                const int k = int((i * 7 + 7) % n);
                const float alpha = float(k + 0.5f) * (1.0f / float(n));
                const float angle = alpha * (float(turns) * 6.28f) + rotation;
                const float radius = sqrtf(alpha);
                const size_t o = (size_t(tile) * kTileSize * n + size_t(i) * kTileSize + s) * 2;
                out[o + 0] = cosf(angle) * radius;
                out[o + 1] = sinf(angle) * radius;
            }
        }
}

void buildSampleSetup(const hvvr_sample* samples, uint32_t count, uint32_t split, const hvvr_float_rect& vp,
                      const hvvr_thin_lens& lens, float fovXDeg, float fovYDeg, uint32_t width, uint32_t height,
                      SampleSetup& out) {
    FtzDazScope ftz;
    const bool spherical = fovXDeg > 0.0f;
    std::vector<Sorted> sorted(count);
    for (uint32_t i = 0; i < count; i++) sorted[i] = Sorted{samples[i], i % split};
    const uint32_t blocks = (count + kBlockSize - 1) / kBlockSize;
    clusterXY(sorted, blocks);
    out.blocks = blocks;
    out.tiles = blocks * kTilesPerBlock;
    out.padded = blocks * kBlockSize;
    out.valid = count;
    // Camera::getSampleToCamera (libraries/hvvr/raycaster/camera.cpp:167-171)
    const M3 S{v3(vp.upper.x - vp.lower.x, 0, 0), v3(0, vp.lower.y - vp.upper.y, 0), v3(vp.lower.x, vp.upper.y, -1)};
    // BeamBatch2D (sample_hierarchy.cpp:154-190): tile rectangles padded by the major axis,
    // blocks as unions, unpacked ellipses; padding samples past the last one stay zero
    std::vector<float> center(2 * size_t(out.padded), 0.0f), major(2 * size_t(out.padded), 0.0f),
        minor(2 * size_t(out.padded), 0.0f);
    out.tileRays.resize(out.tiles);
    out.blockRays.resize(blocks);
    const uint32_t maxIndex = count - 1;
    uint32_t si = 0;
    for (uint32_t b = 0; b < blocks; b++) {
        float bf[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
        for (uint32_t t = 0; t < kTilesPerBlock; t++) {
            float tf[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
            for (uint32_t k = 0; k < kTileSize; k++) {
                const hvvr_sample& s = sorted[si].s;
                const float x = s.position.x, y = s.position.y, mj = s.major_axis_length;
                const float xs[2] = {x + mj, x - mj}, ys[2] = {y + mj, y - mj};
                for (int q = 0; q < 2; q++) {
                    tf[0] = fmin2(tf[0], xs[q]);
                    tf[1] = fmin2(tf[1], -xs[q]);
                    tf[2] = fmin2(tf[2], ys[q]);
                    tf[3] = fmin2(tf[3], -ys[q]);
                }
                // unpackSample (libraries/hvvr/raycaster/samples.cpp:144-159)
                const float ext = 0.70710678118f;
                const float mnx = s.minor_axis.x * ext, mny = s.minor_axis.y * ext;
                const float mlen = sqrtf(s.minor_axis.x * s.minor_axis.x + s.minor_axis.y * s.minor_axis.y);
                const float rescale = s.major_axis_length * ext / mlen;
                center[2 * si] = x;
                center[2 * si + 1] = y;
                minor[2 * si] = mnx;
                minor[2 * si + 1] = mny;
                major[2 * si] = -mny * rescale;
                major[2 * si + 1] = mnx * rescale;
                si = std::min(si + 1, maxIndex);
            }
            for (int j = 0; j < 4; j++) tf[j] = fmax2(tf[j], -INFINITY); // intersect with the +-inf cull rect
            out.tileRays[b * kTilesPerBlock + t] = frustumFrom2D(tf, S, lens, spherical, fovXDeg, fovYDeg);
            for (int j = 0; j < 4; j++) bf[j] = fmin2(bf[j], tf[j]);
        }
        out.blockRays[b] = frustumFrom2D(bf, S, lens, spherical, fovXDeg, fovYDeg);
    }
    // BeamBatch::generateFrom2D beams (sample_hierarchy.cpp:129-152)
    out.beams.assign(size_t(out.padded) * 12, 0.0f);
    for (uint32_t i = 0; i < out.padded; i++) {
        V3 c = mul(S, v3(center[2 * i], center[2 * i + 1], 1.0f));
        V3 du = mul(S, v3(major[2 * i], major[2 * i + 1], 0.0f));
        V3 dv = mul(S, v3(minor[2 * i], minor[2 * i + 1], 0.0f));
        if (spherical) {
            const float cu = center[2 * i], cv = center[2 * i + 1];
            c = sphericalDir(cu, cv, fovXDeg, fovYDeg);
            du = sub(sphericalDir(cu + major[2 * i], cv + major[2 * i + 1], fovXDeg, fovYDeg), c);
            dv = sub(sphericalDir(cu + minor[2 * i], cv + minor[2 * i + 1], fovXDeg, fovYDeg), c);
        }
        float* b = &out.beams[size_t(i) * 12];
        b[0] = c.x; b[1] = c.y; b[2] = c.z; b[3] = du.x;
        b[4] = du.y; b[5] = du.z; b[6] = dv.x; b[7] = dv.y;
        b[8] = dv.z; b[9] = 0.0f; b[10] = 0.0f; b[11] = 0.0f;
    }
    // imageLocationToSampleIndex (camera.cpp:57-63)
    out.remap.assign(size_t(width) * height * split, -1);
    for (uint32_t i = 0; i < count; i++) {
        const hvvr_sample& s = sorted[i].s;
        const size_t idx = (size_t(s.pixel_y) * width + s.pixel_x) * split + sorted[i].channel;
        if (s.pixel_x < width && s.pixel_y < height) out.remap[idx] = int32_t(i);
    }
}

} // namespace hvb
