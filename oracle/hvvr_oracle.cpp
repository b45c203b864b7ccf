// hvvr_oracle.cpp - TEST INFRASTRUCTURE ONLY (see hvvr_oracle.h).
//
// Scalar restatement of the reference primary-visibility path. Every function cites the
// reference lines it restates (paths relative to the reference project root; RC/ =
// libraries/hvvr/raycaster/, SH/ = libraries/hvvr/shared/).
//
// Floating point: built with -ffp-contract=off; MXCSR FTZ|DAZ is set for the duration of
// oracle_render exactly as the reference sets it on its worker threads (RC/raycaster.cpp:21-27).
// fmaf() appears only where the reference issues an explicit FMA (_mm256_fmadd_ps in
// RC/traverse_avx.{h,cpp}) or where its kernel comments mark FMA (RC/prim_tests.h:193-229,
// HVVR_FP_FMA mode).

#include "hvvr_oracle.h"

#include <immintrin.h>
#include <math.h>
#include <float.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <map>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

namespace {

enum { kTileSize = 128, kTilesPerBlock = 64, kBlockSize = kTileSize * kTilesPerBlock };
enum { kBlockStackSize = 64, kTileStackMax = 4096 };

struct V2 { float x, y; };
struct V3 { float x, y, z; };
struct V4 { float x, y, z, w; };

inline V3 mk(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator-(V3 a) { return mk(-a.x, -a.y, -a.z); }
inline V3 operator*(V3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline V3 operator*(V3 a, V3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
// vector3::operator/(float) multiplies by the reciprocal (SH/vector_math.h:210-213)
inline V3 divs(V3 a, float s) { float inv = 1.0f / s; return mk(a.x * inv, a.y * inv, a.z * inv); }
// SH/vector_math.h:262-286
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline float length(V3 v) { return sqrtf(dot(v, v)); }
inline V3 normalize(V3 v) { return divs(v, length(v)); }
// SH/util.h:46-47 (min/max templates)
inline float tmin(float a, float b) { return a < b ? a : b; }
inline float tmax(float a, float b) { return a > b ? a : b; }
inline float sat(float x) { return x > 0.0f ? (x < 1.0f ? x : 1.0f) : 0.0f; } // __saturatef (NaN -> 0)

inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
inline float bitsf(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
// denormals-are-zero view of a float, for comparisons the reference makes under MXCSR.DAZ
inline float daz(float f) { uint32_t u = fbits(f); return (u & 0x7f800000u) == 0 ? bitsf(u & 0x80000000u) : f; }

// column-major matrices (SH/vector_math.h:1003-1133, 1152-1278)
struct M3 { V3 m0, m1, m2; };
struct M4 { V4 m0, m1, m2, m3; };
inline V3 mul(const M3& m, V3 v) {
    return mk(m.m0.x * v.x + m.m1.x * v.y + m.m2.x * v.z, m.m0.y * v.x + m.m1.y * v.y + m.m2.y * v.z,
              m.m0.z * v.x + m.m1.z * v.y + m.m2.z * v.z);
}
inline V4 mul(const M4& m, V4 v) {
    return V4{m.m0.x * v.x + m.m1.x * v.y + m.m2.x * v.z + m.m3.x * v.w,
              m.m0.y * v.x + m.m1.y * v.y + m.m2.y * v.z + m.m3.y * v.w,
              m.m0.z * v.x + m.m1.z * v.y + m.m2.z * v.z + m.m3.z * v.w,
              m.m0.w * v.x + m.m1.w * v.y + m.m2.w * v.z + m.m3.w * v.w};
}
// mul(m, v) as the reference's GPU build (nvcc, -use_fast_math) contracts it in
// SceneTransformVerticesKernel (RC/gpu_scene_state.cu:118): per component, the first column's
// product fused into the rounded second one, then the third and fourth fused in turn
inline V4 mulFma(const M4& m, V4 v) {
    auto row = [&](float a, float b, float c, float d) {
        return fmaf(d, v.w, fmaf(c, v.z, fmaf(a, v.x, b * v.y)));
    };
    return V4{row(m.m0.x, m.m1.x, m.m2.x, m.m3.x), row(m.m0.y, m.m1.y, m.m2.y, m.m3.y),
              row(m.m0.z, m.m1.z, m.m2.z, m.m3.z), row(m.m0.w, m.m1.w, m.m2.w, m.m3.w)};
}
inline M3 m3of(const M4& m) { return M3{mk(m.m0.x, m.m0.y, m.m0.z), mk(m.m1.x, m.m1.y, m.m1.z), mk(m.m2.x, m.m2.y, m.m2.z)}; }

// matrix4x4(const transform&) = matrix4x4(matrix3x3(rotation) * scale, translation)
// (SH/vector_math.h:1021-1037 quaternion->matrix, 1158, 1161)
M4 transformToMatrix(const hvvr_transform& t) {
    float qx = t.rotation.x, qy = t.rotation.y, qz = t.rotation.z, qw = t.rotation.w;
    float x2 = qx + qx, y2 = qy + qy, z2 = qz + qz;
    float xx = qx * x2, yy = qy * y2, zz = qz * z2;
    float xy = qx * y2, yz = qy * z2, xz = qz * x2;
    float wx = qw * x2, wy = qw * y2, wz = qw * z2;
    V3 c0 = mk(1.0f - (yy + zz), xy + wz, xz - wy);
    V3 c1 = mk(xy - wz, 1.0f - (xx + zz), yz + wx);
    V3 c2 = mk(xz + wy, yz - wx, 1.0f - (xx + yy));
    float s = t.scale;
    c0 = c0 * s; c1 = c1 * s; c2 = c2 * s;
    return M4{V4{c0.x, c0.y, c0.z, 0.0f}, V4{c1.x, c1.y, c1.z, 0.0f}, V4{c2.x, c2.y, c2.z, 0.0f},
              V4{t.translation.x, t.translation.y, t.translation.z, 1.0f}};
}

// ------------------------------------------------------------------ BVH node (RC/bvh_node.h:17-36)
struct Node {
    float b[6][4]; // xMax, xNegMin, yMax, yNegMin, zMax, zNegMin
    uint32_t leafMask;
    uint32_t tri[5]; // leaf.triIndex[5]; children.offset[k] aliases tri[k+1]
    uint32_t pad[2];
};
static_assert(sizeof(Node) == 128, "node");
inline uint32_t childOf(const Node* nodes, uint32_t n, int k) { return n + nodes[n].tri[k + 1]; }

struct Tri { V3 v0, e0, e1; };

inline float halfToFloat(uint16_t h) { return _cvtsh_ss(h); }
inline uint16_t floatToHalf(float f) { return (uint16_t)_cvtss_sh(f, 0); }

// ------------------------------------------------------------------ scene build + refit
struct Scene {
    std::vector<Node> nodes;
    std::vector<hvvr_tri_shade> triShade;
    std::vector<hvvr_shading_vertex> verts;     // untransformed, merged
    std::vector<uint32_t> vertModel;
    std::vector<hvvr_material> materials;
    std::vector<hvvr_shading_vertex> world;     // transformed
    std::vector<Tri> tris;
    uint32_t status = 0;
};

// Raycaster::buildScene (RC/scene_update.cpp:22-143)
void buildScene(const oracle_frame_in* in, Scene& s) {
    uint32_t modelCount = in->model_count;
    if (modelCount == 0) {
        s.nodes.assign(1, Node{});
        s.nodes[0].leafMask = 0xf;
        return;
    }
    uint32_t rootNodeCount = (modelCount + 1) / 3;
    uint32_t vc = 0, tc = 0, nc = rootNodeCount, mc = 0;
    for (uint32_t m = 0; m < modelCount; m++) {
        vc += in->models[m].vert_count; tc += in->models[m].tri_count;
        nc += in->models[m].node_count; mc += in->models[m].material_count;
    }
    s.nodes.assign(nc, Node{});
    s.triShade.resize(tc);
    s.verts.resize(vc);
    s.vertModel.resize(vc);
    s.materials.resize(mc);
    std::vector<uint32_t> viewOffsets(modelCount);
    uint32_t vOff = 0, tOff = 0, mOff = 0, nOff = rootNodeCount;
    for (uint32_t m = 0; m < modelCount; m++) {
        const hvvr_mesh_data& md = in->models[m];
        for (uint32_t i = 0; i < md.material_count; i++) s.materials[mOff + i] = md.materials[i];
        for (uint32_t i = 0; i < md.tri_count; i++) {
            hvvr_tri_shade t = md.tri_shade[i];
            t.indices[0] += vOff; t.indices[1] += vOff; t.indices[2] += vOff;
            t.material += mOff;
            s.triShade[tOff + i] = t;
        }
        for (uint32_t i = 0; i < md.vert_count; i++) { s.verts[vOff + i] = md.verts[i]; s.vertModel[vOff + i] = m; }
        viewOffsets[m] = nOff;
        for (uint32_t i = 0; i < md.node_count; i++) {
            const hvvr_topology_node& tn = md.nodes[i];
            Node& n = s.nodes[nOff + i];
            n.leafMask = tn.leaf_mask;
            n.tri[0] = tOff + tn.data[0];
            for (int k = 0; k < 4; k++)
                n.tri[1 + k] = (tn.leaf_mask & (1u << k)) ? tOff + tn.data[1 + k] : tn.data[1 + k];
        }
        vOff += md.vert_count; tOff += md.tri_count; mOff += md.material_count; nOff += md.node_count;
    }
    if (rootNodeCount > 0) {
        // root fix-up nodes: nulls first, then fix-up nodes, then model entry points
        std::vector<int64_t> children(rootNodeCount * 4);
        size_t w = 0;
        for (size_t i = children.size() - modelCount - (rootNodeCount - 1); i != 0; --i) children[w++] = -1;
        for (uint32_t i = 1; i < rootNodeCount; i++) children[w++] = i;
        for (uint32_t m = 0; m < modelCount; m++) children[w++] = viewOffsets[m];
        for (uint32_t i = 0; i < rootNodeCount; i++) {
            Node& n = s.nodes[i];
            n.tri[0] = 0;
            n.leafMask = 0;
            for (int k = 0; k < 4; k++) {
                int64_t c = children[4 * i + k];
                if (c < 0) { n.tri[1 + k] = 0; n.leafMask |= 1u << k; continue; }
                n.tri[1 + k] = uint32_t(c - i);
            }
        }
    }
}

// FloatFlip / IFloatFlip (RC/sort.h:13-32)
inline uint32_t floatFlip(uint32_t f) { uint32_t mask = uint32_t(-int32_t(f >> 31)) | 0x80000000u; return f ^ mask; }
inline uint32_t ifloatFlip(uint32_t f) { uint32_t mask = ((f & 0x80000000u) == 0) ? 0xffffffffu : 0x80000000u; return f ^ mask; }

// GPUSceneState::update (RC/gpu_scene_state.cu:377-451) and setGeometry's task ordering
// (RC/gpu_scene_state.cu:469-599). Bounds use the same max operators: atomicMax on
// float-flipped integers for leaf slots, max(a,b)=a>b?a:b for internal slots.
void refitScene(const oracle_frame_in* in, Scene& s) {
    uint32_t modelCount = in->model_count;
    std::vector<M4> modelToWorld(modelCount);
    for (uint32_t m = 0; m < modelCount; m++) modelToWorld[m] = transformToMatrix(in->model_xf[m]);
    // SceneTransformVerticesKernel (RC/gpu_scene_state.cu:88-132)
    s.world = s.verts;
    for (size_t i = 0; i < s.verts.size(); i++) {
        const M4& t = modelToWorld[s.vertModel[i]];
        const hvvr_shading_vertex& v = s.verts[i];
        const V4 vp = V4{v.pos.x, v.pos.y, v.pos.z, 1.0f};
        V4 fp = in->fp_mode == HVVR_FP_FMA ? mulFma(t, vp) : mul(t, vp);
        V3 p = mk(fp.x, fp.y, fp.z) * (1.0f / fp.w);
        s.world[i].pos = hvvr_vec3{p.x, p.y, p.z};
        V3 n = mk(halfToFloat(v.normal[0]), halfToFloat(v.normal[1]), halfToFloat(v.normal[2]));
        V3 nn = normalize(mul(m3of(t), n));
        s.world[i].normal[0] = floatToHalf(nn.x);
        s.world[i].normal[1] = floatToHalf(nn.y);
        s.world[i].normal[2] = floatToHalf(nn.z);
        s.world[i].normal[3] = floatToHalf(0.0f);
    }
    uint32_t nodeCount = uint32_t(s.nodes.size());
    uint32_t triCount = uint32_t(s.triShade.size());
    // triToNodeChild (RC/gpu_scene_state.cu:538-570): nodes back to front, slots 3..0
    std::vector<uint32_t> triToNodeChild(triCount, 0);
    for (int64_t n = int64_t(nodeCount) - 1; n >= 0; n--) {
        const Node& nd = s.nodes[n];
        for (int k = 3; k >= 0; k--) {
            if (nd.leafMask & (1u << k)) {
                for (uint32_t t = nd.tri[k]; t < nd.tri[k + 1]; t++)
                    if (t < triCount) triToNodeChild[t] = (uint32_t(n) << 2) | uint32_t(k);
            }
        }
    }
    // SceneRefitPreKernel: bounds := FloatFlip(-inf)
    std::vector<uint32_t> fb(size_t(nodeCount) * 24, floatFlip(0xff800000u));
    // ScenePrecomputeTrianglesKernel (RC/gpu_scene_state.cu:167-244)
    s.tris.resize(triCount);
    for (uint32_t i = 0; i < triCount; i++) {
        const hvvr_tri_shade& ts = s.triShade[i];
        V3 v0 = mk(s.world[ts.indices[0]].pos.x, s.world[ts.indices[0]].pos.y, s.world[ts.indices[0]].pos.z);
        V3 v1 = mk(s.world[ts.indices[1]].pos.x, s.world[ts.indices[1]].pos.y, s.world[ts.indices[1]].pos.z);
        V3 v2 = mk(s.world[ts.indices[2]].pos.x, s.world[ts.indices[2]].pos.y, s.world[ts.indices[2]].pos.z);
        s.tris[i] = Tri{v0, v1 - v0, v2 - v0};
        float mx[3] = {tmax(v0.x, tmax(v1.x, v2.x)), tmax(v0.y, tmax(v1.y, v2.y)), tmax(v0.z, tmax(v1.z, v2.z))};
        float nm[3] = {tmax(-v0.x, tmax(-v1.x, -v2.x)), tmax(-v0.y, tmax(-v1.y, -v2.y)), tmax(-v0.z, tmax(-v1.z, -v2.z))};
        uint32_t nc = triToNodeChild[i];
        uint32_t parent = nc >> 2, slot = nc & 3;
        for (int a = 0; a < 3; a++) {
            uint32_t* pMax = &fb[size_t(parent) * 24 + (2 * a) * 4 + slot];
            uint32_t* pNeg = &fb[size_t(parent) * 24 + (2 * a + 1) * 4 + slot];
            *pMax = std::max(*pMax, floatFlip(fbits(mx[a])));
            *pNeg = std::max(*pNeg, floatFlip(fbits(nm[a])));
        }
    }
    // SceneRefitIntFixupKernel
    for (uint32_t n = 0; n < nodeCount; n++)
        for (int j = 0; j < 24; j++) s.nodes[n].b[j / 4][j % 4] = bitsf(ifloatFlip(fb[size_t(n) * 24 + j]));
    // internal refit, deepest parents first (RC/gpu_scene_state.cu:505-589, 273-375)
    std::vector<uint32_t> depth(nodeCount, 0);
    uint32_t maxDepth = 0;
    for (uint32_t n = 0; n < nodeCount; n++) {
        const Node& nd = s.nodes[n];
        for (int k = 3; k >= 0; k--) {
            if (!(nd.leafMask & (1u << k))) {
                uint32_t c = n + nd.tri[k + 1];
                if (c < nodeCount) { depth[c] = depth[n] + 1; maxDepth = std::max(maxDepth, depth[n] + 1); }
            }
        }
    }
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> byDepth(maxDepth + 1);
    for (uint32_t n = 0; n < nodeCount; n++)
        for (int k = 0; k < 4; k++)
            if (!(s.nodes[n].leafMask & (1u << k))) byDepth[depth[n]].push_back({n, uint32_t(k)});
    for (int64_t d = maxDepth; d >= 0; d--) {
        for (auto& task : byDepth[d]) {
            uint32_t c = task.first + s.nodes[task.first].tri[task.second + 1];
            if (c >= nodeCount) { s.status |= 1; continue; }
            const Node& ch = s.nodes[c];
            for (int j = 0; j < 6; j++) {
                float v = tmax(ch.b[j][0], tmax(ch.b[j][1], tmax(ch.b[j][2], ch.b[j][3])));
                s.nodes[task.first].b[j][task.second] = v;
            }
        }
    }
}

// ------------------------------------------------------------------ samples (RC/camera.cpp:21-64)
struct SortedSample { hvvr_sample s; uint32_t channel; };

// naiveXYCluster (RC/sample_clustering.h:17-49)
void naiveXYCluster(std::vector<SortedSample>& v, size_t k) {
    size_t yStrata = (size_t)sqrt((double)k);
    size_t xStrata = (k + yStrata - 1) / yStrata;
    size_t blockYStrata = (size_t)sqrt((double)kTilesPerBlock);
    size_t blockXStrata = (kTilesPerBlock + blockYStrata - 1) / blockYStrata;
    auto yx = [](const SortedSample& a, const SortedSample& b) {
        return (a.s.position.y < b.s.position.y) || (a.s.position.y == b.s.position.y && a.s.position.x < b.s.position.x);
    };
    auto xy = [](const SortedSample& a, const SortedSample& b) {
        return (a.s.position.x < b.s.position.x) || (a.s.position.x == b.s.position.x && a.s.position.y < b.s.position.y);
    };
    size_t n = v.size();
    std::sort(v.begin(), v.end(), yx);
    for (size_t i = 0; i < yStrata; ++i)
        std::sort(v.begin() + (i * kBlockSize * xStrata), v.begin() + std::min((i + 1) * kBlockSize * xStrata, n), xy);
    for (size_t i = 0; i < k; ++i)
        std::sort(v.begin() + (i * kBlockSize), v.begin() + std::min((i + 1) * kBlockSize, n), yx);
    for (size_t i = 0; i < n; i += kTileSize * blockXStrata)
        std::sort(v.begin() + i, v.begin() + std::min(i + kTileSize * blockXStrata, n), xy);
}

struct Frustum2D { float d[4]; }; // xMin, -xMax, yMin, -yMax (RC/sample_hierarchy.h:19-58)
inline void merge2D(Frustum2D& f, float x, float y) {
    f.d[0] = tmin(f.d[0], x); f.d[1] = tmin(f.d[1], -x); f.d[2] = tmin(f.d[2], y); f.d[3] = tmin(f.d[3], -y);
}

struct Rays4 { V3 o[4], d[4]; };

// Camera::getSampleToCamera (RC/camera.cpp:167-171)
M3 sampleToCamera(const hvvr_float_rect& vp) {
    return M3{mk(vp.upper.x - vp.lower.x, 0, 0), mk(0, vp.lower.y - vp.upper.y, 0), mk(vp.lower.x, vp.upper.y, -1)};
}

// get3DFrustumFrom2D, perspective mapping (RC/sample_hierarchy.cpp:46-123)
Rays4 frustumFrom2D(const Frustum2D& f, const M3& S, const hvvr_thin_lens& lens) {
    const float farPlane = -100.0f;
    float xMin = f.d[0], xMax = -f.d[1], yMin = f.d[2], yMax = -f.d[3];
    V3 nearP[4] = {mk(-lens.radius, -lens.radius, 0), mk(+lens.radius, -lens.radius, 0),
                   mk(+lens.radius, +lens.radius, 0), mk(-lens.radius, +lens.radius, 0)};
    V3 rd[4] = {mul(S, mk(xMin, yMax, 1)), mul(S, mk(xMax, yMax, 1)), mul(S, mk(xMax, yMin, 1)), mul(S, mk(xMin, yMin, 1))};
    V3 focus[4];
    for (int i = 0; i < 4; i++) focus[i] = rd[i] * (lens.focal_distance / -rd[i].z);
    float fxMax = -INFINITY, fxMin = INFINITY, fyMax = -INFINITY, fyMin = INFINITY;
    for (int i = 0; i < 4; ++i) {
        for (int j = 0; j < 4; ++j) {
            V3 pos = nearP[i];
            V3 dir = normalize(focus[j] - pos);
            V3 p = pos + dir * (farPlane / dir.z);
            fxMax = tmax(fxMax, p.x); fxMin = tmin(fxMin, p.x);
            fyMax = tmax(fyMax, p.y); fyMin = tmin(fyMin, p.y);
        }
    }
    V3 farP[4] = {mk(fxMin, fyMin, farPlane), mk(fxMax, fyMin, farPlane), mk(fxMax, fyMax, farPlane), mk(fxMin, fyMax, farPlane)};
    Rays4 r;
    for (int i = 0; i < 4; i++) { r.o[i] = nearP[i]; r.d[i] = normalize(farP[i] - nearP[i]); }
    return r;
}

struct Beam { V3 c, du, dv; };

struct SampleSetup {
    uint32_t blocks = 0, tiles = 0, padded = 0, valid = 0;
    std::vector<Rays4> tileRays, blockRays; // camera space
    std::vector<Beam> beams;
    std::vector<int32_t> remap;
};

void setupSamples(const oracle_frame_in* in, SampleSetup& ss) {
    uint32_t n = in->sample_count;
    std::vector<SortedSample> sorted(n);
    for (uint32_t i = 0; i < n; i++) sorted[i] = SortedSample{in->samples[i], i % in->split_color_samples};
    uint32_t blockCount = (n + kBlockSize - 1) / kBlockSize;
    naiveXYCluster(sorted, blockCount);
    ss.blocks = blockCount; ss.tiles = blockCount * kTilesPerBlock; ss.padded = blockCount * kBlockSize; ss.valid = n;
    M3 S = sampleToCamera(in->viewport);
    // BeamBatch2D (RC/sample_hierarchy.cpp:154-190); cullRect is +-inf so intersect() is a no-op
    std::vector<Frustum2D> tile2D(ss.tiles), block2D(blockCount);
    std::vector<V2> center(ss.padded, V2{0, 0}), major(ss.padded, V2{0, 0}), minor(ss.padded, V2{0, 0});
    uint32_t maxIndex = n - 1, si = 0;
    for (uint32_t b = 0; b < blockCount; b++) {
        Frustum2D bf{{INFINITY, INFINITY, INFINITY, INFINITY}};
        for (uint32_t t = 0; t < kTilesPerBlock; t++) {
            Frustum2D tf{{INFINITY, INFINITY, INFINITY, INFINITY}};
            for (uint32_t k = 0; k < kTileSize; k++) {
                const hvvr_sample& s = sorted[si].s;
                float x = s.position.x, y = s.position.y, mj = s.major_axis_length;
                merge2D(tf, x + mj, y + mj);
                merge2D(tf, x - mj, y - mj);
                // unpackSample (RC/samples.cpp:144-159)
                const float EXT = 0.70710678118f;
                V2 mn{s.minor_axis.x * EXT, s.minor_axis.y * EXT};
                float mlen = sqrtf(s.minor_axis.x * s.minor_axis.x + s.minor_axis.y * s.minor_axis.y);
                float rescale = s.major_axis_length * EXT / mlen;
                center[si] = V2{s.position.x, s.position.y};
                minor[si] = mn;
                major[si] = V2{-mn.y * rescale, mn.x * rescale};
                si = std::min(si + 1, maxIndex);
            }
            for (int j = 0; j < 4; j++) tf.d[j] = tmax(tf.d[j], -INFINITY);
            tile2D[b * kTilesPerBlock + t] = tf;
            for (int j = 0; j < 4; j++) bf.d[j] = tmin(bf.d[j], tf.d[j]);
        }
        block2D[b] = bf;
    }
    // BeamBatch::generateFrom2D (RC/sample_hierarchy.cpp:129-152)
    ss.tileRays.resize(ss.tiles);
    ss.blockRays.resize(blockCount);
    for (uint32_t b = 0; b < blockCount; b++) {
        for (uint32_t t = 0; t < kTilesPerBlock; t++)
            ss.tileRays[b * kTilesPerBlock + t] = frustumFrom2D(tile2D[b * kTilesPerBlock + t], S, in->lens);
        ss.blockRays[b] = frustumFrom2D(block2D[b], S, in->lens);
    }
    ss.beams.resize(ss.padded);
    for (uint32_t i = 0; i < ss.padded; i++) {
        ss.beams[i].c = mul(S, mk(center[i].x, center[i].y, 1.0f));
        ss.beams[i].du = mul(S, mk(major[i].x, major[i].y, 0.0f));
        ss.beams[i].dv = mul(S, mk(minor[i].x, minor[i].y, 0.0f));
    }
    uint32_t split = in->split_color_samples;
    ss.remap.assign(size_t(in->width) * in->height * split, -1);
    for (uint32_t i = 0; i < n; i++) {
        const hvvr_sample& s = sorted[i].s;
        size_t idx = (size_t(s.pixel_y) * in->width + s.pixel_x) * split + sorted[i].channel;
        if (idx < ss.remap.size()) ss.remap[idx] = int32_t(i);
    }
}

// ------------------------------------------------------------------ traversal frustum
// Frustum::Frustum (RC/traverse_avx.cpp:22-211), lane by lane.
struct TravFrustum {
    bool degenerate;
    int distIdx; // 0..5: xMax, xNegMin, yMax, yNegMin, zMax, zNegMin
    float tpLo[4][3], tpHi[4][3], w[4];
    float proj[3][8];
    float edge[12][3];
    float minF[12], maxF[12];
    V3 o[4], d[4];
};

void buildTravFrustum(const V3* origin, const V3* dir, TravFrustum& f) {
    V4 plane[4];
    V3 avg = mk(0, 0, 0);
    for (int p = 0; p < 4; p++) {
        f.o[p] = origin[p]; f.d[p] = dir[p];
        if (isinf(origin[0].x)) {
            plane[p] = V4{0, 0, 0, -INFINITY};
        } else {
            V3 n = cross(dir[p], dir[(p + 1) % 4]);
            plane[p] = V4{n.x, n.y, n.z, dot(origin[p], n)};
        }
        avg = avg + dir[p];
    }
    f.degenerate = (plane[0].w == -INFINITY);
    if (fabsf(avg.x) > fabsf(avg.y)) {
        if (fabsf(avg.x) > fabsf(avg.z)) f.distIdx = avg.x < 0 ? 0 : 1;
        else f.distIdx = avg.z < 0 ? 4 : 5;
    } else {
        if (fabsf(avg.y) > fabsf(avg.z)) f.distIdx = avg.y < 0 ? 2 : 3;
        else f.distIdx = avg.z < 0 ? 4 : 5;
    }
    for (int p = 0; p < 4; p++) {
        float c[3] = {plane[p].x, plane[p].y, plane[p].z};
        for (int a = 0; a < 3; a++) {
            f.tpLo[p][a] = c[a] < 0.0f ? c[a] : 0.0f;
            f.tpHi[p][a] = c[a] > 0.0f ? -c[a] : 0.0f;
        }
        f.w[p] = plane[p].w;
    }
    // projections onto the axes: lanes 0-3 max side, lanes 4-7 -min side
    for (int a = 0; a < 3; a++) {
        float lane[8];
        for (int i = 0; i < 4; i++) {
            float oc = (&origin[i].x)[a], dc = (&dir[i].x)[a];
            float so0 = -oc, so1 = -(-oc);
            float nd0 = -dc, nd1 = -(-dc);
            float m0 = (0.0f > nd0) ? 0.0f : nd0; // _mm256_max_ps(zero, v)
            float m1 = (0.0f > nd1) ? 0.0f : nd1;
            lane[i] = so0 + FLT_MAX * m0;
            lane[4 + i] = so1 + FLT_MAX * m1;
        }
        float y[8], z[8];
        static const int p1[4] = {2, 3, 0, 1}, p2[4] = {1, 0, 3, 2};
        for (int h = 0; h < 2; h++)
            for (int i = 0; i < 4; i++) { float a0 = lane[4 * h + i], b0 = lane[4 * h + p1[i]]; y[4 * h + i] = a0 > b0 ? a0 : b0; }
        for (int h = 0; h < 2; h++)
            for (int i = 0; i < 4; i++) { float a0 = y[4 * h + i], b0 = y[4 * h + p2[i]]; z[4 * h + i] = a0 > b0 ? a0 : b0; }
        for (int i = 0; i < 8; i++) f.proj[a][i] = -z[i];
    }
    // edge axes d_i x e_k and the frustum's interval on each (RC/traverse_avx.cpp:152-210)
    const V3 axes[3] = {mk(1, 0, 0), mk(0, 1, 0), mk(0, 0, 1)};
    for (int i = 0; i < 4; i++)
        for (int k = 0; k < 3; k++) {
            V3 e = cross(dir[i], axes[k]);
            f.edge[i * 3 + k][0] = e.x; f.edge[i * 3 + k][1] = e.y; f.edge[i * 3 + k][2] = e.z;
        }
    for (int e = 0; e < 12; e++) {
        float ex = f.edge[e][0], ey = f.edge[e][1], ez = f.edge[e][2];
        float mn = FLT_MAX, mx = -FLT_MAX;
        for (int p = 0; p < 4; p++) {
            float d0 = fmaf(ex, origin[p].x, fmaf(ey, origin[p].y, ez * origin[p].z));
            mn = mn < d0 ? mn : d0;
            mx = mx > d0 ? mx : d0;
            float d1 = fmaf(ex, dir[p].x, fmaf(ey, dir[p].y, ez * dir[p].z));
            const float eps = .000001f;
            float a = d1 + eps, b = d1 - eps;
            float amin = a < 0.0f ? a : 0.0f;  // _mm256_min_ps(a, zero)
            float bmax = b > 0.0f ? b : 0.0f;  // _mm256_max_ps(b, zero)
            mn = amin * FLT_MAX + mn;
            mx = bmax * FLT_MAX + mx;
        }
        f.minF[e] = mn; f.maxF[e] = mx;
    }
}

// Frustum::testBVHNodeChildren (RC/traverse_avx.h:104-164)
uint32_t testChildren(const Node& n, const TravFrustum& f) {
    uint32_t result = 0;
    for (int c = 0; c < 4; c++) {
        bool pass = true;
        for (int p = 0; p < 4; p++) {
            float lo = fmaf(f.tpLo[p][0], n.b[0][c], fmaf(f.tpLo[p][1], n.b[2][c], f.tpLo[p][2] * n.b[4][c]));
            float hi = fmaf(f.tpHi[p][0], n.b[1][c], fmaf(f.tpHi[p][1], n.b[3][c], f.tpHi[p][2] * n.b[5][c]));
            float d = lo + hi;
            if (!(d <= f.w[p])) pass = false;
        }
        if (pass) result |= 1u << c;
    }
    if (!result) return 0;
    uint32_t m = 0;
    for (int c = 0; c < 4; c++) {
        bool ok = true;
        for (int a = 0; a < 3; a++) {
            if (!(n.b[2 * a][c] >= f.proj[a][c])) ok = false;
            if (!(n.b[2 * a + 1][c] >= f.proj[a][4 + c])) ok = false;
        }
        if (ok) m |= 1u << c;
    }
    return result & m;
}

// Frustum::testBVHNodeChildrenRefine (RC/traverse_avx.h:166-217)
uint32_t refineChildren(const Node& n, const TravFrustum& f, uint32_t prev) {
    uint32_t result = prev;
    for (int e = 0; e < 12; e++) {
        float ex = f.edge[e][0], ey = f.edge[e][1], ez = f.edge[e][2];
        bool px = ex > 0.0f, py = ey > 0.0f, pz = ez > 0.0f;
        for (int c = 0; c < 4; c++) {
            float pX = (px ? n.b[0][c] : -n.b[1][c]) + 0.0f;
            float pY = (py ? n.b[2][c] : -n.b[3][c]) + 0.0f;
            float pZ = (pz ? n.b[4][c] : -n.b[5][c]) + 0.0f;
            float nX = (px ? -n.b[1][c] : n.b[0][c]) + 0.0f;
            float nY = (py ? -n.b[3][c] : n.b[2][c]) + 0.0f;
            float nZ = (pz ? -n.b[5][c] : n.b[4][c]) + 0.0f;
            float maxBox = fmaf(ex, pX, fmaf(ey, pY, ez * pZ));
            float minBox = fmaf(ex, nX, fmaf(ey, nY, ez * nZ));
            if ((maxBox < f.minF[e]) || (f.maxF[e] < minBox)) result &= ~(1u << c);
        }
    }
    return result;
}

struct StackEntry { float tMin; uint32_t mask; uint32_t node; };
struct CullEntry { uint32_t tDeltaBits; float tMinTemp; uint32_t node; };

inline bool comigt(float a, float b) { return daz(a) > daz(b); }
inline bool comilt(float a, float b) { return daz(a) < daz(b); }

// traverseBlocks + BlockFrame::sort (RC/traverse_avx.h:293-410)
uint32_t traverseBlock(const Node* nodes, const TravFrustum& f, StackEntry* sorted) {
    if (f.degenerate) return 0;
    CullEntry cull[kBlockStackSize + 4];
    uint32_t top = 0;
    float tMin = 0.0f;
    uint32_t node = 0;
    for (;;) {
        const Node& nd = nodes[node];
        uint32_t mask = testChildren(nd, f);
        mask = refineChildren(nd, f, mask);
        if (mask) {
            uint32_t leaf = mask & nd.leafMask;
            if (leaf) {
                mask &= ~leaf;
                uint32_t i = top;
                while (comigt(i > 0 ? bitsf(cull[i - 1].tDeltaBits) : -1.0f, 0.0f)) { cull[i] = cull[i - 1]; --i; }
                ++top;
                cull[i] = CullEntry{leaf, tMin, node};
            }
            if (mask) {
                float tMinK[4], tDeltaK[4];
                int maxIdx = f.distIdx & ~1;
                for (int k = 0; k < 4; k++) {
                    tMinK[k] = bitsf(fbits(nd.b[f.distIdx][k]) ^ 0x80000000u);
                    tDeltaK[k] = nd.b[maxIdx][k] + nd.b[maxIdx + 1][k];
                }
                do {
                    int k = __builtin_ctz(mask);
                    float td = tDeltaK[k];
                    uint32_t i = top;
                    while (comigt(i > 0 ? bitsf(cull[i - 1].tDeltaBits) : -1.0f, td)) { cull[i] = cull[i - 1]; --i; }
                    cull[i] = CullEntry{fbits(td), tMinK[k], childOf(nodes, node, k)};
                    mask &= mask - 1;
                    ++top;
                } while (mask);
            }
        }
        // POP
        if (top >= kBlockStackSize - 4 || top == 0 || cull[top - 1].tDeltaBits <= 0xf) break;
        --top;
        node = cull[top].node;
        tMin = cull[top].tMinTemp;
    }
    uint32_t stackSize = top;
    for (uint32_t t = 0; t < stackSize; t++) {
        StackEntry data{cull[t].tMinTemp, cull[t].tDeltaBits, cull[t].node};
        uint32_t slot = t;
        while (comilt(slot > 0 ? sorted[slot - 1].tMin : INFINITY, data.tMin)) { sorted[slot] = sorted[slot - 1]; slot--; }
        sorted[slot] = data;
        if (cull[t].tDeltaBits > 0xf) sorted[slot].mask = 0;
    }
    return stackSize;
}

// traverseTiles (RC/traverse_avx.h:412-527)
uint32_t traverseTile(const Node* nodes, const TravFrustum& f, const StackEntry* blockStack, uint32_t stackSize,
                      std::vector<uint32_t>& out, uint32_t& status) {
    out.clear();
    if (f.degenerate || stackSize == 0) return 0;
    std::vector<StackEntry> stack(blockStack, blockStack + stackSize);
    stack.resize(kTileStackMax);
    uint32_t top = stackSize - 1;
    uint32_t node = stack[top].node;
    for (;;) {
        const Node& nd = nodes[node];
        uint32_t mask = testChildren(nd, f);
        bool descend = false;
        if (mask) {
            uint32_t leaf = mask & nd.leafMask;
            if (leaf) {
                mask = refineChildren(nd, f, mask);
                leaf = mask & nd.leafMask;
                uint32_t emit = leaf;
                while (emit) {
                    int k = __builtin_ctz(emit);
                    uint32_t t0 = nd.tri[k], t1 = nd.tri[k + 1];
                    if (t1 <= t0) status |= 2;
                    for (uint32_t t = t0; t < t1; t++) out.push_back(t);
                    emit &= emit - 1;
                }
            }
            mask &= ~nd.leafMask;
            if (mask && !stack[top].mask) {
                float tMinK[4];
                for (int k = 0; k < 4; k++) tMinK[k] = bitsf(fbits(nd.b[f.distIdx][k]) ^ 0x80000000u);
                int k = __builtin_ctz(mask);
                if (!(mask & (mask - 1))) {
                    node = childOf(nodes, node, k);
                    continue; // TEST
                }
                bool first = true;
                do {
                    if (!first) ++top;
                    first = false;
                    k = __builtin_ctz(mask);
                    if (top + 1 >= kTileStackMax) { status |= 4; return uint32_t(out.size()); }
                    float tm = tMinK[k];
                    uint32_t i = top;
                    while (comilt(i > 0 ? stack[i - 1].tMin : INFINITY, tm)) { stack[i] = stack[i - 1]; --i; }
                    stack[i] = StackEntry{tm, 0, childOf(nodes, node, k)};
                    mask &= mask - 1;
                } while (mask);
                descend = true;
            }
        }
        if (descend) { node = stack[top].node; continue; } // POP_LAST
        if (top == 0) break;                                 // POP
        --top;
        node = stack[top].node;
    }
    return uint32_t(out.size());
}

// ------------------------------------------------------------------ intersect (RC/prim_tests.h, RC/intersect.cu)
struct FrustumPlanes { V4 p[4]; };
// FrustumPlanes::FrustumPlanes (RC/prim_tests.h:22-28)
FrustumPlanes makePlanes(const Rays4& r) {
    FrustumPlanes fp;
    for (int n = 0; n < 4; n++) {
        V3 d = cross(r.d[n], r.d[(n + 1) % 4]);
        fp.p[n] = V4{d.x, d.y, d.z, dot(r.o[n], d)};
    }
    return fp;
}
// FrustumPlanes::test (RC/prim_tests.h:30-49)
bool planesTest(const FrustumPlanes& fp, const Tri& t) {
    for (int n = 0; n < 4; n++) {
        V3 dir = mk(fp.p[n].x, fp.p[n].y, fp.p[n].z);
        float dist = fp.p[n].w;
        float d0 = dot(dir, t.v0);
        float d1 = d0 + dot(dir, t.e0);
        float d2 = d0 + dot(dir, t.e1);
        if (d0 > dist && d1 > dist && d2 > dist) return false;
    }
    return true;
}
// TestRayTriangle<false> (RC/prim_tests.h:53-82)
V4 testRayTriangle(V3 ro, V3 rd, const Tri& tri) {
    V3 n = cross(tri.e0, tri.e1);
    float denom = dot(-rd, n);
    V3 v0r = ro - tri.v0;
    float t = dot(v0r, n);
    V3 e = cross(-rd, v0r);
    float v = dot(tri.e1, e);
    float w = -dot(tri.e0, e);
    float ood = 1.0f / denom;
    t *= ood; v *= ood; w *= ood;
    float u = 1.0f - v - w;
    return V4{u, v, w, t};
}
// TestTriangleFrustaUVW (RC/prim_tests.h:89-116); returns true unless all-out
bool uvwNotAllOut(const Rays4& r, const Tri& tri) {
    V4 uvw[4];
    for (int n = 0; n < 4; n++) uvw[n] = testRayTriangle(r.o[n], r.d[n], tri);
    float uMin = FLT_MAX, uMax = -FLT_MAX, vMin = FLT_MAX, vMax = -FLT_MAX, wMin = FLT_MAX, wMax = -FLT_MAX;
    for (int n = 0; n < 4; n++) {
        uMin = tmin(uMin, uvw[n].x); uMax = tmax(uMax, uvw[n].x);
        vMin = tmin(vMin, uvw[n].y); vMax = tmax(vMax, uvw[n].y);
        wMin = tmin(wMin, uvw[n].z); wMax = tmax(wMax, uvw[n].z);
    }
    if (uMax < 0 || uMin > 1 || vMax < 0 || vMin > 1 || wMax < 0 || wMin > 1) return false;
    return true;
}

struct TriTile { float t; V3 e0, e1, v0r; };
// IntersectTriangleTile<false>::setup (RC/prim_tests.h:148-163)
bool tileSetup(const Tri& tri, V3 ro, TriTile& tt) {
    tt.e0 = tri.e0; tt.e1 = tri.e1;
    V3 normal = cross(tt.e0, tt.e1);
    tt.v0r = ro - tri.v0;
    tt.t = dot(tt.v0r, normal);
    return !(tt.t < 0.0f);
}

struct TriThread { float dc, vc, wc; V2 dd, dv, dw; };
// IntersectTriangleThread ctor + GetDifferentials (RC/prim_tests.h:118-134, 175-188)
TriThread threadSetup(const TriTile& tt, V3 c, V3 du, V3 dv) {
    TriThread r;
    V3 normal = cross(tt.e0, tt.e1);
    r.dc = dot(-c, normal);
    V3 ec = cross(-c, tt.v0r);
    r.vc = dot(tt.e1, ec);
    r.wc = -dot(tt.e0, ec);
    V3 n2 = cross(tt.e0, tt.e1);
    r.dd = V2{dot(-du, n2), dot(-dv, n2)};
    r.dv = V2{dot(tt.e1, cross(-du, tt.v0r)), dot(tt.e1, cross(-dv, tt.v0r))};
    r.dw = V2{-dot(tt.e0, cross(-du, tt.v0r)), -dot(tt.e0, cross(-dv, tt.v0r))};
    return r;
}
// IntersectTriangleThread::test (RC/prim_tests.h:192-231)
inline bool threadTest(const TriThread& th, float tt_t, V2 a, float& depth, bool fma) {
    float denom, depthDelta, v, w;
    if (fma) {
        denom = fmaf(th.dd.y, a.y, fmaf(th.dd.x, a.x, th.dc));
        depthDelta = fmaf(depth, denom, -tt_t);
        v = fmaf(th.dv.y, a.y, fmaf(th.dv.x, a.x, th.vc));
        w = fmaf(th.dw.y, a.y, fmaf(th.dw.x, a.x, th.wc));
    } else {
        denom = th.dc + th.dd.x * a.x + th.dd.y * a.y;
        depthDelta = depth * denom - tt_t;
        v = th.vc + th.dv.x * a.x + th.dv.y * a.y;
        w = th.wc + th.dw.x * a.x + th.dw.y * a.y;
    }
    float u = denom - v - w;
    int32_t test = int32_t(fbits(depthDelta) | fbits(u) | fbits(v) | fbits(w));
    if (test < 0) return false;
    depth = tt_t * (1.0f / denom);
    return true;
}
// IntersectTriangleThread::calcUVW (RC/prim_tests.h:233-245)
inline V3 calcUVW(const TriThread& th, V2 a, bool fma) {
    float denom, v, w;
    if (fma) {
        denom = fmaf(th.dd.y, a.y, fmaf(th.dd.x, a.x, th.dc));
        v = fmaf(th.dv.y, a.y, fmaf(th.dv.x, a.x, th.vc));
        w = fmaf(th.dw.y, a.y, fmaf(th.dw.x, a.x, th.wc));
    } else {
        denom = th.dc + th.dd.x * a.x + th.dd.y * a.y;
        v = th.vc + th.dv.x * a.x + th.dv.y * a.y;
        w = th.wc + th.dw.x * a.x + th.dw.y * a.y;
    }
    float u = denom - v - w;
    float inv = 1.0f / denom;
    return mk(u * inv, v * inv, w * inv);
}

// ------------------------------------------------------------------ depth of field
// IntersectTriangleTile<true>, IntersectTriangleThreadDoF (RC/prim_tests.h:247-392), TileData<true>
// (RC/tile_data.h:33-60), GetSampleUVsDoF (RC/gpu_samples.h:84-103), initLookupTables
// (RC/gpu_camera.cu:59-88). fma selects the contraction the kernel comments mark (HVVR_FP_FMA).
inline V3 fma3(float s, V3 a, V3 c) { return mk(fmaf(s, a.x, c.x), fmaf(s, a.y, c.y), fmaf(s, a.z, c.z)); }

struct DofTile { V3 lensU, lensV; V2 focalToLensScale; };
// TileData<true>::load. The kernels call it with the world-space beam of GetDirectionalSample3D and
// rotate it again (cameraToWorldRotation * sample.du); kept. rsqrtf is taken as 1/sqrtf.
DofTile dofTileData(const M3& R, const Beam& bmCam, const hvvr_thin_lens& lens) {
    V3 focalU = mul(R, mul(R, bmCam.du)), focalV = mul(R, mul(R, bmCam.dv));
    float uInv = 1.0f / sqrtf(dot(focalU, focalU)), vInv = 1.0f / sqrtf(dot(focalV, focalV));
    float uMag = 1.0f / uInv, vMag = 1.0f / vInv;
    DofTile d;
    d.lensU = focalU * (lens.radius * uInv);
    d.lensV = focalV * (lens.radius * vInv);
    float sc = lens.focal_distance / lens.radius;
    d.focalToLensScale = V2{sc * uMag, sc * vMag};
    return d;
}

struct DofTri { V3 e0, e1, v0l; float tC, tU, tV; V2 dd; };
enum { kAllOut = 0, kPartial = 1, kAllIn = 2 };
// IntersectTriangleTile<true>::setup
int dofSetup(const Tri& tri, V3 lensCenter, V3 lensU, V3 lensV, DofTri& d) {
    d.e0 = tri.e0; d.e1 = tri.e1;
    V3 normal = cross(d.e0, d.e1);
    d.v0l = lensCenter - tri.v0;
    d.tC = dot(d.v0l, normal);
    d.tU = dot(lensU, normal);
    d.tV = dot(lensV, normal);
    float tExtent = fabsf(d.tU) + fabsf(d.tV);
    float tMax = d.tC + tExtent;
    if (tMax < 0.0f) return kAllOut;
    d.dd = V2{dot(-lensU, normal), dot(-lensV, normal)};
    float tMin = d.tC - tExtent;
    if (tMin < 0.0f) return kPartial;
    return kAllIn;
}
// IntersectTriangleThreadDoF ctor
inline float dofDenomCenter(const DofTri& d, V3 lc2fc) { return dot(-lc2fc, cross(d.e0, d.e1)); }

// GetSampleUVsDoF: lens position from the table, direction offset from the MSAA pattern
inline void dofSampleUVs(const V2* table, uint32_t n, uint32_t lensTile, uint32_t s, uint32_t i, V2 aa, V2 fls,
                         bool fma, V2& lensUV, V2& dirUV) {
    lensUV = table[size_t(lensTile) * kTileSize * n + size_t(i) * kTileSize + s];
    if (fma) dirUV = V2{fmaf(aa.x, fls.x, -lensUV.x), fmaf(aa.y, fls.y, -lensUV.y)};
    else dirUV = V2{aa.x * fls.x - lensUV.x, aa.y * fls.y - lensUV.y};
}

// the scaled barycentrics of IntersectTriangleThreadDoF::test / calcUVW
inline void dofBary(const DofTri& d, float denomCenter, V3 lc2fc, V3 lensU, V3 lensV, V2 lensUV, V2 dirUV,
                    bool fma, float& denom, float& v, float& w) {
    V3 o, rd, e;
    if (fma) {
        denom = fmaf(d.dd.y, dirUV.y, fmaf(d.dd.x, dirUV.x, denomCenter));
        o = fma3(lensUV.y, lensV, fma3(lensUV.x, lensU, d.v0l));
        rd = fma3(dirUV.y, lensV, fma3(dirUV.x, lensU, lc2fc));
        V3 a = -rd;
        e = mk(fmaf(a.y, o.z, -(a.z * o.y)), fmaf(a.z, o.x, -(a.x * o.z)), fmaf(a.x, o.y, -(a.y * o.x)));
        v = fmaf(d.e1.z, e.z, fmaf(d.e1.y, e.y, d.e1.x * e.x));
        w = -fmaf(d.e0.z, e.z, fmaf(d.e0.y, e.y, d.e0.x * e.x));
    } else {
        denom = denomCenter + d.dd.x * dirUV.x + d.dd.y * dirUV.y;
        o = d.v0l + lensU * lensUV.x + lensV * lensUV.y;
        rd = lc2fc + lensU * dirUV.x + lensV * dirUV.y;
        e = cross(-rd, o);
        v = dot(d.e1, e);
        w = -dot(d.e0, e);
    }
}

// IntersectTriangleThreadDoF::test
inline bool dofTest(const DofTri& d, float denomCenter, V3 lc2fc, V3 lensU, V3 lensV, V2 lensUV, V2 dirUV,
                    float& depth, bool fma) {
    float t = fma ? fmaf(d.tV, lensUV.y, fmaf(d.tU, lensUV.x, d.tC)) : d.tC + d.tU * lensUV.x + d.tV * lensUV.y;
    float denom, v, w;
    dofBary(d, denomCenter, lc2fc, lensU, lensV, lensUV, dirUV, fma, denom, v, w);
    float depthDelta = fma ? fmaf(depth, denom, -t) : depth * denom - t;
    float u = denom - v - w;
    int32_t test = int32_t(fbits(t) | fbits(depthDelta) | fbits(u) | fbits(v) | fbits(w));
    if (test < 0) return false;
    // a NaN (the zero beam of a padding sample normalises to NaN) fails: the sign-bit test alone
    // depends on which NaN the platform produces (x86's default NaN is negative)
    if (u != u || depthDelta != depthDelta) return false;
    depth = t * (1.0f / denom);
    return true;
}

// IntersectTriangleThreadDoF::calcUVW
inline V3 dofUVW(const DofTri& d, float denomCenter, V3 lc2fc, V3 lensU, V3 lensV, V2 lensUV, V2 dirUV, bool fma) {
    float denom, v, w;
    dofBary(d, denomCenter, lc2fc, lensU, lensV, lensUV, dirUV, fma, denom, v, w);
    float u = denom - v - w;
    float inv = 1.0f / denom;
    return mk(u * inv, v * inv, w * inv);
}

// ------------------------------------------------------------------ shading (RC/shading.h, RC/shading_helpers.h)
const int kTau[] = {1,  1,  1,  2,  3,  2,  5,  2,  3,  2,  3,  3,  5,  5,  3,  4,  7,  5,  5,  7,
                    9,  8,  5,  5,  7,  7,  7,  8,  5,  8,  11, 12, 7,  10, 13, 8,  11, 8,  7,  14};

struct Material { V3 emissive, diffuse, specular; float glossiness; uint64_t code; };

struct LightEnv {
    int nd = 0, np = 0, ns = 0;
    hvvr_light_directional dir[1];
    hvvr_light_point pt[4];
    hvvr_light_spot spot[4];
};

inline V3 v3(hvvr_vec3 v) { return mk(v.x, v.y, v.z); }
inline float pow5(float x) { float x2 = x * x; return x2 * x2 * x; }

// GGX_SchlickFresnel_SchlickSmithGGX (RC/shading_helpers.h:89-112)
V3 ggxSpec(V3 N, V3 L, V3 V, float roughness, V3 F0) {
    float alpha = roughness * roughness;
    V3 H = normalize(L + V);
    float alpha2 = alpha * alpha;
    float NdotH = sat(dot(N, H));
    float nh2 = NdotH * NdotH;
    float q = nh2 * (alpha2 - 1.0f) + 1.0f;
    float D = alpha2 / (3.141592653589f * (q * q));
    float LdotH = sat(dot(L, H));
    V3 F = F0 + (mk(1, 1, 1) - F0) * pow5(1.0f - LdotH);
    float NdotL = sat(dot(N, L));
    float NdotV = sat(dot(N, V));
    float k = alpha * 0.5f;
    float vis = (1.0f / (NdotL * (1.0f - k) + k)) * (1.0f / (NdotV * (1.0f - k) + k));
    return divs((F * D) * vis, 4.0f);
}
// PBR_BRDF1 (RC/shading_helpers.h:115-122)
V3 pbr(V3 L, V3 N, V3 V, V3 base, float roughness, V3 F0, V3 lightColor) {
    V3 spec = ggxSpec(N, L, V, roughness, F0);
    float NdotL = sat(dot(N, L));
    V3 diffuse = ((base * lightColor) * (mk(1, 1, 1) - spec)) * NdotL;
    V3 glossy = lightColor * spec;
    return diffuse + glossy;
}
// the texture reads of one shading point: uv, its screen derivatives and the sampler
struct TexRead {
    V2 uv, dx, dy;
    const oracle_frame_in* in;
    // ReadTexture (RC/shading.h:45-47) for material texture slot `id`; false (the constant
    // stays) for badTextureIndex and for an id with no live texture
    bool read(uint32_t id, float* rgba) const {
        if (id == 0xffffu || id >= in->texture_count || !in->texture_sample) return false;
        const float q[6] = {uv.x, uv.y, dx.x, dx.y, dy.x, dy.y};
        in->texture_sample(in->texture_ctx, id, q, rgba);
        return true;
    }
};
// true when GGXShade reads a texture for m (the emissive texture for the emissive model, else
// any of diffuse, specular, glossiness; SimpleMaterial bit layout, RC/material.h:22-49)
bool readsTextures(const Material& m) {
    uint32_t model = uint32_t(m.code & 0xffff);
    uint32_t gl = uint32_t(m.code >> 16) & 0xffff, sp = uint32_t(m.code >> 32) & 0xffff, di = uint32_t(m.code >> 48);
    return model == 2 ? di != 0xffff : (di != 0xffff || sp != 0xffff || gl != 0xffff);
}
// GGXShade (RC/shading.h:84-161); tex NULL: no texture reads (the constants stay)
V3 ggxShade(const Material& m, V3 pos, V3 nrm, V3 camPos, const LightEnv& env, const TexRead* tex) {
    V3 normal = normalize(nrm);
    uint32_t model = uint32_t(m.code & 0xffff);
    const uint32_t texGloss = uint32_t(m.code >> 16) & 0xffff, texSpec = uint32_t(m.code >> 32) & 0xffff,
                   texDiffuse = uint32_t(m.code >> 48) & 0xffff;
    float t[4];
    if (model == 2) { // emissive
        if (tex && tex->read(texDiffuse, t)) return mk(t[0], t[1], t[2]);
        return m.emissive;
    }
    V3 base = m.diffuse;
    if (tex && tex->read(texDiffuse, t)) base = mk(t[0], t[1], t[2]);
    V3 V = normalize(camPos - pos);
    V3 F0 = m.specular;
    if (tex && tex->read(texSpec, t)) F0 = mk(t[0], t[1], t[2]);
    float roughness = 1.0f - m.glossiness;
    if (tex && tex->read(texGloss, t)) roughness = 1.0f - t[0];
    V3 radiance = m.emissive;
    radiance = radiance + base * mk(.15f, .15f, .165f);
    for (int i = 0; i < env.nd && i < 1; i++)
        radiance = radiance + pbr(v3(env.dir[i].direction), normal, V, base, roughness, F0, v3(env.dir[i].power));
    for (int i = 0; i < env.np && i < 4; i++) {
        const hvvr_light_point& l = env.pt[i];
        V3 delta = v3(l.position) - pos;
        float r = length(delta);
        V3 L = normalize(delta);
        float fd = sat((l.falloff_end - r) * l.falloff_scale);
        radiance = radiance + pbr(L, normal, V, base, roughness, F0, v3(l.color) * fd);
    }
    for (int i = 0; i < env.ns && i < 4; i++) {
        const hvvr_light_spot& l = env.spot[i];
        V3 delta = v3(l.position) - pos;
        float r = length(delta);
        V3 L = normalize(delta);
        float fd = sat((l.falloff_end - r) * l.falloff_scale);
        V3 lit = pbr(L, normal, V, base, roughness, F0, v3(l.color) * fd);
        float cosA = dot(v3(l.direction), -L);
        float fa = sat((cosA - l.cos_outer_angle) * l.cos_angle_scale);
        radiance = radiance + lit * fa;
    }
    return mk(tmax(radiance.x, 0.0f), tmax(radiance.y, 0.0f), tmax(radiance.z, 0.0f));
}
// ACESFilm + linearToSRgb + ToColor4Unorm8SRgb (RC/shading_helpers.h:158-200; SH/util_graphics.h:26-28)
inline float aces(float x) {
    float r = (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
    return sat(r);
}
inline float toSrgb(float x) { return (x <= 0.0031308f) ? (x * 12.92f) : (powf(x, (1.0f / 2.4f)) * 1.055f - .055f); }
inline uint32_t packColor(V3 c) {
    uint32_t r = uint32_t(toSrgb(c.x) * 255.0f), g = uint32_t(toSrgb(c.y) * 255.0f), b = uint32_t(toSrgb(c.z) * 255.0f);
    uint32_t a = uint32_t(1.0f * 255.0f);
    return r | (g << 8) | (b << 16) | (a << 24);
}

struct MxcsrScope {
    unsigned saved;
    MxcsrScope() { saved = _mm_getcsr(); _mm_setcsr(saved | 0x8040); }
    ~MxcsrScope() { _mm_setcsr(saved); }
};

} // namespace

extern "C" void oracle_msaa_offsets(uint32_t n, float* out) {
    // tapLocation / getSubsampleUnitOffset with JITTER_SAMPLES=0 (RC/gpu_samples.h:35-61)
    int turns = kTau[n];
    for (uint32_t i = 0; i < n; i++) {
        float alpha = float(int(i) + 0.5f) * (1.0f / float(n));
        float angle = alpha * (float(turns) * 6.28f) + 0.0f;
        float radius = sqrtf(alpha);
        out[2 * i + 0] = cosf(angle) * radius;
        out[2 * i + 1] = sinf(angle) * radius;
    }
}

// The library's alternative MSAA pattern (no counterpart in the reference, whose only pattern is
// the spiral above): an n-rooks lattice, subsample i in column i and row (k i) mod n of an n x n
// grid over [-1, 1]^2 (k = 1, 3, 5, 9, 19 for n = 2, 4, 8, 16, 32), scaled by 1/sqrt(2) into the
// unit disk; n = 1 is the sample's centre.
extern "C" void oracle_msaa_offsets_rotated_grid(uint32_t n, float* out) {
    const uint32_t k = n == 2 ? 1u : n == 4 ? 3u : n == 8 ? 5u : n == 16 ? 9u : n == 32 ? 19u : 0u;
    for (uint32_t i = 0; i < n; i++) {
        const float x = float(2 * i + 1) / float(n) - 1.0f;
        const float y = float(2 * ((k * i) % n) + 1) / float(n) - 1.0f;
        out[2 * i + 0] = x * 0.70710677f;
        out[2 * i + 1] = y * 0.70710677f;
    }
}

// GPUCamera::initLookupTables (RC/gpu_camera.cu:59-88): DOF_LENS_POS_LOOKUP_TABLE_TILES (4) tiles of
// per-sample random rotations of the spiral, subsample i taking spiral position (7 i + 7) mod n,
// laid out [tile][subsample][sample]; std::mt19937 default seed, uniform_real_distribution<float>.
extern "C" void oracle_lens_table(uint32_t n, float* out) {
    std::uniform_real_distribution<float> dist(0.0f, 1.0f);
    std::mt19937 gen;
    const float tauF = 6.283185307180f; // Tau (SH/constants_math.h:16)
    int turns = kTau[n];
    for (uint32_t tile = 0; tile < 4; tile++)
        for (uint32_t s = 0; s < kTileSize; s++) {
            float rotation = dist(gen) * tauF;
            for (uint32_t i = 0; i < n; i++) {
                int k = int((i * 7 + 7) % n);
                float alpha = float(k + 0.5f) * (1.0f / float(n));
                float angle = alpha * (float(turns) * 6.28f) + rotation;
                float radius = sqrtf(alpha);
                size_t o = (size_t(tile) * kTileSize * n + size_t(i) * kTileSize + s) * 2;
                out[o + 0] = cosf(angle) * radius;
                out[o + 1] = sinf(angle) * radius;
            }
        }
}

extern "C" void oracle_layout(uint32_t sample_count, uint32_t* blocks, uint32_t* tiles, uint32_t* padded) {
    uint32_t b = (sample_count + kBlockSize - 1) / kBlockSize;
    if (blocks) *blocks = b;
    if (tiles) *tiles = b * kTilesPerBlock;
    if (padded) *padded = b * kBlockSize;
}

extern "C" void oracle_scene_counts(const oracle_frame_in* in, uint32_t* nodes, uint32_t* tris, uint32_t* verts) {
    uint32_t n = in->model_count ? (in->model_count + 1) / 3 : 1, t = 0, v = 0;
    for (uint32_t m = 0; m < in->model_count; m++) {
        n += in->models[m].node_count; t += in->models[m].tri_count; v += in->models[m].vert_count;
    }
    if (nodes) *nodes = n;
    if (tris) *tris = t;
    if (verts) *verts = v;
}

namespace {
int renderCore(const oracle_frame_in* in, const SampleSetup& ss, const M4& c2w, const float* cullPlanes,
               oracle_frame_out* out);
}

extern "C" int oracle_render(const oracle_frame_in* in, oracle_frame_out* out) {
    MxcsrScope mx;
    if (!in || !out || in->sample_count == 0) return 1;
    SampleSetup ss;
    setupSamples(in, ss);
    if (out->remap) memcpy(out->remap, ss.remap.data(), ss.remap.size() * sizeof(int32_t));
    if (out->beams) memcpy(out->beams, ss.beams.data(), ss.beams.size() * sizeof(Beam));
    if (out->tile_rays) memcpy(out->tile_rays, ss.tileRays.data(), ss.tileRays.size() * sizeof(Rays4));
    return renderCore(in, ss, transformToMatrix(in->cam_xf), nullptr, out);
}

extern "C" int oracle_render_beams(const oracle_frame_in* in, const oracle_beams_in* bi, oracle_frame_out* out) {
    MxcsrScope mx;
    if (!in || !bi || !out || bi->blocks == 0) return 1;
    SampleSetup ss;
    ss.blocks = bi->blocks;
    ss.tiles = bi->blocks * kTilesPerBlock;
    ss.padded = bi->blocks * kBlockSize;
    ss.valid = ss.padded;
    ss.beams.resize(ss.padded);
    memcpy(ss.beams.data(), bi->beams, ss.beams.size() * sizeof(Beam));
    ss.tileRays.resize(ss.tiles);
    memcpy(ss.tileRays.data(), bi->tile_rays, ss.tileRays.size() * sizeof(Rays4));
    ss.blockRays.resize(ss.blocks);
    memcpy(ss.blockRays.data(), bi->block_rays, ss.blockRays.size() * sizeof(Rays4));
    M4 m;
    memcpy(&m, bi->batch_to_world, sizeof(M4));
    return renderCore(in, ss, m, bi->cull_planes, out);
}

namespace {
int renderCore(const oracle_frame_in* in, const SampleSetup& ss, const M4& c2w, const float* cullPlanes,
               oracle_frame_out* out) {
    uint32_t N = in->msaa;
    if (!(N == 1 || N == 2 || N == 4 || N == 8 || N == 16 || N == 32)) return 1;
    bool useFma = in->fp_mode == HVVR_FP_FMA;
    out->status = 0;

    Scene scene;
    buildScene(in, scene);
    refitScene(in, scene);
    out->status |= scene.status;
    if (out->nodes) memcpy(out->nodes, scene.nodes.data(), scene.nodes.size() * sizeof(Node));
    if (out->tris) memcpy(out->tris, scene.tris.data(), scene.tris.size() * sizeof(Tri));

    // per-frame transform (RC/render.cpp:282-365, RC/traversal.h:38-47)
    M3 R = m3of(c2w);
    auto xformRays = [&](const Rays4& r) {
        Rays4 w;
        for (int v = 0; v < 4; v++) {
            V4 o = mul(c2w, V4{r.o[v].x, r.o[v].y, r.o[v].z, 1.0f});
            w.o[v] = mk(o.x, o.y, o.z);
            w.d[v] = mul(R, r.d[v]);
        }
        return w;
    };
    std::vector<Rays4> tileW(ss.tiles), blockW(ss.blocks);
    for (uint32_t i = 0; i < ss.tiles; i++) tileW[i] = xformRays(ss.tileRays[i]);
    for (uint32_t i = 0; i < ss.blocks; i++) blockW[i] = xformRays(ss.blockRays[i]);
    // blockTransformAndCullTask: a tile frustum entirely beyond one of the cull planes becomes
    // degenerate (origin at infinity); planeCullsFrustum (RC/render.cpp:270-279)
    if (cullPlanes) {
        for (uint32_t t = 0; t < ss.tiles; t++) {
            bool culled = false;
            for (int p = 0; p < 4; p++) {
                V3 n = mk(cullPlanes[4 * p], cullPlanes[4 * p + 1], cullPlanes[4 * p + 2]);
                float dist = cullPlanes[4 * p + 3];
                bool allout = true;
                for (int i = 0; i < 4; i++) {
                    allout = allout && dot(n, tileW[t].o[i]) > dist;
                    allout = allout && dot(n, tileW[t].o[i] + tileW[t].d[i] * 10000.0f) > dist;
                }
                culled = culled || allout;
            }
            if (culled)
                for (int i = 0; i < 4; i++) {
                    tileW[t].o[i] = mk(INFINITY, INFINITY, INFINITY);
                    tileW[t].d[i] = mk(0.0f, 0.0f, 0.0f);
                }
        }
    }

    const Node* nodes = scene.nodes.data();
    std::vector<StackEntry> blockStacks(size_t(ss.blocks) * kBlockStackSize);
    std::vector<uint32_t> blockSizes(ss.blocks);
    for (uint32_t b = 0; b < ss.blocks; b++) {
        TravFrustum f;
        buildTravFrustum(blockW[b].o, blockW[b].d, f);
        blockSizes[b] = traverseBlock(nodes, f, &blockStacks[size_t(b) * kBlockStackSize]);
        if (out->block_sizes) out->block_sizes[b] = blockSizes[b];
        if (out->block_entries) {
            for (uint32_t i = 0; i < kBlockStackSize; i++) {
                const StackEntry& e = blockStacks[size_t(b) * kBlockStackSize + i];
                uint32_t* dst = out->block_entries + (size_t(b) * kBlockStackSize + i) * 3;
                if (i < blockSizes[b]) { dst[0] = fbits(e.tMin); dst[1] = e.mask; dst[2] = e.node; }
                else { dst[0] = dst[1] = dst[2] = 0; }
            }
        }
    }

    // MSAA offsets and the lighting environment (GPUSceneState::updateLighting, RC/gpu_scene_state.cu:47-81)
    std::vector<float> off(2 * N);
    // thin-lens views keep the spiral, which their lens table is built on
    if (in->msaa_pattern == HVVR_MSAA_ROTATED_GRID && !(in->lens.radius > 0.0f))
        oracle_msaa_offsets_rotated_grid(N, off.data());
    else oracle_msaa_offsets(N, off.data());
    LightEnv env;
    for (uint32_t i = 0; i < in->light_count; i++) {
        const hvvr_light_union& l = in->lights[i];
        if (l.type == HVVR_LIGHT_DIRECTIONAL && env.nd < 1) env.dir[env.nd++] = l.u.directional;
        else if (l.type == HVVR_LIGHT_POINT && env.np < 4) env.pt[env.np++] = l.u.point;
        else if (l.type == HVVR_LIGHT_SPOT && env.ns < 4) env.spot[env.ns++] = l.u.spot;
    }
    std::vector<Material> mats(scene.materials.size());
    for (size_t i = 0; i < mats.size(); i++) {
        const hvvr_material& m = scene.materials[i];
        mats[i] = Material{mk(m.emissive.x, m.emissive.y, m.emissive.z), mk(m.diffuse.x, m.diffuse.y, m.diffuse.z),
                           mk(m.specular.x, m.specular.y, m.specular.z), m.glossiness, m.texture_ids_and_shading_model};
    }
    V3 camPos = mk(c2w.m3.x, c2w.m3.y, c2w.m3.z);
    V3 lookVec = -mk(c2w.m2.x, c2w.m2.y, c2w.m2.z); // cameraLookVector = -vector3(cameraToWorld.m2)

    // tiles: traversal of every tile first (the reference's lists are complete before its
    // intersect launch), then intersect + shade (RC/intersect.cu:171-342, RC/resolve.cu:161-458)
    std::vector<std::vector<uint32_t>> lists(ss.tiles);
    std::vector<uint32_t> colors(ss.padded, 0xFF000000u);
    std::atomic<uint32_t> next(0), status(0);
    uint32_t nt = in->threads ? in->threads : 1;
    auto runPool = [&](auto&& fn) {
        next = 0;
        std::vector<std::thread> pool;
        for (uint32_t t = 1; t < nt; t++) pool.emplace_back(fn);
        fn();
        for (auto& th : pool) th.join();
    };
    runPool([&]() {
        MxcsrScope mxw;
        for (;;) {
            uint32_t tile = next.fetch_add(1);
            if (tile >= ss.tiles) break;
            uint32_t b = tile / kTilesPerBlock;
            TravFrustum f;
            buildTravFrustum(tileW[tile].o, tileW[tile].d, f);
            uint32_t st = 0;
            traverseTile(nodes, f, &blockStacks[size_t(b) * kBlockStackSize], blockSizes[b], lists[tile], st);
            if (st) status.fetch_or(st);
        }
    });

    // depth of field (lens radius > 0): the lens-position table is indexed by the intersect/resolve
    // CTA index, which is the tile's rank among the occupied tiles (tileIndexRemapOccupied,
    // RC/traversal.cpp:213-330); the per-tile lens values come from the tile's middle sample
    const bool dof = in->lens.radius > 0.0f;
    std::vector<V2> lensTab;
    std::vector<uint32_t> occRank(ss.tiles, 0);
    V3 look = mul(R, mk(0.0f, 0.0f, -1.0f));
    if (dof) {
        lensTab.resize(size_t(kTileSize) * 4 * N);
        oracle_lens_table(N, &lensTab[0].x);
        uint32_t r = 0;
        for (uint32_t t = 0; t < ss.tiles; t++) {
            occRank[t] = r;
            if (!lists[t].empty()) r++;
        }
    }

    runPool([&]() {
        MxcsrScope mxw;
        for (;;) {
            uint32_t tile = next.fetch_add(1);
            if (tile >= ss.tiles) break;
            const std::vector<uint32_t>& list = lists[tile];
            uint32_t base = tile * kTileSize;
            if (list.empty()) {
                // ClearEmptyKernel (RC/resolve.cu:527-542)
                for (uint32_t s = 0; s < kTileSize; s++) {
                    for (uint32_t i = 0; i < N; i++) {
                        size_t o = size_t(base + s) * N + i;
                        if (out->hit_ids) out->hit_ids[o] = ~0u;
                        if (out->depth) out->depth[o] = INFINITY;
                        if (out->depth64) out->depth64[o] = NAN;
                        if (out->gb_tri) out->gb_tri[o] = (i == 0) ? ~0u : 0u;
                        if (out->gb_mask) out->gb_mask[o] = (i == 0) ? (N == 32 ? ~0u : ((1u << N) - 1)) : 0u;
                    }
                    if (out->gb_n) out->gb_n[base + s] = 1;
                    if (out->tmax) out->tmax[base + s] = INFINITY;
                    colors[base + s] = 0xFF000000u;
                }
                continue;
            }
            FrustumPlanes fp = makePlanes(tileW[tile]);
            DofTile dt{};
            const uint32_t lensTile = occRank[tile] % 4;
            if (dof) dt = dofTileData(R, ss.beams[base + kTileSize / 2], in->lens);
            // per-chunk culling and compaction preserves list order, so the surviving sequence is
            // the list filtered by the three pre-tests
            std::vector<uint32_t> surv;
            std::vector<TriTile> survTT;
            std::vector<DofTri> survDT;
            surv.reserve(list.size());
            for (uint32_t idx : list) {
                const Tri& tri = scene.tris[idx];
                if (!planesTest(fp, tri)) continue;
                if (dof) {
                    DofTri d;
                    int r = dofSetup(tri, camPos, dt.lensU, dt.lensV, d);
                    if (r == kAllOut) continue;
                    // the corner-ray test only when every lens position sees the front of the plane
                    if (r == kAllIn && !uvwNotAllOut(tileW[tile], tri)) continue;
                    surv.push_back(idx);
                    survDT.push_back(d);
                } else {
                    TriTile tt;
                    if (!tileSetup(tri, camPos, tt)) continue;
                    if (!uvwNotAllOut(tileW[tile], tri)) continue;
                    surv.push_back(idx);
                    survTT.push_back(tt);
                }
            }
            for (uint32_t s = 0; s < kTileSize; s++) {
                uint32_t sid = base + s;
                const Beam& bm = ss.beams[sid];
                V3 c = mul(R, bm.c), du = mul(R, bm.du), dv = mul(R, bm.dv);
                V3 lc2fc{};
                if (dof) {
                    V3 centerDir = normalize(c);
                    float zed = dot(look, centerDir);
                    lc2fc = centerDir * (in->lens.focal_distance / zed);
                }
                float tmaxv[32];
                uint32_t hit[32];
                for (uint32_t i = 0; i < N; i++) { tmaxv[i] = FLT_MAX; hit[i] = ~0u; }
                for (size_t j = 0; j < surv.size(); j++) {
                    if (dof) {
                        float dc = dofDenomCenter(survDT[j], lc2fc);
                        for (uint32_t i = 0; i < N; i++) {
                            V2 lensUV, dirUV;
                            dofSampleUVs(lensTab.data(), N, lensTile, s, i, V2{off[2 * i], off[2 * i + 1]},
                                         dt.focalToLensScale, useFma, lensUV, dirUV);
                            if (dofTest(survDT[j], dc, lc2fc, dt.lensU, dt.lensV, lensUV, dirUV, tmaxv[i], useFma))
                                hit[i] = surv[j];
                        }
                    } else {
                        TriThread th = threadSetup(survTT[j], c, du, dv);
                        for (uint32_t i = 0; i < N; i++) {
                            V2 a{off[2 * i], off[2 * i + 1]};
                            if (threadTest(th, survTT[j].t, a, tmaxv[i], useFma)) hit[i] = surv[j];
                        }
                    }
                }
                for (uint32_t i = 0; i < N; i++) {
                    size_t o = size_t(sid) * N + i;
                    if (out->hit_ids) out->hit_ids[o] = hit[i];
                    if (out->depth) out->depth[o] = hit[i] == ~0u ? INFINITY : tmaxv[i];
                    if (out->depth64) {
                        if (hit[i] == ~0u || dof) out->depth64[o] = NAN;
                        else {
                            const Tri& t = scene.tris[hit[i]];
                            double D[3] = {double(c.x) + double(off[2 * i]) * du.x + double(off[2 * i + 1]) * dv.x,
                                           double(c.y) + double(off[2 * i]) * du.y + double(off[2 * i + 1]) * dv.y,
                                           double(c.z) + double(off[2 * i]) * du.z + double(off[2 * i + 1]) * dv.z};
                            double e0[3] = {t.e0.x, t.e0.y, t.e0.z}, e1[3] = {t.e1.x, t.e1.y, t.e1.z};
                            double n[3] = {e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2],
                                           e0[0] * e1[1] - e0[1] * e1[0]};
                            double w0[3] = {double(camPos.x) - t.v0.x, double(camPos.y) - t.v0.y, double(camPos.z) - t.v0.z};
                            double num = w0[0] * n[0] + w0[1] * n[1] + w0[2] * n[2];
                            double den = -(D[0] * n[0] + D[1] * n[1] + D[2] * n[2]);
                            out->depth64[o] = num / den;
                        }
                    }
                }
                // TMaxBuffer (RC/resolve.cu:386-457): view depth of subsample 0's triangle at subsample 0
                if (out->tmax) {
                    float tv = INFINITY;
                    if (hit[0] != ~0u && !dof) {
                        const Tri& tri = scene.tris[hit[0]];
                        TriTile tt;
                        tileSetup(tri, camPos, tt);
                        V3 uvw = calcUVW(threadSetup(tt, c, du, dv), V2{off[0], off[1]}, useFma);
                        V3 p = (tri.v0 * uvw.x + (tri.v0 + tri.e0) * uvw.y) + (tri.v0 + tri.e1) * uvw.z;
                        tv = dot(p - camPos, lookVec);
                    }
                    out->tmax[sid] = tv;
                }
                // G-buffer compression (EmitGBuffer, RC/intersect.cu:28-89): pairs sorted by tri, misses last
                uint32_t keys[32];
                for (uint32_t i = 0; i < N; i++) keys[i] = (hit[i] << 5) | i;
                std::sort(keys, keys + N);
                uint32_t gtri[32], gmask[32], gn = 0;
                for (uint32_t i = 0; i < N; i++) {
                    uint32_t t = uint32_t(int32_t(keys[i]) >> 5);
                    uint32_t m = 1u << (keys[i] & 31);
                    if (gn && gtri[gn - 1] == t) gmask[gn - 1] |= m;
                    else { gtri[gn] = t; gmask[gn] = m; gn++; }
                }
                if (out->gb_n) out->gb_n[sid] = gn;
                for (uint32_t i = 0; i < N; i++) {
                    if (out->gb_tri) out->gb_tri[size_t(sid) * N + i] = i < gn ? gtri[i] : 0;
                    if (out->gb_mask) out->gb_mask[size_t(sid) * N + i] = i < gn ? gmask[i] : 0;
                }
                // ShadeMSAA (RC/resolve.cu:161-284), centroid shading per unique triangle
                float res[4] = {0, 0, 0, 0};
                uint32_t all = N == 32 ? ~0u : ((1u << N) - 1), combined = 0;
                for (uint32_t g = 0; g < gn; g++) {
                    if (combined == all) break;
                    uint32_t triIndex = gtri[g];
                    if (triIndex == ~0u) break;
                    uint32_t sm = gmask[g];
                    combined |= sm;
                    float inv = 1.0f / float(__builtin_popcount(sm));
                    V2 ca{0.0f, 0.0f}, cl{0.0f, 0.0f}, cd{0.0f, 0.0f};
                    for (uint32_t cm = sm; cm;) {
                        int si = __builtin_ctz(cm);
                        cm &= ~(1u << si);
                        ca.x = ca.x + off[2 * si] * inv;
                        ca.y = ca.y + off[2 * si + 1] * inv;
                        if (dof) {
                            V2 lensUV, dirUV;
                            dofSampleUVs(lensTab.data(), N, lensTile, s, uint32_t(si), V2{off[2 * si], off[2 * si + 1]},
                                         dt.focalToLensScale, useFma, lensUV, dirUV);
                            cl.x = cl.x + lensUV.x * inv; cl.y = cl.y + lensUV.y * inv;
                            cd.x = cd.x + dirUV.x * inv; cd.y = cd.y + dirUV.y * inv;
                        }
                    }
                    const Tri& tri = scene.tris[triIndex];
                    const hvvr_tri_shade& ts = scene.triShade[triIndex];
                    const bool textured = in->texture_count && readsTextures(mats[ts.material]);
                    // bx, by: barycentrics one sample step along x and y, for the texture
                    // derivatives (centroid alpha + (1,0) / (0,1); the DoF branch steps the
                    // centroid direction the same way, RC/resolve.cu:232-262)
                    V3 bc, bx{}, by{};
                    if (dof) {
                        DofTri d;
                        dofSetup(tri, camPos, dt.lensU, dt.lensV, d);
                        const float dcen = dofDenomCenter(d, lc2fc);
                        bc = dofUVW(d, dcen, lc2fc, dt.lensU, dt.lensV, cl, cd, useFma);
                        if (textured) {
                            bx = dofUVW(d, dcen, lc2fc, dt.lensU, dt.lensV, cl, V2{cd.x + 1.0f, cd.y + 0.0f}, useFma);
                            by = dofUVW(d, dcen, lc2fc, dt.lensU, dt.lensV, cl, V2{cd.x + 0.0f, cd.y + 1.0f}, useFma);
                        }
                    } else {
                        TriTile tt;
                        tileSetup(tri, camPos, tt);
                        TriThread th = threadSetup(tt, c, du, dv);
                        bc = calcUVW(th, ca, useFma);
                        if (textured) {
                            bx = calcUVW(th, V2{ca.x + 1.0f, ca.y + 0.0f}, useFma);
                            by = calcUVW(th, V2{ca.x + 0.0f, ca.y + 1.0f}, useFma);
                        }
                    }
                    const hvvr_shading_vertex& a0 = scene.world[ts.indices[0]];
                    const hvvr_shading_vertex& a1 = scene.world[ts.indices[1]];
                    const hvvr_shading_vertex& a2 = scene.world[ts.indices[2]];
                    V3 pos = (v3(a0.pos) * bc.x + v3(a1.pos) * bc.y) + v3(a2.pos) * bc.z;
                    V3 n0 = mk(halfToFloat(a0.normal[0]), halfToFloat(a0.normal[1]), halfToFloat(a0.normal[2]));
                    V3 n1 = mk(halfToFloat(a1.normal[0]), halfToFloat(a1.normal[1]), halfToFloat(a1.normal[2]));
                    V3 n2 = mk(halfToFloat(a2.normal[0]), halfToFloat(a2.normal[1]), halfToFloat(a2.normal[2]));
                    V3 nrm = (n0 * bc.x + n1 * bc.y) + n2 * bc.z;
                    TexRead tr;
                    if (textured) {
                        // interpolate (RC/shading.h:18-36) of uv at bc, bx, by; dUVdX/dUVdY as differences
                        auto uvAt = [&](V3 b) {
                            return V2{(a0.uv.x * b.x + a1.uv.x * b.y) + a2.uv.x * b.z,
                                      (a0.uv.y * b.x + a1.uv.y * b.y) + a2.uv.y * b.z};
                        };
                        const V2 uv = uvAt(bc), ux = uvAt(bx), uy = uvAt(by);
                        tr = TexRead{uv, V2{ux.x - uv.x, ux.y - uv.y}, V2{uy.x - uv.x, uy.y - uv.y}, in};
                    }
                    V3 col = ggxShade(mats[ts.material], pos, nrm, camPos, env, textured ? &tr : nullptr);
                    float pc = float(__builtin_popcount(sm));
                    res[0] = res[0] + col.x * pc; res[1] = res[1] + col.y * pc; res[2] = res[2] + col.z * pc;
                }
                float sN = 1.0f / float(N);
                V3 lin = mk(res[0] * sN, res[1] * sN, res[2] * sN);
                colors[sid] = packColor(mk(aces(lin.x), aces(lin.y), aces(lin.z)));
            }
        }
    });
    out->status |= status.load();

    uint64_t total = 0;
    for (uint32_t t = 0; t < ss.tiles; t++) {
        if (out->tile_counts) out->tile_counts[t] = uint32_t(lists[t].size());
        if (out->tile_indices) {
            for (uint32_t v : lists[t]) {
                if (total < out->tile_capacity) out->tile_indices[total] = v;
                total++;
            }
        } else {
            total += lists[t].size();
        }
    }
    out->tile_total = total;
    if (out->tile_indices && total > out->tile_capacity) out->status |= 8;
    if (out->colors) memcpy(out->colors, colors.data(), colors.size() * 4);
    // RemapKernel (RC/remap.cu:35-77)
    if (out->image && !ss.remap.empty()) {
        uint32_t split = in->split_color_samples;
        for (uint32_t y = 0; y < in->height; y++)
            for (uint32_t x = 0; x < in->width; x++) {
                size_t p = size_t(y) * in->width + x;
                if (split == 1) {
                    int32_t o = ss.remap[p];
                    if (o >= 0) out->image[p] = colors[o];
                } else {
                    uint32_t c[3] = {0, 0, 0};
                    for (uint32_t ch = 0; ch < split; ch++) {
                        int32_t o = ss.remap[p * split + ch];
                        if (o >= 0) c[ch] = colors[o];
                    }
                    out->image[p] = split == 2 ? ((c[1] & 0xff) | (c[0] & 0xff00) | (c[1] & 0xff0000) | 0xff000000u)
                                               : ((c[0] & 0xff) | (c[1] & 0xff00) | (c[2] & 0xff0000) | 0xff000000u);
                }
            }
    }
    return 0;
}
} // namespace

// ------------------------------------------------------------------ foveated resolve
// Restatement, texel by texel and pixel by pixel, of the reference's foveated resolve in the
// pass order of GPUCamera::foveatedPolarToScreenSpace (RC/gpu_foveated.cu:335-375):
//   RemapPolarFoveatedKernel            RC/remap.cu:127-141
//   ComputeMoments                      RC/gpu_foveated.cu:124-139, 159-172
//   FoveatedPolarToScreenSpaceKernel    RC/gpu_foveated.cu:36-122, 141-157, 174-249
//   SeparableFilterUsingEccentricity    RC/gpu_foveated.cu:251-294, steps {0,1} then {1,0}
//   FinishConstrastEnhancement          RC/gpu_foveated.cu:296-333
// with the colour conversions of shared/util_graphics.h:16-33 and RC/shading_helpers.h:
// 178-224, the eccentricity map of RC/foveated.h:32-113 and the texture setup of
// RC/gpu_camera.cu:174-230. The reference reads CUDA texture objects; a fetch here is the
// texture unit's documented behaviour: normalized coordinates, wrap (u - floor(u)) or clamp
// addressing, linear filtering between floor(x) and floor(x) + 1 at x = u * n - 0.5 with the
// fraction held to 1/256, point sampling at floor(u * n), sRGB texels decoded by sRgbToLinear
// (alpha linear) and unorm16 texels as v / 65535. acos, atan2, log, cos, sin and pow are
// taken in double and rounded to float (the reference's single-precision device functions
// are within a few ulp of that).
namespace {

struct C4 {
    float x, y, z, w;
};
inline C4 c4(float x, float y, float z, float w) { return C4{x, y, z, w}; }
inline C4 operator+(C4 a, C4 b) { return c4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline C4 operator-(C4 a, C4 b) { return c4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
inline C4 operator*(C4 a, C4 b) { return c4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
inline C4 operator*(C4 a, float s) { return c4(a.x * s, a.y * s, a.z * s, a.w * s); }
// device min/max: a NaN operand yields the other one
inline float dmin(float a, float b) { return fminf(a, b); }
inline float dmax(float a, float b) { return fmaxf(a, b); }
inline float clampF(float x, float lo, float hi) { return dmin(hi, dmax(lo, x)); }
inline C4 clampC(C4 a, C4 lo, C4 hi) {
    return c4(clampF(a.x, lo.x, hi.x), clampF(a.y, lo.y, hi.y), clampF(a.z, lo.z, hi.z), clampF(a.w, lo.w, hi.w));
}
inline C4 clampC(C4 a, float lo, float hi) { return clampC(a, c4(lo, lo, lo, lo), c4(hi, hi, hi, hi)); }

inline float acosD(float x) { return float(acos(double(x))); }
inline float atan2D(float y, float x) { return float(atan2(double(y), double(x))); }
inline float logD(float x) { return float(log(double(x))); }
inline float cosD(float x) { return float(cos(double(x))); }
inline float sinD(float x) { return float(sin(double(x))); }
inline float powD(float x, float y) { return float(pow(double(x), double(y))); }

// sRgbToLinear / linearToSRgb (shared/util_graphics.h:16-33)
inline float sRgbToLinear(float x) {
    return (x <= 0.04045f) ? x * (1.0f / 12.92f) : powD((x + .055f) * (1.0f / 1.055f), 2.4f);
}
inline float linearToSRgb(float x) {
    return (x <= 0.0031308f) ? (x * 12.92f) : (powD(x, (1.0f / 2.4f)) * 1.055f - .055f);
}
// uint32_t(float) / uint64_t(float) as the device converts (truncate, saturate, NaN -> 0)
inline uint32_t toU32(float v) {
    if (!(v > 0.0f)) return 0;
    return v >= 4294967296.0f ? 0xffffffffu : uint32_t(v);
}
inline uint64_t toU64(float v) {
    if (!(v > 0.0f)) return 0;
    return v >= 18446744073709551616.0f ? ~0ull : uint64_t(v);
}
// ToColor4Unorm8SRgb(vector4), ToColor4Unorm16, FromColor4Unorm8SRgb (RC/shading_helpers.h)
inline uint32_t toColor4Unorm8SRgb(C4 c) {
    const uint32_t r = toU32(linearToSRgb(c.x) * 255.0f), g = toU32(linearToSRgb(c.y) * 255.0f);
    const uint32_t b = toU32(linearToSRgb(c.z) * 255.0f), a = toU32(c.w * 255.0f);
    return (r) | (g << 8) | (b << 16) | (a << 24);
}
inline uint64_t toColor4Unorm16(C4 c) {
    const float C = 65535.0f;
    const uint64_t r = toU64(c.x * C), g = toU64(c.y * C), b = toU64(c.z * C), a = toU64(c.w * C);
    return (r) | (g << 16) | (b << 32) | (a << 48);
}
inline C4 fromColor4Unorm8SRgb(uint32_t c) {
    const float r = (c & 0xFF) / 255.0f, g = ((c >> 8) & 0xFF) / 255.0f, b = ((c >> 16) & 0xFF) / 255.0f;
    const float a = ((c >> 24) & 0xFF) / 255.0f;
    return c4(sRgbToLinear(r), sRgbToLinear(g), sRgbToLinear(b), a);
}

// a texture: RGBA8 sRGB (uint32 texels), RGBA16 unorm (uint64 texels) or R32F
enum TexFormat { kSrgb8, kUnorm16, kR32f };
struct Tex {
    const void* data;
    int w, h;
    bool wrapX, wrapY;
    TexFormat fmt;
};
inline int address(int i, int n, bool wrap) {
    if (wrap) return ((i % n) + n) % n;
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}
inline C4 texel(const Tex& t, int x, int y) {
    const size_t o = size_t(address(y, t.h, t.wrapY)) * t.w + address(x, t.w, t.wrapX);
    if (t.fmt == kSrgb8) return fromColor4Unorm8SRgb(static_cast<const uint32_t*>(t.data)[o]);
    if (t.fmt == kUnorm16) {
        const uint64_t v = static_cast<const uint64_t*>(t.data)[o];
        return c4(float(v & 0xffff) / 65535.0f, float((v >> 16) & 0xffff) / 65535.0f,
                  float((v >> 32) & 0xffff) / 65535.0f, float((v >> 48) & 0xffff) / 65535.0f);
    }
    const float f = static_cast<const float*>(t.data)[o];
    return c4(f, 0.0f, 0.0f, 0.0f);
}
// one axis of a linear fetch: base texel and the 1/256-quantised fraction (in 256ths)
inline void linearTap(float u, int n, bool wrap, int& i0, int& a8) {
    if (wrap) u = u - floorf(u);
    float x = u * float(n) - 0.5f;
    x = dmax(dmin(x, float(n)), -1.0f);
    const float fl = floorf(x);
    i0 = int(fl);
    a8 = int(nearbyintf((x - fl) * 256.0f));
}
// tex2D with linear filtering at normalized (u, v)
inline C4 tex2DLinear(const Tex& t, float u, float v) {
    int x0, y0, ax, ay;
    linearTap(u, t.w, t.wrapX, x0, ax);
    linearTap(v, t.h, t.wrapY, y0, ay);
    const float wx1 = float(ax) * (1.0f / 256.0f), wx0 = float(256 - ax) * (1.0f / 256.0f);
    const float wy1 = float(ay) * (1.0f / 256.0f), wy0 = float(256 - ay) * (1.0f / 256.0f);
    return ((texel(t, x0, y0) * (wx0 * wy0) + texel(t, x0 + 1, y0) * (wx1 * wy0)) + texel(t, x0, y0 + 1) * (wx0 * wy1)) +
           texel(t, x0 + 1, y0 + 1) * (wx1 * wy1);
}
// tex2D with point filtering at normalized (u, v)
inline float tex2DPoint(const Tex& t, float u, float v) {
    auto idx = [](float c, int n, bool wrap) {
        if (wrap) c = c - floorf(c);
        return int(floorf(dmax(dmin(c * float(n), float(n)), -1.0f)));
    };
    return texel(t, idx(u, t.w, t.wrapX), idx(v, t.h, t.wrapY)).x;
}

constexpr float kPiF = 3.141592653589f;  // shared/constants_math.h:15

struct EccMapping {
    // EccentricityMap (RC/foveated.h:46-55) and EccentricityToTexCoordMapping (RC/gpu_foveated.cu:73-85)
    float m, w0, S, invLogA, invW0, invM, texMapSize, invTexMapSize, invMaxEccentricity;
    float applyInverse(float E) const {
        const float i0 = E * invW0;
        const float sDivW = S * invW0;
        const float x = logD((m * (i0 - sDivW)) + 1.0f) * invLogA;
        const float i1 = x + sDivW;
        return (E < S) ? i0 : i1;
    }
};

// getNormalizedCoord + sampleSpaceToEyeSpaceMatrix * point + eyeSpaceDirectionToAngularEyeCoord
inline void eyeCoord(const float* S, uint32_t i, uint32_t j, uint32_t w, uint32_t h, float& theta, float& ecc) {
    const float nx = (float(i) + 0.5f) / float(w), ny = (float(j) + 0.5f) / float(h);
    const float dx = S[0] * nx + S[3] * ny + S[6] * 1.0f;
    const float dy = S[1] * nx + S[4] * ny + S[7] * 1.0f;
    const float dz = S[2] * nx + S[5] * ny + S[8] * 1.0f;
    const float inv = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
    const float ex = dx * inv, ey = dy * inv, ez = dz * inv;
    ecc = acosD(-ez);
    theta = -atan2D(ey, ex);
}

// bicubicFast (RC/gpu_foveated.cu:36-71)
C4 bicubicFast(const Tex& tex, float cx, float cy) {
    const float W = float(tex.w), H = float(tex.h);
    const float pcx = cx * W, pcy = cy * H;
    const float ctx = floorf(pcx - 0.5f) + 0.5f, cty = floorf(pcy - 0.5f) + 0.5f;
    const float iDx = 1.0f / W, iDy = 1.0f / H;
    float s0[2], s1[2], t0[2], t1[2];
    const float fv[2] = {pcx - ctx, pcy - cty}, cv[2] = {ctx, cty}, iv[2] = {iDx, iDy};
    for (int k = 0; k < 2; k++) {
        const float f = fv[k], f2 = f * f, f3 = f2 * f;
        const float omf2 = (1.0f - f) * (1.0f - f);
        const float omf3 = omf2 * (1.0f - f);
        const float sixth = (1.0f / 6.0f);
        const float w0 = omf3 * sixth;
        const float w1 = ((4.0f / 6.0f) * 1.0f + f3 * 0.5f) - f2;
        const float w3 = f3 * sixth;
        const float w2 = ((1.0f - w0) - w1) - w3;
        s0[k] = w0 + w1;
        s1[k] = w2 + w3;
        const float f0 = w1 / (w0 + w1), f1 = w3 / (w2 + w3);
        t0[k] = ((cv[k] - 1.0f) + f0) * iv[k];
        t1[k] = ((cv[k] + 1.0f) + f1) * iv[k];
    }
    return tex2DLinear(tex, t0[0], t0[1]) * s0[0] * s0[1] + tex2DLinear(tex, t1[0], t0[1]) * s1[0] * s0[1] +
           tex2DLinear(tex, t0[0], t1[1]) * s0[0] * s1[1] + tex2DLinear(tex, t1[0], t1[1]) * s1[0] * s1[1];
}

template <class Fn>
void forRows(uint32_t rows, uint32_t threads, Fn fn) {
    std::atomic<uint32_t> next(0);
    auto work = [&]() {
        MxcsrScope mx;
        for (uint32_t r; (r = next.fetch_add(1)) < rows;) fn(r);
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < (threads ? threads : 1); t++) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
}

} // namespace

extern "C" int oracle_foveated_resolve(const oracle_fov_in* in, oracle_fov_out* out) {
    MxcsrScope mx;
    const uint32_t W = in->samples_per_ring, H = in->ring_count, w = in->width, h = in->height;
    if (!W || !H || !w || !h || !out->result || !out->image) return 1;
    const float radPerDeg = kPiF / 180.0f;
    EccMapping em;
    em.m = in->mar_slope;
    em.w0 = in->foveal_mar_degrees * radPerDeg;
    em.S = in->degree_tracking_error * radPerDeg;
    em.invLogA = float(1.0 / log(1.0 + double(em.m)));
    em.invW0 = float(1.0 / em.w0);
    em.invM = float(1.0 / em.m);
    em.texMapSize = float(H);
    em.invTexMapSize = 1.0f / float(H);
    em.invMaxEccentricity = 1.0f / (in->max_fov_degrees * radPerDeg);
    // RemapPolarFoveatedKernel
    std::vector<uint32_t> raw(size_t(W) * H, 0u);
    std::vector<float> depth(size_t(W) * H, 0.0f);
    for (uint32_t s = 0; s < in->valid; s++) {
        const size_t o = size_t(in->remap[2 * s + 1]) * W + in->remap[2 * s];
        raw[o] = toColor4Unorm8SRgb(fromColor4Unorm8SRgb(in->colors[s]));
        depth[o] = in->tmax[s];
    }
    const Tex rawTex{raw.data(), int(W), int(H), true, false, kSrgb8};
    const Tex depthTex{depth.data(), int(W), int(H), true, false, kR32f};
    // ComputeMoments
    std::vector<uint64_t> m1(size_t(W) * H), m2(size_t(W) * H);
    forRows(H, in->threads, [&](uint32_t j) {
        const float idx = 1.0f / float(W), idy = 1.0f / float(H);
        const float offsets[3] = {-1.0f, 0.0f, 1.0f};
        for (uint32_t i = 0; i < W; i++) {
            const float cx = idx * float(i), cy = idy * float(j);
            C4 a = c4(0, 0, 0, 0), b = c4(0, 0, 0, 0);
            for (int x = 0; x < 3; ++x)
                for (int y = 0; y < 3; ++y) {
                    const C4 c = tex2DLinear(rawTex, cx + (offsets[x] * idx), cy + (offsets[y] * idy));
                    a = a + c;
                    b = b + c * c;
                }
            const float weight = 1.0f / 9.0f;
            m1[size_t(j) * W + i] = toColor4Unorm16(a * weight);
            m2[size_t(j) * W + i] = toColor4Unorm16(b * weight);
        }
    });
    const Tex m1Tex{m1.data(), int(W), int(H), true, false, kUnorm16};
    const Tex m2Tex{m2.data(), int(W), int(H), true, false, kUnorm16};
    const Tex prevTex{in->history, int(w), int(h), false, false, kSrgb8};
    // FoveatedPolarToScreenSpaceKernel (RGBA8_SRGB): the result texture
    uint32_t* result = out->result;
    forRows(h, in->threads, [&](uint32_t j) {
        for (uint32_t i = 0; i < w; i++) {
            float theta, ecc;
            eyeCoord(in->sample_to_eye, i, j, w, h, theta, ecc);
            const float cx = (theta + kPiF) / (2.0f * kPiF);
            const float cy = (em.applyInverse(ecc) + 0.5f) * em.invTexMapSize;
            const C4 newValue = bicubicFast(rawTex, cx, cy);
            C4 surfaceResult = newValue;
            const float tValue = tex2DPoint(depthTex, cx, cy);
            if (tValue < INFINITY) {
                // angularEyeCoordToDirection(theta, eccentricity) * tValue
                const float z = -cosD(ecc);
                const float xyLength = sqrtf(1.0f - z * z);
                const float px = (cosD(-theta) * xyLength) * tValue, py = (sinD(-theta) * xyLength) * tValue;
                const float pz = z * tValue;
                const float* M = in->eye_to_sample_prev;
                const float qx = M[0] * px + M[4] * py + M[8] * pz + M[12] * 1.0f;
                const float qy = M[1] * px + M[5] * py + M[9] * pz + M[13] * 1.0f;
                const float qz = M[2] * px + M[6] * py + M[10] * pz + M[14] * 1.0f;
                const float ox = qx * (1.0f / qz), oy = qy * (1.0f / qz);
                float alpha = 0.05f;
                C4 oldValue = newValue;
                if (ox > 0 && oy > 0 && ox < 1 && oy < 1 && tValue > 0) oldValue = tex2DLinear(prevTex, ox, oy);
                // clampToNeighborhood (stddevMultiplier 1)
                const C4 a = tex2DLinear(m1Tex, cx, cy), b = tex2DLinear(m2Tex, cx, cy);
                const C4 var = b - (a * a);
                const C4 sd = c4(sqrtf(var.x), sqrtf(var.y), sqrtf(var.z), sqrtf(var.w));
                const float scaleFactor = 1.0f;
                C4 clampedOld = clampC(oldValue, a - (sd * scaleFactor), a + (sd * scaleFactor));
                float normalizedE = ecc * em.invMaxEccentricity;
                const float mn = 0.2f, mxv = 0.35f;
                const float t = clampF((normalizedE - mn) / (mxv - mn), 0.f, 1.f);
                alpha = 0.5f + (alpha - 0.5f) * t;
                normalizedE = sqrtf(sqrtf(sqrtf(sqrtf(normalizedE))));
                clampedOld.x = clampedOld.x + (oldValue.x - clampedOld.x) * normalizedE;
                clampedOld.y = clampedOld.y + (oldValue.y - clampedOld.y) * normalizedE;
                clampedOld.z = clampedOld.z + (oldValue.z - clampedOld.z) * normalizedE;
                clampedOld.w = clampedOld.w + (oldValue.w - clampedOld.w) * normalizedE;
                surfaceResult = newValue * alpha + clampedOld * (1.0f - alpha);
            }
            result[size_t(j) * w + i] = toColor4Unorm8SRgb(surfaceResult);
        }
    });
    // SeparableFilterUsingEccentricity: step {0, 1} into horizontallyFiltered, then {1, 0}
    auto separable = [&](const uint32_t* input, uint32_t* output, int sx, int sy) {
        const Tex inTex{input, int(w), int(h), false, false, kSrgb8};
        forRows(h, in->threads, [&](uint32_t j) {
            for (uint32_t i = 0; i < w; i++) {
                float theta, ecc;
                eyeCoord(in->sample_to_eye, i, j, w, h, theta, ecc);
                const int filterRadius = 5;
                C4 valueSum = c4(0.0f, 0.0f, 0.0f, 0.0f);
                float weightSum = 0.0f;
                for (int R = -filterRadius; R <= filterRadius; ++R) {
                    const int tx = std::min(std::max(int(i) + R * sx, 0), int(w) - 1);
                    const int ty = std::min(std::max(int(j) + R * sy, 0), int(h) - 1);
                    const float normDist = fabsf(float(R)) / float(filterRadius + 0.1);
                    const float weight = powD(1.0f - normDist, sqrtf(ecc));
                    // texelFetch: a linear fetch at the texel centre
                    valueSum = valueSum + tex2DLinear(inTex, (float(tx) + 0.5f) / float(w),
                                                      (float(ty) + 0.5f) / float(h)) * weight;
                    weightSum += weight;
                }
                output[size_t(j) * w + i] = toColor4Unorm8SRgb(valueSum * (1.0f / weightSum));
            }
        });
    };
    std::vector<uint32_t> hFiltered(size_t(w) * h), fFiltered(size_t(w) * h);
    separable(result, hFiltered.data(), 0, 1);
    separable(hFiltered.data(), fFiltered.data(), 1, 0);
    if (out->filtered) memcpy(out->filtered, hFiltered.data(), hFiltered.size() * 4);
    // FinishConstrastEnhancement (f_e = 1)
    const Tex unfTex{result, int(w), int(h), false, false, kSrgb8};
    const Tex filTex{fFiltered.data(), int(w), int(h), false, false, kSrgb8};
    forRows(h, in->threads, [&](uint32_t j) {
        for (uint32_t i = 0; i < w; i++) {
            float theta, ecc;
            eyeCoord(in->sample_to_eye, i, j, w, h, theta, ecc);
            float sigma = 8.0f;
            const float t = ecc * em.invMaxEccentricity;
            sigma *= dmax(0.001f, clampF(t * t, 0.f, 1.f));
            const float u = (float(i) + 0.5f) / float(w), v = (float(j) + 0.5f) / float(h);
            const C4 pix = tex2DLinear(unfTex, u, v), pmean = tex2DLinear(filTex, u, v);
            const float cScale = 1.f + sigma * 1.0f;
            const C4 scaled = pmean + (pix - pmean) * cScale;
            out->image[size_t(j) * w + i] = toColor4Unorm8SRgb(clampC(scaled, 0.0f, 1.0f));
        }
    });
    if (out->polar_color) memcpy(out->polar_color, raw.data(), raw.size() * 4);
    if (out->moments)
        for (size_t k = 0; k < m1.size(); k++) {
            memcpy(out->moments + 8 * k, &m1[k], 8);
            memcpy(out->moments + 8 * k + 4, &m2[k], 8);
        }
    return 0;
}

// ---------------------------------------------------------------- texture samplers
// Test samplers behind oracle_frame_in.texture_sample; see hvvr_oracle.h.
namespace {
typedef std::array<uint32_t, 7> TexKey; // id and the query's six float bit patterns
std::mutex gTexMutex;
std::map<TexKey, std::array<float, 4>> gTexTable;
bool gTexRecord = false;
std::atomic<uint32_t> gTexMissing{0};
TexKey texKey(uint32_t id, const float* q) {
    TexKey k;
    k[0] = id;
    memcpy(&k[1], q, 6 * sizeof(float));
    return k;
}
} // namespace

extern "C" {

void oracle_texture_hash(void*, uint32_t id, const float* q, float* rgba) {
    uint64_t h = 0x9E3779B97F4A7C15ull ^ id;
    for (int i = 0; i < 6; i++) {
        uint32_t b;
        memcpy(&b, &q[i], 4);
        h = (h ^ b) * 0x100000001B3ull;
        h ^= h >> 29;
    }
    for (int c = 0; c < 4; c++) {
        h = h * 6364136223846793005ull + 1442695040888963407ull;
        rgba[c] = float((h >> 40) & 0xffffffu) / 16777216.0f;
    }
}

void oracle_texture_table(void*, uint32_t id, const float* q, float* rgba) {
    const TexKey k = texKey(id, q);
    std::lock_guard<std::mutex> lock(gTexMutex);
    if (gTexRecord) {
        gTexTable.emplace(k, std::array<float, 4>{0.0f, 0.0f, 0.0f, 0.0f});
        for (int c = 0; c < 4; c++) rgba[c] = 0.0f;
        return;
    }
    auto it = gTexTable.find(k);
    if (it == gTexTable.end()) {
        gTexMissing++;
        for (int c = 0; c < 4; c++) rgba[c] = NAN;
        return;
    }
    for (int c = 0; c < 4; c++) rgba[c] = it->second[c];
}

void oracle_texture_table_reset(int record) {
    std::lock_guard<std::mutex> lock(gTexMutex);
    gTexTable.clear();
    gTexRecord = record != 0;
    gTexMissing = 0;
}

uint32_t oracle_texture_table_queries(uint32_t* ids, float* q, uint32_t capacity) {
    std::lock_guard<std::mutex> lock(gTexMutex);
    uint32_t n = 0;
    for (const auto& e : gTexTable) {
        if (n < capacity) {
            if (ids) ids[n] = e.first[0];
            if (q) memcpy(q + 6 * size_t(n), &e.first[1], 6 * sizeof(float));
        }
        n++;
    }
    return n;
}

void oracle_texture_table_set(uint32_t n, const uint32_t* ids, const float* q, const float* rgba) {
    std::lock_guard<std::mutex> lock(gTexMutex);
    gTexRecord = false;
    for (uint32_t i = 0; i < n; i++)
        gTexTable[texKey(ids[i], q + 6 * size_t(i))] = {rgba[4 * i], rgba[4 * i + 1], rgba[4 * i + 2], rgba[4 * i + 3]};
}

uint32_t oracle_texture_table_missing(void) { return gTexMissing.load(); }

} // extern "C"

// ------------------------------------------------------------------ device BVH build (restated)
// The linear BVH build of the library's bvh_device.cu, step for step on the CPU. It has no
// counterpart in the reference, whose GenerateTopology (libraries/hvvr/shared/bvh.cpp:542-556) is a
// host SAH build; the output uses the reference's TopologyNode layout (leaf slots before internal
// slots, so that leaf slot k spans [data[k], data[k+1])) and its depth-first node order.
namespace {

constexpr uint32_t kLbvhLeafTris = 4;

inline uint32_t spreadBits10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

inline uint32_t quantize10(float c, float lo, float scale) {
    float q = (c - lo) * scale;
    q = q > 0.0f ? q : 0.0f;
    q = q < 1023.0f ? q : 1023.0f;
    return uint32_t(q);
}

struct LbvhTree {
    std::vector<uint32_t> keys;              // sorted Morton codes
    std::vector<uint32_t> order;             // sorted position -> triangle
    std::vector<uint32_t> left, right;       // internal node children (bit 31: a sorted position, i.e. a single triangle)
    std::vector<uint32_t> first, last;       // internal node ranges
};

inline int lbvhDelta(const LbvhTree& t, int i, int j) {
    const int n = int(t.keys.size());
    if (j < 0 || j >= n) return -1;
    const uint32_t a = t.keys[size_t(i)], b = t.keys[size_t(j)];
    if (a == b) return 32 + __builtin_clz(uint32_t(i) ^ uint32_t(j));
    return __builtin_clz(a ^ b);
}

// the binary radix tree of the sorted keys (one internal node per i in [0, n-2])
void lbvhRadixTree(LbvhTree& t) {
    const int n = int(t.keys.size());
    t.left.assign(size_t(n > 1 ? n - 1 : 0), 0u);
    t.right = t.left;
    t.first = t.left;
    t.last = t.left;
    for (int i = 0; i + 1 < n; i++) {
        const int d = lbvhDelta(t, i, i + 1) - lbvhDelta(t, i, i - 1) > 0 ? 1 : -1;
        const int dmin = lbvhDelta(t, i, i - d);
        int lmax = 2;
        while (lbvhDelta(t, i, i + lmax * d) > dmin) lmax *= 2;
        int l = 0;
        for (int s = lmax / 2; s >= 1; s /= 2)
            if (lbvhDelta(t, i, i + (l + s) * d) > dmin) l += s;
        const int j = i + l * d;
        const int dnode = lbvhDelta(t, i, j);
        int s = 0;
        for (int div = 2;; div *= 2) {
            const int step = (l + div - 1) / div;
            if (lbvhDelta(t, i, i + (s + step) * d) > dnode) s += step;
            if (step <= 1) break;
        }
        const int gamma = i + s * d + (d < 0 ? -1 : 0);
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        t.left[size_t(i)] = lo == gamma ? (0x80000000u | uint32_t(gamma)) : uint32_t(gamma);
        t.right[size_t(i)] = hi == gamma + 1 ? (0x80000000u | uint32_t(gamma + 1)) : uint32_t(gamma + 1);
        t.first[size_t(i)] = uint32_t(lo);
        t.last[size_t(i)] = uint32_t(hi);
    }
}

struct LbvhEntry {
    uint32_t node;      // internal node id, or bit 31 + sorted position for a single triangle
    uint32_t lo, hi;    // sorted range [lo, hi]
    uint32_t count() const { return hi - lo + 1; }
    bool internal() const { return count() > kLbvhLeafTris; }
};

LbvhEntry lbvhEntry(const LbvhTree& t, uint32_t c) {
    if (c & 0x80000000u) return LbvhEntry{c, c & 0x7fffffffu, c & 0x7fffffffu};
    return LbvhEntry{c, t.first[c], t.last[c]};
}

// the 4-wide node of internal node x: its two children, the child with the most triangles
// expanded until there are four or none can be, then leaf slots before internal slots
int lbvhCollapse(const LbvhTree& t, uint32_t x, LbvhEntry* out) {
    LbvhEntry e[4];
    int n = 2;
    e[0] = lbvhEntry(t, t.left[x]);
    e[1] = lbvhEntry(t, t.right[x]);
    while (n < 4) {
        int best = -1;
        for (int k = 0; k < n; k++)
            if (e[k].internal() && (best < 0 || e[k].count() > e[best].count())) best = k;
        if (best < 0) break;
        const uint32_t id = e[best].node;
        for (int k = n; k > best + 1; k--) e[k] = e[k - 1];
        e[best] = lbvhEntry(t, t.left[id]);
        e[best + 1] = lbvhEntry(t, t.right[id]);
        n++;
    }
    int m = 0;
    for (int k = 0; k < n; k++)
        if (!e[k].internal()) out[m++] = e[k];
    const int leaves = m;
    for (int k = 0; k < n; k++)
        if (e[k].internal()) out[m++] = e[k];
    (void)leaves;
    return n;
}

struct LbvhWriter {
    const LbvhTree& t;
    const hvvr_tri_shade* tris;
    hvvr_tri_shade* trisOut;
    hvvr_topology_node* nodes;
    uint32_t capacity, nodeCount = 0, triCount = 0;
    bool overflow = false;

    // writes the node of entry list e[0, n) (n <= 4) at the next index; returns its index
    uint32_t emit(const LbvhEntry* e, int n) {
        const uint32_t index = nodeCount++;
        if (index >= capacity) {
            overflow = true;
            return index;
        }
        hvvr_topology_node out{};
        out.leaf_mask = 0;
        out.data[0] = triCount;
        uint32_t children[4];
        int internalCount = 0;
        for (int k = 0; k < 4; k++) {
            if (k >= n) { // empty leaf slot
                out.leaf_mask |= 1u << k;
                out.data[1 + k] = triCount;
                continue;
            }
            if (e[k].internal()) {
                children[internalCount++] = uint32_t(k);
                continue;
            }
            out.leaf_mask |= 1u << k;
            for (uint32_t p = e[k].lo; p <= e[k].hi; p++) trisOut[triCount++] = tris[t.order[p]];
            out.data[1 + k] = triCount;
        }
        nodes[index] = out;
        for (int c = 0; c < internalCount; c++) {
            const int k = int(children[c]);
            LbvhEntry sub[4];
            const int m = lbvhCollapse(t, e[k].node, sub);
            const uint32_t child = emit(sub, m);
            if (!overflow) nodes[index].data[1 + k] = child - index;
        }
        return index;
    }
};

} // namespace

extern "C" int oracle_lbvh_build(const hvvr_shading_vertex* verts, uint32_t vert_count, const hvvr_tri_shade* tris,
                                 uint32_t tri_count, hvvr_tri_shade* tris_out, hvvr_topology_node* nodes_out,
                                 uint32_t capacity, uint32_t* node_count) {
    if (!verts || !tris || !tris_out || !nodes_out || !node_count || tri_count == 0) return 1;
    for (uint32_t i = 0; i < tri_count; i++)
        for (int k = 0; k < 3; k++)
            if (tris[i].indices[k] >= vert_count) return 1;
    // centroids (IEEE single, no contraction) and their bounds
    std::vector<float> cen(size_t(tri_count) * 3);
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = 0; i < tri_count; i++) {
        const hvvr_vec3& a = verts[tris[i].indices[0]].pos;
        const hvvr_vec3& b = verts[tris[i].indices[1]].pos;
        const hvvr_vec3& c = verts[tris[i].indices[2]].pos;
        const float v[3] = {((a.x + b.x) + c.x) * (1.0f / 3.0f), ((a.y + b.y) + c.y) * (1.0f / 3.0f),
                            ((a.z + b.z) + c.z) * (1.0f / 3.0f)};
        for (int k = 0; k < 3; k++) {
            cen[size_t(i) * 3 + k] = v[k];
            lo[k] = v[k] < lo[k] ? v[k] : lo[k];
            hi[k] = v[k] > hi[k] ? v[k] : hi[k];
        }
    }
    float scale[3];
    for (int k = 0; k < 3; k++) {
        const float ext = hi[k] - lo[k];
        scale[k] = ext > 0.0f ? 1024.0f / ext : 0.0f;
    }
    LbvhTree t;
    std::vector<uint32_t> codes(tri_count);
    for (uint32_t i = 0; i < tri_count; i++) {
        const float* c = &cen[size_t(i) * 3];
        codes[i] = (spreadBits10(quantize10(c[0], lo[0], scale[0])) << 2) |
                   (spreadBits10(quantize10(c[1], lo[1], scale[1])) << 1) |
                   spreadBits10(quantize10(c[2], lo[2], scale[2]));
    }
    t.order.resize(tri_count);
    for (uint32_t i = 0; i < tri_count; i++) t.order[i] = i;
    std::stable_sort(t.order.begin(), t.order.end(), [&](uint32_t a, uint32_t b) { return codes[a] < codes[b]; });
    t.keys.resize(tri_count);
    for (uint32_t i = 0; i < tri_count; i++) t.keys[i] = codes[t.order[i]];
    lbvhRadixTree(t);
    LbvhWriter w{t, tris, tris_out, nodes_out, capacity};
    LbvhEntry root[4];
    int n;
    if (tri_count <= kLbvhLeafTris) {
        root[0] = LbvhEntry{0x80000000u, 0, tri_count - 1};
        n = 1;
    } else {
        n = lbvhCollapse(t, 0, root);
    }
    w.emit(root, n);
    *node_count = w.nodeCount;
    return w.overflow ? 2 : 0;
}
