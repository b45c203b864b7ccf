// ref_harness.cpp - TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own sources (compiled unmodified from the reference tree by
// oracle/refshim/ref.mk) through the same C API as the oracle, so tests can pin the
// oracle restatement against the reference's code:
//   * SampleData (RC/camera.cpp:21-64) for sorting, 2D->3D frusta and beams;
//   * frustumTransform (RC/traversal.h:38-47) and traverse::avx::Frustum (RC/traverse_avx.cpp);
//   * traverseBlocks / BlockFrame::sort / traverseTiles (RC/traverse_avx.h) driven exactly
//     like cullThread (RC/traversal.cpp:99-190);
//   * the kernels' per-thread math compiled for the host: FrustumPlanes,
//     IntersectTriangleTile<false>, TestTriangleFrustaUVW, IntersectTriangleThread
//     (RC/prim_tests.h), getSubsampleUnitOffset (RC/gpu_samples.h), sortBitonic (RC/sort.h),
//     interpolate / GGXShade / ACESFilm / ToColor4Unorm8SRgb (RC/shading*.h);
//   * GenerateTopology (SH/bvh.cpp).
// The kernel control structure (128-triangle chunks, order-preserving compaction, the
// G-buffer grouping and the MSAA resolve loop of RC/intersect.cu and RC/resolve.cu) and the
// GPU refit kernels cannot run on a CPU as written; they are restated here around the
// reference functions, with -ffp-contract=off (the HVVR_FP_STRICT arithmetic).

#define TRAVERSAL_IMP 1
#include "traversal.h"

#include "bvh.h"
#include "bvh_node.h"
#include "camera.h"
#include "gpu_samples.h"
#include "graphics_types.h"
#include "light.h"
#include "lighting_env.h"
#include "material.h"
#include "model.h"
#include "prim_tests.h"
#include "shading.h"
#include "sort.h"
#include "tile_data.h"
#include "foveated.h"
#include "gpu_buffer.h"

#include "../hvvr_oracle.h"

#include <atomic>
#include <memory>
#include <functional>
#include <random>
#include <thread>

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
hv_texture_hook_fn hv_texture_hook = nullptr;
void* hv_texture_hook_ctx = nullptr;

namespace hvvr {
// Link stubs for GPU-side classes referenced by camera.cpp's Camera methods. The harness
// only constructs SampleData, so none of these run.
class GPUCamera;
class GPUContext;
} // namespace hvvr

using namespace hvvr;

namespace {

struct MxcsrScope {
    unsigned saved;
    MxcsrScope() { saved = _mm_getcsr(); _mm_setcsr(saved | 0x8040); }
    ~MxcsrScope() { _mm_setcsr(saved); }
};

inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
inline float bitsf(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

template <uint32_t N> vector2 subOffset(int i) { return getSubsampleUnitOffset<N>(vector2(0.0f, 0.0f), i); }
template <uint32_t N> vector2 lensOffset(int i, float rot) { return getSubsampleUnitOffset<N>(vector2(0.0f, 0.0f), i, rot); }
vector2 lensOffsetN(uint32_t n, int i, float rot) {
    switch (n) {
    case 1: return lensOffset<1>(i, rot);
    case 2: return lensOffset<2>(i, rot);
    case 4: return lensOffset<4>(i, rot);
    case 8: return lensOffset<8>(i, rot);
    case 16: return lensOffset<16>(i, rot);
    default: return lensOffset<32>(i, rot);
    }
}
// GetSampleUVsDoF for a run-time rate (it reads blockIdx.x and threadIdx.x like the kernels)
void sampleUVsDoF(uint32_t n, const vector2* tab, vector2 fls, int i, vector2& lensUV, vector2& dirUV) {
    switch (n) {
    case 1: GetSampleUVsDoF<1, TILE_SIZE>(tab, vector2(0.0f, 0.0f), fls, i, lensUV, dirUV); break;
    case 2: GetSampleUVsDoF<2, TILE_SIZE>(tab, vector2(0.0f, 0.0f), fls, i, lensUV, dirUV); break;
    case 4: GetSampleUVsDoF<4, TILE_SIZE>(tab, vector2(0.0f, 0.0f), fls, i, lensUV, dirUV); break;
    case 8: GetSampleUVsDoF<8, TILE_SIZE>(tab, vector2(0.0f, 0.0f), fls, i, lensUV, dirUV); break;
    case 16: GetSampleUVsDoF<16, TILE_SIZE>(tab, vector2(0.0f, 0.0f), fls, i, lensUV, dirUV); break;
    default: GetSampleUVsDoF<32, TILE_SIZE>(tab, vector2(0.0f, 0.0f), fls, i, lensUV, dirUV); break;
    }
}
vector2 subsampleOffset(uint32_t n, int i) {
    switch (n) {
    case 1: return subOffset<1>(i);
    case 2: return subOffset<2>(i);
    case 4: return subOffset<4>(i);
    case 8: return subOffset<8>(i);
    case 16: return subOffset<16>(i);
    default: return subOffset<32>(i);
    }
}

} // namespace

extern "C" int ref_generate_topology(hvvr_shading_vertex* verts, uint32_t vert_count, hvvr_tri_shade* tri_shade,
                                     uint32_t tri_count, hvvr_topology_node* nodes_out, uint32_t capacity,
                                     uint32_t* node_count) {
    MeshData mesh;
    mesh.verts.assign((ShadingVertex*)verts, (ShadingVertex*)verts + vert_count);
    mesh.triShade.assign((PrecomputedTriangleShade*)tri_shade, (PrecomputedTriangleShade*)tri_shade + tri_count);
    if (!GenerateTopology(mesh)) return 1;
    if (mesh.nodes.size() > capacity) return 2;
    memcpy(verts, mesh.verts.data(), vert_count * sizeof(ShadingVertex));
    memcpy(tri_shade, mesh.triShade.data(), tri_count * sizeof(PrecomputedTriangleShade));
    memcpy(nodes_out, mesh.nodes.data(), mesh.nodes.size() * sizeof(TopologyNode));
    *node_count = uint32_t(mesh.nodes.size());
    return 0;
}

namespace {

// What the reference keeps from one frame to the next: the uploaded and refit scene
// (Raycaster::buildScene / GPUSceneState, RC/scene_update.cpp:22-143, RC/gpu_scene_state.cu), its
// lighting environment, and a camera's SampleData (Camera::setSamples, RC/camera.cpp:104-164).
struct RefSession {
    uint32_t N = 1, width = 0, height = 0, split = 1;
    ThinLens lens{0.0f, 1.0f};
    DynamicArray<BVHNode> nodes;
    std::vector<ShadingVertex> world;
    std::vector<PrecomputedTriangleIntersect> tris;
    std::vector<PrecomputedTriangleShade> triShade;
    std::vector<SimpleMaterial> materials;
    LightingEnvironment env;
    std::unique_ptr<SampleData> sd;
    uint32_t textureCount = 0;
    hv_texture_hook_fn textureSample = nullptr;
    void* textureCtx = nullptr;
};

// scene upload and refit, lighting environment and sample set of one camera
int refSetup(const oracle_frame_in* in, oracle_frame_out* out, RefSession& S) {
    if (in->model_count != 1 || in->sample_count == 0) return 1; // harness covers single-model scenes
    const hvvr_mesh_data& md = in->models[0];
    S.N = in->msaa;
    S.width = in->width;
    S.height = in->height;
    S.split = in->split_color_samples;
    S.lens = ThinLens{in->lens.radius, in->lens.focal_distance};
    S.textureCount = in->texture_count;
    S.textureSample = in->texture_sample;
    S.textureCtx = in->texture_ctx;
    S.materials.assign((const SimpleMaterial*)md.materials, (const SimpleMaterial*)md.materials + md.material_count);

    // scene build for one model (RC/scene_update.cpp:86-101 with offsets 0, no root fix-up)
    S.nodes = DynamicArray<BVHNode>(md.node_count);
    DynamicArray<BVHNode>& nodes = S.nodes;
    memset(nodes.data(), 0, md.node_count * sizeof(BVHNode));
    for (uint32_t n = 0; n < md.node_count; n++) {
        const TopologyNode& tn = ((const TopologyNode*)md.nodes)[n];
        BVHNode& node = nodes[n];
        node.boxData.leafMask = tn.leafMask;
        node.boxData.leaf.triIndex[0] = tn.getFirstTriangleIndex(0);
        for (size_t k = 0; k < 4; k++) {
            if (tn.isLeaf(k)) node.boxData.leaf.triIndex[1 + k] = tn.getBoundTriangleIndex(k);
            else node.boxData.children.offset[k] = tn.getChildOffset(k);
        }
    }
    // refit (restatement of RC/gpu_scene_state.cu:88-375 with the reference's types and operators)
    matrix4x4 modelToWorld = matrix4x4(*(const transform*)&in->model_xf[0]);
    S.world.resize(md.vert_count);
    std::vector<ShadingVertex>& world = S.world;
    for (uint32_t i = 0; i < md.vert_count; i++) {
        ShadingVertex vertex = ((const ShadingVertex*)md.verts)[i];
        vector4 fp = modelToWorld * vector4(vertex.pos, 1.0);
        vertex.pos = vector3(fp) * (1.0f / fp.w);
        vertex.normal = vector4h(normalize(matrix3x3(modelToWorld) * vector3(vertex.normal)));
        world[i] = vertex;
    }
    S.triShade.assign((const PrecomputedTriangleShade*)md.tri_shade, (const PrecomputedTriangleShade*)md.tri_shade + md.tri_count);
    const PrecomputedTriangleShade* triShade = S.triShade.data();
    std::vector<uint32_t> triToNodeChild(md.tri_count, 0);
    for (int64_t n = int64_t(md.node_count) - 1; n >= 0; --n) {
        for (int k = 3; k >= 0; k--) {
            if (_bittest((const long*)&nodes[n].boxData.leafMask, k)) {
                for (uint32_t t = nodes[n].boxData.leaf.triIndex[k]; t < nodes[n].boxData.leaf.triIndex[k + 1]; t++)
                    triToNodeChild[t] = (uint32_t(n) << 2) | uint32_t(k);
            }
        }
    }
    std::vector<uint32_t> flip(size_t(md.node_count) * 24, FloatFlip(0xff800000));
    S.tris.resize(md.tri_count);
    std::vector<PrecomputedTriangleIntersect>& tris = S.tris;
    for (uint32_t i = 0; i < md.tri_count; i++) {
        vector3 v0 = world[triShade[i].indices[0]].pos, v1 = world[triShade[i].indices[1]].pos,
                v2 = world[triShade[i].indices[2]].pos;
        tris[i].v0 = v0; tris[i].edge0 = v1 - v0; tris[i].edge1 = v2 - v0;
        float mx3[3] = {max(v0.x, max(v1.x, v2.x)), max(v0.y, max(v1.y, v2.y)), max(v0.z, max(v1.z, v2.z))};
        float nm3[3] = {max(-v0.x, max(-v1.x, -v2.x)), max(-v0.y, max(-v1.y, -v2.y)), max(-v0.z, max(-v1.z, -v2.z))};
        uint32_t parent = triToNodeChild[i] >> 2, slot = triToNodeChild[i] & 3;
        for (int a = 0; a < 3; a++) {
            uint32_t& m = flip[size_t(parent) * 24 + 8 * a + slot];
            uint32_t& g = flip[size_t(parent) * 24 + 8 * a + 4 + slot];
            m = std::max(m, FloatFlipF(mx3[a]));
            g = std::max(g, FloatFlipF(nm3[a]));
        }
    }
    for (uint32_t n = 0; n < md.node_count; n++) {
        float* b = nodes[n].xMax;
        for (int j = 0; j < 24; j++) b[j] = IFloatFlipF(flip[size_t(n) * 24 + j]);
    }
    std::vector<uint32_t> depthOf(md.node_count, 0);
    uint32_t maxDepth = 0;
    for (uint32_t n = 0; n < md.node_count; n++)
        for (int k = 3; k >= 0; k--)
            if (!_bittest((const long*)&nodes[n].boxData.leafMask, k)) {
                uint32_t c = n + nodes[n].boxData.children.offset[k];
                depthOf[c] = depthOf[n] + 1;
                maxDepth = std::max(maxDepth, depthOf[c]);
            }
    for (int64_t d = maxDepth; d >= 0; d--)
        for (uint32_t n = 0; n < md.node_count; n++) {
            if (depthOf[n] != d) continue;
            for (int k = 0; k < 4; k++) {
                if (_bittest((const long*)&nodes[n].boxData.leafMask, k)) continue;
                const float* bp = nodes[n + nodes[n].boxData.children.offset[k]].xMax;
                float* pb = nodes[n].xMax;
                for (int j = 0; j < 6; j++)
                    pb[j * 4 + k] = max(bp[j * 4 + 0], max(bp[j * 4 + 1], max(bp[j * 4 + 2], bp[j * 4 + 3])));
            }
        }
    if (out->nodes) memcpy(out->nodes, nodes.data(), md.node_count * sizeof(BVHNode));
    if (out->tris) memcpy(out->tris, tris.data(), md.tri_count * sizeof(PrecomputedTriangleIntersect));

    // lighting environment (GPUSceneState::updateLighting, RC/gpu_scene_state.cu:47-81)
    LightingEnvironment& env = S.env;
    memset(&env, 0, sizeof(env));
    for (uint32_t i = 0; i < in->light_count; i++) {
        const LightUnion& l = ((const LightUnion*)in->lights)[i];
        if (l.type == LightType::directional && env.directionalLightCount < int(MAX_DIRECTIONAL_LIGHTS))
            env.directionalLights[env.directionalLightCount++] = l.directional;
        else if (l.type == LightType::point && env.pointLightCount < int(MAX_POINT_LIGHTS))
            env.pointLights[env.pointLightCount++] = l.point;
        else if (l.type == LightType::spot && env.spotLightCount < int(MAX_SPOT_LIGHTS))
            env.spotLights[env.spotLightCount++] = l.spot;
    }
    // samples: the reference's SampleData with Camera::getSampleToCamera (RC/camera.cpp:167-171)
    const FloatRect vp(vector2(in->viewport.lower.x, in->viewport.lower.y), vector2(in->viewport.upper.x, in->viewport.upper.y));
    matrix3x3 sampleToCamera(vector3(vp.upper.x - vp.lower.x, 0, 0), vector3(0, vp.lower.y - vp.upper.y, 0),
                             vector3(vp.lower.x, vp.upper.y, -1));
    S.sd.reset(new SampleData((const Sample*)in->samples, in->sample_count, in->split_color_samples,
                              Sample2Dto3DMappingSettings(sampleToCamera, S.lens), in->width, in->height));
    const SampleData& sd = *S.sd;
    const uint32_t padded = uint32_t(sd.samples.directionalBeams.size());
    if (out->remap) memcpy(out->remap, sd.imageLocationToSampleIndex.data(), sd.imageLocationToSampleIndex.size() * 4);
    if (out->beams) memcpy(out->beams, sd.samples.directionalBeams.data(), size_t(padded) * sizeof(DirectionalBeam));
    return 0;
}

// one frame of a camera: world-space frusta, traversal, intersect, G-buffer, shading, remap
int refFrame(RefSession& S, const hvvr_transform& camXf, uint32_t threads, oracle_frame_out* out) {
    out->status = 0;
    const SampleData& sd = *S.sd;
    const BeamBatch& batch = sd.samples;
    const uint32_t N = S.N;
    const uint32_t nt = threads ? threads : 1;
    const LightingEnvironment& env = S.env;
    uint32_t blockCount = uint32_t(batch.blockFrusta3D.size());
    uint32_t tileCount = uint32_t(batch.tileFrusta3D.size());
    uint32_t padded = uint32_t(batch.directionalBeams.size());

    // per-frame transform (transformHierarchyCameraToWorld without cull planes, RC/render.cpp:293-310)
    matrix4x4 cameraToWorld = matrix4x4(*(const transform*)&camXf);
    DynamicArray<Frustum> blocksW(blockCount), tilesW(tileCount);
    std::vector<SimpleRayFrustum> simple(tileCount);
    for (uint32_t b = 0; b < blockCount; b++) blocksW[b] = frustumTransform(batch.blockFrusta3D[b], cameraToWorld);
    for (uint32_t t = 0; t < tileCount; t++) {
        tilesW[t] = frustumTransform(batch.tileFrusta3D[t], cameraToWorld);
        for (int n = 0; n < Frustum::pointCount; n++) {
            simple[t].origins[n] = tilesW[t].pointOrigin[n];
            simple[t].directions[n] = tilesW[t].pointDir[n];
        }
    }
    static_assert(sizeof(SimpleRayFrustum) == 96, "SimpleRayFrustum");
    if (out->tile_frusta) memcpy(out->tile_frusta, simple.data(), size_t(tileCount) * sizeof(SimpleRayFrustum));

    // cullThread (RC/traversal.cpp:99-190): the blocks are traversed on `threads` threads, each
    // taking the next block (a tile's list depends only on its block, so the lists are the same
    // for any assignment of blocks to threads)
    std::vector<std::vector<uint32_t>> lists(tileCount);
    std::atomic<uint32_t> nextBlock(0);
    auto cullWorker = [&]() {
        MxcsrScope mxc;
        std::vector<uint32_t> scratch(1 << 20);
        for (;;) {
            const uint32_t b = nextBlock.fetch_add(1);
            if (b >= blockCount) break;
            BlockFrame blockFrame;
            uint32_t stackSize = traverseBlocks(blockFrame, S.nodes.data(), blocksW[b]);
            if (out->block_sizes) out->block_sizes[b] = stackSize;
            if (!stackSize) {
                if (out->block_entries) memset(out->block_entries + size_t(b) * 64 * 3, 0, 64 * 3 * 4);
                continue;
            }
            blockFrame.sort(stackSize);
            if (out->block_entries) {
                for (uint32_t i = 0; i < 64; i++) {
                    uint32_t* dst = out->block_entries + (size_t(b) * 64 + i) * 3;
                    if (i < stackSize) {
                        dst[0] = fbits(blockFrame.sortedStack[i].tMin);
                        dst[1] = blockFrame.sortedStack[i].mask;
                        dst[2] = uint32_t(blockFrame.sortedStack[i].node - S.nodes.data());
                    } else {
                        dst[0] = dst[1] = dst[2] = 0;
                    }
                }
            }
            for (uint32_t ti = 0; ti < TILES_PER_BLOCK; ti++) {
                uint32_t tile = b * TILES_PER_BLOCK + ti;
                TileFrame tileFrame;
                for (uint32_t slot = 0; slot != stackSize; ++slot)
                    store(&(tileFrame.stack + slot)->tMin, load_m128(&(blockFrame.sortedStack + slot)->tMin));
                uint32_t count = traverseTiles(scratch.data(), uint32_t(scratch.size()), tileFrame, stackSize, tilesW[tile]);
                lists[tile].assign(scratch.begin(), scratch.begin() + count);
            }
        }
    };
    {
        std::vector<std::thread> cullPool;
        for (uint32_t t = 1; t < nt; t++) cullPool.emplace_back(cullWorker);
        cullWorker();
        for (auto& th : cullPool) th.join();
    }

    const SimpleMaterial* materials = S.materials.data();
    // material textures: the texture object of id i is i, and ReadTexture's tex2DGrad goes to the
    // frame's texture sampler
    hv_texture_hook = S.textureCount ? S.textureSample : nullptr;
    hv_texture_hook_ctx = S.textureCtx;
    std::vector<cudaTextureObject_t> textureObjects(SimpleMaterial::maxTextureCount);
    for (uint32_t i = 0; i < SimpleMaterial::maxTextureCount; i++) textureObjects[i] = cudaTextureObject_t(i);
    vector3 cameraPos = vector3(cameraToWorld.m3);
    std::vector<vector2> alphaTab(N);
    for (uint32_t i = 0; i < N; i++) alphaTab[i] = subsampleOffset(N, int(i));
    uint32_t maskAll = N < 32 ? ((1u << N) - 1) : ~0u;
    std::vector<uint32_t> colors(padded, 0xFF000000u);

    // depth of field: the lens table of GPUCamera::initLookupTables (RC/gpu_camera.cu:59-88) and the
    // occupied-tile index the intersect/resolve kernels run under (tileIndexRemapOccupied)
    const bool dof = S.lens.radius > 0.0f;
    std::vector<vector2> lensTab;
    std::vector<uint32_t> occRank(tileCount, 0);
    alignas(CameraBeams) unsigned char cbStorage[sizeof(CameraBeams)];
    memset(cbStorage, 0, sizeof(cbStorage));
    CameraBeams& cameraBeams = *reinterpret_cast<CameraBeams*>(cbStorage); // TileData<true>::load reads .lens only
    cameraBeams.lens = S.lens;
    if (dof) {
        std::uniform_real_distribution<float> uniformRandomDist(0.0f, 1.0f);
        std::mt19937 generator;
        auto r = std::bind(uniformRandomDist, std::ref(generator));
        lensTab.resize(size_t(TILE_SIZE) * DOF_LENS_POS_LOOKUP_TABLE_TILES * N);
        for (int tile = 0; tile < DOF_LENS_POS_LOOKUP_TABLE_TILES; tile++)
            for (int sample = 0; sample < int(TILE_SIZE); sample++) {
                float rotation = r() * Tau;
                for (int subsample = 0; subsample < int(N); subsample++)
                    lensTab[tile * TILE_SIZE * N + subsample * TILE_SIZE + sample] =
                        lensOffsetN(N, (subsample * 7 + 7) % int(N), rotation);
            }
        uint32_t rank = 0;
        for (uint32_t t = 0; t < tileCount; t++) {
            occRank[t] = rank;
            if (!lists[t].empty()) rank++;
        }
    }

    std::atomic<uint32_t> next(0);
    auto worker = [&]() {
        MxcsrScope mxw;
        for (;;) {
            uint32_t tile = next.fetch_add(1);
            if (tile >= tileCount) break;
            const std::vector<uint32_t>& list = lists[tile];
            uint32_t base = tile * TILE_SIZE;
            blockIdx.x = occRank[tile];
            if (list.empty()) {
                for (uint32_t s = 0; s < TILE_SIZE; s++) {
                    for (uint32_t i = 0; i < N; i++) {
                        size_t o = size_t(base + s) * N + i;
                        if (out->hit_ids) out->hit_ids[o] = ~0u;
                        if (out->depth) out->depth[o] = INFINITY;
                        if (out->gb_tri) out->gb_tri[o] = i == 0 ? ~0u : 0u;
                        if (out->gb_mask) out->gb_mask[o] = i == 0 ? maskAll : 0u;
                    }
                    if (out->gb_n) out->gb_n[base + s] = 1;
                }
                continue;
            }
            // IntersectKernel / IntersectTile (RC/intersect.cu:171-342)
            FrustumPlanes planes(simple[tile]);
            std::vector<uint32_t> survIdx;
            std::vector<IntersectTriangleTile<false>> survTile;
            std::vector<IntersectTriangleTile<true>> survTileDoF;
            // TileData<true>::load by thread BlockSize/2 on its world-space beam (RC/intersect.cu:182-186)
            TileData<true> tileDoF;
            if (dof) tileDoF.load(cameraBeams, cameraToWorld,
                                  matrix3x3(cameraToWorld) * batch.directionalBeams[base + TILE_SIZE / 2]);
            for (uint32_t idx : list) {
                const PrecomputedTriangleIntersect& tri = S.tris[idx];
                if (!planes.test(tri)) continue;
                if (dof) {
                    IntersectTriangleTile<true> tt;
                    IntersectResult r0 = tt.setup(tri, cameraPos, tileDoF.lensU, tileDoF.lensV);
                    if (r0 == intersect_all_out) continue;
                    if (r0 != intersect_partial && TestTriangleFrustaUVW(simple[tile], tri) == intersect_all_out) continue;
                    survIdx.push_back(idx);
                    survTileDoF.push_back(tt);
                    continue;
                }
                IntersectTriangleTile<false> tt;
                if (tt.setup(tri, cameraPos) == intersect_all_out) continue;
                if (TestTriangleFrustaUVW(simple[tile], tri) == intersect_all_out) continue;
                survIdx.push_back(idx);
                survTile.push_back(tt);
            }
            for (uint32_t s = 0; s < TILE_SIZE; s++) {
                uint32_t sid = base + s;
                DirectionalBeam sample = matrix3x3(cameraToWorld) * batch.directionalBeams[sid];
                threadIdx.x = s;
                // IntersectSamples (RC/intersect.cu:117-168)
                vector3 centerDir = normalize(sample.centerRay);
                float zed = dot(matrix3x3(cameraToWorld) * vector3(0, 0, -1.0f), centerDir);
                vector3 lensCenterToFocalCenter = (S.lens.focalDistance / zed) * centerDir;
                float tmaxv[32];
                uint32_t hit[32];
                for (uint32_t i = 0; i < N; i++) { tmaxv[i] = FLT_MAX; hit[i] = ~0u; }
                for (size_t j = 0; j < survIdx.size(); j++) {
                    if (dof) {
                        IntersectTriangleThreadDoF th(survTileDoF[j], lensCenterToFocalCenter);
                        for (uint32_t i = 0; i < N; i++) {
                            vector2 lensUV, dirUV;
                            sampleUVsDoF(N, lensTab.data(), tileDoF.focalToLensScale, int(i), lensUV, dirUV);
                            if (th.test(survTileDoF[j], lensCenterToFocalCenter, tileDoF.lensU, tileDoF.lensV, lensUV,
                                        dirUV, tmaxv[i]))
                                hit[i] = survIdx[j];
                        }
                        continue;
                    }
                    IntersectTriangleThread th(survTile[j], sample.centerRay, sample.du, sample.dv);
                    for (uint32_t i = 0; i < N; i++)
                        if (th.test(survTile[j], alphaTab[i], tmaxv[i])) hit[i] = survIdx[j];
                }
                for (uint32_t i = 0; i < N; i++) {
                    size_t o = size_t(sid) * N + i;
                    if (out->hit_ids) out->hit_ids[o] = hit[i];
                    if (out->depth) out->depth[o] = hit[i] == ~0u ? INFINITY : tmaxv[i];
                }
                // EmitGBuffer grouping (RC/intersect.cu:51-87) with the reference's sortBitonic
                uint32_t keys[32];
                for (uint32_t i = 0; i < N; i++) keys[i] = (hit[i] << 5) | i;
                sortBitonic(keys, int(N));
                uint32_t gtri[32], gmask[32], gn = 0;
                gtri[0] = uint32_t(int32_t(keys[0]) >> 5);
                gmask[0] = 1u << (keys[0] & 31);
                gn = 1;
                for (uint32_t i = 1; i < N; i++) {
                    uint32_t t = uint32_t(int32_t(keys[i]) >> 5), m = 1u << (keys[i] & 31);
                    if (gtri[gn - 1] == t) gmask[gn - 1] |= m;
                    else { gtri[gn] = t; gmask[gn] = m; gn++; }
                }
                if (out->gb_n) out->gb_n[sid] = gn;
                for (uint32_t i = 0; i < N; i++) {
                    if (out->gb_tri) out->gb_tri[size_t(sid) * N + i] = i < gn ? gtri[i] : 0;
                    if (out->gb_mask) out->gb_mask[size_t(sid) * N + i] = i < gn ? gmask[i] : 0;
                }
                // ShadeMSAA, non-DoF branch (RC/resolve.cu:161-284)
                vector4 result(0.0f, 0.0f, 0.0f, 0.0f);
                uint32_t combined = 0;
                for (uint32_t g = 0; g < gn; g++) {
                    if (combined == maskAll) break;
                    uint32_t triIndex = gtri[g];
                    if (triIndex == ~0u) break;
                    uint32_t sampleMask = gmask[g];
                    combined |= sampleMask;
                    float sampleCountInv = 1.0f / __builtin_popcount(sampleMask);
                    vector2 centroidAlpha(0.0f, 0.0f);
                    vector2 centroidLensUV(0.0f, 0.0f), centroidDirUV(0.0f, 0.0f);
                    for (uint32_t cm = sampleMask; cm != 0;) {
                        int si = __builtin_ctz(cm);
                        cm &= ~(1u << si);
                        centroidAlpha += alphaTab[si] * sampleCountInv;
                        if (dof) {
                            vector2 lensUV, dirUV;
                            sampleUVsDoF(N, lensTab.data(), tileDoF.focalToLensScale, si, lensUV, dirUV);
                            centroidLensUV += lensUV * sampleCountInv;
                            centroidDirUV += dirUV * sampleCountInv;
                        }
                    }
                    vector3 b, bOffX, bOffY;
                    if (dof) {
                        IntersectTriangleTile<true> tt;
                        tt.setup(S.tris[triIndex], cameraPos, tileDoF.lensU, tileDoF.lensV);
                        IntersectTriangleThreadDoF th(tt, lensCenterToFocalCenter);
                        th.calcUVW(tt, lensCenterToFocalCenter, tileDoF.lensU, tileDoF.lensV, centroidLensUV,
                                   centroidDirUV, b);
                        vector2 derivScale = vector2(1.0f, 1.0f);
                        vector2 dirUV_dX = centroidDirUV + vector2(derivScale.x, 0.0f);
                        th.calcUVW(tt, lensCenterToFocalCenter, tileDoF.lensU, tileDoF.lensV, centroidLensUV, dirUV_dX,
                                   bOffX);
                        vector2 dirUV_dY = centroidDirUV + vector2(0.0f, derivScale.y);
                        th.calcUVW(tt, lensCenterToFocalCenter, tileDoF.lensU, tileDoF.lensV, centroidLensUV, dirUV_dY,
                                   bOffY);
                    } else {
                        IntersectTriangleTile<false> tt;
                        tt.setup(S.tris[triIndex], cameraPos);
                        IntersectTriangleThread th(tt, sample.centerRay, sample.du, sample.dv);
                        th.calcUVW(tt, centroidAlpha, b);
                        vector2 alpha_dX = centroidAlpha + vector2(1.0f, 0.0f);
                        th.calcUVW(tt, alpha_dX, bOffX);
                        vector2 alpha_dY = centroidAlpha + vector2(0.0f, 1.0f);
                        th.calcUVW(tt, alpha_dY, bOffY);
                    }
                    InterpolatedVertex vI = interpolate(S.world.data(), S.triShade[triIndex], b);
                    InterpolatedVertex vInterpX = interpolate(S.world.data(), S.triShade[triIndex], bOffX);
                    InterpolatedVertex vInterpY = interpolate(S.world.data(), S.triShade[triIndex], bOffY);
                    vector2 dUVdX = vInterpX.uv - vI.uv;
                    vector2 dUVdY = vInterpY.uv - vI.uv;
                    vector4 shaded = GGXShade(S.triShade[triIndex].material, vI, dUVdX, dUVdY, cameraPos, materials,
                                              textureObjects.data(), env);
                    result += shaded * float(__builtin_popcount(sampleMask));
                }
                result *= 1.0f / N;
                result.w = 1.0f;
                colors[sid] = ToColor4Unorm8SRgb(ACESFilm(result));
            }
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nt; t++) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();

    uint64_t total = 0;
    for (uint32_t t = 0; t < tileCount; t++) {
        if (out->tile_counts) out->tile_counts[t] = uint32_t(lists[t].size());
        for (uint32_t v : lists[t]) {
            if (out->tile_indices && total < out->tile_capacity) out->tile_indices[total] = v;
            total++;
        }
    }
    out->tile_total = total;
    if (out->colors) memcpy(out->colors, colors.data(), size_t(padded) * 4);
    if (out->image) {
        for (uint32_t y = 0; y < S.height; y++)
            for (uint32_t x = 0; x < S.width; x++) {
                int32_t o = sd.imageLocationToSampleIndex[size_t(y) * S.width + x];
                if (o >= 0 && S.split == 1) out->image[size_t(y) * S.width + x] = colors[o];
            }
    }
    return 0;
}

} // namespace


extern "C" int ref_render(const oracle_frame_in* in, oracle_frame_out* out) {
    MxcsrScope mx;
    RefSession S;
    const int rc = refSetup(in, out, S);
    if (rc) return rc;
    return refFrame(S, in->cam_xf, in->threads, out);
}

// A camera kept across frames, as the reference's Raycaster keeps it: ref_session_create does the
// scene upload and the sample setup once; each ref_session_frame renders one frame (frusta to
// world, traversal, intersect and shading on `threads` threads, remap) into colors [padded] and
// image [height*width] (either may be NULL).
extern "C" int ref_session_create(const oracle_frame_in* in, void** session) {
    MxcsrScope mx;
    std::unique_ptr<RefSession> S(new RefSession());
    oracle_frame_out none;
    memset(&none, 0, sizeof(none));
    const int rc = refSetup(in, &none, *S);
    if (rc) return rc;
    *session = S.release();
    return 0;
}

extern "C" int ref_session_frame(void* session, const hvvr_transform* cam_xf, uint32_t threads, uint32_t* colors,
                                 uint32_t* image) {
    MxcsrScope mx;
    oracle_frame_out out;
    memset(&out, 0, sizeof(out));
    out.colors = colors;
    out.image = image;
    return refFrame(*static_cast<RefSession*>(session), *cam_xf, threads, &out);
}

extern "C" void ref_session_destroy(void* session) { delete static_cast<RefSession*>(session); }

// ------------------------------------------------------------------ foveated sample set
// polarSpaceFoveatedSetup's sample-set part (libraries/hvvr/raycaster/foveated.cpp:47-110):
// the reference's generateEyeSpacePolarFoveatedSampleData and ComputeEyeSpaceFrusta, run here
// on the host (GPUBuffer over host memory, see ref_stubs.cpp). Counts first (null outputs).
namespace hvvr {
void ComputeEyeSpaceFrusta(const GPUBuffer<DirectionalBeam>& dirSamples, GPUBuffer<SimpleRayFrustum>& tileFrusta,
                           GPUBuffer<SimpleRayFrustum>& blockFrusta);
}
extern "C" int ref_polar_foveated(float degreeTrackingError, float maxFOVDegrees, float marSlope,
                                  float fovealMARDegrees, uint32_t* counts4, float* beams9, uint32_t* remap2,
                                  float* tileRays24, float* blockRays24) {
    MxcsrScope mx;
    FoveatedSampleData fsd;
    std::vector<vector2ui> polarRemapToPixel;
    EccentricityMap emap;
    size_t samplesPerRing = 0;
    RayCasterSpecification::FoveatedSamplePattern pattern;
    pattern.degreeTrackingError = degreeTrackingError;
    pattern.maxFOVDegrees = maxFOVDegrees;
    pattern.marSlope = marSlope;
    pattern.fovealMARDegrees = fovealMARDegrees;
    generateEyeSpacePolarFoveatedSampleData(fsd, polarRemapToPixel, emap, samplesPerRing, pattern);
    const DynamicArray<DirectionalBeam>& beams = fsd.samples.directionalBeams;
    const uint32_t valid = uint32_t(beams.size());
    const uint32_t blocks = uint32_t(fsd.blockCount);
    if (counts4) {
        counts4[0] = uint32_t(samplesPerRing);
        counts4[1] = uint32_t(valid / samplesPerRing);
        counts4[2] = valid;
        counts4[3] = blocks * BLOCK_SIZE;
    }
    if (beams9) memcpy(beams9, beams.data(), size_t(valid) * sizeof(DirectionalBeam));
    if (remap2) memcpy(remap2, polarRemapToPixel.data(), size_t(valid) * sizeof(vector2ui));
    if (tileRays24 || blockRays24) {
        GPUBuffer<DirectionalBeam> d(beams.data(), beams.data() + valid);
        GPUBuffer<SimpleRayFrustum> t(size_t(blocks) * TILES_PER_BLOCK), b(blocks);
        ComputeEyeSpaceFrusta(d, t, b);
        if (tileRays24) t.readback((SimpleRayFrustum*)tileRays24);
        if (blockRays24) b.readback((SimpleRayFrustum*)blockRays24);
    }
    return 0;
}

// ------------------------------------------------------------------ foveated frame matrices
// The per-frame matrices of Raycaster::renderFoveatedPolarSpaceCudaReconstruct
// (RC/render.cpp:454-487) with the reference's own vector algebra: eyeToWorld, the cull planes
// of cullRectToCullPlanes (RC/render.cpp:397-416, a file-static function, so its ten lines are
// restated here on the reference's types), sampleToEye, and eyeToSamplePrevious as
// GPUCamera::foveatedPolarToScreenSpace forms it (RC/gpu_foveated.cu:341); then the history
// update. Column-major in and out.
static_assert(sizeof(matrix4x4) == 64 && sizeof(matrix3x3) == 36, "column-major float matrices");
extern "C" int ref_foveated_frame_matrices(const hvvr_transform* cameraToWorldXf, const float* eyeDir3,
                                           const float* sampleBounds4, const float* viewport4,
                                           float* worldToEyePrev16, float* eyePrevToSamplePrev9, float* eyeToWorld16,
                                           float* cullPlanes16, float* sampleToEye9, float* eyeToSamplePrev16) {
    MxcsrScope mx;
    const FloatRect vp(vector2(viewport4[0], viewport4[1]), vector2(viewport4[2], viewport4[3]));
    const FloatRect sb(vector2(sampleBounds4[0], sampleBounds4[1]), vector2(sampleBounds4[2], sampleBounds4[3]));
    matrix3x3 sampleToCamera(vector3(vp.upper.x - vp.lower.x, 0, 0), vector3(0, vp.lower.y - vp.upper.y, 0),
                             vector3(vp.lower.x, vp.upper.y, -1));
    const vector3 eyeDirection(eyeDir3[0], eyeDir3[1], eyeDir3[2]);
    matrix3x3 eyeToCamera = matrix3x3::rotationFromZAxis(-eyeDirection);
    matrix4x4 cameraToWorld = matrix4x4(*(const transform*)cameraToWorldXf);
    matrix4x4 eyeToWorld = cameraToWorld * matrix4x4(eyeToCamera);
    {
        const matrix3x3 cameraToEye = invert(eyeToCamera);
        auto U = sb.upper;
        auto L = sb.lower;
        vector2 sampleDirs[4] = {{U.x, U.y}, {L.x, U.y}, {L.x, L.y}, {U.x, L.y}};
        for (int i = 0; i < 4; ++i) {
            vector3 dir0 = sampleToCamera * vector3(sampleDirs[i], 1.0f);
            vector3 dir1 = sampleToCamera * vector3(sampleDirs[(i + 1) % 4], 1.0f);
            Plane eyeSpacePlane;
            eyeSpacePlane.normal = cameraToEye * normalize(cross(dir1, dir0));
            eyeSpacePlane.dist = -0.01f;
            Plane p = eyeToWorld * eyeSpacePlane;
            cullPlanes16[4 * i + 0] = p.normal.x;
            cullPlanes16[4 * i + 1] = p.normal.y;
            cullPlanes16[4 * i + 2] = p.normal.z;
            cullPlanes16[4 * i + 3] = p.dist;
        }
    }
    matrix4x4 worldToEyePrevious;
    matrix3x3 eyePreviousToSamplePrevious;
    memcpy(&worldToEyePrevious, worldToEyePrev16, 64);
    memcpy(&eyePreviousToSamplePrevious, eyePrevToSamplePrev9, 36);
    matrix3x3 sampleToEye = invert(eyeToCamera) * sampleToCamera;
    matrix4x4 eyeToEyePrevious = worldToEyePrevious * eyeToWorld;
    matrix4x4 eyeToSamplePrevious = matrix4x4(eyePreviousToSamplePrevious) * eyeToEyePrevious;
    memcpy(eyeToWorld16, &eyeToWorld, 64);
    memcpy(sampleToEye9, &sampleToEye, 36);
    memcpy(eyeToSamplePrev16, &eyeToSamplePrevious, 64);
    worldToEyePrevious = invert(eyeToWorld);
    eyePreviousToSamplePrevious = invert(sampleToEye);
    memcpy(worldToEyePrev16, &worldToEyePrevious, 64);
    memcpy(eyePrevToSamplePrev9, &eyePreviousToSamplePrevious, 36);
    return 0;
}

// ------------------------------------------------------------------ scene and sample files
// The reference's own model_import::saveBin / loadBin (SS/model_import_bin.cpp) and
// saveSamples / loadSamples (RC/samples.cpp:161-187), for checking the library's file formats
// byte for byte in both directions.
#include "model_import.h"
namespace hvvr {
void saveSamples(const std::vector<hvvr::Sample>& samples, const std::string& filename);
}
static_assert(sizeof(hvvr::ShadingVertex) == 32 && sizeof(hvvr::PrecomputedTriangleShade) == 16 &&
                  sizeof(hvvr::SimpleMaterial) == 64 && sizeof(hvvr::LightUnion) == 56 &&
                  sizeof(hvvr::transform) == 32 && sizeof(hvvr::TopologyNode) == 32,
              "record layouts");

// saveBin of the given meshes and lights, plus one r8g8b8a8_unorm texture when texels != NULL
extern "C" int ref_bin_save(const char* path, const hvvr_mesh_data* meshes, const hvvr_transform* xfs,
                            uint32_t meshCount, const hvvr_light_union* lights, uint32_t lightCount,
                            const uint8_t* texels, uint32_t texWidth, uint32_t texHeight) {
    model_import::Model model;
    if (texels) {
        hvvr::TextureData td = {};
        td.format = hvvr::TextureFormat::r8g8b8a8_unorm;
        td.width = texWidth;
        td.height = texHeight;
        td.strideElements = texWidth;
        uint8_t* data = new uint8_t[size_t(texWidth) * texHeight * 4];
        memcpy(data, texels, size_t(texWidth) * texHeight * 4);
        td.data = data;
        model.textures.emplace_back(model_import::Texture(td));
    }
    for (uint32_t i = 0; i < lightCount; i++) model.lights.push_back(*reinterpret_cast<const hvvr::LightUnion*>(&lights[i]));
    for (uint32_t i = 0; i < meshCount; i++) {
        const hvvr_mesh_data& md = meshes[i];
        model_import::Mesh mesh;
        mesh.transform = *reinterpret_cast<const hvvr::transform*>(&xfs[i]);
        const auto* v = reinterpret_cast<const hvvr::ShadingVertex*>(md.verts);
        const auto* t = reinterpret_cast<const hvvr::PrecomputedTriangleShade*>(md.tri_shade);
        const auto* n = reinterpret_cast<const hvvr::TopologyNode*>(md.nodes);
        const auto* m = reinterpret_cast<const hvvr::SimpleMaterial*>(md.materials);
        mesh.data.verts.assign(v, v + md.vert_count);
        mesh.data.triShade.assign(t, t + md.tri_count);
        if (md.node_count) mesh.data.nodes.assign(n, n + md.node_count);
        mesh.data.materials.assign(m, m + md.material_count);
        model.meshes.emplace_back(std::move(mesh));
    }
    return model_import::saveBin(path, model) ? 0 : 1;
}

// loadBin: counts[4] = {textures, lights, meshes, total bytes}; with out != NULL every texture's
// {format, width, height, stride} and texels (getTextureSize), then the lights, then every mesh's
// transform and arrays are packed into out in file order
extern "C" int ref_bin_load(const char* path, uint64_t* counts, uint8_t* out) {
    model_import::Model model;
    if (!model_import::loadBin(path, model)) return 1;
    uint64_t bytes = model.lights.size() * sizeof(hvvr::LightUnion);
    for (const auto& t : model.textures)
        bytes += 16 + hvvr::getTextureSize(t.tex.strideElements, t.tex.height, t.tex.format);
    for (const auto& m : model.meshes)
        bytes += sizeof(hvvr::transform) + m.data.verts.size() * 32 + m.data.triShade.size() * 16 +
                 m.data.nodes.size() * 32 + m.data.materials.size() * 64;
    counts[0] = model.textures.size();
    counts[1] = model.lights.size();
    counts[2] = model.meshes.size();
    counts[3] = bytes;
    if (!out) return 0;
    auto put = [&](const void* p, size_t n) { memcpy(out, p, n); out += n; };
    for (const auto& t : model.textures) {
        const uint32_t rec[4] = {uint32_t(t.tex.format), t.tex.width, t.tex.height, t.tex.strideElements};
        put(rec, sizeof(rec));
        put(t.tex.data, hvvr::getTextureSize(t.tex.strideElements, t.tex.height, t.tex.format));
    }
    put(model.lights.data(), model.lights.size() * sizeof(hvvr::LightUnion));
    for (const auto& m : model.meshes) {
        put(&m.transform, sizeof(hvvr::transform));
        put(m.data.verts.data(), m.data.verts.size() * 32);
        put(m.data.triShade.data(), m.data.triShade.size() * 16);
        put(m.data.nodes.data(), m.data.nodes.size() * 32);
        put(m.data.materials.data(), m.data.materials.size() * 64);
    }
    return 0;
}

extern "C" int ref_samples_save(const char* path, const hvvr_sample* samples, uint32_t count) {
    const auto* s = reinterpret_cast<const hvvr::Sample*>(samples);
    hvvr::saveSamples(std::vector<hvvr::Sample>(s, s + count), path);
    return 0;
}

extern "C" int ref_samples_load(const char* path, hvvr_sample* out, uint32_t capacity, uint32_t* count) {
    hvvr::DynamicArray<hvvr::Sample> samples;
    hvvr::loadSamples(samples, path);
    *count = uint32_t(samples.size());
    if (out && capacity >= samples.size()) memcpy(out, samples.data(), samples.size() * sizeof(hvvr::Sample));
    return 0;
}
