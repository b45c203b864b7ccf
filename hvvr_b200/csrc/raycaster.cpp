// raycaster.cpp - the C ABI (include/hvvr_c.h) and the host frame driver.
//
// Object model and frame order follow the reference's Raycaster (libraries/hvvr/raycaster/
// raycaster.h, render.cpp:204-451, scene_update.cpp:22-174): models, lights and cameras are
// owned by the raycaster; render() rebuilds and refits the scene when it is dirty, then per
// enabled camera runs block cull -> tile cull -> intersect/shade/resolve -> remap. Unlike
// the reference, traversal runs on the GPU, the refit BVH never returns to the host, and
// the per-tile triangle lists never cross PCIe.
#include <cuda_runtime.h>

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <iterator>
#include <cmath>
#include <atomic>
#include <mutex>
#include <memory>
#include <string>
#include <vector>

#include "foveated.h"
#include "host_objects.h"
#include "sample_setup.h"

using namespace hvb;

namespace hvb {

thread_local std::string gLastError;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    gLastError = buf;
    return code;
}

} // namespace hvb


int hvb::setLastError(int code, const char* msg) {
    gLastError = msg ? msg : "";
    return code;
}

namespace hvb {

const char* kEmpty = "";

bool validRate(uint32_t r) { return r == 1 || r == 2 || r == 4 || r == 8 || r == 16 || r == 32; }

// Raycaster::buildScene (libraries/hvvr/raycaster/scene_update.cpp:22-143), plus validation
// that every leaf range lies inside the model and every child offset inside its node array.
int buildScene(hvvr_raycaster* rc, std::vector<Node>& nodes, std::vector<uint4>& triShade,
               std::vector<float4>& verts, std::vector<uint32_t>& vertModel, std::vector<float4>& materials) {
    const uint32_t modelCount = uint32_t(rc->models.size());
    nodes.clear();
    triShade.clear();
    verts.clear();
    vertModel.clear();
    materials.clear();
    // Models without triangles have no nodes: they take no child slot of the root fix-up nodes. A
    // scene with no triangles at all gets one root whose four leaf slots are empty; the refit gives
    // empty ranges -inf bounds, which fail every frustum test, so every tile's list is empty and the
    // frame clears its samples to the background.
    uint32_t liveCount = 0;
    for (auto& m : rc->models) liveCount += m->nodes.empty() ? 0u : 1u;
    if (liveCount == 0) {
        nodes.assign(1, Node{});
        nodes[0].leafMask = 0xf;
        return HVVR_OK;
    }
    const uint32_t rootNodeCount = (liveCount + 1) / 3;
    size_t nc = rootNodeCount;
    for (auto& m : rc->models) nc += m->nodes.size();
    nodes.assign(nc, Node{});
    std::vector<uint32_t> viewOffsets(modelCount);
    uint32_t vOff = 0, tOff = 0, mOff = 0, nOff = rootNodeCount;
    for (uint32_t mi = 0; mi < modelCount; mi++) {
        const hvvr_model& m = *rc->models[mi];
        const uint32_t tc = uint32_t(m.triShade.size()), vc = uint32_t(m.verts.size());
        for (const hvvr_material& mat : m.materials) {
            const float4* q = reinterpret_cast<const float4*>(&mat);
            materials.insert(materials.end(), q, q + 4);
        }
        for (const hvvr_tri_shade& t : m.triShade) {
            if (t.indices[0] >= vc || t.indices[1] >= vc || t.indices[2] >= vc)
                return fail(HVVR_ERR_INVALID, "model %u: vertex index out of range", mi);
            if (t.material >= m.materials.size()) return fail(HVVR_ERR_INVALID, "model %u: material out of range", mi);
            triShade.push_back(make_uint4(t.indices[0] + vOff, t.indices[1] + vOff, t.indices[2] + vOff, t.material + mOff));
        }
        for (const hvvr_shading_vertex& v : m.verts) {
            const float4* q = reinterpret_cast<const float4*>(&v);
            verts.push_back(q[0]);
            verts.push_back(q[1]);
            vertModel.push_back(mi);
        }
        viewOffsets[mi] = nOff;
        std::vector<uint32_t> cover(tc, 0);
        for (size_t i = 0; i < m.nodes.size(); i++) {
            const hvvr_topology_node& tn = m.nodes[i];
            Node& n = nodes[nOff + i];
            n.leafMask = tn.leaf_mask & 0xfu;
            n.tri[0] = tOff + tn.data[0];
            for (int k = 0; k < 4; k++) {
                if (tn.leaf_mask & (1u << k)) {
                    n.tri[1 + k] = tOff + tn.data[1 + k];
                    const uint32_t a = tn.data[k], b = tn.data[1 + k];
                    if (a > b || b > tc) return fail(HVVR_ERR_INVALID, "model %u node %zu: bad leaf range", mi, i);
                    for (uint32_t t = a; t < b; t++) cover[t]++;
                } else {
                    n.tri[1 + k] = tn.data[1 + k];
                    if (tn.data[1 + k] == 0 || i + tn.data[1 + k] >= m.nodes.size())
                        return fail(HVVR_ERR_INVALID, "model %u node %zu: bad child offset", mi, i);
                }
            }
        }
        for (uint32_t t = 0; t < tc; t++)
            if (cover[t] != 1)
                return fail(HVVR_ERR_INVALID, "model %u: triangle %u covered by %u leaves (topology must partition)",
                            mi, t, cover[t]);
        vOff += vc;
        tOff += tc;
        mOff += uint32_t(m.materials.size());
        nOff += uint32_t(m.nodes.size());
    }
    if (rootNodeCount > 0) {
        std::vector<int64_t> children(rootNodeCount * 4);
        size_t w = 0;
        for (size_t i = children.size() - liveCount - (rootNodeCount - 1); i != 0; --i) children[w++] = -1;
        for (uint32_t i = 1; i < rootNodeCount; i++) children[w++] = i;
        for (uint32_t mi = 0; mi < modelCount; mi++)
            if (!rc->models[mi]->nodes.empty()) children[w++] = viewOffsets[mi];
        for (uint32_t i = 0; i < rootNodeCount; i++) {
            Node& n = nodes[i];
            n.tri[0] = 0;
            n.leafMask = 0;
            for (int k = 0; k < 4; k++) {
                const int64_t c = children[4 * i + k];
                if (c < 0) {
                    n.tri[1 + k] = 0;
                    n.leafMask |= 1u << k;
                    continue;
                }
                n.tri[1 + k] = uint32_t(c - i);
            }
        }
    }
    return HVVR_OK;
}

int uploadScene(hvvr_raycaster* rc, cudaStream_t st) {
    std::vector<Node> nodes;
    std::vector<uint4> triShade;
    std::vector<float4> verts, materials;
    std::vector<uint32_t> vertModel;
    TRY(buildScene(rc, nodes, triShade, verts, vertModel, materials));
    const uint32_t nodeCount = uint32_t(nodes.size());
    // refit order: parent slot of every internal child, internal child counts, start nodes
    std::vector<uint32_t> parentSlot(nodeCount, 0xffffffffu), internalCount(nodeCount, 0), depth(nodeCount, 0), starts;
    uint32_t maxDepth = 0;
    for (uint32_t n = 0; n < nodeCount; n++) {
        for (int k = 0; k < 4; k++) {
            if (nodes[n].leafMask & (1u << k)) continue;
            const uint32_t c = n + nodes[n].tri[k + 1];
            if (c >= nodeCount || c <= n) return fail(HVVR_ERR_INVALID, "node %u: child offset out of range", n);
            parentSlot[c] = (n << 2) | uint32_t(k);
            internalCount[n]++;
            depth[c] = depth[n] + 1;
            maxDepth = std::max(maxDepth, depth[c]);
        }
    }
    for (uint32_t n = 0; n < nodeCount; n++)
        if (internalCount[n] == 0) starts.push_back(n);
    std::vector<Mat4> xf(std::max<size_t>(rc->models.size(), 1));
    for (size_t i = 0; i < rc->models.size(); i++) xf[i] = transformToMatrix(rc->models[i]->xf);

    TRY(rc->nodes.upload(nodes.data(), nodes.size(), st));
    TRY(rc->triShade.upload(triShade.data(), triShade.size(), st));
    TRY(rc->vertsIn.upload(verts.data(), verts.size(), st));
    TRY(rc->verts.alloc(verts.size()));
    TRY(rc->vertModel.upload(vertModel.data(), vertModel.size(), st));
    TRY(rc->materials.upload(materials.data(), materials.size(), st));
    TRY(rc->tris.alloc(triShade.size() * 3));
    TRY(rc->modelToWorld.upload(xf.data(), xf.size(), st));
    TRY(rc->parentSlot.upload(parentSlot.data(), parentSlot.size(), st));
    TRY(rc->internalCount.upload(internalCount.data(), internalCount.size(), st));
    TRY(rc->arrivals.alloc(size_t(nodeCount) + 1));
    TRY(rc->refitStarts.upload(starts.data(), starts.size(), st));
    SceneDev& s = rc->scene;
    s.nodes = rc->nodes.p;
    s.nodeCount = nodeCount;
    s.tris = rc->tris.p;
    s.triShade = rc->triShade.p;
    s.triCount = uint32_t(triShade.size());
    s.vertsIn = rc->vertsIn.p;
    s.verts = rc->verts.p;
    s.vertModel = rc->vertModel.p;
    s.vertCount = uint32_t(vertModel.size());
    s.modelToWorld = rc->modelToWorld.p;
    s.modelCount = uint32_t(rc->models.size());
    s.materials = rc->materials.p;
    s.materialCount = uint32_t(materials.size() / 4);
    s.parentSlot = rc->parentSlot.p;
    s.internalCount = rc->internalCount.p;
    s.arrivals = rc->arrivals.p;
    s.refitStarts = rc->refitStarts.p;
    s.refitStartCount = uint32_t(starts.size());
    s.maxDepth = maxDepth;
    rc->hostNodes = std::move(nodes);
    // GPUSceneState::updateLighting (libraries/hvvr/raycaster/gpu_scene_state.cu:47-81)
    LightEnvDev& env = s.env;
    memset(&env, 0, sizeof(env));
    for (auto& l : rc->lights) {
        const hvvr_light_union& u = l->light;
        if (u.type == HVVR_LIGHT_DIRECTIONAL && env.nd < 1) {
            const hvvr_light_directional& d = u.u.directional;
            float* o = env.dir[env.nd++];
            o[0] = d.direction.x; o[1] = d.direction.y; o[2] = d.direction.z;
            o[3] = d.power.x; o[4] = d.power.y; o[5] = d.power.z;
        } else if (u.type == HVVR_LIGHT_POINT && env.np < 4) {
            const hvvr_light_point& p = u.u.point;
            float* o = env.pt[env.np++];
            o[0] = p.position.x; o[1] = p.position.y; o[2] = p.position.z; o[3] = p.falloff_end;
            o[4] = p.color.x; o[5] = p.color.y; o[6] = p.color.z; o[7] = p.falloff_scale;
        } else if (u.type == HVVR_LIGHT_SPOT && env.ns < 4) {
            const hvvr_light_spot& p = u.u.spot;
            float* o = env.spot[env.ns++];
            o[0] = p.position.x; o[1] = p.position.y; o[2] = p.position.z; o[3] = p.falloff_end;
            o[4] = p.direction.x; o[5] = p.direction.y; o[6] = p.direction.z; o[7] = p.falloff_scale;
            o[8] = p.color.x; o[9] = p.color.y; o[10] = p.color.z; o[11] = p.cos_outer_angle; o[12] = p.cos_angle_scale;
        }
    }
    return HVVR_OK;
}

int uploadTransforms(hvvr_raycaster* rc, cudaStream_t st) {
    std::vector<Mat4> xf(std::max<size_t>(rc->models.size(), 1));
    for (size_t i = 0; i < rc->models.size(); i++) xf[i] = transformToMatrix(rc->models[i]->xf);
    return rc->modelToWorld.upload(xf.data(), xf.size(), st);
}

std::atomic<uint64_t> gSetupGen{0};

int setupFoveatedCamera(hvvr_camera* cam, cudaStream_t st);

int setupCamera(hvvr_camera* cam, cudaStream_t st) {
    if (cam->samples.empty()) return fail(HVVR_ERR_STATE, "camera has no samples");
    if (cam->rc->spec.mode == HVVR_MODE_FOVEATED_POLAR) return setupFoveatedCamera(cam, st);
    const uint32_t w = cam->target.width, h = cam->target.height;
    // the sample hierarchy: on the device unless the spec asks for the host, the spherical
    // mapping is on (its sin/cos follow the host's libm), or two samples share a position
    bool host = cam->rc->spec.sample_setup == HVVR_SETUP_HOST || cam->fovX > 0.0f;
    if (!host) {
        DeviceSampleSetup ds{&cam->tileRays, &cam->blockRays, &cam->beams, &cam->remap};
        TRY(buildSampleSetupDevice(cam->samples.data(), uint32_t(cam->samples.size()), cam->split, cam->viewport,
                                   cam->lens, w, h, ds, st, host));
        if (!host) {
            cam->setup = SampleSetup{};
            cam->setup.blocks = ds.blocks;
            cam->setup.tiles = ds.tiles;
            cam->setup.padded = ds.padded;
            cam->setup.valid = ds.valid;
        }
    }
    if (host) {
        buildSampleSetup(cam->samples.data(), uint32_t(cam->samples.size()), cam->split, cam->viewport, cam->lens,
                         cam->fovX, cam->fovY, w, h, cam->setup);
        SampleSetup& hs = cam->setup;
        TRY(cam->tileRays.upload(hs.tileRays.data(), hs.tileRays.size(), st));
        TRY(cam->blockRays.upload(hs.blockRays.data(), hs.blockRays.size(), st));
        TRY(cam->beams.upload(hs.beams.data(), hs.beams.size() / 4, st));
        TRY(cam->remap.upload(hs.remap.data(), hs.remap.size(), st));
        CUDA_TRY(cudaStreamSynchronize(st));  // the host arrays are released next
        hs.tileRays = {};
        hs.blockRays = {};
        hs.beams = {};
        hs.remap = {};
    }
    cam->setupOnHost = host;
    const SampleSetup& ss = cam->setup;
    TRY(cam->blockStacks.alloc(size_t(ss.blocks) * kBlockStack));
    TRY(cam->blockSizes.alloc(ss.blocks));
    TRY(cam->tileLists.alloc(ss.tiles));
    TRY(cam->colors.alloc(ss.padded));
    TRY(cam->tileCost.alloc(ss.tiles));
    CUDA_TRY(cudaMemsetAsync(cam->tileCost.p, 0, size_t(ss.tiles) * 4, st));
    const bool cpuTarget = cam->target.memory_type == HVVR_MEMORY_CPU;
    if (cpuTarget && w && h) TRY(cam->image.alloc(size_t(w) * h));
    CameraDev& d = cam->dev;
    d.blocks = ss.blocks;
    d.tiles = ss.tiles;
    d.padded = ss.padded;
    d.valid = ss.valid;
    d.tileRays = cam->tileRays.p;
    d.blockRays = cam->blockRays.p;
    d.beams = cam->beams.p;
    d.remap = cam->remap.p;
    d.width = w;
    d.height = h;
    d.split = cam->split;
    d.blockStacks = cam->blockStacks.p;
    d.blockSizes = cam->blockSizes.p;
    d.tileLists = cam->tileLists.p;
    d.tileCost = cam->tileCost.p;
    d.colors = cam->colors.p;
    if (cpuTarget) {
        d.image = cam->image.p;
        d.imageStride = w;
    } else {
        d.image = static_cast<uint32_t*>(cam->target.data);
        d.imageStride = cam->target.stride ? cam->target.stride : w;
    }
    cam->setupDirty = false;
    cam->setupGen = ++gSetupGen;
    cam->costFrames = 0;
    return HVVR_OK;
}

void resetFoveatedHistory(hvvr_camera* cam) {
    // a new camera's state (libraries/hvvr/raycaster/camera.h:121-122: _worldToEyePrevious
    // zero, _eyePreviousToSamplePrevious identity)
    memset(cam->worldToEyePrev, 0, sizeof(cam->worldToEyePrev));
    const float id[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    memcpy(cam->eyePrevToSamplePrev, id, sizeof(id));
}

// A camera of a foveated-polar raycaster (renderFoveatedPolarSpaceCudaReconstruct,
// libraries/hvvr/raycaster/render.cpp:454-492): traversal and shading run on the raycaster's
// polar sample set in eye space; the camera's own samples only bound the screen (sampleBounds,
// libraries/hvvr/raycaster/camera.cpp:36-42) for the tile cull planes.
int setupFoveatedCamera(hvvr_camera* cam, cudaStream_t st) {
    hvvr_raycaster* rc = cam->rc;
    if (!rc->polar) {
        rc->polar = std::make_unique<PolarSetup>();
        buildPolarFoveatedSetup(rc->spec.foveated_degree_tracking_error, rc->spec.foveated_max_fov_degrees,
                                rc->spec.foveated_mar_slope, rc->spec.foveated_foveal_mar_degrees, *rc->polar);
    }
    const PolarSetup& ps = *rc->polar;
    hvvr_float_rect b{{1.0f, 1.0f}, {0.0f, 0.0f}};
    for (const hvvr_sample& smp : cam->samples) {
        b.lower.x = std::min(b.lower.x, smp.position.x);
        b.lower.y = std::min(b.lower.y, smp.position.y);
        b.upper.x = std::max(b.upper.x, smp.position.x);
        b.upper.y = std::max(b.upper.y, smp.position.y);
    }
    cam->sampleBounds = b;
    std::vector<float4> beams(size_t(ps.padded) * 3, make_float4(0, 0, 0, 0));
    for (size_t i = 0; i < ps.beams.size(); i++) {
        const PolarBeam& pb = ps.beams[i];
        beams[3 * i + 0] = make_float4(pb.c[0], pb.c[1], pb.c[2], pb.du[0]);
        beams[3 * i + 1] = make_float4(pb.du[1], pb.du[2], pb.dv[0], pb.dv[1]);
        beams[3 * i + 2] = make_float4(pb.dv[2], 0.0f, 0.0f, 0.0f);
    }
    TRY(cam->tileRays.upload(ps.tileRays.data(), ps.tileRays.size(), st));
    TRY(cam->blockRays.upload(ps.blockRays.data(), ps.blockRays.size(), st));
    TRY(cam->beams.upload(beams.data(), beams.size(), st));
    TRY(cam->polarRemap.upload(ps.remap.data(), ps.padded, st));
    CUDA_TRY(cudaStreamSynchronize(st)); // host staging goes out of scope
    TRY(cam->blockStacks.alloc(size_t(ps.blocks) * kBlockStack));
    TRY(cam->blockSizes.alloc(ps.blocks));
    TRY(cam->tileLists.alloc(ps.tiles));
    TRY(cam->colors.alloc(ps.padded));
    TRY(cam->tmax.alloc(ps.padded));
    TRY(cam->tileCost.alloc(ps.tiles));
    CUDA_TRY(cudaMemsetAsync(cam->tileCost.p, 0, size_t(ps.tiles) * 4, st));
    // the resolve (GPUCamera::registerPolarFoveatedSamples and the image-sized textures,
    // libraries/hvvr/raycaster/gpu_camera.cu:174-183, 194-230; getEccentricityMap,
    // gpu_foveated.cu:80-85)
    const uint32_t w = cam->target.width, h = cam->target.height;
    const bool cpuTarget = cam->target.memory_type == HVVR_MEMORY_CPU;
    FoveaDev& fv = cam->fovStatic;
    fv = FoveaDev{};
    if (w && h) {
        const size_t npix = size_t(w) * h;
        const uint32_t spr = ps.samplesPerRing, rings = ps.ringCount;
        const cudaChannelFormatDesc rgba8 = cudaCreateChannelDesc(8, 8, 8, 8, cudaChannelFormatKindUnsigned);
        const cudaChannelFormatDesc rgba16 = cudaCreateChannelDesc(16, 16, 16, 16, cudaChannelFormatKindUnsigned);
        const cudaChannelFormatDesc r32f = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
        const cudaTextureAddressMode wrap = cudaAddressModeWrap, clamp = cudaAddressModeClamp;
        // polar textures: wrap in azimuth, clamp in eccentricity; depth point-sampled
        TRY(cam->polarRaw.create(spr, rings, rgba8, 4, cudaReadModeNormalizedFloat, true, wrap, clamp, true));
        TRY(cam->polarDepth.create(spr, rings, r32f, 4, cudaReadModeElementType, false, wrap, clamp, false));
        TRY(cam->moment1.create(spr, rings, rgba16, 8, cudaReadModeNormalizedFloat, false, wrap, clamp, true));
        TRY(cam->moment2.create(spr, rings, rgba16, 8, cudaReadModeNormalizedFloat, false, wrap, clamp, true));
        // screen textures (createImageSizedTexture: clamp, linear)
        for (int k = 0; k < 2; k++)
            TRY(cam->fovResult[k].create(w, h, rgba8, 4, cudaReadModeNormalizedFloat, true, clamp, clamp, true));
        for (TexArray* t : {&cam->polarRaw, &cam->polarDepth, &cam->moment1, &cam->moment2, &cam->fovResult[0],
                            &cam->fovResult[1]})
            TRY(t->clear(st));
        // the texture unit's read of each 8-bit code of a screen texture (for the fused filter and
        // contrast pass): a 256-texel texture made like the screen textures, texel i = (i, i, i, i)
        {
            TexArray codes;
            TRY(codes.create(256, 1, rgba8, 4, cudaReadModeNormalizedFloat, true, clamp, clamp, true));
            uint32_t texels[256];
            for (uint32_t i = 0; i < 256; i++) texels[i] = i * 0x01010101u;
            CUDA_TRY(cudaMemcpy2DToArrayAsync(codes.array, 0, 0, texels, sizeof(texels), sizeof(texels), 1,
                                              cudaMemcpyHostToDevice, st));
            TRY(cam->fovDecode.alloc(256));
            CUDA_TRY(launchSrgbDecodeTable(codes.tex, cam->fovDecode.p, st));
            CUDA_TRY(cudaStreamSynchronize(st)); // before the probe texture and the host texels go
        }
        if (cpuTarget) TRY(cam->image.alloc(npix));
        fv.remap = cam->polarRemap.p;
        fv.rawTex = cam->polarRaw.tex;
        fv.rawSurf = cam->polarRaw.surf;
        fv.depthTex = cam->polarDepth.tex;
        fv.depthSurf = cam->polarDepth.surf;
        fv.m1Tex = cam->moment1.tex;
        fv.m1Surf = cam->moment1.surf;
        fv.m2Tex = cam->moment2.tex;
        fv.m2Surf = cam->moment2.surf;
        fv.srgbDecode = cam->fovDecode.p;
        fv.image = cpuTarget ? cam->image.p : static_cast<uint32_t*>(cam->target.data);
        fv.imageStride = cpuTarget ? w : (cam->target.stride ? uint32_t(cam->target.stride) : w);
        fv.width = w;
        fv.height = h;
        fv.spr = ps.samplesPerRing;
        fv.rings = ps.ringCount;
        fv.valid = ps.valid;
        fv.eccM = ps.eccM;
        fv.eccW0 = ps.eccW0;
        fv.eccS = ps.eccS;
        fv.eccInvLogA = ps.eccInvLogA;
        fv.eccInvW0 = ps.eccInvW0;
        fv.eccInvM = ps.eccInvM;
        fv.texMapSize = float(ps.ringCount);
        fv.invTexMapSize = 1.0f / float(ps.ringCount);
        fv.invMaxEcc = 1.0f / ps.maxEccentricity;
    }
    resetFoveatedHistory(cam);
    CameraDev& d = cam->dev;
    d = CameraDev{};
    d.blocks = ps.blocks;
    d.tiles = ps.tiles;
    d.padded = ps.padded;
    d.valid = ps.valid;
    d.tileRays = cam->tileRays.p;
    d.blockRays = cam->blockRays.p;
    d.beams = cam->beams.p;
    d.blockStacks = cam->blockStacks.p;
    d.blockSizes = cam->blockSizes.p;
    d.tileLists = cam->tileLists.p;
    d.tileCost = cam->tileCost.p;
    d.colors = cam->colors.p;
    d.width = w;
    d.height = h;
    d.image = fv.image;
    d.imageStride = fv.imageStride;
    cam->setup = SampleSetup{};
    cam->setup.blocks = ps.blocks;
    cam->setup.tiles = ps.tiles;
    cam->setup.padded = ps.padded;
    cam->setup.valid = ps.valid;
    cam->foveated = true;
    cam->setupDirty = false;
    cam->setupGen = ++gSetupGen;
    cam->costFrames = 0;
    return HVVR_OK;
}

// CPU_MEMORY render targets are page-locked while they are bound, so the per-frame image
// copy runs at pinned-memory bandwidth; if registration fails the copy stays pageable.
void unregisterTarget(hvvr_camera* cam) {
    if (cam->registered) {
        cudaHostUnregister(cam->registered);
        cam->registered = nullptr;
    }
}

void releaseCamera(hvvr_camera* cam) { unregisterTarget(cam); }

uint32_t rateIndex(uint32_t rate) { return rate <= 1 ? 0u : uint32_t(31 - __builtin_clz(rate)); }

bool hasLens(const hvvr_camera* c) { return c->lens.radius > 0.0f; }
// launches are grouped by rate class: log2(msaa), + 6 for a thin-lens view (a separate kernel)
// rate class: log2(msaa); + 6 for a thin-lens view; + 12 for a pinhole view with the rotated grid
uint32_t rateClass(const hvvr_camera* c) {
    if (hasLens(c)) return rateIndex(c->msaa) + 6u;
    return rateIndex(c->msaa) + (c->msaaPattern == HVVR_MSAA_ROTATED_GRID ? 12u : 0u);
}

// the offset tables live in one __constant__ array per device, written once per rate
int ensureMsaaTable(uint32_t rate, cudaStream_t st) {
    static std::mutex mu;
    static bool uploaded[64][6] = {};
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(HVVR_ERR_INVALID, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(mu);
    bool& done = uploaded[dev][rateIndex(rate)];
    if (done) return HVVR_OK;
    float off[64];
    msaaOffsets(rate, off);
    CUDA_TRY(uploadMsaaTable(rate, 0, off, st));
    msaaOffsetsRotatedGrid(rate, off);
    CUDA_TRY(uploadMsaaTable(rate, 1, off, st));
    CUDA_TRY(cudaStreamSynchronize(st)); // visible before any other stream can use the rate
    done = true;
    return HVVR_OK;
}

size_t cameraBytes(const hvvr_camera* cam, uint32_t msaa) {
    if (cam->foveated) {
        const CameraDev& d = cam->dev;
        const FoveaDev& f = cam->fovStatic;
        size_t b = size_t(d.tiles) * (sizeof(Rays4) + sizeof(TileList) + 4) +
                   size_t(d.blocks) * (sizeof(Rays4) + kBlockStack * sizeof(StackEntry) + 4) +
                   size_t(d.padded) * (48 + 8 + 4 + 4);
        b += size_t(f.spr) * f.rings * (4 + 4 + 8 + 8) + size_t(f.width) * f.height * (4 * 4);
        if (cam->target.memory_type == HVVR_MEMORY_CPU) b += size_t(f.width) * f.height * 4;
        if (cam->capture & HVVR_CAPTURE_HITS) b += size_t(d.padded) * msaa * 8;
        return b;
    }
    const SampleSetup& ss = cam->setup;
    size_t b = cam->tileRays.n * sizeof(Rays4) + cam->blockRays.n * sizeof(Rays4) + cam->beams.n * sizeof(float4) +
               cam->remap.n * 4;
    b += size_t(ss.blocks) * kBlockStack * sizeof(StackEntry) + size_t(ss.blocks) * 4;
    b += size_t(ss.tiles) * (sizeof(TileList) + 4) + size_t(ss.padded) * 4;
    if (cam->target.memory_type == HVVR_MEMORY_CPU) b += size_t(cam->target.width) * cam->target.height * 4;
    if (cam->capture & HVVR_CAPTURE_HITS) b += size_t(ss.padded) * msaa * 8;
    return b;
}

int cloneCamera(const hvvr_camera* src, hvvr_camera** out) {
    if (src->setupDirty) return fail(HVVR_ERR_STATE, "camera to clone has no setup yet");
    if (src->foveated) {
        // a polar-mode camera's samples are the raycaster's polar set: set the clone up from it
        auto c = std::make_unique<hvvr_camera>();
        c->rc = src->rc;
        c->viewport = src->viewport;
        c->lens = src->lens;
        c->eyeDir = src->eyeDir;
        c->target = src->target;
        c->target.data = nullptr;
        c->samples = src->samples;
        c->split = src->split;
        c->xf = src->xf;
        c->msaa = src->msaa;
        const cudaStream_t st = src->rc->stream;
        TRY(setupFoveatedCamera(c.get(), st));
        CUDA_TRY(cudaMemcpyAsync(c->tileCost.p, src->tileCost.p, size_t(c->dev.tiles) * 4, cudaMemcpyDeviceToDevice, st));
        c->costFrames = src->costFrames;
        CUDA_TRY(cudaStreamSynchronize(st));
        *out = c.get();
        src->rc->cameras.push_back(std::move(c));
        return HVVR_OK;
    }
    auto c = std::make_unique<hvvr_camera>();
    c->rc = src->rc;
    c->viewport = src->viewport;
    c->lens = src->lens;
    c->eyeDir = src->eyeDir;
    c->fovX = src->fovX;
    c->fovY = src->fovY;
    c->target = src->target;
    c->target.data = nullptr;
    c->samples = src->samples;
    c->split = src->split;
    c->xf = src->xf;
    c->msaa = src->msaa;
    c->setup = src->setup;
    c->setupOnHost = src->setupOnHost;
    const SampleSetup& ss = c->setup;
    const cudaStream_t st = src->rc->stream;
    TRY(c->tileRays.alloc(src->tileRays.n));
    TRY(c->blockRays.alloc(src->blockRays.n));
    TRY(c->beams.alloc(src->beams.n));
    TRY(c->remap.alloc(src->remap.n));
    CUDA_TRY(cudaMemcpyAsync(c->tileRays.p, src->tileRays.p, src->tileRays.n * sizeof(Rays4), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(c->blockRays.p, src->blockRays.p, src->blockRays.n * sizeof(Rays4), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(c->beams.p, src->beams.p, src->beams.n * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(c->remap.p, src->remap.p, src->remap.n * 4, cudaMemcpyDeviceToDevice, st));
    TRY(c->blockStacks.alloc(size_t(ss.blocks) * kBlockStack));
    TRY(c->blockSizes.alloc(ss.blocks));
    TRY(c->tileLists.alloc(ss.tiles));
    TRY(c->colors.alloc(ss.padded));
    TRY(c->tileCost.alloc(ss.tiles));
    CUDA_TRY(cudaMemcpyAsync(c->tileCost.p, src->tileCost.p, size_t(ss.tiles) * 4, cudaMemcpyDeviceToDevice, st));
    c->dev = src->dev;
    CameraDev& d = c->dev;
    d.tileRays = c->tileRays.p;
    d.blockRays = c->blockRays.p;
    d.beams = c->beams.p;
    d.remap = c->remap.p;
    d.blockStacks = c->blockStacks.p;
    d.blockSizes = c->blockSizes.p;
    d.tileLists = c->tileLists.p;
    d.tileCost = c->tileCost.p;
    d.colors = c->colors.p;
    d.hitIds = nullptr;
    d.depth = nullptr;
    d.image = nullptr;
    c->costFrames = src->costFrames;
    c->setupDirty = false;
    c->setupGen = ++gSetupGen;
    CUDA_TRY(cudaStreamSynchronize(st));
    *out = c.get();
    src->rc->cameras.push_back(std::move(c));
    return HVVR_OK;
}

// rate groups with fewer tiles are not split
constexpr uint32_t kSplitMinTiles = 32;

void batchConfigDefault(hvvr_batch_config* c) {
    // On the 1M-triangle stereo 2x1080x1200 8xMSAA frame, one-warp cull CTAs with the slowest 1/8
    // of the tiles as the heavy part, cull -> shade pipeline on, were fastest: 4.92 ms against 5.50
    // with 2-warp CTAs (a warp that runs out of tiles frees its registers for the shade of finished
    // tiles at once); heavy shares 1/4, 1/6, 1/12 and 1/16 were 5.17, 5.05, 5.19 and 5.3-5.4 ms;
    // without the pipeline 5.99. Streaming the lists of the first 400 tiles of each rate class's first
    // part: 4.86 ms against 4.99 without (16, 48, 148, 1000, 2544 tiles: 4.99, 4.99, 4.89, 4.87, 5.00)
    c->tile_cull_warps = 1;
    c->heavy_divisor = 8;
    c->tri_index_capacity = kDefaultCapacity;
    c->use_graph = 1;
    c->frame_ms = 0.0f;
    c->tile_stack_entries = 0;
    c->timing = 0;
    c->pipeline = 1;
    c->tile_cull_ctas_per_sm = 0;
    c->tile_cull_persistent = 1;
    c->stream_tiles = 400;
}

int checkConfig(const hvvr_batch_config& c) {
    if (c.tile_cull_warps != 1 && c.tile_cull_warps != 2 && c.tile_cull_warps != 4 && c.tile_cull_warps != 8)
        return fail(HVVR_ERR_INVALID, "tile_cull_warps must be 1, 2, 4 or 8");
    const uint64_t chunks = (c.tri_index_capacity + kChunk - 1) / kChunk;
    if (c.tri_index_capacity == 0 || chunks > 0xfffffff0ull) return fail(HVVR_ERR_INVALID, "bad tri_index_capacity");
    if (c.tile_stack_entries && (c.tile_stack_entries < 8 || c.tile_stack_entries > kTileStack))
        return fail(HVVR_ERR_INVALID, "tile_stack_entries must be 0 or in [8, 256]");
    if (c.timing > 1) return fail(HVVR_ERR_INVALID, "timing must be 0 or 1");
    if (c.pipeline > 1) return fail(HVVR_ERR_INVALID, "pipeline must be 0 or 1");
    if (c.tile_cull_persistent > 1) return fail(HVVR_ERR_INVALID, "tile_cull_persistent must be 0 or 1");
    return HVVR_OK;
}

void dropGraph(hvvr_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graphKey.clear();
}

// The side streams of the rate classes that this frame renders, made on first use: the device has a
// fixed number of hardware work queues (CUDA_DEVICE_MAX_CONNECTIONS, 8 unless the process sets more
// before CUDA starts) that all streams share, so a batch keeps no idle streams, and streams of
// different priorities (a server's latency and throughput slots) share a queue as rarely as the
// count allows.
int ensureSideStreams(hvvr_batch* b) {
    int leastPriority = 0, greatestPriority = 0;
    for (uint32_t r = 0; r < kRateClasses; r++) {
        if (!b->rateTiles[r]) continue;
        // the heavy part's stream only where a heavy part can run
        const bool heavy = b->cfg.heavy_divisor != 0 && !(r >= 6 && r < 12);
        if (b->side[2 * r + 1] && (b->side[2 * r] || !heavy)) continue;
        if (leastPriority == 0 && greatestPriority == 0)
            CUDA_TRY(cudaDeviceGetStreamPriorityRange(&leastPriority, &greatestPriority));
        const int heavyPrio = b->streamPriorities == 2 ? leastPriority : greatestPriority;
        const int restPrio = b->streamPriorities == 1 ? greatestPriority : leastPriority;
        if (heavy && !b->side[2 * r])
            CUDA_TRY(cudaStreamCreateWithPriority(&b->side[2 * r], cudaStreamNonBlocking, heavyPrio));
        if (!b->side[2 * r + 1])
            CUDA_TRY(cudaStreamCreateWithPriority(&b->side[2 * r + 1], cudaStreamNonBlocking, restPrio));
    }
    return HVVR_OK;
}

int batchResources(hvvr_batch* b) {
    if (!b->forkEv) {
        CUDA_TRY(cudaEventCreateWithFlags(&b->rankEv, cudaEventDisableTiming));
        for (auto& e : b->cullEv) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&b->forkEv, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&b->orderForkEv, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&b->orderDoneEv, cudaEventDisableTiming));
        for (auto& e : b->doneEv) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (auto& e : b->hostViewsEv) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (auto& e : b->ev) CUDA_TRY(cudaEventCreate(&e));
        for (auto& k : b->kev)
            for (auto& e : k) CUDA_TRY(cudaEventCreate(&e));
        CUDA_TRY(cudaMallocHost((void**)&b->hostCounters, kCounterWords * sizeof(uint32_t)));
        memset(b->hostCounters, 0, kCounterWords * sizeof(uint32_t));
    }
    const uint64_t chunks = (b->cfg.tri_index_capacity + kChunk - 1) / kChunk;
    if (b->chunkNext.n != chunks) {
        b->chunkNext.release();
        b->pool.release();
        TRY(b->pool.alloc(size_t(chunks) * kChunk));
        TRY(b->chunkNext.alloc(size_t(chunks)));
        b->poolChunks = uint32_t(chunks);
        dropGraph(b);
    }
    TRY(b->counters.alloc(kCounterWords));
    return HVVR_OK;
}

void releaseBatch(hvvr_batch* b) {
    dropGraph(b);
    for (auto& t : b->side)
        if (t) cudaStreamDestroy(t), t = nullptr;
    for (cudaEvent_t* e : {&b->forkEv, &b->orderForkEv, &b->orderDoneEv})
        if (*e) cudaEventDestroy(*e), *e = nullptr;
    for (auto& e : b->doneEv)
        if (e) cudaEventDestroy(e), e = nullptr;
    for (auto& e : b->cullEv)
        if (e) cudaEventDestroy(e), e = nullptr;
    if (b->rankEv) cudaEventDestroy(b->rankEv), b->rankEv = nullptr;
    for (auto& e : b->hostViewsEv)
        if (e) cudaEventDestroy(e), e = nullptr;
    for (auto& e : b->ev)
        if (e) cudaEventDestroy(e), e = nullptr;
    for (auto& k : b->kev)
        for (auto& e : k)
            if (e) cudaEventDestroy(e), e = nullptr;
    for (auto& h : b->hostViews)
        if (h) cudaFreeHost(h), h = nullptr;
    if (b->hostCounters) cudaFreeHost(b->hostCounters), b->hostCounters = nullptr;
}

int checkStatus(const hvvr_batch* b) {
    if (!b || !b->counterValid || !b->hostCounters) return HVVR_OK;
    const uint32_t s = b->hostCounters[1];
    if (s & kStatusPoolOverflow)
        return fail(HVVR_ERR_OVERFLOW, "triangle-index pool exhausted (%u chunks); raise tri_index_capacity",
                    b->poolChunks);
    if (s & kStatusStackOverflow) return fail(HVVR_ERR_OVERFLOW, "tile traversal stack exhausted");
    if (s & kStatusBadLeaf) return fail(HVVR_ERR_INVALID, "BVH leaf with an empty triangle range passed the cull");
    if (s & kStatusPipelineTimeout)
        return fail(HVVR_ERR_TIMEOUT, "intersect/shade gave up waiting for a tile's list (cull -> shade pipeline)");
    return HVVR_OK;
}

uint32_t heavyTiles(const hvvr_batch* b, uint32_t n) {
    if (!b->costValid || !b->cfg.heavy_divisor || n < kSplitMinTiles) return 0;
    return std::max<uint32_t>(1u, n / b->cfg.heavy_divisor);
}

// a stage-timing event: inside a stream capture it must be recorded as an external event so
// that the graph records it on every replay (a plain record only orders the capture)
cudaError_t recordStage(cudaEvent_t ev, cudaStream_t s, bool capturing) {
    return capturing ? cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal) : cudaEventRecord(ev, s);
}

// Enqueues one frame on st (and the side streams, forked from and joined back to st), recording
// the stage and per-part events (as graph nodes when capturing).
int enqueueFrame(hvvr_batch* b, const FrameDev& fr, cudaStream_t st, bool capturing) {
    const bool stages = b->cfg.timing != 0;
    CUDA_TRY(recordStage(b->ev[0], st, capturing));
    CUDA_TRY(cudaMemsetAsync(fr.counters, 0, kCounterWords * sizeof(uint32_t), st));
    if (b->cfg.pipeline && fr.tiles) CUDA_TRY(cudaMemsetAsync(fr.ready, 0xff, size_t(fr.tiles) * sizeof(uint32_t), st));
    // The tile order reads only last frame's costs, so it runs beside the block cull, and the tile
    // culls wait for both. It borrows the side stream of the first rate class (heavy part's if
    // there is one): idle at the top of the frame, it has the priority the batch gives its culls
    // (a latency-class batch's order must not queue behind other batches' work), and it adds no
    // stream to share the device's hardware queues.
    cudaStream_t os = st;
    for (uint32_t r = 0; r < kRateClasses; r++) {
        if (!b->rateTiles[r]) continue;
        cudaStream_t c = b->side[2 * r] ? b->side[2 * r] : b->side[2 * r + 1];
        if (c) os = c;
        break;
    }
    if (os != st) {
        CUDA_TRY(cudaEventRecord(b->orderForkEv, st));
        CUDA_TRY(cudaStreamWaitEvent(os, b->orderForkEv, 0));
    }
    CUDA_TRY(launchTileOrder(fr, os));
    if (os != st) CUDA_TRY(cudaEventRecord(b->orderDoneEv, os));
    CUDA_TRY(launchBlockCull(fr, st));
    if (stages) CUDA_TRY(recordStage(b->ev[1], st, capturing));
    if (os != st) CUDA_TRY(cudaStreamWaitEvent(st, b->orderDoneEv, 0));
    CUDA_TRY(cudaEventRecord(b->forkEv, st));
    bool first = true;
    for (auto& u : b->kevUsed) u = false;
    for (auto& u : b->kevPipelined) u = false;
    // Pinhole classes: per part, tile cull then intersect on the part's stream, or (config.pipeline)
    // one cull -> shade pipeline per part. Thin-lens classes (one part each) need the occupied-tile
    // ranks of the whole view, so all their culls finish before one rank launch, and their
    // intersects follow it.
    for (uint32_t r = 0; r < kRateClasses; r++) {
        const uint32_t n = b->rateTiles[r];
        if (!n) continue;
        const bool lens = r >= 6 && r < 12;
        const uint32_t pattern = r >= 12 ? 1u : 0u;
        const uint32_t rs = b->rateStart[r], heavy = lens ? 0u : heavyTiles(b, n), msaa = 1u << (r % 6);
        // part 0: last frame's slowest tiles on the high-priority stream; part 1: the rest
        for (uint32_t part = heavy ? 0u : 1u; part < 2; part++) {
            const uint32_t k = 2 * r + part;
            const uint32_t p0 = part ? rs + heavy : rs, pn = part ? n - heavy : heavy;
            cudaStream_t ps = b->side[k];
            CUDA_TRY(cudaStreamWaitEvent(ps, b->forkEv, 0));
            if (stages) CUDA_TRY(recordStage(b->kev[k][0], ps, capturing));
            if (!lens && b->cfg.pipeline) {
                // the class's first part holds its longest tiles: those stream their lists
                FrameDev fp = fr;
                fp.streamTiles = part == (heavy ? 0u : 1u) ? b->cfg.stream_tiles : 0u;
                CUDA_TRY(launchCullShadePipeline(fp, msaa, pattern, b->fpStrict, p0, pn, fr.counters + kQueueBase + kQueueWords * k,
                                                 fr.counters + kPipeBase + k, b->cfg.tile_cull_warps,
                                                 b->cfg.tile_stack_entries, ps));
                // the cull and the shade overlap: one event marks the end of both (and of the retry
                // passes); no event sits between the two launches, which would serialise them
                if (stages) {
                    CUDA_TRY(recordStage(b->kev[k][1], ps, capturing));
                    CUDA_TRY(recordStage(b->kev[k][2], ps, capturing));
                    if (part == 1 && first) CUDA_TRY(recordStage(b->ev[2], ps, capturing));
                }
                b->kevUsed[k] = true;
                b->kevPipelined[k] = true;
                CUDA_TRY(cudaEventRecord(b->doneEv[k], ps));
                CUDA_TRY(cudaStreamWaitEvent(st, b->doneEv[k], 0));
                continue;
            }
            CUDA_TRY(launchTileCull(fr, fr.order, p0, pn, fr.counters + kQueueBase + kQueueWords * k,
                                    b->cfg.tile_cull_warps, b->cfg.tile_stack_entries, ps));
            if (stages) CUDA_TRY(recordStage(b->kev[k][1], ps, capturing));
            if (stages && part == 1 && first) CUDA_TRY(recordStage(b->ev[2], ps, capturing));
            if (lens) {
                CUDA_TRY(cudaEventRecord(b->cullEv[k], ps));
                continue;
            }
            CUDA_TRY(launchIntersectShade(fr, msaa, pattern, b->fpStrict, false, fr.order, p0, pn, ps));
            if (stages) CUDA_TRY(recordStage(b->kev[k][2], ps, capturing));
            b->kevUsed[k] = true;
            CUDA_TRY(cudaEventRecord(b->doneEv[k], ps));
            CUDA_TRY(cudaStreamWaitEvent(st, b->doneEv[k], 0));
        }
        first = false;
    }
    if (b->anyLens) {
        for (uint32_t r = 6; r < 12; r++)
            if (b->rateTiles[r]) CUDA_TRY(cudaStreamWaitEvent(st, b->cullEv[2 * r + 1], 0));
        CUDA_TRY(launchOccupiedRank(fr, st));
        CUDA_TRY(cudaEventRecord(b->rankEv, st));
        for (uint32_t r = 6; r < 12; r++) {
            const uint32_t n = b->rateTiles[r];
            if (!n) continue;
            const uint32_t k = 2 * r + 1;
            cudaStream_t ps = b->side[k];
            CUDA_TRY(cudaStreamWaitEvent(ps, b->rankEv, 0));
            CUDA_TRY(launchIntersectShade(fr, 1u << (r % 6), 0, b->fpStrict, true, fr.order, b->rateStart[r], n, ps));
            if (stages) CUDA_TRY(recordStage(b->kev[k][2], ps, capturing));
            b->kevUsed[k] = true;
            CUDA_TRY(cudaEventRecord(b->doneEv[k], ps));
            CUDA_TRY(cudaStreamWaitEvent(st, b->doneEv[k], 0));
        }
    }
    if (stages) CUDA_TRY(recordStage(b->ev[3], st, capturing));
    for (uint32_t i = 0; i < b->views.size(); i++) {
        const hvvr_camera* c = b->views[i].cam;
        if (c->foveated) CUDA_TRY(launchFoveatedResolve(fr, i, c->fovStatic, st));
        else CUDA_TRY(launchRemap(c->dev, st));
    }
    if (stages) CUDA_TRY(recordStage(b->ev[4], st, capturing));
    CUDA_TRY(cudaMemcpyAsync(b->hostCounters, fr.counters, kCounterWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    for (const auto& v : b->views) {
        const hvvr_camera* c = v.cam;
        const CameraDev& d = c->dev;
        if (c->target.memory_type == HVVR_MEMORY_CPU && c->target.data && d.image && d.width && d.height) {
            const uint64_t stride = c->target.stride ? c->target.stride : d.width;
            CUDA_TRY(cudaMemcpy2DAsync(c->target.data, stride * 4, d.image, size_t(d.width) * 4, size_t(d.width) * 4,
                                       d.height, cudaMemcpyDeviceToHost, st));
        }
    }
    CUDA_TRY(recordStage(b->ev[5], st, capturing));
    return HVVR_OK;
}

int reserveBatch(hvvr_batch* b, size_t tiles, size_t blocks, size_t views) {
    TRY(b->blockView.ensure(blocks));
    TRY(b->order.ensure(tiles));
    TRY(b->retry.ensure(tiles));
    TRY(b->ready.ensure(tiles));
    TRY(b->viewsDev.ensure(views));
    if (b->hostViewsCap < views) {
        for (int k = 0; k < 2; k++) {
            if (b->hostViewsUsed[k]) CUDA_TRY(cudaEventSynchronize(b->hostViewsEv[k]));
            if (b->hostViews[k]) cudaFreeHost(b->hostViews[k]);
            b->hostViews[k] = nullptr;
            b->hostViewsUsed[k] = false;
        }
        b->hostViewsCap = 0;
        for (int k = 0; k < 2; k++) CUDA_TRY(cudaMallocHost((void**)&b->hostViews[k], views * sizeof(ViewDev)));
        b->hostViewsCap = views;
    }
    return HVVR_OK;
}

// Scene update and refit of every raycaster, then one frame of all their enabled cameras.
int renderBatch(hvvr_batch* b, cudaStream_t st, bool skipScenes) {
    if (b->detached) return fail(HVVR_ERR_STATE, "a raycaster of this batch was destroyed");
    if (b->rcs.empty()) return HVVR_OK;
    const int device = b->rcs[0]->spec.device;
    const bool strict = b->rcs[0]->spec.fp_mode == HVVR_FP_STRICT;
    CUDA_TRY(cudaSetDevice(device));
    for (hvvr_raycaster* rc : b->rcs) {
        if (rc->spec.device != device) return fail(HVVR_ERR_INVALID, "batched raycasters must share one device");
        if ((rc->spec.fp_mode == HVVR_FP_STRICT) != strict)
            return fail(HVVR_ERR_INVALID, "batched raycasters must share one fp_mode");
        if (skipScenes) continue;
        if (rc->sceneDirty) {
            TRY(uploadScene(rc, st));
            rc->sceneDirty = false;
            rc->refitDirty = true;
        }
        if (rc->scene.nodeCount && rc->refitDirty) {
            CUDA_TRY(launchRefit(rc->scene, rc->spec.fp_mode == HVVR_FP_FMA, st));
            rc->refitDirty = false;
        }
    }
    std::vector<hvvr_camera*> candidates, cams;
    if (b->fixedViews) {
        candidates = b->cams;
    } else {
        for (hvvr_raycaster* rc : b->rcs)
            for (auto& cp : rc->cameras)
                if (!cp->hidden) candidates.push_back(cp.get());
    }
    bool cpuTargets = false, capturable = true;
    {
        for (hvvr_camera* c : candidates) {
            hvvr_raycaster* rc = c->rc;
            if (rc->scene.nodeCount == 0 || !c->enabled || c->samples.empty()) continue;
            if (c->setupDirty) TRY(setupCamera(c, st));
            TRY(ensureMsaaTable(c->msaa, st));
            CameraDev& d = c->dev;
            d.msaa = c->msaa;
            if (c->capture & HVVR_CAPTURE_HITS) {
                TRY(c->hitIds.alloc(size_t(d.padded) * d.msaa));
                TRY(c->depth.alloc(size_t(d.padded) * d.msaa));
                d.hitIds = c->hitIds.p;
                d.depth = c->depth.p;
            } else {
                d.hitIds = nullptr;
                d.depth = nullptr;
            }
            if (hasLens(c)) {
                if (c->lensRate != c->msaa || !c->lensPos.p) {
                    std::vector<float> tab(size_t(kTileSize) * 4 * c->msaa * 2);
                    lensTable(c->msaa, tab.data());
                    TRY(c->lensPos.upload(tab.data(), tab.size() / 2, st));
                    CUDA_TRY(cudaStreamSynchronize(st)); // the host table goes out of scope
                    c->lensRate = c->msaa;
                }
                TRY(c->occRank.alloc(d.tiles));
            }
            if (c->target.memory_type == HVVR_MEMORY_CPU && c->target.data) {
                cpuTargets = true;
                if (!c->registered) capturable = false; // pageable copies cannot be captured
            }
            cams.push_back(c);
        }
    }
    if (cams.empty()) return HVVR_OK;
    TRY(batchResources(b));

    std::vector<uint64_t> key;
    for (const hvvr_camera* c : cams) {
        const uint64_t k[] = {uint64_t(uintptr_t(c)), c->setupGen, c->msaa, uint64_t(uintptr_t(c->dev.hitIds)),
                              uint64_t(uintptr_t(c->target.data)), c->target.memory_type, c->target.stride,
                              uint64_t(uintptr_t(c->registered)), uint64_t(hasLens(c)),
                              uint64_t(uintptr_t(c->lensPos.p)), uint64_t(uintptr_t(c->occRank.p))};
        key.insert(key.end(), k, k + 11);
    }
    if (key != b->layoutKey) {
        b->views.clear();
        b->tiles = b->blocks = 0;
        uint32_t rateTiles[kRateClasses] = {};
        std::vector<uint32_t> blockView;
        b->anyLens = false;
        for (const hvvr_camera* c : cams) {
            rateTiles[rateClass(c)] += c->dev.tiles;
            b->anyLens = b->anyLens || hasLens(c);
        }
        for (uint32_t i = 0; i < cams.size(); i++) {
            hvvr_camera* c = cams[i];
            b->views.push_back(hvvr_batch::View{c, b->tiles, b->blocks});
            blockView.insert(blockView.end(), c->dev.blocks, i);
            b->tiles += c->dev.tiles;
            b->blocks += c->dev.blocks;
        }
        uint32_t run = 0;
        for (uint32_t r = 0; r < kRateClasses; r++) {
            b->rateTiles[r] = rateTiles[r];
            b->rateStart[r] = run;
            run += rateTiles[r];
        }
        TRY(reserveBatch(b, b->tiles, b->blocks, b->views.size()));
        CUDA_TRY(cudaMemcpyAsync(b->blockView.p, blockView.data(), blockView.size() * 4, cudaMemcpyHostToDevice, st));
        b->layoutKey = key;
        // scheduling by last frame's cost needs a previous frame of every camera in the layout
        b->costValid = std::all_of(cams.begin(), cams.end(), [](const hvvr_camera* c) { return c->costFrames > 0; });
        dropGraph(b);
    }
    TRY(ensureSideStreams(b));
    b->fpStrict = strict;

    // this frame's view table (transforms, scene pointers), staged in pinned memory that the
    // frame before last has finished reading
    const int slot = b->hostSlot;
    b->hostSlot ^= 1;
    if (b->hostViewsUsed[slot]) CUDA_TRY(cudaEventSynchronize(b->hostViewsEv[slot]));
    ViewDev* hv = b->hostViews[slot];
    // scenes whose BVH nodes the block-cull launch prefetches into L2, at most half of a B200's
    // 126 MB L2 per frame (a served batch over several large scenes would only evict its own lines)
    std::vector<const Node*> prefetched;
    size_t prefetchBytes = 0;
    constexpr size_t kPrefetchBudget = size_t(64) << 20;
    for (size_t i = 0; i < b->views.size(); i++) {
        const hvvr_camera* c = b->views[i].cam;
        const SceneDev& sc = c->rc->scene;
        const CameraDev& d = c->dev;
        ViewDev v{};
        v.M = transformToMatrix(c->xf);
        v.env = sc.env;
        v.nodes = sc.nodes;
        if (sc.nodes && std::find(prefetched.begin(), prefetched.end(), sc.nodes) == prefetched.end() &&
            prefetchBytes + size_t(sc.nodeCount) * sizeof(Node) <= kPrefetchBudget) {
            v.prefetchNodes = sc.nodeCount;
            prefetched.push_back(sc.nodes);
            prefetchBytes += size_t(sc.nodeCount) * sizeof(Node);
        }
        v.tris = sc.tris;
        v.triShade = sc.triShade;
        v.verts = sc.verts;
        v.materials = sc.materials;
        v.textures = sc.textures;
        v.textureCount = sc.textureCount;
        v.tileRays = d.tileRays;
        v.blockRays = d.blockRays;
        v.beams = d.beams;
        v.blockStacks = d.blockStacks;
        v.blockSizes = d.blockSizes;
        v.tileLists = d.tileLists;
        v.tileCost = d.tileCost;
        v.colors = d.colors;
        v.hitIds = d.hitIds;
        v.depth = d.depth;
        v.tileStart = b->views[i].tileStart;
        v.blockStart = b->views[i].blockStart;
        v.msaa = c->msaa;
        v.rateIdx = rateClass(c);
        v.lensRadius = hasLens(c) ? c->lens.radius : 0.0f;
        v.focalDistance = c->lens.focal_distance;
        v.lensPos = hasLens(c) ? c->lensPos.p : nullptr;
        v.occRank = hasLens(c) ? c->occRank.p : nullptr;
        if (c->foveated) {
            hvvr_camera* cm = b->views[i].cam;
            float c2w[16];
            memcpy(c2w, &v.M, sizeof(c2w));
            foveatedFrame(c2w, c->eyeDir, c->sampleBounds, c->viewport, cm->eyeToWorld, cm->cullPlanes);
            memcpy(&v.M, cm->eyeToWorld, sizeof(v.M));
            memcpy(v.cull, cm->cullPlanes, sizeof(v.cull));
            v.hasCull = 1;
            v.tmaxOut = c->tmax.p;
            if (cm->fovStatic.image) {
                // resolve into fovResult[fovCur] against the other buffer (the previous frame's
                // result), then swap (GPUCamera::foveatedPolarToScreenSpace's std::swap)
                v.fov = cm->fovStatic;
                foveatedResolveFrame(cm->eyeToWorld, c->eyeDir, c->viewport, cm->worldToEyePrev,
                                     cm->eyePrevToSamplePrev, v.fov.sampleToEye, v.fov.eyeToSamplePrev);
                memcpy(cm->lastSampleToEye, v.fov.sampleToEye, sizeof(cm->lastSampleToEye));
                memcpy(cm->lastEyeToSamplePrev, v.fov.eyeToSamplePrev, sizeof(cm->lastEyeToSamplePrev));
                v.fov.resultTex = cm->fovResult[cm->fovCur].tex;
                v.fov.resultSurf = cm->fovResult[cm->fovCur].surf;
                v.fov.prevTex = cm->fovResult[cm->fovCur ^ 1u].tex;
                cm->fovCur ^= 1u;
            }
        }
        hv[i] = v;
    }
    CUDA_TRY(cudaMemcpyAsync(b->viewsDev.p, hv, b->views.size() * sizeof(ViewDev), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaEventRecord(b->hostViewsEv[slot], st));
    b->hostViewsUsed[slot] = true;

    FrameDev fr;
    fr.views = b->viewsDev.p;
    fr.blockView = b->blockView.p;
    fr.viewCount = uint32_t(b->views.size());
    fr.tiles = b->tiles;
    fr.blocks = b->blocks;
    fr.pool = b->pool.p;
    fr.chunkNext = b->chunkNext.p;
    fr.poolChunks = b->poolChunks;
    fr.counters = b->counters.p;
    fr.order = b->order.p;
    fr.retry = b->retry.p;
    fr.ready = b->ready.p;
    fr.cullCtasPerSm = b->cfg.tile_cull_ctas_per_sm;
    fr.cullPersistent = b->cfg.tile_cull_persistent;
    if (b->cfg.use_graph && b->costValid && capturable) {
        std::vector<uint64_t> gkey = b->layoutKey;
        const uint64_t extra[] = {b->cfg.tile_cull_warps, b->cfg.heavy_divisor, b->poolChunks, strict ? 1u : 0u,
                                  uint64_t(uintptr_t(st)), b->cfg.tile_stack_entries, b->cfg.timing,
                                  b->cfg.pipeline, b->cfg.tile_cull_ctas_per_sm, b->cfg.tile_cull_persistent,
                                  b->cfg.stream_tiles};
        gkey.insert(gkey.end(), std::begin(extra), std::end(extra));
        if (!b->graph || gkey != b->graphKey) {
            dropGraph(b);
            CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
            const int r = enqueueFrame(b, fr, st, true);
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(st, &g);
            if (r != HVVR_OK) {
                if (g) cudaGraphDestroy(g);
                return r;
            }
            CUDA_TRY(e);
            const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) b->graph = nullptr;
            CUDA_TRY(ie);
            b->graphKey = gkey;
        }
        CUDA_TRY(cudaGraphLaunch(b->graph, st));
    } else {
        TRY(enqueueFrame(b, fr, st, false));
    }
    b->stageTimes = b->cfg.timing != 0;
    for (hvvr_camera* c : cams) {
        c->lastBatch = b;
        c->rendered = true;
        c->costFrames++;
    }
    b->costValid = true; // the next frame schedules its tiles by this frame's visit counts
    b->counterValid = true;
    if (cpuTargets) {
        CUDA_TRY(cudaStreamSynchronize(st));
        TRY(checkStatus(b));
    }
    return HVVR_OK;
}

} // namespace hvb

extern "C" {

const char* hvvr_last_error(void) { return gLastError.empty() ? kEmpty : gLastError.c_str(); }
int hvvr_version(void) { return 10000; }

void hvvr_spec_default(hvvr_spec* spec) {
    if (!spec) return;
    memset(spec, 0, sizeof(*spec));
    spec->mode = HVVR_MODE_DEFERRED_MSAA_RESOLVE;
    spec->foveated_degree_tracking_error = 0.5f;
    spec->foveated_max_fov_degrees = 110.0f;
    spec->foveated_mar_slope = 0.022f;
    spec->foveated_foveal_mar_degrees = 1.0f / 60.0f;
    spec->fp_mode = HVVR_FP_FMA;
}

int hvvr_raycaster_create(const hvvr_spec* spec, hvvr_raycaster** out) {
    if (!out) return fail(HVVR_ERR_INVALID, "out is NULL");
    *out = nullptr;
    hvvr_spec s;
    if (spec) s = *spec;
    else hvvr_spec_default(&s);
    if (s.output_to_3d_api) return fail(HVVR_ERR_INVALID, "output to a 3D API is not available: no graphics stack");
    if (s.mode != HVVR_MODE_DEFERRED_MSAA_RESOLVE && s.mode != HVVR_MODE_FOVEATED_POLAR)
        return fail(HVVR_ERR_INVALID, "unknown mode");
    if (s.fp_mode != HVVR_FP_FMA && s.fp_mode != HVVR_FP_STRICT) return fail(HVVR_ERR_INVALID, "bad fp_mode");
    if (s.sample_setup != HVVR_SETUP_DEVICE && s.sample_setup != HVVR_SETUP_HOST)
        return fail(HVVR_ERR_INVALID, "bad sample_setup");
    if (s.bvh_build != HVVR_BVH_HOST && s.bvh_build != HVVR_BVH_DEVICE) return fail(HVVR_ERR_INVALID, "bad bvh_build");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return fail(HVVR_ERR_CUDA, "no CUDA device available");
    if (s.device < 0 || s.device >= count) return fail(HVVR_ERR_INVALID, "device %d out of range", s.device);
    CUDA_TRY(cudaSetDevice(s.device));
    auto rc = std::make_unique<hvvr_raycaster>();
    rc->spec = s;
    CUDA_TRY(cudaStreamCreateWithFlags(&rc->stream, cudaStreamNonBlocking));
    *out = rc.release();
    return HVVR_OK;
}

int hvvr_raycaster_destroy(hvvr_raycaster* rc) {
    if (!rc) return fail(HVVR_ERR_INVALID, "NULL raycaster");
    cudaSetDevice(rc->spec.device);
    cudaStreamSynchronize(rc->stream);
    cudaDeviceSynchronize();
    for (hvvr_batch* b : rc->batches) {
        // the batch stays a valid handle (destroy still works) but can no longer render
        b->detached = true;
        for (hvvr_raycaster* other : b->rcs) {
            if (other == rc) continue;
            other->batches.erase(std::remove(other->batches.begin(), other->batches.end(), b), other->batches.end());
            for (auto& c : other->cameras) {
                if (c->lastBatch == b) c->lastBatch = nullptr;
                c->batches.erase(std::remove(c->batches.begin(), c->batches.end(), b), c->batches.end());
            }
        }
        b->rcs.clear();
        b->cams.clear();
    }
    for (auto& c : rc->cameras) releaseCamera(c.get());
    if (rc->own) releaseBatch(rc->own.get());
    cudaStreamDestroy(rc->stream);
    delete rc;
    return HVVR_OK;
}

int hvvr_raycaster_set_scene_dirty(hvvr_raycaster* rc) {
    if (!rc) return fail(HVVR_ERR_INVALID, "NULL raycaster");
    rc->sceneDirty = true;
    return HVVR_OK;
}

// the raycaster's own batch (made on first use)
hvvr_batch* ownBatch(hvvr_raycaster* rc) {
    if (!rc->own) {
        rc->own = std::make_unique<hvvr_batch>();
        hvvr_batch* b = rc->own.get();
        b->rcs.push_back(rc);
        b->internal = true;
        batchConfigDefault(&b->cfg);
        if (rc->spec.tri_index_capacity) b->cfg.tri_index_capacity = rc->spec.tri_index_capacity;
    }
    return rc->own.get();
}

int hvvr_raycaster_render(hvvr_raycaster* rc, double elapsed_time, void* stream) {
    (void)elapsed_time;
    if (!rc) return fail(HVVR_ERR_INVALID, "NULL raycaster");
    return renderBatch(ownBatch(rc), stream ? static_cast<cudaStream_t>(stream) : rc->stream);
}

int hvvr_raycaster_get_batch_config(hvvr_raycaster* rc, hvvr_batch_config* cfg) {
    if (!rc || !cfg) return fail(HVVR_ERR_INVALID, "NULL argument");
    *cfg = ownBatch(rc)->cfg;
    return HVVR_OK;
}

int hvvr_raycaster_set_batch_config(hvvr_raycaster* rc, const hvvr_batch_config* cfg) {
    if (!rc || !cfg) return fail(HVVR_ERR_INVALID, "NULL argument");
    TRY(checkConfig(*cfg));
    ownBatch(rc)->cfg = *cfg; // the pool follows tri_index_capacity on the next frame
    return HVVR_OK;
}

int hvvr_raycaster_synchronize(hvvr_raycaster* rc) {
    if (!rc) return fail(HVVR_ERR_INVALID, "NULL raycaster");
    CUDA_TRY(cudaSetDevice(rc->spec.device));
    CUDA_TRY(cudaStreamSynchronize(rc->stream));
    CUDA_TRY(cudaDeviceSynchronize());
    return checkStatus(rc->own.get());
}

void hvvr_batch_config_default(hvvr_batch_config* cfg) {
    if (cfg) batchConfigDefault(cfg);
}

int hvvr_batch_create(hvvr_raycaster* const* raycasters, uint32_t count, const hvvr_batch_config* cfg,
                      hvvr_batch** out) {
    if (!out) return fail(HVVR_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!raycasters || count == 0) return fail(HVVR_ERR_INVALID, "no raycasters");
    for (uint32_t i = 0; i < count; i++) {
        if (!raycasters[i]) return fail(HVVR_ERR_INVALID, "NULL raycaster %u", i);
        for (uint32_t k = 0; k < i; k++)
            if (raycasters[k] == raycasters[i]) return fail(HVVR_ERR_INVALID, "raycaster %u listed twice", i);
        if (raycasters[i]->spec.device != raycasters[0]->spec.device)
            return fail(HVVR_ERR_INVALID, "batched raycasters must share one device");
        if (raycasters[i]->spec.fp_mode != raycasters[0]->spec.fp_mode)
            return fail(HVVR_ERR_INVALID, "batched raycasters must share one fp_mode");
    }
    auto b = std::make_unique<hvvr_batch>();
    batchConfigDefault(&b->cfg);
    if (cfg) {
        b->cfg = *cfg;
        TRY(checkConfig(b->cfg));
    }
    b->rcs.assign(raycasters, raycasters + count);
    for (hvvr_raycaster* rc : b->rcs) rc->batches.push_back(b.get());
    *out = b.release();
    return HVVR_OK;
}

int hvvr_batch_create_views(hvvr_camera* const* cameras, uint32_t count, const hvvr_batch_config* cfg,
                            hvvr_batch** out) {
    if (!out) return fail(HVVR_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!cameras || count == 0) return fail(HVVR_ERR_INVALID, "no cameras");
    auto b = std::make_unique<hvvr_batch>();
    batchConfigDefault(&b->cfg);
    if (cfg) {
        b->cfg = *cfg;
        TRY(checkConfig(b->cfg));
    }
    for (uint32_t i = 0; i < count; i++) {
        hvvr_camera* c = cameras[i];
        if (!c) return fail(HVVR_ERR_INVALID, "NULL camera %u", i);
        if (std::find(b->cams.begin(), b->cams.end(), c) != b->cams.end())
            return fail(HVVR_ERR_INVALID, "camera %u listed twice", i);
        hvvr_raycaster* rc = c->rc;
        if (rc->spec.device != cameras[0]->rc->spec.device)
            return fail(HVVR_ERR_INVALID, "batched cameras must share one device");
        if (rc->spec.fp_mode != cameras[0]->rc->spec.fp_mode)
            return fail(HVVR_ERR_INVALID, "batched cameras must share one fp_mode");
        b->cams.push_back(c);
        if (std::find(b->rcs.begin(), b->rcs.end(), rc) == b->rcs.end()) b->rcs.push_back(rc);
    }
    b->fixedViews = true;
    for (hvvr_raycaster* rc : b->rcs) rc->batches.push_back(b.get());
    for (hvvr_camera* c : b->cams) c->batches.push_back(b.get());
    *out = b.release();
    return HVVR_OK;
}

int hvvr_batch_destroy(hvvr_batch* b) {
    if (!b || b->internal) return fail(HVVR_ERR_INVALID, "not a batch");
    if (!b->rcs.empty()) cudaSetDevice(b->rcs[0]->spec.device);
    cudaDeviceSynchronize();
    for (hvvr_raycaster* rc : b->rcs) {
        rc->batches.erase(std::remove(rc->batches.begin(), rc->batches.end(), b), rc->batches.end());
        for (auto& c : rc->cameras) {
            if (c->lastBatch == b) c->lastBatch = nullptr;
            c->batches.erase(std::remove(c->batches.begin(), c->batches.end(), b), c->batches.end());
        }
    }
    releaseBatch(b);
    delete b;
    return HVVR_OK;
}

int hvvr_batch_render(hvvr_batch* b, double elapsed_time, void* stream) {
    (void)elapsed_time;
    if (!b || b->internal) return fail(HVVR_ERR_INVALID, "not a batch");
    if (b->detached || b->rcs.empty()) return fail(HVVR_ERR_STATE, "a raycaster of this batch was destroyed");
    return renderBatch(b, stream ? static_cast<cudaStream_t>(stream) : b->rcs[0]->stream);
}

int hvvr_batch_synchronize(hvvr_batch* b) {
    if (!b || b->internal) return fail(HVVR_ERR_INVALID, "not a batch");
    if (b->detached || b->rcs.empty()) return fail(HVVR_ERR_STATE, "a raycaster of this batch was destroyed");
    CUDA_TRY(cudaSetDevice(b->rcs[0]->spec.device));
    CUDA_TRY(cudaDeviceSynchronize());
    return checkStatus(b);
}

int hvvr_batch_get_config(const hvvr_batch* b, hvvr_batch_config* cfg) {
    if (!b || !cfg) return fail(HVVR_ERR_INVALID, "NULL argument");
    *cfg = b->cfg;
    return HVVR_OK;
}

int hvvr_batch_set_config(hvvr_batch* b, const hvvr_batch_config* cfg) {
    if (!b || !cfg || b->internal) return fail(HVVR_ERR_INVALID, "NULL argument");
    TRY(checkConfig(*cfg));
    b->cfg = *cfg;
    return HVVR_OK;
}

int hvvr_batch_read_timings(const hvvr_batch* b, float* ms5) {
    if (!b || !ms5) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (!b->counterValid) return fail(HVVR_ERR_STATE, "the batch has not rendered a frame");
    CUDA_TRY(cudaEventSynchronize(b->ev[5]));
    CUDA_TRY(cudaEventElapsedTime(&ms5[0], b->ev[0], b->ev[5]));
    for (int i = 1; i < 5; i++) {
        ms5[i] = 0.0f;
        if (b->stageTimes) CUDA_TRY(cudaEventElapsedTime(&ms5[i], b->ev[i == 4 ? 3 : i - 1], b->ev[i == 4 ? 5 : i]));
    }
    return HVVR_OK;
}

namespace {
int kernelTimes(const hvvr_batch* b, float* ms4) {
    if (!b || !b->counterValid) return fail(HVVR_ERR_STATE, "no frame rendered");
    if (!b->stageTimes) return fail(HVVR_ERR_STATE, "the last frame was rendered without per-launch events (config.timing = 0)");
    CUDA_TRY(cudaEventSynchronize(b->ev[5]));
    float cull = 0.0f, isect = 0.0f, t = 0.0f;
    for (uint32_t k = 0; k < 2 * kRateClasses; k++) {
        if (!b->kevUsed[k]) continue;
        if (b->kevPipelined[k]) {
            // cull and shade overlap: the span of the pipeline counts as intersect/shade time
            CUDA_TRY(cudaEventElapsedTime(&t, b->kev[k][0], b->kev[k][2]));
            isect += t;
            continue;
        }
        CUDA_TRY(cudaEventElapsedTime(&t, b->kev[k][0], b->kev[k][1]));
        cull += t;
        CUDA_TRY(cudaEventElapsedTime(&t, b->kev[k][1], b->kev[k][2]));
        isect += t;
    }
    ms4[0] = cull;
    ms4[1] = isect;
    CUDA_TRY(cudaEventElapsedTime(&ms4[2], b->ev[0], b->ev[1]));
    CUDA_TRY(cudaEventElapsedTime(&ms4[3], b->ev[3], b->ev[4]));
    return HVVR_OK;
}
} // namespace

static int frameCounters(const hvvr_batch* b, uint64_t* out, uint32_t count) {
    if (!b || !out) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (!b->counterValid || !b->hostCounters) return fail(HVVR_ERR_STATE, "the batch has not rendered a frame");
    CUDA_TRY(cudaEventSynchronize(b->ev[5]));
    uint64_t retried = 0;
    for (uint32_t k = 0; k < 2 * kRateClasses; k++) retried += b->hostCounters[kQueueBase + kQueueWords * k + 1];
    const uint64_t v[6] = {uint64_t(std::min(b->hostCounters[0], b->poolChunks)) * kChunk, retried, b->hostCounters[1],
                           b->views.size(), b->hostCounters[kSurvivorWord], b->hostCounters[kTestedWord]};
    for (uint32_t i = 0; i < count; i++) out[i] = i < 6 ? v[i] : 0u;
    return HVVR_OK;
}

static int partTimes(const hvvr_batch* b, float* ms108) {
    if (!b || !b->counterValid) return fail(HVVR_ERR_STATE, "no frame rendered");
    if (!b->stageTimes) return fail(HVVR_ERR_STATE, "the last frame was rendered without per-launch events (config.timing = 0)");
    CUDA_TRY(cudaEventSynchronize(b->ev[5]));
    for (uint32_t k = 0; k < 2 * kRateClasses; k++) {
        float* o = ms108 + 3 * k;
        o[0] = o[1] = o[2] = -1.0f;
        if (!b->kevUsed[k]) continue;
        for (int i = 0; i < 3; i++) CUDA_TRY(cudaEventElapsedTime(&o[i], b->ev[0], b->kev[k][i]));
        if (b->kevPipelined[k]) o[1] = -1.0f; // the cull's own end is not observed in a pipeline
    }
    return HVVR_OK;
}
int hvvr_batch_read_stats(const hvvr_batch* b, uint64_t* out4) {
    if (!b || !out4) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (!b->counterValid || !b->hostCounters) return fail(HVVR_ERR_STATE, "the batch has not rendered a frame");
    CUDA_TRY(cudaEventSynchronize(b->ev[5]));
    uint64_t retried = 0;
    for (uint32_t k = 0; k < 2 * kRateClasses; k++) retried += b->hostCounters[kQueueBase + kQueueWords * k + 1];
    out4[0] = uint64_t(std::min(b->hostCounters[0], b->poolChunks)) * kChunk;
    out4[1] = retried;
    out4[2] = b->hostCounters[1];
    out4[3] = b->views.size();
    return HVVR_OK;
}

int hvvr_raycaster_read_kernel_times(const hvvr_raycaster* rc, float* ms4) {
    if (!rc || !ms4) return fail(HVVR_ERR_INVALID, "NULL argument");
    return kernelTimes(rc->own.get(), ms4);
}

int hvvr_batch_read_counters(const hvvr_batch* b, uint64_t* out, uint32_t count) {
    return frameCounters(b, out, count);
}

int hvvr_raycaster_read_counters(const hvvr_raycaster* rc, uint64_t* out, uint32_t count) {
    if (!rc) return fail(HVVR_ERR_INVALID, "NULL argument");
    return frameCounters(rc->own.get(), out, count);
}

int hvvr_raycaster_read_part_times(const hvvr_raycaster* rc, float* ms108) {
    if (!rc || !ms108) return fail(HVVR_ERR_INVALID, "NULL argument");
    return partTimes(rc->own.get(), ms108);
}

int hvvr_batch_read_part_times(const hvvr_batch* b, float* ms108) {
    if (!ms108) return fail(HVVR_ERR_INVALID, "NULL argument");
    return partTimes(b, ms108);
}

int hvvr_batch_read_kernel_times(const hvvr_batch* b, float* ms4) {
    if (!ms4) return fail(HVVR_ERR_INVALID, "NULL argument");
    return kernelTimes(b, ms4);
}

int hvvr_batch_autotune(hvvr_batch* b, uint32_t frames, hvvr_batch_config* out) {
    if (!b || b->internal) return fail(HVVR_ERR_INVALID, "not a batch");
    if (b->detached || b->rcs.empty()) return fail(HVVR_ERR_STATE, "a raycaster of this batch was destroyed");
    if (frames == 0) frames = 5;
    cudaStream_t st = b->rcs[0]->stream;
    const hvvr_batch_config base = b->cfg;
    hvvr_batch_config best = base;
    float bestMs = INFINITY;
    uint32_t maxChunks = 0;
    // per cull CTA width: the cull -> shade pipeline, and the split path with each heavy share
    // (heavy_divisor 0 = no split); the pipeline does not use the heavy share
    struct Candidate { uint32_t pipeline, div; };
    const Candidate candidates[] = {{1u, base.heavy_divisor}, {0u, 0u}, {0u, 16u}, {0u, 8u}, {0u, 4u}};
    for (uint32_t warps : {1u, 2u, 4u, 8u}) {
        for (const Candidate& cand : candidates) {
            b->cfg = base;
            b->cfg.tile_cull_warps = warps;
            b->cfg.pipeline = cand.pipeline;
            b->cfg.heavy_divisor = cand.div;
            std::vector<float> ms;
            for (uint32_t f = 0; f <= frames; f++) {
                int r = renderBatch(b, st);
                if (r == HVVR_OK && cudaStreamSynchronize(st) != cudaSuccess) r = fail(HVVR_ERR_CUDA, "frame failed");
                if (r == HVVR_OK) r = checkStatus(b);
                if (r != HVVR_OK) {
                    b->cfg = base;
                    return r;
                }
                maxChunks = std::max(maxChunks, b->hostCounters[0]);
                float t = 0.0f;
                CUDA_TRY(cudaEventElapsedTime(&t, b->ev[0], b->ev[5]));
                if (f > 0) ms.push_back(t);
            }
            std::sort(ms.begin(), ms.end());
            const float med = ms[ms.size() / 2];
            if (med < bestMs) {
                bestMs = med;
                best = b->cfg;
            }
        }
    }
    const uint64_t unit = 1ull << 20;
    const uint64_t want = (uint64_t(maxChunks) * kChunk * 5 / 4 + unit - 1) / unit * unit;
    best.tri_index_capacity = std::max<uint64_t>(want, unit);
    best.frame_ms = bestMs;
    b->cfg = best;
    if (out) *out = best;
    return HVVR_OK;
}

int hvvr_model_create(hvvr_raycaster* rc, const hvvr_mesh_data* mesh, hvvr_model** out) {
    if (!rc || !mesh || !out) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (mesh->tri_count && (!mesh->verts || !mesh->tri_shade)) return fail(HVVR_ERR_INVALID, "missing arrays");
    if (mesh->tri_count >= (1u << 27)) return fail(HVVR_ERR_INVALID, "at most 2^27-1 triangles (G-buffer key width)");
    auto m = std::make_unique<hvvr_model>();
    m->rc = rc;
    m->verts.assign(mesh->verts, mesh->verts + mesh->vert_count);
    m->triShade.assign(mesh->tri_shade, mesh->tri_shade + mesh->tri_count);
    if (mesh->materials) m->materials.assign(mesh->materials, mesh->materials + mesh->material_count);
    if (mesh->tri_count == 0) {
        // a model without triangles (MeshData may be empty): no nodes; the scene merge skips it
    } else if (mesh->nodes && mesh->node_count) {
        m->nodes.assign(mesh->nodes, mesh->nodes + mesh->node_count);
    } else {
        std::vector<hvvr_topology_node> nodes(size_t(mesh->tri_count) + 4);
        uint32_t count = 0;
        if (rc->spec.bvh_build == HVVR_BVH_DEVICE) {
            CUDA_TRY(cudaSetDevice(rc->spec.device));
            TRY(hvvr_generate_topology_device(m->verts.data(), uint32_t(m->verts.size()), m->triShade.data(),
                                              uint32_t(m->triShade.size()), nodes.data(), uint32_t(nodes.size()), &count,
                                              rc->stream));
        } else {
            TRY(hvvr_generate_topology(m->verts.data(), uint32_t(m->verts.size()), m->triShade.data(),
                                       uint32_t(m->triShade.size()), nodes.data(), uint32_t(nodes.size()), &count));
        }
        nodes.resize(count);
        m->nodes = std::move(nodes);
    }
    m->xf.rotation = hvvr_vec4{0.0f, 0.0f, 0.0f, 1.0f};
    m->xf.scale = 1.0f;
    *out = m.get();
    rc->models.push_back(std::move(m));
    rc->sceneDirty = true;
    return HVVR_OK;
}

int hvvr_model_destroy(hvvr_raycaster* rc, hvvr_model* model) {
    if (!rc) return fail(HVVR_ERR_INVALID, "NULL raycaster");
    for (auto it = rc->models.begin(); it != rc->models.end(); ++it) {
        if (it->get() == model) {
            rc->models.erase(it);
            rc->sceneDirty = true;
            return HVVR_OK;
        }
    }
    return fail(HVVR_ERR_NOT_FOUND, "model not owned by this raycaster");
}

int hvvr_model_set_transform(hvvr_model* model, const hvvr_transform* xf) {
    if (!model || !xf) return fail(HVVR_ERR_INVALID, "NULL argument");
    model->xf = *xf;
    hvvr_raycaster* rc = model->rc;
    if (!rc->sceneDirty) {
        int r = uploadTransforms(rc, rc->stream);
        if (r != HVVR_OK) return r;
        rc->refitDirty = true;
    }
    return HVVR_OK;
}

int hvvr_model_update_vertices(hvvr_model* model, const hvvr_shading_vertex* verts, uint32_t count) {
    if (!model || !verts) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (count != model->verts.size()) return fail(HVVR_ERR_INVALID, "vertex count mismatch");
    model->verts.assign(verts, verts + count);
    hvvr_raycaster* rc = model->rc;
    if (rc->sceneDirty) return HVVR_OK;
    size_t off = 0;
    for (auto& m : rc->models) {
        if (m.get() == model) break;
        off += m->verts.size();
    }
    CUDA_TRY(cudaMemcpyAsync(rc->vertsIn.p + 2 * off, verts, size_t(count) * sizeof(hvvr_shading_vertex),
                             cudaMemcpyHostToDevice, rc->stream));
    rc->refitDirty = true;
    return HVVR_OK;
}

int hvvr_model_update_vertices_device(hvvr_model* model, uint32_t first, uint32_t count, const void* device_verts,
                                      void* stream) {
    if (!model || (count && !device_verts)) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (uint64_t(first) + count > model->verts.size()) return fail(HVVR_ERR_INVALID, "vertex range out of bounds");
    hvvr_raycaster* rc = model->rc;
    if (rc->sceneDirty) return fail(HVVR_ERR_STATE, "the scene is not on the device yet (render once first)");
    size_t off = 0;
    for (auto& m : rc->models) {
        if (m.get() == model) break;
        off += m->verts.size();
    }
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : rc->stream;
    if (count)
        CUDA_TRY(cudaMemcpyAsync(rc->vertsIn.p + 2 * (off + first), device_verts,
                                 size_t(count) * sizeof(hvvr_shading_vertex), cudaMemcpyDeviceToDevice, st));
    rc->refitDirty = true;
    return HVVR_OK;
}

int hvvr_light_create(hvvr_raycaster* rc, const hvvr_light_union* light, hvvr_light** out) {
    if (!rc || !light || !out) return fail(HVVR_ERR_INVALID, "NULL argument");
    auto l = std::make_unique<hvvr_light>();
    l->rc = rc;
    l->light = *light;
    *out = l.get();
    rc->lights.push_back(std::move(l));
    rc->sceneDirty = true;
    return HVVR_OK;
}

int hvvr_light_destroy(hvvr_raycaster* rc, hvvr_light* light) {
    if (!rc) return fail(HVVR_ERR_INVALID, "NULL raycaster");
    for (auto it = rc->lights.begin(); it != rc->lights.end(); ++it) {
        if (it->get() == light) {
            rc->lights.erase(it);
            rc->sceneDirty = true;
            return HVVR_OK;
        }
    }
    return fail(HVVR_ERR_NOT_FOUND, "light not owned by this raycaster");
}

int hvvr_camera_create(hvvr_raycaster* rc, const hvvr_float_rect* viewport, float aperture_radius, hvvr_camera** out) {
    if (!rc || !viewport || !out) return fail(HVVR_ERR_INVALID, "NULL argument");
    auto c = std::make_unique<hvvr_camera>();
    c->rc = rc;
    c->viewport = *viewport;
    c->lens = hvvr_thin_lens{aperture_radius, 1.0f};
    c->xf.rotation = hvvr_vec4{0.0f, 0.0f, 0.0f, 1.0f};
    c->xf.scale = 1.0f;
    *out = c.get();
    rc->cameras.push_back(std::move(c));
    return HVVR_OK;
}

int hvvr_camera_destroy(hvvr_raycaster* rc, hvvr_camera* cam) {
    if (!rc) return fail(HVVR_ERR_INVALID, "NULL raycaster");
    for (auto it = rc->cameras.begin(); it != rc->cameras.end(); ++it) {
        if (it->get() == cam) {
            cudaDeviceSynchronize();
            for (hvvr_batch* b : cam->batches) b->cams.erase(std::remove(b->cams.begin(), b->cams.end(), cam), b->cams.end());
            releaseCamera(cam);
            rc->cameras.erase(it);
            return HVVR_OK;
        }
    }
    return fail(HVVR_ERR_NOT_FOUND, "camera not owned by this raycaster");
}

#define CAM_CHECK(c) \
    if (!(c)) return fail(HVVR_ERR_INVALID, "NULL camera")

int hvvr_camera_set_enabled(hvvr_camera* cam, int enabled) {
    CAM_CHECK(cam);
    cam->enabled = enabled != 0;
    return HVVR_OK;
}
int hvvr_camera_set_viewport(hvvr_camera* cam, const hvvr_float_rect* viewport) {
    CAM_CHECK(cam);
    if (!viewport) return fail(HVVR_ERR_INVALID, "NULL viewport");
    cam->viewport = *viewport;
    cam->setupDirty = true;
    return HVVR_OK;
}
int hvvr_camera_set_lens(hvvr_camera* cam, const hvvr_thin_lens* lens) {
    CAM_CHECK(cam);
    if (!lens) return fail(HVVR_ERR_INVALID, "NULL lens");
    if (!(lens->radius >= 0.0f) || !std::isfinite(lens->radius) || !(lens->focal_distance > 0.0f) ||
        !std::isfinite(lens->focal_distance))
        return fail(HVVR_ERR_INVALID, "lens radius must be >= 0 and the focal distance > 0");
    cam->lens = *lens;
    cam->setupDirty = true;
    return HVVR_OK;
}
int hvvr_camera_set_aperture(hvvr_camera* cam, float radius) {
    CAM_CHECK(cam);
    hvvr_thin_lens l = cam->lens;
    l.radius = radius;
    return hvvr_camera_set_lens(cam, &l);
}
int hvvr_camera_set_focal_depth(hvvr_camera* cam, float depth) {
    CAM_CHECK(cam);
    hvvr_thin_lens l = cam->lens;
    l.focal_distance = depth;
    return hvvr_camera_set_lens(cam, &l);
}
int hvvr_camera_set_eye_dir(hvvr_camera* cam, const hvvr_vec3* eye_dir) {
    CAM_CHECK(cam);
    if (!eye_dir) return fail(HVVR_ERR_INVALID, "NULL eye_dir");
    cam->eyeDir = *eye_dir;
    return HVVR_OK;
}
int hvvr_camera_set_spherical_warp(hvvr_camera* cam, float fov_x_degrees, float fov_y_degrees) {
    CAM_CHECK(cam);
    cam->fovX = fov_x_degrees;
    cam->fovY = fov_y_degrees;
    cam->setupDirty = true;
    return HVVR_OK;
}
int hvvr_camera_set_render_target(hvvr_camera* cam, const hvvr_image_desc* target) {
    CAM_CHECK(cam);
    if (!target) return fail(HVVR_ERR_INVALID, "NULL target");
    if (target->memory_type != HVVR_MEMORY_CPU && target->memory_type != HVVR_MEMORY_CUDA)
        return fail(HVVR_ERR_INVALID, "render target must be CPU or CUDA memory (no graphics API here)");
    if (target->pixel_format != HVVR_PIXEL_RGBA8_SRGB) return fail(HVVR_ERR_INVALID, "pixel format must be RGBA8 sRGB");
    if (target->stride && target->stride < target->width) return fail(HVVR_ERR_INVALID, "stride < width");
    cudaDeviceSynchronize();
    unregisterTarget(cam);
    cam->target = *target;
    if (target->memory_type == HVVR_MEMORY_CPU && target->data && target->width && target->height) {
        const size_t bytes = size_t(target->stride ? target->stride : target->width) * target->height * 4;
        if (cudaHostRegister(target->data, bytes, cudaHostRegisterDefault) == cudaSuccess) cam->registered = target->data;
        else cudaGetLastError();
    }
    cam->setupDirty = true;
    return HVVR_OK;
}
int hvvr_camera_set_samples(hvvr_camera* cam, const hvvr_sample* samples, uint32_t count, uint32_t split) {
    CAM_CHECK(cam);
    if (!samples || count == 0) return fail(HVVR_ERR_INVALID, "no samples");
    if (split < 1 || split > 3) return fail(HVVR_ERR_INVALID, "splitColorSamples must be 1, 2 or 3");
    cam->samples.assign(samples, samples + count);
    cam->split = split;
    cam->setupDirty = true;
    return HVVR_OK;
}
int hvvr_camera_set_camera_to_world(hvvr_camera* cam, const hvvr_transform* xf) {
    CAM_CHECK(cam);
    if (!xf) return fail(HVVR_ERR_INVALID, "NULL transform");
    cam->xf = *xf;
    return HVVR_OK;
}
int hvvr_camera_set_msaa(hvvr_camera* cam, uint32_t rate) {
    CAM_CHECK(cam);
    if (!validRate(rate)) return fail(HVVR_ERR_INVALID, "MSAA rate must be 1, 2, 4, 8, 16 or 32");
    cam->msaa = rate;
    return HVVR_OK;
}

int hvvr_camera_set_msaa_pattern(hvvr_camera* cam, uint32_t pattern) {
    if (!cam) return fail(HVVR_ERR_INVALID, "NULL camera");
    if (pattern != HVVR_MSAA_SPIRAL && pattern != HVVR_MSAA_ROTATED_GRID) return fail(HVVR_ERR_INVALID, "unknown MSAA pattern");
    cam->msaaPattern = pattern;
    return HVVR_OK;
}
int hvvr_camera_get_sample_count(const hvvr_camera* cam, uint32_t* count) {
    CAM_CHECK(cam);
    if (!count) return fail(HVVR_ERR_INVALID, "NULL count");
    *count = uint32_t(cam->samples.size());
    return HVVR_OK;
}
int hvvr_camera_set_capture(hvvr_camera* cam, uint32_t flags) {
    CAM_CHECK(cam);
    cam->capture = flags;
    if (!(flags & HVVR_CAPTURE_HITS)) {
        cam->dev.hitIds = nullptr;
        cam->dev.depth = nullptr;
    }
    return HVVR_OK;
}
int hvvr_camera_get_layout(const hvvr_camera* cam, uint32_t* block_count, uint32_t* tile_count,
                           uint32_t* padded_sample_count, uint32_t* msaa_rate) {
    CAM_CHECK(cam);
    uint32_t n = uint32_t(cam->samples.size());
    hvvr_raycaster* rc = cam->rc;
    if (rc->spec.mode == HVVR_MODE_FOVEATED_POLAR) {
        // the raycaster's polar sample set replaces the camera's samples
        if (!rc->polar) {
            rc->polar = std::make_unique<PolarSetup>();
            buildPolarFoveatedSetup(rc->spec.foveated_degree_tracking_error, rc->spec.foveated_max_fov_degrees,
                                    rc->spec.foveated_mar_slope, rc->spec.foveated_foveal_mar_degrees, *rc->polar);
        }
        n = rc->polar->valid;
    }
    const uint32_t blocks = (n + kBlockSize - 1) / kBlockSize;
    if (block_count) *block_count = blocks;
    if (tile_count) *tile_count = blocks * kTilesPerBlock;
    if (padded_sample_count) *padded_sample_count = blocks * kBlockSize;
    if (msaa_rate) *msaa_rate = cam->msaa;
    return HVVR_OK;
}

static int requireRendered(const hvvr_camera* cam) {
    if (!cam) return fail(HVVR_ERR_INVALID, "NULL camera");
    if (!cam->rendered) return fail(HVVR_ERR_STATE, "camera has not rendered a frame");
    cudaError_t e = cudaStreamSynchronize(cam->rc->stream);
    if (e != cudaSuccess) return fail(HVVR_ERR_CUDA, "sync: %s", cudaGetErrorString(e));
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail(HVVR_ERR_CUDA, "sync: %s", cudaGetErrorString(e));
    return HVVR_OK;
}

int hvvr_camera_read_tile_lists(const hvvr_camera* cam, uint32_t* counts, uint32_t* indices, uint64_t capacity,
                                uint64_t* total) {
    TRY(requireRendered(cam));
    const CameraDev& d = cam->dev;
    std::vector<TileList> lists(d.tiles);
    CUDA_TRY(cudaMemcpy(lists.data(), d.tileLists, sizeof(TileList) * d.tiles, cudaMemcpyDeviceToHost));
    uint64_t sum = 0;
    for (uint32_t t = 0; t < d.tiles; t++) {
        if (counts) counts[t] = lists[t].count;
        sum += lists[t].count;
    }
    if (total) *total = sum;
    if (!indices) return HVVR_OK;
    if (capacity < sum) return fail(HVVR_ERR_OVERFLOW, "capacity %llu < %llu entries", (unsigned long long)capacity,
                                    (unsigned long long)sum);
    const hvvr_batch* b = cam->lastBatch;
    if (!b) return fail(HVVR_ERR_STATE, "the batch that rendered this camera's lists was destroyed");
    uint32_t used = 0;
    CUDA_TRY(cudaMemcpy(&used, b->counters.p, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    used = std::min(used, b->poolChunks);
    std::vector<uint32_t> pool(size_t(used) * kChunk), next(used);
    if (used) {
        CUDA_TRY(cudaMemcpy(pool.data(), b->pool.p, pool.size() * 4, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(next.data(), b->chunkNext.p, next.size() * 4, cudaMemcpyDeviceToHost));
    }
    uint64_t w = 0;
    for (uint32_t t = 0; t < d.tiles; t++) {
        uint32_t c = lists[t].first, left = lists[t].count;
        while (left) {
            if (c >= used) return fail(HVVR_ERR_STATE, "broken chunk chain in tile %u", t);
            const uint32_t n = std::min<uint32_t>(left, kChunk);
            memcpy(indices + w, &pool[size_t(c) * kChunk], n * 4);
            w += n;
            left -= n;
            c = next[c];
        }
    }
    return HVVR_OK;
}

int hvvr_camera_read_block_stacks(const hvvr_camera* cam, uint32_t* sizes, uint32_t* entries) {
    TRY(requireRendered(cam));
    const CameraDev& d = cam->dev;
    std::vector<uint32_t> sz(d.blocks);
    CUDA_TRY(cudaMemcpy(sz.data(), d.blockSizes, 4 * size_t(d.blocks), cudaMemcpyDeviceToHost));
    if (sizes) memcpy(sizes, sz.data(), 4 * size_t(d.blocks));
    if (entries) {
        std::vector<StackEntry> e(size_t(d.blocks) * kBlockStack);
        CUDA_TRY(cudaMemcpy(e.data(), d.blockStacks, e.size() * sizeof(StackEntry), cudaMemcpyDeviceToHost));
        for (uint32_t b = 0; b < d.blocks; b++)
            for (uint32_t i = 0; i < kBlockStack; i++) {
                uint32_t* dst = entries + (size_t(b) * kBlockStack + i) * 3;
                if (i < sz[b]) {
                    const StackEntry& s = e[size_t(b) * kBlockStack + i];
                    memcpy(&dst[0], &s.tMin, 4);
                    dst[1] = s.mask;
                    dst[2] = s.node;
                } else {
                    dst[0] = dst[1] = dst[2] = 0;
                }
            }
    }
    return HVVR_OK;
}

int hvvr_camera_read_hits(const hvvr_camera* cam, uint32_t* tri_ids, float* depth) {
    TRY(requireRendered(cam));
    const CameraDev& d = cam->dev;
    if (!d.hitIds) return fail(HVVR_ERR_STATE, "hit capture was not enabled for the last frame");
    const size_t n = size_t(d.padded) * d.msaa;
    if (tri_ids) CUDA_TRY(cudaMemcpy(tri_ids, d.hitIds, n * 4, cudaMemcpyDeviceToHost));
    if (depth) CUDA_TRY(cudaMemcpy(depth, d.depth, n * 4, cudaMemcpyDeviceToHost));
    return HVVR_OK;
}

int hvvr_camera_read_gbuffer(const hvvr_camera* cam, uint32_t* n, uint32_t* tri, uint32_t* mask) {
    TRY(requireRendered(cam));
    const CameraDev& d = cam->dev;
    if (!d.hitIds) return fail(HVVR_ERR_STATE, "hit capture was not enabled for the last frame");
    const uint32_t N = d.msaa;
    std::vector<uint32_t> hits(size_t(d.padded) * N);
    CUDA_TRY(cudaMemcpy(hits.data(), d.hitIds, hits.size() * 4, cudaMemcpyDeviceToHost));
    for (uint32_t s = 0; s < d.padded; s++) {
        uint32_t keys[32];
        for (uint32_t i = 0; i < N; i++) keys[i] = (hits[size_t(s) * N + i] << 5) | i;
        std::sort(keys, keys + N);
        uint32_t gn = 0, gt[32], gm[32];
        for (uint32_t i = 0; i < N; i++) {
            const uint32_t t = uint32_t(int32_t(keys[i]) >> 5), m = 1u << (keys[i] & 31);
            if (gn && gt[gn - 1] == t) gm[gn - 1] |= m;
            else { gt[gn] = t; gm[gn] = m; gn++; }
        }
        if (n) n[s] = gn;
        for (uint32_t i = 0; i < N; i++) {
            if (tri) tri[size_t(s) * N + i] = i < gn ? gt[i] : 0;
            if (mask) mask[size_t(s) * N + i] = i < gn ? gm[i] : 0;
        }
    }
    return HVVR_OK;
}

int hvvr_camera_read_sample_colors(const hvvr_camera* cam, uint32_t* rgba) {
    TRY(requireRendered(cam));
    if (!rgba) return fail(HVVR_ERR_INVALID, "NULL output");
    CUDA_TRY(cudaMemcpy(rgba, cam->dev.colors, size_t(cam->dev.padded) * 4, cudaMemcpyDeviceToHost));
    return HVVR_OK;
}

int hvvr_camera_prepare(hvvr_camera* cam, uint32_t* on_host) {
    CAM_CHECK(cam);
    CUDA_TRY(cudaSetDevice(cam->rc->spec.device));
    if (cam->setupDirty) {
        TRY(setupCamera(cam, cam->rc->stream));
        CUDA_TRY(cudaStreamSynchronize(cam->rc->stream));
    }
    if (on_host) *on_host = cam->setupOnHost ? 1u : 0u;
    return HVVR_OK;
}

int hvvr_camera_read_sample_remap(const hvvr_camera* cam, int32_t* remap, uint64_t count) {
    CAM_CHECK(cam);
    if (cam->setupDirty) return fail(HVVR_ERR_STATE, "sample setup not built yet (render once first)");
    if (!remap || count < cam->remap.n) return fail(HVVR_ERR_INVALID, "remap buffer too small");
    if (cam->remap.n) CUDA_TRY(cudaMemcpy(remap, cam->remap.p, cam->remap.n * 4, cudaMemcpyDeviceToHost));
    return HVVR_OK;
}

int hvvr_camera_read_beams(const hvvr_camera* cam, float* beams9) {
    CAM_CHECK(cam);
    if (cam->setupDirty) return fail(HVVR_ERR_STATE, "sample setup not built yet (render once first)");
    if (!beams9) return fail(HVVR_ERR_INVALID, "NULL output");
    if (cam->foveated) {
        const PolarSetup& ps = *cam->rc->polar;
        memset(beams9, 0, size_t(ps.padded) * 9 * 4);
        memcpy(beams9, ps.beams.data(), ps.beams.size() * sizeof(PolarBeam));
        return HVVR_OK;
    }
    std::vector<float4> b(cam->beams.n);
    CUDA_TRY(cudaMemcpy(b.data(), cam->beams.p, b.size() * sizeof(float4), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < cam->setup.padded; i++) memcpy(beams9 + 9 * i, &b[3 * i], 9 * 4);
    return HVVR_OK;
}

int hvvr_camera_read_timings(const hvvr_camera* cam, float* ms6) {
    TRY(requireRendered(cam));
    if (!ms6) return fail(HVVR_ERR_INVALID, "NULL output");
    const hvvr_batch* b = cam->lastBatch;
    if (!b) return fail(HVVR_ERR_STATE, "the batch that rendered this camera was destroyed");
    ms6[0] = 0.0f;
    for (int i = 1; i < 5; i++) {
        ms6[i] = 0.0f;
        if (b->stageTimes) CUDA_TRY(cudaEventElapsedTime(&ms6[i], b->ev[i - 1], b->ev[i]));
    }
    CUDA_TRY(cudaEventElapsedTime(&ms6[5], b->ev[0], b->ev[5]));
    return HVVR_OK;
}

int hvvr_camera_read_tile_costs(const hvvr_camera* cam, uint32_t* visits) {
    TRY(requireRendered(cam));
    if (!visits) return fail(HVVR_ERR_INVALID, "NULL output");
    CUDA_TRY(cudaMemcpy(visits, cam->dev.tileCost, size_t(cam->dev.tiles) * 4, cudaMemcpyDeviceToHost));
    return HVVR_OK;
}

int hvvr_camera_read_foveated_frame(const hvvr_camera* cam, float* eye_to_world16, float* cull_planes16,
                                    float* view_depth) {
    TRY(requireRendered(cam));
    if (!cam->foveated) return fail(HVVR_ERR_STATE, "not a foveated camera");
    if (eye_to_world16) memcpy(eye_to_world16, cam->eyeToWorld, 16 * 4);
    if (cull_planes16) memcpy(cull_planes16, cam->cullPlanes, 16 * 4);
    if (view_depth) CUDA_TRY(cudaMemcpy(view_depth, cam->tmax.p, size_t(cam->dev.padded) * 4, cudaMemcpyDeviceToHost));
    return HVVR_OK;
}

int hvvr_camera_read_foveated_resolve(const hvvr_camera* cam, float* sample_to_eye9, float* eye_to_sample_prev16,
                                      uint32_t* result, uint32_t* history) {
    TRY(requireRendered(cam));
    if (!cam->foveated || !cam->fovStatic.image) return fail(HVVR_ERR_STATE, "not a foveated camera with a render target");
    if (sample_to_eye9) memcpy(sample_to_eye9, cam->lastSampleToEye, 9 * 4);
    if (eye_to_sample_prev16) memcpy(eye_to_sample_prev16, cam->lastEyeToSamplePrev, 16 * 4);
    // the last frame wrote fovResult[fovCur ^ 1] and read fovResult[fovCur] (legacy default
    // stream: ordered after the frame's work)
    if (result) TRY(cam->fovResult[cam->fovCur ^ 1u].download(result, 0));
    if (history) TRY(cam->fovResult[cam->fovCur].download(history, 0));
    return HVVR_OK;
}

int hvvr_camera_read_polar_textures(const hvvr_camera* cam, uint32_t* color, float* depth, uint16_t* moments) {
    TRY(requireRendered(cam));
    if (!cam->foveated || !cam->fovStatic.image) return fail(HVVR_ERR_STATE, "not a foveated camera with a render target");
    const size_t texels = size_t(cam->fovStatic.spr) * cam->fovStatic.rings;
    if (color) TRY(cam->polarRaw.download(color, 0));
    if (depth) TRY(cam->polarDepth.download(depth, 0));
    if (moments) {
        // [texel][first, second][rgba] from the two RGBA16 textures
        std::vector<uint64_t> m1(texels), m2(texels);
        TRY(cam->moment1.download(m1.data(), 0));
        TRY(cam->moment2.download(m2.data(), 0));
        for (size_t k = 0; k < texels; k++) {
            memcpy(moments + 8 * k, &m1[k], 8);
            memcpy(moments + 8 * k + 4, &m2[k], 8);
        }
    }
    return HVVR_OK;
}

int hvvr_foveated_frame_matrices(const hvvr_transform* camera_to_world, const hvvr_vec3* eye_dir,
                                 const hvvr_float_rect* sample_bounds, const hvvr_float_rect* viewport,
                                 float* world_to_eye_prev16, float* eye_prev_to_sample_prev9, float* eye_to_world16,
                                 float* cull_planes16, float* sample_to_eye9, float* eye_to_sample_prev16) {
    if (!camera_to_world || !eye_dir || !sample_bounds || !viewport || !world_to_eye_prev16 ||
        !eye_prev_to_sample_prev9 || !eye_to_world16 || !cull_planes16 || !sample_to_eye9 || !eye_to_sample_prev16)
        return fail(HVVR_ERR_INVALID, "null argument");
    const Mat4 c2w = transformToMatrix(*camera_to_world);
    float planes[4][4];
    foveatedFrame(&c2w.m[0][0], *eye_dir, *sample_bounds, *viewport, eye_to_world16, planes);
    memcpy(cull_planes16, planes, sizeof(planes));
    foveatedResolveFrame(eye_to_world16, *eye_dir, *viewport, world_to_eye_prev16, eye_prev_to_sample_prev9,
                         sample_to_eye9, eye_to_sample_prev16);
    return HVVR_OK;
}

int hvvr_camera_read_list_total(const hvvr_camera* cam, uint64_t* total) {
    return hvvr_camera_read_tile_lists(cam, nullptr, nullptr, 0, total);
}

int hvvr_scene_get_counts(const hvvr_raycaster* rc, uint32_t* node_count, uint32_t* tri_count, uint32_t* vert_count) {
    if (!rc) return fail(HVVR_ERR_INVALID, "NULL raycaster");
    if (node_count) *node_count = rc->scene.nodeCount;
    if (tri_count) *tri_count = rc->scene.triCount;
    if (vert_count) *vert_count = rc->scene.vertCount;
    return HVVR_OK;
}

int hvvr_scene_read_nodes(hvvr_raycaster* rc, void* nodes128) {
    if (!rc || !nodes128) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (rc->scene.nodeCount == 0) return fail(HVVR_ERR_STATE, "no scene uploaded");
    CUDA_TRY(cudaStreamSynchronize(rc->stream));
    CUDA_TRY(cudaDeviceSynchronize());
    CUDA_TRY(cudaMemcpy(nodes128, rc->scene.nodes, size_t(rc->scene.nodeCount) * sizeof(Node), cudaMemcpyDeviceToHost));
    return HVVR_OK;
}

int hvvr_scene_read_triangles(hvvr_raycaster* rc, float* tris9) {
    if (!rc || !tris9) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (rc->scene.nodeCount == 0) return fail(HVVR_ERR_STATE, "no scene uploaded");
    CUDA_TRY(cudaDeviceSynchronize());
    std::vector<float4> t(size_t(rc->scene.triCount) * 3);
    CUDA_TRY(cudaMemcpy(t.data(), rc->scene.tris, t.size() * sizeof(float4), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < rc->scene.triCount; i++) memcpy(tris9 + 9 * i, &t[3 * i], 9 * 4);
    return HVVR_OK;
}

int hvvr_polar_foveated_layout(const hvvr_spec* spec, uint32_t* samples_per_ring, uint32_t* ring_count,
                               uint32_t* valid, uint32_t* padded) {
    hvvr_spec d;
    hvvr_spec_default(&d);
    const hvvr_spec& s = spec ? *spec : d;
    PolarSetup ps;
    buildPolarFoveatedSetup(s.foveated_degree_tracking_error, s.foveated_max_fov_degrees, s.foveated_mar_slope,
                            s.foveated_foveal_mar_degrees, ps);
    if (samples_per_ring) *samples_per_ring = ps.samplesPerRing;
    if (ring_count) *ring_count = ps.ringCount;
    if (valid) *valid = ps.valid;
    if (padded) *padded = ps.padded;
    return HVVR_OK;
}

int hvvr_polar_foveated_samples(const hvvr_spec* spec, float* beams9, uint32_t* remap2, float* tile_rays24,
                                float* block_rays24) {
    hvvr_spec d;
    hvvr_spec_default(&d);
    const hvvr_spec& s = spec ? *spec : d;
    PolarSetup ps;
    buildPolarFoveatedSetup(s.foveated_degree_tracking_error, s.foveated_max_fov_degrees, s.foveated_mar_slope,
                            s.foveated_foveal_mar_degrees, ps);
    if (beams9) memcpy(beams9, ps.beams.data(), ps.beams.size() * sizeof(PolarBeam));
    if (remap2) memcpy(remap2, ps.remap.data(), ps.remap.size() * 4);
    if (tile_rays24) memcpy(tile_rays24, ps.tileRays.data(), ps.tileRays.size() * sizeof(Rays4));
    if (block_rays24) memcpy(block_rays24, ps.blockRays.data(), ps.blockRays.size() * sizeof(Rays4));
    return HVVR_OK;
}

int hvvr_grid_samples(uint32_t width, uint32_t height, hvvr_sample* out) {
    if (!out || !width || !height) return fail(HVVR_ERR_INVALID, "bad arguments");
    // getGridSamples (libraries/hvvr/raycaster/samples.cpp:21-42)
    const float invW = 1.0f / width, invH = 1.0f / height;
    for (uint32_t y = 0; y < height; y++)
        for (uint32_t x = 0; x < width; x++) {
            hvvr_sample& s = out[size_t(y) * width + x];
            s.pixel_x = x;
            s.pixel_y = y;
            s.position.x = (float(x) + 0.5f) * invW;
            s.position.y = (float(y) + 0.5f) * invH;
            if (width > height) {
                s.minor_axis = hvvr_vec2{invW, 0.0f};
                s.major_axis_length = invH;
            } else {
                s.minor_axis = hvvr_vec2{0.0f, invH};
                s.major_axis_length = invW;
            }
        }
    return HVVR_OK;
}

} // extern "C"
