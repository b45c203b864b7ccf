// GPU-side harness around the reference's own intersect and shade/resolve kernels
// (libraries/hvvr/raycaster/intersect.cu IntersectKernel, resolve.cu ResolveKernel), built with
// nvcc for sm_100a into oracle/_ref/libhvvr_ref_gpu.so. Test infrastructure only. The kernels
// are compiled from the reference's source files, included here so that this translation unit
// instantiates them for every MSAA rate (the reference fixes one at compile time,
// COLOR_MODE_MSAA_RATE) and launches them the way GPUCamera::intersect and
// GPUCamera::shadeAndResolve do (intersect.cu:358-385, resolve.cu:460-502), on inputs given
// by the caller: the camera-space beams, the world-space tile frusta, the per-tile triangle
// lists and the scene arrays the reference's host code produced.
#include "intersect.cu"
#include "resolve.cu"

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

namespace hvvr {
// GPUCamera-bound constructor the included GPUCamera methods refer to; the harness builds its
// CameraBeams field by field, so this is never called.
CameraBeams::CameraBeams(const GPUCamera&) {
    fprintf(stderr, "ref_gpu_intersect: CameraBeams(const GPUCamera&) is not part of the harness\n");
    abort();
}
} // namespace hvvr

namespace {

template <class T>
struct Dev {
    T* p = nullptr;
    ~Dev() { cudaFree(p); }
    cudaError_t up(const void* src, size_t count) {
        cudaError_t e = cudaMalloc((void**)&p, (count ? count : 1) * sizeof(T));
        if (e == cudaSuccess && count) e = cudaMemcpy(p, src, count * sizeof(T), cudaMemcpyHostToDevice);
        return e;
    }
    cudaError_t alloc(size_t count) { return cudaMalloc((void**)&p, (count ? count : 1) * sizeof(T)); }
};

template <uint32_t N>
cudaError_t launch(uint32_t occupied, hvvr::RaycasterGBufferSubsample* gb, const hvvr::CameraBeams& beams,
                   const hvvr::matrix4x4& c2w, const uint32_t* remap, const hvvr::TileTriRange* ranges,
                   const uint32_t* triIndices, const hvvr::SimpleRayFrustum* frusta,
                   const hvvr::PrecomputedTriangleIntersect* tris, const hvvr::PrecomputedTriangleShade* shade,
                   const hvvr::ShadingVertex* verts, const hvvr::SimpleMaterial* mats,
                   const hvvr::LightingEnvironment& env, uint32_t* colors, float* tmax) {
    using namespace hvvr;
    KernelDim dim(occupied * TILE_SIZE, TILE_SIZE);
    IntersectKernel<N, TILE_SIZE, false><<<dim.grid, dim.block>>>(gb, beams, c2w, nullptr, remap, ranges, triIndices,
                                                                 frusta, tris);
    ResolveKernel<true, false, N, TILE_SIZE><<<dim.grid, dim.block>>>(colors, tmax, gb, beams, c2w, nullptr, remap,
                                                                      tris, shade, verts, mats, gDeviceTextureArray,
                                                                      env, nullptr);
    return cudaGetLastError();
}

} // namespace

extern "C" {

// One pinhole frame of the reference's intersect + resolve kernels. beams: [padded][9] camera-space
// DirectionalBeam; frusta: [tiles][24] world-space SimpleRayFrustum; tile_counts [tiles] and
// tile_indices (concatenated lists); tris [tri][9] PrecomputedTriangleIntersect; tri_shade [tri][4];
// verts [n] ShadingVertex (world space, 32 B); materials [m] SimpleMaterial (64 B); lights [l]
// LightUnion (56 B); cam_xf the camera transform (32 B). Outputs: gb_tri / gb_mask [padded][msaa]
// (the G-buffer unpacked from its warp-interleaved layout; written for occupied tiles only, the
// rest read ~0), colors [padded] (RGBA8) and tmax [padded] (the TMaxBuffer depth), empty tiles
// cleared by ClearEmptyKernel.
int ref_gpu_intersect_resolve(uint32_t msaa, const float* beams, uint32_t padded, const float* frusta, uint32_t tiles,
                              const uint32_t* tile_counts, const uint32_t* tile_indices, const float* tris,
                              const uint32_t* tri_shade, uint32_t tri_count, const void* verts, uint32_t vert_count,
                              const void* materials, uint32_t material_count, const void* lights, uint32_t light_count,
                              const void* cam_xf, uint32_t* gb_tri, uint32_t* gb_mask, uint32_t* colors, float* tmax) {
    using namespace hvvr;
    if (padded % TILE_SIZE || padded / TILE_SIZE != tiles) return -1;
    // occupied tiles, their triangle ranges and the concatenated indices (GPUCamera's streamed data)
    std::vector<uint32_t> remap, empty;
    std::vector<TileTriRange> ranges;
    uint64_t offset = 0;
    for (uint32_t t = 0; t < tiles; t++) {
        if (tile_counts[t]) {
            remap.push_back(t);
            ranges.push_back(TileTriRange{uint32_t(offset), uint32_t(offset + tile_counts[t])});
        } else {
            empty.push_back(t);
        }
        offset += tile_counts[t];
    }
    const uint32_t occupied = uint32_t(remap.size()), emptyCount = uint32_t(empty.size());
    // LightingEnvironment from the lights (GPUSceneState::updateLighting, gpu_scene_state.cu:47-81)
    LightingEnvironment env;
    memset(&env, 0, sizeof(env));
    for (uint32_t i = 0; i < light_count; i++) {
        const LightUnion& l = ((const LightUnion*)lights)[i];
        if (l.type == LightType::directional && env.directionalLightCount < int(MAX_DIRECTIONAL_LIGHTS))
            env.directionalLights[env.directionalLightCount++] = l.directional;
        else if (l.type == LightType::point && env.pointLightCount < int(MAX_POINT_LIGHTS))
            env.pointLights[env.pointLightCount++] = l.point;
        else if (l.type == LightType::spot && env.spotLightCount < int(MAX_SPOT_LIGHTS))
            env.spotLights[env.spotLightCount++] = l.spot;
    }
    const matrix4x4 cameraToWorld = matrix4x4(*(const transform*)cam_xf);

    Dev<DirectionalBeam> dBeams;
    Dev<SimpleRayFrustum> dFrusta;
    Dev<uint32_t> dRemap, dEmpty, dIdx, dColors;
    Dev<TileTriRange> dRanges;
    Dev<PrecomputedTriangleIntersect> dTris;
    Dev<PrecomputedTriangleShade> dShade;
    Dev<ShadingVertex> dVerts;
    Dev<SimpleMaterial> dMats;
    Dev<RaycasterGBufferSubsample> dGb;
    Dev<float> dTmax;
    cudaError_t e = dBeams.up(beams, padded);
    if (e == cudaSuccess) e = dFrusta.up(frusta, tiles);
    if (e == cudaSuccess) e = dRemap.up(remap.data(), remap.size());
    if (e == cudaSuccess) e = dEmpty.up(empty.data(), empty.size());
    if (e == cudaSuccess) e = dRanges.up(ranges.data(), ranges.size());
    if (e == cudaSuccess) e = dIdx.up(tile_indices, offset);
    if (e == cudaSuccess) e = dTris.up(tris, tri_count);
    if (e == cudaSuccess) e = dShade.up(tri_shade, tri_count);
    if (e == cudaSuccess) e = dVerts.up(verts, vert_count);
    if (e == cudaSuccess) e = dMats.up(materials, material_count);
    if (e == cudaSuccess) e = dGb.alloc(size_t(padded) * msaa);
    if (e == cudaSuccess) e = dColors.alloc(padded);
    if (e == cudaSuccess) e = dTmax.alloc(padded);
    if (e == cudaSuccess) e = cudaMemset(dGb.p, 0xff, size_t(padded) * msaa * sizeof(RaycasterGBufferSubsample));
    if (e != cudaSuccess) return int(e);
    // CameraBeams: its GPUCamera constructor is bypassed; the kernels read these three fields
    alignas(CameraBeams) unsigned char storage[sizeof(CameraBeams)];
    memset(storage, 0, sizeof(storage));
    CameraBeams& cb = *reinterpret_cast<CameraBeams*>(storage);
    cb.directionalBeams = dBeams.p;
    cb.frameJitter = vector2(0.0f, 0.0f);
    cb.lens = ThinLens{0.0f, 1.0f};
    if (occupied) {
        switch (msaa) {
#define HV_RATE(N)                                                                                                    \
    case N:                                                                                                            \
        e = launch<N>(occupied, dGb.p, cb, cameraToWorld, dRemap.p, dRanges.p, dIdx.p, dFrusta.p, dTris.p, dShade.p,  \
                      dVerts.p, dMats.p, env, dColors.p, dTmax.p);                                                     \
        break;
            HV_RATE(1) HV_RATE(2) HV_RATE(4) HV_RATE(8) HV_RATE(16) HV_RATE(32)
#undef HV_RATE
        default:
            return -2;
        }
    }
    // empty tiles: ClearEmptyKernel (resolve.cu:527-541) as GPUCamera::clearEmpty launches it
    if (e == cudaSuccess && emptyCount) {
        ClearEmptyKernel<<<(emptyCount * TILE_SIZE + CUDA_GROUP_SIZE - 1) / CUDA_GROUP_SIZE, CUDA_GROUP_SIZE>>>(
            dColors.p, dTmax.p, dEmpty.p, emptyCount);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return int(e);
    std::vector<RaycasterGBufferSubsample> gb(size_t(padded) * msaa);
    e = cudaMemcpy(gb.data(), dGb.p, gb.size() * sizeof(RaycasterGBufferSubsample), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(colors, dColors.p, size_t(padded) * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(tmax, dTmax.p, size_t(padded) * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return int(e);
    // entry (slot s, lane l) of warp w sits at w * 32 * msaa + s * 32 + l (EmitGBuffer)
    for (uint32_t s = 0; s < padded; s++) {
        const size_t base = size_t(s / WARP_SIZE) * WARP_SIZE * msaa + (s % WARP_SIZE);
        for (uint32_t k = 0; k < msaa; k++) {
            gb_tri[size_t(s) * msaa + k] = gb[base + size_t(k) * WARP_SIZE].triIndex;
            gb_mask[size_t(s) * msaa + k] = gb[base + size_t(k) * WARP_SIZE].sampleMask;
        }
    }
    return 0;
}

} // extern "C"
