// GPU-side harness around the reference's own scene update kernels (libraries/hvvr/raycaster/
// gpu_scene_state.cu: SceneTransformVerticesKernel, SceneRefitPreKernel, ScenePrecomputeTrianglesKernel,
// SceneRefitIntFixupKernel, SceneRefitNodeMultiPassKernel), built with nvcc for sm_100a into
// oracle/_ref/libhvvr_ref_gpu.so. Test infrastructure only. The kernels are compiled from the
// reference's source file, included here, and launched in the order GPUSceneState::update
// (gpu_scene_state.cu:377-451) launches them. The internal nodes are refit by the multi-pass kernel
// (one launch per BVH depth, the reference's path above 64K refit tasks): it takes no spin-wait,
// and a slot's bound is a max over the same child bounds either way. The refit task list follows
// GPUSceneState::setGeometry's rules (gpu_scene_state.cu:517-587): internal children grouped by
// their parent's depth, deepest first, by child index within a depth; each leaf slot's triangles
// point at that slot.
// the reference file sorts with std::sort without including <algorithm>
#include <algorithm>

#include "gpu_scene_state.cu"

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

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

} // namespace

extern "C" {

// One scene update of the reference's GPU path. Inputs: the BVH [nodeCount] (BVHNode; only the
// child and leaf data are read), the untransformed vertices [vertexCount] (ShadingVertex), the
// model of each vertex, the model transforms [modelCount] (transform: rotation quaternion,
// translation, scale; converted by matrix4x4(const transform&) as Raycaster's scene update does,
// scene_update.cpp:153-156) and the triangles [triangleCount] (PrecomputedTriangleShade).
// Outputs: the world-space vertices, the precomputed triangles (PrecomputedTriangleIntersect)
// and the refit BVH.
int ref_gpu_scene_update(const void* nodesIn, uint32_t nodeCount, const void* vertices, uint32_t vertexCount,
                         const uint32_t* vertexModel, const void* transforms, uint32_t modelCount,
                         const void* trianglesShade, uint32_t triangleCount, void* worldVertices,
                         void* trianglesIntersect, void* nodesOut) {
    using namespace hvvr;
    static_assert(sizeof(BVHNode) == 128 && sizeof(ShadingVertex) == 32, "layouts");
    static_assert(sizeof(transform) == 32 && sizeof(matrix4x4) == 64, "layouts");
    static_assert(sizeof(hvvr::PrecomputedTriangleShade) == 16 && sizeof(hvvr::PrecomputedTriangleIntersect) == 36, "layouts");
    if (!nodeCount || !vertexCount || !triangleCount || !modelCount) return -1;
    std::vector<BVHNode> nodes(nodeCount);
    memcpy(nodes.data(), nodesIn, size_t(nodeCount) * sizeof(BVHNode));
    std::vector<matrix4x4> modelToWorld(modelCount);
    for (uint32_t m = 0; m < modelCount; m++) {
        transform t;
        memcpy(&t, (const char*)transforms + size_t(m) * sizeof(transform), sizeof(transform));
        modelToWorld[m] = matrix4x4(t);
    }

    // parent depth of every node, then the refit tasks and each triangle's leaf slot
    std::vector<uint32_t> depth(nodeCount, 0);
    for (uint32_t n = 0; n < nodeCount; n++) {
        for (int k = 0; k < 4; k++) {
            if (nodes[n].boxData.leafMask & (1u << k)) continue;
            const uint32_t c = n + nodes[n].boxData.children.offset[k];
            if (c >= nodeCount) return -2;
            depth[c] = depth[n] + 1;
        }
    }
    std::vector<SceneRefitTaskNode> tasks;
    std::vector<uint32_t> triToNodeChild(triangleCount, 0);
    for (uint32_t n = nodeCount; n-- > 0;) {
        for (int k = 3; k >= 0; k--) {
            const uint32_t nodeChild = (n << 2) | uint32_t(k);
            if (!(nodes[n].boxData.leafMask & (1u << k))) {
                tasks.push_back({n + nodes[n].boxData.children.offset[k], nodeChild});
            } else {
                const uint32_t t0 = nodes[n].boxData.leaf.triIndex[k], t1 = nodes[n].boxData.leaf.triIndex[k + 1];
                if (t1 > triangleCount || t0 > t1) return -3;
                for (uint32_t t = t0; t < t1; t++) triToNodeChild[t] = nodeChild;
            }
        }
    }
    std::sort(tasks.begin(), tasks.end(), [&](const SceneRefitTaskNode& a, const SceneRefitTaskNode& b) {
        const uint32_t da = depth[a.nodeChild >> 2], db = depth[b.nodeChild >> 2];
        return da != db ? da > db : a.childIndex < b.childIndex;
    });

    Dev<BVHNode> dNodes;
    Dev<ShadingVertex> dVerts, dWorld;
    Dev<uint32_t> dVertModel, dTriToNode;
    Dev<matrix4x4> dXf;
    Dev<hvvr::PrecomputedTriangleShade> dShade;
    Dev<hvvr::PrecomputedTriangleIntersect> dIsect;
    Dev<SceneRefitTaskNode> dTasks;
    cudaError_t e = dNodes.up(nodes.data(), nodeCount);
    if (e == cudaSuccess) e = dVerts.up(vertices, vertexCount);
    if (e == cudaSuccess) e = dWorld.alloc(vertexCount);
    if (e == cudaSuccess) e = dVertModel.up(vertexModel, vertexCount);
    if (e == cudaSuccess) e = dXf.up(modelToWorld.data(), modelCount);
    if (e == cudaSuccess) e = dShade.up(trianglesShade, triangleCount);
    if (e == cudaSuccess) e = dIsect.alloc(triangleCount);
    if (e == cudaSuccess) e = dTriToNode.up(triToNodeChild.data(), triangleCount);
    if (e == cudaSuccess) e = dTasks.up(tasks.data(), tasks.size());
    for (uint32_t v = 0; e == cudaSuccess && v < vertexCount; v++)
        if (vertexModel[v] >= modelCount) e = cudaErrorInvalidValue;
    for (uint32_t t = 0; e == cudaSuccess && t < triangleCount; t++) {
        const uint32_t* ix = (const uint32_t*)trianglesShade + 4 * size_t(t);
        if (ix[0] >= vertexCount || ix[1] >= vertexCount || ix[2] >= vertexCount) e = cudaErrorInvalidValue;
    }
    if (e == cudaSuccess) {
        KernelDim vdim(vertexCount, WARP_SIZE), ndim(nodeCount, WARP_SIZE), tdim(triangleCount, WARP_SIZE);
        SceneTransformVerticesKernel<<<vdim.grid, vdim.block>>>(dVerts.p, dWorld.p, dVertModel.p, dXf.p, vertexCount);
        SceneRefitPreKernel<false><<<ndim.grid, ndim.block>>>(nodeCount, dNodes.p, nullptr);
        ScenePrecomputeTrianglesKernel<<<tdim.grid, tdim.block>>>(triangleCount, dWorld.p, dShade.p, dTriToNode.p,
                                                                 dIsect.p, dNodes.p);
        SceneRefitIntFixupKernel<<<ndim.grid, ndim.block>>>(nodeCount, dNodes.p);
        size_t start = 0;
        while (start < tasks.size()) {
            size_t end = start;
            const uint32_t d = depth[tasks[start].nodeChild >> 2];
            while (end < tasks.size() && depth[tasks[end].nodeChild >> 2] == d) end++;
            KernelDim dim(end - start, WARP_SIZE);
            SceneRefitNodeMultiPassKernel<<<dim.grid, dim.block>>>(dTasks.p + start, uint32_t(end - start), dNodes.p);
            start = end;
        }
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(worldVertices, dWorld.p, size_t(vertexCount) * 32, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(trianglesIntersect, dIsect.p, size_t(triangleCount) * 36, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(nodesOut, dNodes.p, size_t(nodeCount) * 128, cudaMemcpyDeviceToHost);
    return int(e);
}

} // extern "C"
