// refit.cu - device scene update: vertex transform, triangle precompute and BVH refit.
//
// Restates GPUSceneState::update (libraries/hvvr/raycaster/gpu_scene_state.cu:377-451):
//   transformVertsKernel  <- SceneTransformVerticesKernel (gpu_scene_state.cu:88-132)
//   precomputeTrisKernel  <- ScenePrecomputeTrianglesKernel (gpu_scene_state.cu:167-244)
//   leafBoundsKernel      <- the leaf-slot atomicMax on float-flipped integers (gpu_scene_state.cu:214-235)
//                            plus SceneRefitIntFixupKernel; a leaf slot owns a contiguous
//                            triangle range, so one thread reduces it without atomics, using
//                            the same ordering (per-triangle max3, then the float-flip order)
//   internalRefitKernel   <- SceneRefitNode{SinglePass,MultiPass}Kernel (gpu_scene_state.cu:273-375):
//                            bottom-up from the nodes without internal children; each node's
//                            arrival counter is bumped by its children and the last child to
//                            arrive continues with the parent, so no thread ever waits.
#include "dev_common.cuh"

#include <cuda_fp16.h>

namespace hvb {

namespace {

__device__ __forceinline__ uint32_t floatFlip(uint32_t f) {
    const uint32_t mask = uint32_t(-int32_t(f >> 31)) | 0x80000000u;
    return f ^ mask;
}
__device__ __forceinline__ uint32_t ifloatFlip(uint32_t f) {
    const uint32_t mask = ((f & 0x80000000u) == 0) ? 0xffffffffu : 0x80000000u;
    return f ^ mask;
}

// matrix4x4 * vector4(p, 1), one output component: the columns summed left to right, or, for the
// fused mode, as the reference's GPU build (nvcc, -use_fast_math) contracts that sum in
// SceneTransformVerticesKernel (gpu_scene_state.cu:118): the first column's product fused into the
// rounded second one, the third fused into that, then the fourth (times w = 1) added. Matched
// bit for bit against that kernel's output on rotated and scaled models.
template <bool Fma>
__device__ __forceinline__ float xformRow(const Mat4& M, int r, float x, float y, float z) {
    if (Fma) return fmaf(M.m[3][r], 1.0f, fmaf(M.m[2][r], z, fmaf(M.m[0][r], x, M.m[1][r] * y)));
    return M.m[0][r] * x + M.m[1][r] * y + M.m[2][r] * z + M.m[3][r] * 1.0f;
}

template <bool Fma>
__global__ void transformVertsKernel(const float4* __restrict__ in, float4* __restrict__ out,
                                     const uint32_t* __restrict__ vertModel, const Mat4* __restrict__ xf,
                                     uint32_t count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float4 a = in[2 * size_t(i)], b = in[2 * size_t(i) + 1];
    const Mat4 M = xf[vertModel[i]];
    const float w = xformRow<Fma>(M, 3, a.x, a.y, a.z);
    const F3 p = f3(xformRow<Fma>(M, 0, a.x, a.y, a.z), xformRow<Fma>(M, 1, a.x, a.y, a.z),
                    xformRow<Fma>(M, 2, a.x, a.y, a.z));
    const float iw = 1.0f / w;
    const uint32_t n01 = __float_as_uint(a.w), n23 = __float_as_uint(b.x);
    const F3 n = f3(__half2float(__ushort_as_half((unsigned short)(n01 & 0xffffu))),
                    __half2float(__ushort_as_half((unsigned short)(n01 >> 16))),
                    __half2float(__ushort_as_half((unsigned short)(n23 & 0xffffu))));
    const F3 nn = normalize3(xformDir(M, n));
    const uint32_t hx = __half_as_ushort(__float2half_rn(nn.x));
    const uint32_t hy = __half_as_ushort(__float2half_rn(nn.y));
    const uint32_t hz = __half_as_ushort(__float2half_rn(nn.z));
    const uint32_t hw = __half_as_ushort(__float2half_rn(0.0f));
    out[2 * size_t(i)] = make_float4(p.x * iw, p.y * iw, p.z * iw, __uint_as_float(hx | (hy << 16)));
    out[2 * size_t(i) + 1] = make_float4(__uint_as_float(hz | (hw << 16)), b.y, b.z, b.w);
}

__global__ void precomputeTrisKernel(const uint4* __restrict__ triShade, const float4* __restrict__ verts,
                                     float4* __restrict__ tris, uint32_t count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint4 t = triShade[i];
    const float4 p0 = verts[2 * size_t(t.x)], p1 = verts[2 * size_t(t.y)], p2 = verts[2 * size_t(t.z)];
    const F3 v0 = f3(p0.x, p0.y, p0.z);
    const F3 e0 = f3(p1.x, p1.y, p1.z) - v0;
    const F3 e1 = f3(p2.x, p2.y, p2.z) - v0;
    tris[3 * size_t(i) + 0] = make_float4(v0.x, v0.y, v0.z, e0.x);
    tris[3 * size_t(i) + 1] = make_float4(e0.y, e0.z, e1.x, e1.y);
    tris[3 * size_t(i) + 2] = make_float4(e1.z, 0.0f, 0.0f, 0.0f);
}

__global__ void leafBoundsKernel(Node* __restrict__ nodes, uint32_t nodeCount, const uint4* __restrict__ triShade,
                                 const float4* __restrict__ verts) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nodeCount) return;
    Node& node = nodes[n];
    const uint32_t leafMask = node.leafMask;
    for (int k = 0; k < 4; k++) {
        if (!(leafMask & (1u << k))) continue;
        uint32_t acc[6];
        for (int j = 0; j < 6; j++) acc[j] = floatFlip(0xff800000u);
        const uint32_t t0 = node.tri[k], t1 = node.tri[k + 1];
        for (uint32_t t = t0; t < t1; t++) {
            const uint4 ts = triShade[t];
            const float4 a = verts[2 * size_t(ts.x)], b = verts[2 * size_t(ts.y)], c = verts[2 * size_t(ts.z)];
            const float mx[3] = {tmaxf(a.x, tmaxf(b.x, c.x)), tmaxf(a.y, tmaxf(b.y, c.y)), tmaxf(a.z, tmaxf(b.z, c.z))};
            const float nm[3] = {tmaxf(-a.x, tmaxf(-b.x, -c.x)), tmaxf(-a.y, tmaxf(-b.y, -c.y)),
                                 tmaxf(-a.z, tmaxf(-b.z, -c.z))};
            for (int ax = 0; ax < 3; ax++) {
                acc[2 * ax] = max(acc[2 * ax], floatFlip(__float_as_uint(mx[ax])));
                acc[2 * ax + 1] = max(acc[2 * ax + 1], floatFlip(__float_as_uint(nm[ax])));
            }
        }
        for (int j = 0; j < 6; j++) node.b[j][k] = __uint_as_float(ifloatFlip(acc[j]));
    }
}

__global__ void internalRefitKernel(Node* nodes, const uint32_t* __restrict__ starts, uint32_t startCount,
                                    const uint32_t* __restrict__ parentSlot, const uint32_t* __restrict__ internalCount,
                                    uint32_t* arrivals, uint32_t maxSteps, uint32_t* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= startCount) return;
    uint32_t n = starts[i];
    for (uint32_t step = 0; step <= maxSteps; step++) {
        const uint32_t ps = parentSlot[n];
        if (ps == 0xffffffffu) return; // reached a root
        const float* bp = nodes[n].b[0];
        float s[6];
        for (int j = 0; j < 6; j++) {
            const float b0 = __ldcg(bp + 4 * j + 0), b1 = __ldcg(bp + 4 * j + 1);
            const float b2 = __ldcg(bp + 4 * j + 2), b3 = __ldcg(bp + 4 * j + 3);
            s[j] = tmaxf(b0, tmaxf(b1, tmaxf(b2, b3)));
        }
        const uint32_t parent = ps >> 2, slot = ps & 3u;
        for (int j = 0; j < 6; j++) __stcg(&nodes[parent].b[j][slot], s[j]);
        __threadfence();
        const uint32_t old = atomicAdd(&arrivals[parent], 1u);
        if (old + 1u != internalCount[parent]) return; // a sibling is still on its way up
        __threadfence();
        n = parent;
    }
    atomicOr(status, kStatusRefitTimeout);
}

} // namespace

cudaError_t launchRefit(const SceneDev& s, bool fma, cudaStream_t st) {
    if (s.vertCount) {
        auto k = fma ? transformVertsKernel<true> : transformVertsKernel<false>;
        k<<<(s.vertCount + 255) / 256, 256, 0, st>>>(s.vertsIn, s.verts, s.vertModel, s.modelToWorld, s.vertCount);
    }
    if (s.triCount) {
        precomputeTrisKernel<<<(s.triCount + 255) / 256, 256, 0, st>>>(s.triShade, s.verts, s.tris, s.triCount);
    }
    if (s.nodeCount) {
        leafBoundsKernel<<<(s.nodeCount + 127) / 128, 128, 0, st>>>(s.nodes, s.nodeCount, s.triShade, s.verts);
        cudaError_t e = cudaMemsetAsync(s.arrivals, 0, sizeof(uint32_t) * (size_t(s.nodeCount) + 1), st);
        if (e != cudaSuccess) return e;
        if (s.refitStartCount) {
            internalRefitKernel<<<(s.refitStartCount + 127) / 128, 128, 0, st>>>(
                s.nodes, s.refitStarts, s.refitStartCount, s.parentSlot, s.internalCount, s.arrivals, s.maxDepth + 1,
                s.arrivals + s.nodeCount);
        }
    }
    return cudaGetLastError();
}

} // namespace hvb
