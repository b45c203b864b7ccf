// GPU-side harness around the reference's own texture code (libraries/hvvr/raycaster/texture.cu
// and ReadTexture, shading.h:45-47), built with nvcc for sm_100a into oracle/_ref/libhvvr_ref_gpu.so.
// Test infrastructure only: the GPU tests use it to pin the library's texture objects (mip chain
// and tex2DGrad results) against the reference's texture creation and sampling on the same GPU,
// and to sample the oracle's texture queries through the reference's code.
#include "cuda_decl.h"
#include "graphics_types.h"
#include "shading.h"
#include "texture.h"
#include "texture_internal.h"

#include <cuda_runtime.h>
#include <stdint.h>

namespace hvvr {
extern cudaTextureObject_t* gDeviceTextureArray;
extern Texture2D gTextureAtlas[SimpleMaterial::maxTextureCount];
} // namespace hvvr

namespace {

// one thread per query: ReadTexture (shading.h:45-47) at q[i] = {u, v, ddx.x, ddx.y, ddy.x, ddy.y}
__global__ void sampleKernel(uint32_t n, const uint32_t* ids, const float* q, float4* out,
                             cudaTextureObject_t* textures) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = q + 6 * size_t(i);
    const hvvr::vector4 c = hvvr::ReadTexture(textures, ids[i], hvvr::vector2(p[0], p[1]), hvvr::vector2(p[2], p[3]),
                                              hvvr::vector2(p[4], p[5]));
    out[i] = make_float4(c.x, c.y, c.z, c.w);
}

} // namespace

extern "C" {

// hvvr::CreateTexture (texture.cu:201-272): upload, reference mip generation, texture object.
// Returns the texture's index in the reference's global atlas. The reference prints one line
// per texture and exits the process on a CUDA error.
int ref_gpu_texture_create(const uint8_t* data, uint32_t format, uint32_t width, uint32_t height,
                           uint32_t strideElements) {
    hvvr::TextureData td;
    td.data = data;
    td.format = hvvr::TextureFormat(format);
    td.width = width;
    td.height = height;
    td.strideElements = strideElements;
    return int(hvvr::CreateTexture(td));
}

// mip level `level` of atlas texture `id` into out (rows of width * elementSize bytes)
int ref_gpu_texture_read_level(uint32_t id, uint32_t level, void* out, uint64_t capacity, uint32_t* w, uint32_t* h) {
    const hvvr::Texture2D& t = hvvr::gTextureAtlas[id];
    cudaArray_t a = nullptr;
    cudaError_t e = cudaGetMipmappedArrayLevel(&a, t.d_rawMipMappedMemory, level);
    if (e != cudaSuccess) return int(e);
    cudaExtent ext;
    e = cudaArrayGetInfo(nullptr, &ext, nullptr, a);
    if (e != cudaSuccess) return int(e);
    const size_t hh = ext.height ? ext.height : 1;
    *w = uint32_t(ext.width);
    *h = uint32_t(hh);
    const size_t row = ext.width * t.elementSize;
    if (!out) return 0;
    if (row * hh > capacity) return -1;
    return int(cudaMemcpy2DFromArray(out, row, a, 0, 0, row, hh, cudaMemcpyDeviceToHost));
}

// n texture reads through ReadTexture on the default stream; q is [n][6], out is [n][4]
int ref_gpu_texture_sample(uint32_t n, const uint32_t* ids, const float* q, float* out) {
    if (n == 0) return 0;
    uint32_t* dIds = nullptr;
    float* dQ = nullptr;
    float4* dOut = nullptr;
    cudaError_t e = cudaMalloc((void**)&dIds, n * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dQ, size_t(n) * 6 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dOut, size_t(n) * sizeof(float4));
    if (e == cudaSuccess) e = cudaMemcpy(dIds, ids, n * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dQ, q, size_t(n) * 6 * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        sampleKernel<<<(n + 127) / 128, 128>>>(n, dIds, dQ, dOut, hvvr::gDeviceTextureArray);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dOut, size_t(n) * sizeof(float4), cudaMemcpyDeviceToHost);
    cudaFree(dIds);
    cudaFree(dQ);
    cudaFree(dOut);
    return int(e);
}

} // extern "C"
