// texture.cu - material texture kernels: the mip chain generator and the parity read-back of
// texture reads. Texture objects and arrays are made on the host (texture.cpp).
#include "dev_common.cuh"
#include "texture_dev.h"

#include <cuda_runtime.h>

namespace hvb {
namespace {

// d_mipmap (libraries/hvvr/raycaster/texture.cu:78-104): level + 1 texel (x, y) is the mean of
// four bilinear reads of the level above at normalized ((x + i) / w, (y + j) / h), w x h being
// the new level's size, through a clamp-addressed linear-filtered texture object without sRGB
// decode. The 8-bit formats store min(mean * 255, 255) truncated, as the reference does; the
// 16-bit unorm format stores min(mean * 65535, 65535) truncated and the float formats the mean
// itself (the reference's 8-bit store into their wider texels is not a defined operation).
template <uint32_t Format>
__global__ void mipLevelKernel(cudaSurfaceObject_t out, cudaTextureObject_t in, uint32_t w, uint32_t h) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    // float px = 1.0 / float(imageW): a double quotient rounded to float
    const float px = float(1.0 / double(float(w)));
    const float py = float(1.0 / double(float(h)));
    if (x >= w || y >= h) return;
    const float4 a = tex2D<float4>(in, float(x + 0) * px, float(y + 0) * py);
    const float4 b = tex2D<float4>(in, float(x + 1) * px, float(y + 0) * py);
    const float4 c = tex2D<float4>(in, float(x + 1) * px, float(y + 1) * py);
    const float4 d = tex2D<float4>(in, float(x + 0) * px, float(y + 1) * py);
    float4 m = make_float4(((a.x + b.x) + c.x) + d.x, ((a.y + b.y) + c.y) + d.y, ((a.z + b.z) + c.z) + d.z,
                           ((a.w + b.w) + c.w) + d.w);
    m = make_float4(m.x / 4.0f, m.y / 4.0f, m.z / 4.0f, m.w / 4.0f);
    if (Format == kTexRgba8Srgb || Format == kTexRgba8) {
        const float r = fminf(m.x * 255.0f, 255.0f), g = fminf(m.y * 255.0f, 255.0f);
        const float bb = fminf(m.z * 255.0f, 255.0f), al = fminf(m.w * 255.0f, 255.0f);
        surf2Dwrite(make_uchar4((unsigned char)r, (unsigned char)g, (unsigned char)bb, (unsigned char)al), out,
                    x * 4, y);
    } else if (Format == kTexRgba16) {
        const float r = fminf(m.x * 65535.0f, 65535.0f), g = fminf(m.y * 65535.0f, 65535.0f);
        const float bb = fminf(m.z * 65535.0f, 65535.0f), al = fminf(m.w * 65535.0f, 65535.0f);
        surf2Dwrite(make_ushort4((unsigned short)r, (unsigned short)g, (unsigned short)bb, (unsigned short)al), out,
                    x * 8, y);
    } else if (Format == kTexRgba32f) {
        surf2Dwrite(m, out, x * 16, y);
    } else if (Format == kTexRgba16f) {
        surf2Dwrite(make_ushort4(__half_as_ushort(__float2half_rn(m.x)), __half_as_ushort(__float2half_rn(m.y)),
                                 __half_as_ushort(__float2half_rn(m.z)), __half_as_ushort(__float2half_rn(m.w))),
                    out, x * 8, y);
    } else {
        surf2Dwrite(m.x, out, x * 4, y);
    }
}

__global__ void textureSampleKernel(cudaTextureObject_t t, uint32_t n, const float* __restrict__ q,
                                    float4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = q + 6 * size_t(i);
    out[i] = readTexture(t, p[0], p[1], make_float2(p[2], p[3]), make_float2(p[4], p[5]));
}

} // namespace

cudaError_t launchMipLevel(uint32_t format, cudaSurfaceObject_t out, cudaTextureObject_t in, uint32_t w, uint32_t h,
                           cudaStream_t st) {
    const dim3 block(16, 16, 1);
    const dim3 grid((w + 15) / 16, (h + 15) / 16, 1);
    switch (format) {
    case kTexRgba8Srgb: mipLevelKernel<kTexRgba8Srgb><<<grid, block, 0, st>>>(out, in, w, h); break;
    case kTexRgba8: mipLevelKernel<kTexRgba8><<<grid, block, 0, st>>>(out, in, w, h); break;
    case kTexRgba16: mipLevelKernel<kTexRgba16><<<grid, block, 0, st>>>(out, in, w, h); break;
    case kTexRgba32f: mipLevelKernel<kTexRgba32f><<<grid, block, 0, st>>>(out, in, w, h); break;
    case kTexRgba16f: mipLevelKernel<kTexRgba16f><<<grid, block, 0, st>>>(out, in, w, h); break;
    case kTexR32f: mipLevelKernel<kTexR32f><<<grid, block, 0, st>>>(out, in, w, h); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launchTextureSample(cudaTextureObject_t t, uint32_t n, const float* q, float4* out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    textureSampleKernel<<<(n + 127) / 128, 128, 0, st>>>(t, n, q, out);
    return cudaGetLastError();
}

} // namespace hvb
