// texture_dev.h - the texture kernels' launchers (texture.cu) and the format values they take.
// Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hvb {

// TextureFormat values (libraries/hvvr/raycaster/texture.h:16-27)
enum : uint32_t {
    kTexRgba8Srgb = 1,
    kTexRgba8 = 2,
    kTexRgba16 = 3,
    kTexRgba32f = 4,
    kTexRgba16f = 5,
    kTexR11G11B10f = 6,
    kTexR32f = 7,
};

// one mip level: out (w x h) from the level above, read through `in`
cudaError_t launchMipLevel(uint32_t format, cudaSurfaceObject_t out, cudaTextureObject_t in, uint32_t w, uint32_t h,
                           cudaStream_t st);
// n texture reads q[i] = {u, v, ddx.x, ddx.y, ddy.x, ddy.y} (device arrays) through t
cudaError_t launchTextureSample(cudaTextureObject_t t, uint32_t n, const float* q, float4* out, cudaStream_t st);

} // namespace hvb
