// GPU-side harness around the reference's own foveated resolve kernels (libraries/hvvr/raycaster/
// gpu_foveated.cu: ComputeMoments, FoveatedPolarToScreenSpaceKernel, SeparableFilterUsingEccentricity,
// FinishConstrastEnhancement), built with nvcc for sm_100a into oracle/_ref/libhvvr_ref_gpu.so.
// Test infrastructure only. The kernels are compiled from the reference's source files (and
// RemapPolarFoveatedKernel from remap.cu), included
// here so that this translation unit can instantiate and launch them the way
// GPUCamera::foveatedPolarToScreenSpace (gpu_foveated.cu:335-375) does, on textures made by the
// reference's createEmptyTexture with the formats and addressing of GPUCamera's foveated setup
// (gpu_camera.cu:170-230).
#include "gpu_foveated.cu"
#include "remap.cu"

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

namespace hvvr {
// Setup-time functions GPUCamera methods in gpu_foveated.cu refer to; the harness launches the
// resolve kernels only, so these are never called.
void ComputeEyeSpaceFrusta(const GPUBuffer<DirectionalBeam>&, GPUBuffer<SimpleRayFrustum>&,
                           GPUBuffer<SimpleRayFrustum>&) {
    fprintf(stderr, "ref_gpu_foveated: ComputeEyeSpaceFrusta is not part of the harness\n");
    abort();
}
namespace traverse {
namespace avx {
Frustum::Frustum(const vector3*, const vector3*) {
    fprintf(stderr, "ref_gpu_foveated: traverse::avx::Frustum is not part of the harness\n");
    abort();
}
} // namespace avx
} // namespace traverse
} // namespace hvvr

namespace {

cudaError_t upload(const hvvr::Texture2D& t, const void* src, size_t texelBytes) {
    return cudaMemcpy2DToArray(t.d_rawMemory, 0, 0, src, t.width * texelBytes, t.width * texelBytes, t.height,
                               cudaMemcpyHostToDevice);
}
cudaError_t download(void* dst, const hvvr::Texture2D& t, size_t texelBytes) {
    return cudaMemcpy2DFromArray(dst, t.width * texelBytes, t.d_rawMemory, 0, 0, t.width * texelBytes, t.height,
                                 cudaMemcpyDeviceToHost);
}
void release(hvvr::Texture2D& t) {
    cudaDestroyTextureObject(t.d_texObject);
    cudaDestroySurfaceObject(t.d_surfaceObject);
    cudaFreeArray(t.d_rawMemory);
}

} // namespace

extern "C" {

// One resolve of the reference's foveated path on given polar textures. Inputs: the foveated
// pattern parameters (RayCasterSpecification::foveatedSamplePattern), the raw polar colour
// [rings][samplesPerRing] (RGBA8 sRGB) and depth (float), the output size, sampleToEye (3x3) and
// eyeToSamplePrevious (4x4) as the reference's column-major matrices, and the previous result
// [height][width] (RGBA8 sRGB). Outputs: the moments [rings][samplesPerRing][2][4] (unorm16), the
// temporally filtered result texture and the first (vertical) filter pass [height][width]
// (RGBA8 sRGB), and the final image [height][width].
int ref_gpu_foveated_resolve(float degreeTrackingError, float maxFovDegrees, float marSlope, float fovealMarDegrees,
                             uint32_t samplesPerRing, uint32_t ringCount, const uint32_t* polarColor,
                             const float* polarDepth, uint32_t width, uint32_t height, const float* sampleToEye9,
                             const float* eyeToSamplePrev16, const uint32_t* history, uint16_t* moments,
                             uint32_t* result, uint32_t* filtered, uint32_t* image);

// RemapPolarFoveatedKernel (remap.cu:126-141) as GPUCamera::remapPolarFoveated launches it: the
// sample colours (RGBA8 sRGB) and view depths [valid] scattered by remap [valid] (x, y) into
// polar textures [ringCount][samplesPerRing] made as GPUCamera's (initially zero), read back into
// polarColor and polarDepth. valid must equal samplesPerRing * ringCount (the polar set fills its
// texture).
int ref_gpu_foveated_scatter(uint32_t samplesPerRing, uint32_t ringCount, uint32_t valid, const uint32_t* colors,
                             const float* tmax, const uint32_t* remap, uint32_t* polarColor, float* polarDepth) {
    using namespace hvvr;
    if (size_t(valid) != size_t(samplesPerRing) * ringCount) return -1;
    Texture2D raw = createEmptyTexture(samplesPerRing, ringCount, TextureFormat::r8g8b8a8_unorm_srgb,
                                       cudaAddressModeWrap, cudaAddressModeClamp, true);
    Texture2D depth = createEmptyTexture(samplesPerRing, ringCount, TextureFormat::r32_float, cudaAddressModeWrap,
                                         cudaAddressModeClamp, false);
    const size_t n = valid;
    std::vector<uint32_t> zeros(n, 0u);
    cudaError_t e = upload(raw, zeros.data(), 4);
    if (e == cudaSuccess) e = upload(depth, zeros.data(), 4);
    uint32_t *dColors = nullptr, *dRemap = nullptr;
    float* dTmax = nullptr;
    if (e == cudaSuccess) e = cudaMalloc((void**)&dColors, n * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&dTmax, n * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&dRemap, n * 8);
    if (e == cudaSuccess) e = cudaMemcpy(dColors, colors, n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dTmax, tmax, n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dRemap, remap, n * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        KernelDim dim = KernelDim(valid, CUDA_GROUP_SIZE);
        RemapPolarFoveatedKernel<<<dim.grid, dim.block>>>(dColors, dTmax, (vector2ui*)dRemap, raw, depth, n);
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = download(polarColor, raw, 4);
    if (e == cudaSuccess) e = download(polarDepth, depth, 4);
    cudaFree(dColors);
    cudaFree(dTmax);
    cudaFree(dRemap);
    release(raw);
    release(depth);
    return int(e);
}

int ref_gpu_foveated_resolve(float degreeTrackingError, float maxFovDegrees, float marSlope, float fovealMarDegrees,
                             uint32_t samplesPerRing, uint32_t ringCount, const uint32_t* polarColor,
                             const float* polarDepth, uint32_t width, uint32_t height, const float* sampleToEye9,
                             const float* eyeToSamplePrev16, const uint32_t* history, uint16_t* moments,
                             uint32_t* result, uint32_t* filtered, uint32_t* image) {
    using namespace hvvr;
    GPUCamera::PolarTextures polar;
    auto polarImage = [&](TextureFormat f, bool linear) {
        return createEmptyTexture(samplesPerRing, ringCount, f, cudaAddressModeWrap, cudaAddressModeClamp, linear);
    };
    polar.raw = polarImage(TextureFormat::r8g8b8a8_unorm_srgb, true);
    polar.depth = polarImage(TextureFormat::r32_float, false);
    polar.moment1 = polarImage(TextureFormat::r16g16b16a16_unorm, true);
    polar.moment2 = polarImage(TextureFormat::r16g16b16a16_unorm, true);
    auto screenImage = [&]() {
        return createEmptyTexture(width, height, TextureFormat::r8g8b8a8_unorm_srgb, cudaAddressModeClamp,
                                  cudaAddressModeClamp);
    };
    Texture2D resultTexture = screenImage(), previousResultTexture = screenImage();
    Texture2D horizontallyFiltered = screenImage(), fullyFiltered = screenImage();
    GPUImage resultImage;
    resultImage.update(width, height, width, PixelFormat::RGBA8_SRGB);

    cudaError_t e = upload(polar.raw, polarColor, 4);
    if (e == cudaSuccess) e = upload(polar.depth, polarDepth, 4);
    if (e == cudaSuccess) e = upload(previousResultTexture, history, 4);

    EccentricityToTexCoordMapping eToTexMap;
    eToTexMap.eccentricityMap = EccentricityMap(marSlope, fovealMarDegrees, degreeTrackingError);
    eToTexMap.texMapSize = (float)polar.raw.height;
    eToTexMap.invTexMapSize = 1.0f / polar.raw.height;
    eToTexMap.invMaxEccentricity = 1.0f / (maxFovDegrees * RadiansPerDegree);
    matrix3x3 sampleToEye;
    matrix4x4 eyeToSamplePrevious;
    static_assert(sizeof(matrix3x3) == 36 && sizeof(matrix4x4) == 64, "matrix layouts");
    memcpy(&sampleToEye, sampleToEye9, 36);
    memcpy(&eyeToSamplePrevious, eyeToSamplePrev16, 64);
    TemporalFilterSettings temporal;
    ContrastEnhancementSettings contrast;
    contrast.enable = true;
    contrast.f_e = 1.0f;

    if (e == cudaSuccess) {
        KernelDim dim = KernelDim(width, height, CUDA_GROUP_WIDTH, CUDA_GROUP_HEIGHT);
        KernelDim polDim = KernelDim(samplesPerRing, ringCount, CUDA_GROUP_WIDTH, CUDA_GROUP_HEIGHT);
        ComputeMoments<PixelFormat::RGBA16><<<polDim.grid, polDim.block>>>(polar);
        FoveatedPolarToScreenSpaceKernel<PixelFormat::RGBA8_SRGB><<<dim.grid, dim.block>>>(
            polar, resultTexture, resultImage, sampleToEye, eToTexMap, previousResultTexture, eyeToSamplePrevious,
            temporal);
        SeparableFilterUsingEccentricity<PixelFormat::RGBA8_SRGB><<<dim.grid, dim.block>>>(
            horizontallyFiltered, resultTexture, {0, 1}, contrast, sampleToEye);
        SeparableFilterUsingEccentricity<PixelFormat::RGBA8_SRGB><<<dim.grid, dim.block>>>(
            fullyFiltered, horizontallyFiltered, {1, 0}, contrast, sampleToEye);
        FinishConstrastEnhancement<PixelFormat::RGBA8_SRGB><<<dim.grid, dim.block>>>(
            resultImage, resultTexture, fullyFiltered, contrast, sampleToEye, eToTexMap);
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess && moments) {
        const size_t n = size_t(samplesPerRing) * ringCount;
        uint64_t* m1 = (uint64_t*)malloc(n * 8);
        uint64_t* m2 = (uint64_t*)malloc(n * 8);
        e = download(m1, polar.moment1, 8);
        if (e == cudaSuccess) e = download(m2, polar.moment2, 8);
        for (size_t k = 0; e == cudaSuccess && k < n; k++) {
            memcpy(moments + 8 * k, &m1[k], 8);
            memcpy(moments + 8 * k + 4, &m2[k], 8);
        }
        free(m1);
        free(m2);
    }
    if (e == cudaSuccess && result) e = download(result, resultTexture, 4);
    if (e == cudaSuccess && filtered) e = download(filtered, horizontallyFiltered, 4);
    if (e == cudaSuccess && image)
        e = cudaMemcpy(image, resultImage.data(), size_t(width) * height * 4, cudaMemcpyDeviceToHost);
    cudaFree(resultImage.data());
    release(polar.raw);
    release(polar.depth);
    release(polar.moment1);
    release(polar.moment2);
    release(resultTexture);
    release(previousResultTexture);
    release(horizontallyFiltered);
    release(fullyFiltered);
    return int(e);
}

} // extern "C"
