// foveated_resolve.cu - the foveated resolve: polar sample texture -> screen image.
//
// The reference's resolve (GPUCamera::remapPolarFoveated and
// ::foveatedPolarToScreenSpace, libraries/hvvr/raycaster/remap.cu:143-156 and
// gpu_foveated.cu:335-375):
//   polarScatterKernel     RemapPolarFoveatedKernel          remap.cu:126-141
//   momentsKernel          ComputeMoments                    gpu_foveated.cu:124-139, 159-172
//   polarToScreenKernel    FoveatedPolarToScreenSpaceKernel  gpu_foveated.cu:36-122, 141-157, 174-249
//   filterEnhanceKernel    SeparableFilterUsingEccentricity  gpu_foveated.cu:251-294 (vertical, then horizontal)
//                          and FinishConstrastEnhancement    gpu_foveated.cu:296-333, fused (below)
//
// Every texture is a CUDA array read through a texture object and written through a surface
// object, made with the reference's texture setup (createEmptyTexture, texture.cu:283-321, with
// the formats and addressing of gpu_camera.cu:174-183, 217-227): the filtering, the sRGB decode
// and the unorm16 conversion are the texture unit's own. This file is compiled with fast math as
// the reference's kernels are (powf, logf, cosf, sinf, sqrtf and divisions take the fast forms),
// and every expression keeps the reference's operation order, so that the resolve reproduces the
// reference's kernels on the same GPU.
#include "dev_common.cuh"

namespace hvb {

namespace {

constexpr float kPi = 3.141592653589f;  // libraries/hvvr/shared/constants_math.h:15

struct V2 {
    float x, y;
};
struct V4 {
    float x, y, z, w;
};
__device__ __forceinline__ V4 v4(float4 c) { return V4{c.x, c.y, c.z, c.w}; }
__device__ __forceinline__ V4 operator+(V4 a, V4 b) { return V4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
__device__ __forceinline__ V4 operator-(V4 a, V4 b) { return V4{a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
__device__ __forceinline__ V4 operator*(V4 a, V4 b) { return V4{a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
__device__ __forceinline__ V4 operator*(V4 a, float s) { return V4{a.x * s, a.y * s, a.z * s, a.w * s}; }
// vector4 / float multiplies by the reciprocal (libraries/hvvr/shared/vector_math.h:359-362)
__device__ __forceinline__ V4 divs(V4 a, float s) {
    const float inv = 1.0f / s;
    return a * inv;
}
// clamp(x, lo, hi) = min(hi, max(lo, x)) (libraries/hvvr/shared/util.h:56)
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(hi, fmaxf(lo, x)); }
__device__ __forceinline__ int clampi(int x, int lo, int hi) { return min(hi, max(lo, x)); }
// lerp(a, b, t) = a + (b - a) t (util.h:58)
__device__ __forceinline__ float lerpf(float a, float b, float t) { return a + (b - a) * t; }

// linearToSRgb / sRgbToLinear (libraries/hvvr/shared/util_graphics.h:16-33)
__device__ __forceinline__ float toSrgb(float x) {
    return (x <= 0.0031308f) ? (x * 12.92f) : (powf(x, (1.0f / 2.4f)) * 1.055f - .055f);
}
__device__ __forceinline__ float fromSrgb(float x) {
    return (x <= 0.04045f) ? x * (1.0f / 12.92f) : powf((x + .055f) * (1.0f / 1.055f), 2.4f);
}
// ToColor4Unorm8SRgb(vector4) (shading_helpers.h:193-200): sRGB rgb, linear alpha, truncating * 255
__device__ __forceinline__ uint32_t encodeSrgb(V4 c) {
    const uint32_t r = uint32_t(toSrgb(c.x) * 255.0f);
    const uint32_t g = uint32_t(toSrgb(c.y) * 255.0f);
    const uint32_t b = uint32_t(toSrgb(c.z) * 255.0f);
    const uint32_t a = uint32_t(c.w * 255.0f);
    return r | (g << 8) | (b << 16) | (a << 24);
}
// FromColor4Unorm8SRgb (shading_helpers.h:218-225)
__device__ __forceinline__ V4 decodeSrgb(uint32_t c) {
    const float r = (c & 0xFF) / 255.0f;
    const float g = ((c >> 8) & 0xFF) / 255.0f;
    const float b = ((c >> 16) & 0xFF) / 255.0f;
    const float a = ((c >> 24) & 0xFF) / 255.0f;
    return V4{fromSrgb(r), fromSrgb(g), fromSrgb(b), a};
}
// ToColor4Unorm16 (shading_helpers.h:201-208): truncating * 65535, packed r | g << 16 | b << 32 | a << 48
__device__ __forceinline__ unsigned long long encodeUnorm16(V4 c) {
    const float C = 65535.0f;
    const unsigned long long r = (unsigned long long)(c.x * C);
    const unsigned long long g = (unsigned long long)(c.y * C);
    const unsigned long long b = (unsigned long long)(c.z * C);
    const unsigned long long a = (unsigned long long)(c.w * C);
    return r | (g << 16) | (b << 32) | (a << 48);
}

__device__ __forceinline__ V4 fetch(cudaTextureObject_t t, float u, float v) { return v4(tex2D<float4>(t, u, v)); }

// getNormalizedCoord (gpu_foveated.cu:92-94)
__device__ __forceinline__ V2 normalizedCoord(int x, int y, int width, int height) {
    return V2{((float)x + 0.5f) / (float)width, ((float)y + 0.5f) / (float)height};
}
// texelFetch (gpu_foveated.cu:260-263): a linear read at the texel's centre
__device__ __forceinline__ V4 texelFetch(cudaTextureObject_t t, uint32_t w, uint32_t h, int i, int j) {
    const V2 c = normalizedCoord(i, j, int(w), int(h));
    return fetch(t, c.x, c.y);
}
// sampleSpaceToEyeSpaceMatrix * (coord, 1), normalized (vector_math.h:273-275, 1129-1132), then
// eyeSpaceDirectionToAngularEyeCoord (gpu_foveated.cu:103-107)
__device__ __forceinline__ void eyeCoord(const float* S, V2 nc, float& theta, float& ecc) {
    const float vx = S[0] * nc.x + S[3] * nc.y + S[6] * 1.0f;
    const float vy = S[1] * nc.x + S[4] * nc.y + S[7] * 1.0f;
    const float vz = S[2] * nc.x + S[5] * nc.y + S[8] * 1.0f;
    const float len = sqrtf(vx * vx + vy * vy + vz * vz);
    const float inv = 1.0f / len;
    const float dx = vx * inv, dy = vy * inv, dz = vz * inv;
    ecc = acosf(-dz);
    theta = -atan2f(dy, dx);
}
// getEccentricity (gpu_foveated.cu:251-258)
__device__ __forceinline__ float pixelEccentricity(const FoveaDev& f, uint32_t i, uint32_t j) {
    float theta, ecc;
    eyeCoord(f.sampleToEye, normalizedCoord(int(i), int(j), int(f.width), int(f.height)), theta, ecc);
    return ecc;
}

// EccentricityMap::applyInverse (libraries/hvvr/raycaster/foveated.h:106-112)
__device__ __forceinline__ float eccApplyInverse(const FoveaDev& f, float E) {
    const float i0 = E * f.eccInvW0;
    const float sDivW = f.eccS * f.eccInvW0;
    const float x = logf((f.eccM * (i0 - sDivW)) + 1.0f) * f.eccInvLogA;
    const float i1 = x + sDivW;
    return (E < f.eccS) ? i0 : i1;
}

// RemapPolarFoveatedKernel: each sample's colour (through an sRGB decode/encode round trip)
// and view depth to its polar texel
__global__ void __launch_bounds__(256) polarScatterKernel(const ViewDev* views, uint32_t view) {
    const ViewDev& V = views[view];
    const FoveaDev& f = V.fov;
    const uint32_t n = f.valid;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const uint2 tx = f.remap[s];
        const V4 p = decodeSrgb(V.colors[s]);
        const float t = V.tmaxOut[s];
        surf2Dwrite(encodeSrgb(p), f.rawSurf, int(tx.x * 4), int(tx.y));
        surf2Dwrite(t, f.depthSurf, int(tx.x * 4), int(tx.y));
    }
}

// ComputeMoments: mean and mean square of the 3x3 window of bilinear reads around the texel
// (computeMoments3x3Window)
__global__ void __launch_bounds__(256) momentsKernel(const ViewDev* views, uint32_t view) {
    const FoveaDev& f = views[view].fov;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= f.spr || j >= f.rings) return;
    const V2 invDim{1.0f / f.spr, 1.0f / f.rings};
    const V2 coord{invDim.x * i, invDim.y * j};
    const float offsets[3] = {-1.0f, 0.0f, 1.0f};
    V4 m1{0.0f, 0.0f, 0.0f, 0.0f}, m2{0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int x = 0; x < 3; ++x) {
#pragma unroll
        for (int y = 0; y < 3; ++y) {
            const V4 c = fetch(f.rawTex, coord.x + (offsets[x] * invDim.x), coord.y + (offsets[y] * invDim.y));
            m1 = m1 + c;
            m2 = m2 + c * c;
        }
    }
    const float weight = 1.0f / 9.0f;
    m1 = m1 * weight;
    m2 = m2 * weight;
    surf2Dwrite(encodeUnorm16(m1), f.m1Surf, int(i * 8), int(j));
    surf2Dwrite(encodeUnorm16(m2), f.m2Surf, int(i * 8), int(j));
}

// bicubicFast (gpu_foveated.cu:36-71): 4-tap B-spline on the polar colour texture
__device__ __forceinline__ V4 bicubicFast(const FoveaDev& f, V2 coord) {
    const V2 pixCoord{coord.x * float(f.spr), coord.y * float(f.rings)};
    const V2 pixCenter{floorf(pixCoord.x - 0.5f) + 0.5f, floorf(pixCoord.y - 0.5f) + 0.5f};
    const V2 iDim{1.0f / f.spr, 1.0f / f.rings};
    float s0[2], s1[2], t0[2], t1[2];
    const float pc[2] = {pixCoord.x, pixCoord.y}, ctr[2] = {pixCenter.x, pixCenter.y}, id[2] = {iDim.x, iDim.y};
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const float fk = pc[k] - ctr[k];
        const float f2 = fk * fk;
        const float f3 = f2 * fk;
        const float omf2 = (1.0f - fk) * (1.0f - fk);
        const float omf3 = omf2 * (1.0f - fk);
        const float sixth = (1.0f / 6.0f);
        const float w0 = omf3 * sixth;
        const float w1 = ((1.0f * (4.0f / 6.0f)) + f3 * 0.5f) - f2;
        const float w3 = f3 * sixth;
        const float w2 = ((1.0f - w0) - w1) - w3;
        s0[k] = w0 + w1;
        s1[k] = w2 + w3;
        const float f0 = w1 / (w0 + w1);
        const float f1 = w3 / (w2 + w3);
        t0[k] = ((ctr[k] - 1.0f) + f0) * id[k];
        t1[k] = ((ctr[k] + 1.0f) + f1) * id[k];
    }
    const cudaTextureObject_t T = f.rawTex;
    return fetch(T, t0[0], t0[1]) * s0[0] * s0[1] + fetch(T, t1[0], t0[1]) * s1[0] * s0[1] +
           fetch(T, t0[0], t1[1]) * s0[0] * s1[1] + fetch(T, t1[0], t1[1]) * s1[0] * s1[1];
}

// FoveatedPolarToScreenSpaceKernel: bicubic polar lookup, temporal reprojection of the
// previous frame's result clamped to the moments' neighbourhood (clampToNeighborhood),
// eccentricity-dependent blend. The image itself is written by enhanceContrastKernel, which
// overwrites every pixel the reference's kernel writes here.
__global__ void __launch_bounds__(256) polarToScreenKernel(const ViewDev* views, uint32_t view) {
    const FoveaDev& f = views[view].fov;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= f.width || j >= f.height) return;
    float theta, ecc;
    eyeCoord(f.sampleToEye, normalizedCoord(int(i), int(j), int(f.width), int(f.height)), theta, ecc);
    // angularEyeCoordToPolarTextureCoord, eccentricityToTexCoord (gpu_foveated.cu:88-90, 117-122)
    const V2 coord{(theta + kPi) / (2.0f * kPi), (eccApplyInverse(f, ecc) + 0.5f) * f.invTexMapSize};
    const V4 newValue = bicubicFast(f, coord);
    V4 surfaceResult = newValue;
    const float tValue = tex2D<float>(f.depthTex, coord.x, coord.y);
    if (tValue < INFINITY) {
        // angularEyeCoordToDirection (gpu_foveated.cu:96-101) * tValue
        const float z = -cosf(ecc);
        const float xyLength = sqrtf(1.0f - z * z);
        const float px = cosf(-theta) * xyLength, py = sinf(-theta) * xyLength;
        const float ex = px * tValue, ey = py * tValue, ez = z * tValue;
        const float* M = f.eyeToSamplePrev;
        const float qx = M[0] * ex + M[4] * ey + M[8] * ez + M[12] * 1.0f;
        const float qy = M[1] * ex + M[5] * ey + M[9] * ez + M[13] * 1.0f;
        const float qz = M[2] * ex + M[6] * ey + M[10] * ez + M[14] * 1.0f;
        const float iz = 1.0f / qz;
        const float ox = qx * iz, oy = qy * iz;
        float alpha = 0.05f;  // TemporalFilterSettings::alpha (gpu_camera.h:41-45)
        V4 oldValue = newValue;
        if (ox > 0 && oy > 0 && ox < 1 && oy < 1 && tValue > 0) oldValue = fetch(f.prevTex, ox, oy);
        // clampToNeighborhood (stddevMultiplier 1)
        const V4 m1 = fetch(f.m1Tex, coord.x, coord.y);
        const V4 m2 = fetch(f.m2Tex, coord.x, coord.y);
        const V4 var = m2 - (m1 * m1);
        const V4 sd{sqrtf(var.x), sqrtf(var.y), sqrtf(var.z), sqrtf(var.w)};
        const float scaleFactor = 1.0f;
        const V4 minC = m1 - (sd * scaleFactor);
        const V4 maxC = m1 + (sd * scaleFactor);
        V4 co{clampf(oldValue.x, minC.x, maxC.x), clampf(oldValue.y, minC.y, maxC.y),
              clampf(oldValue.z, minC.z, maxC.z), clampf(oldValue.w, minC.w, maxC.w)};
        float normalizedE = ecc * f.invMaxEcc;
        const float mn = 0.2f, mx = 0.35f;
        const float t = clampf((normalizedE - mn) / (mx - mn), 0.f, 1.f);
        alpha = lerpf(0.5f, alpha, t);
        normalizedE = sqrtf(sqrtf(sqrtf(sqrtf(normalizedE))));
        co.x = lerpf(co.x, oldValue.x, normalizedE);
        co.y = lerpf(co.y, oldValue.y, normalizedE);
        co.z = lerpf(co.z, oldValue.z, normalizedE);
        co.w = lerpf(co.w, oldValue.w, normalizedE);
        surfaceResult = newValue * alpha + co * (1.0f - alpha);
    }
    surf2Dwrite(encodeSrgb(surfaceResult), f.resultSurf, int(i * 4), int(j));
}

// The texture unit's value for an RGBA8 sRGB texel read at its centre, per 8-bit code: .x/.y/.z the
// sRGB decode of the code in the red/green/blue channel, .w the linear alpha (read once per
// camera from a 256-texel texture made like the screen textures, decodeTableKernel)
__device__ __forceinline__ V4 decodeTexel(const float4* table, uint32_t c) {
    return V4{table[c & 0xFFu].x, table[(c >> 8) & 0xFFu].y, table[(c >> 16) & 0xFFu].z, table[c >> 24].w};
}

// SeparableFilterUsingEccentricity at pixel (i, j): 11 taps along (sx, sy), clamped at the image
// edges, with weights pow(1 - |R| / 5.1, sqrt(eccentricity)); tap(x, y) is the input value there
template <class Tap>
__device__ __forceinline__ uint32_t eccFilter(const FoveaDev& f, uint32_t i, uint32_t j, int sx, int sy,
                                              float eccentricity, Tap tap) {
    const int filterRadius = 5;
    V4 valueSum{0.0f, 0.0f, 0.0f, 0.0f};
    float weightSum = 0.0f;
#pragma unroll
    for (int R = -filterRadius; R <= filterRadius; ++R) {
        const int tx = clampi(int(i) + R * sx, 0, int(f.width) - 1);
        const int ty = clampi(int(j) + R * sy, 0, int(f.height) - 1);
        const float normDist = fabsf(float(R)) / float(filterRadius + 0.1);
        const float weight = powf(1.0f - normDist, sqrtf(eccentricity));
        valueSum = valueSum + tap(tx, ty) * weight;
        weightSum += weight;
    }
    return encodeSrgb(divs(valueSum, weightSum));
}

// The vertical eccentricity filter, the horizontal one and FinishConstrastEnhancement with
// enhanceContrast (gpu_foveated.cu:251-333; sigma = 8 max(0.001, t^2), f_e = 1, gpu_camera.cu:181)
// in one pass over a tile of 64 x 4 pixels. The reference writes each filter pass to an RGBA8 sRGB
// texture and the next pass reads it at texel centres; here the vertical pass's encoded values for
// the tile and a 5-column halo on each side stay in shared memory, and the horizontal pass and the
// enhancement decode the encoded values through the texture unit's own decode table, so every
// value equals what the texture reads return. The result texture (this frame's temporal result,
// the next frame's history) is still read through its texture object.
constexpr int kFeW = 64, kFeH = 4, kFeRadius = 5, kFeHaloW = kFeW + 2 * kFeRadius;

__global__ void __launch_bounds__(kFeW * kFeH) filterEnhanceKernel(const ViewDev* views, uint32_t view) {
    const FoveaDev& f = views[view].fov;
    __shared__ float4 table[256];
    __shared__ uint32_t vq[kFeH][kFeHaloW];
    const uint32_t tid = threadIdx.y * kFeW + threadIdx.x;
    table[tid] = f.srgbDecode[tid];
    const int x0 = int(blockIdx.x) * kFeW, y0 = int(blockIdx.y) * kFeH;
    // vertical pass of this frame's result over the tile and its halo columns
    for (uint32_t p = tid; p < uint32_t(kFeH * kFeHaloW); p += kFeW * kFeH) {
        const int r = int(p) / kFeHaloW, c = int(p) % kFeHaloW;
        const int j = y0 + r;
        if (j >= int(f.height)) continue;
        const uint32_t ic = uint32_t(clampi(x0 - kFeRadius + c, 0, int(f.width) - 1));
        const float eccentricity = pixelEccentricity(f, ic, uint32_t(j));
        vq[r][c] = eccFilter(f, ic, uint32_t(j), 0, 1, eccentricity, [&](int tx, int ty) {
            return texelFetch(f.resultTex, f.width, f.height, tx, ty);
        });
    }
    __syncthreads();
    const uint32_t i = uint32_t(x0) + threadIdx.x, j = uint32_t(y0) + threadIdx.y;
    if (i >= f.width || j >= f.height) return;
    const float eccentricity = pixelEccentricity(f, i, j);
    // horizontal pass, reading the vertical pass's encoded values as the texture would return them
    const uint32_t hq = eccFilter(f, i, j, 1, 0, eccentricity, [&](int tx, int ty) {
        return decodeTexel(table, vq[ty - y0][tx - (x0 - kFeRadius)]);
    });
    float sigma = 8.0f;
    const float t = eccentricity * f.invMaxEcc;
    sigma *= fmaxf(0.001f, clampf(t * t, 0.f, 1.f));
    const V4 pix = texelFetch(f.resultTex, f.width, f.height, int(i), int(j));
    const V4 pmean = decodeTexel(table, hq);
    const float f_e = 1.0f;
    const float cScale = 1.f + sigma * f_e;
    const V4 scaled = pmean + (pix - pmean) * cScale;
    const V4 r{clampf(scaled.x, 0.0f, 1.0f), clampf(scaled.y, 0.0f, 1.0f), clampf(scaled.z, 0.0f, 1.0f),
               clampf(scaled.w, 0.0f, 1.0f)};
    f.image[size_t(f.imageStride) * j + i] = encodeSrgb(r);
}

// The decode table of filterEnhanceKernel: texel i of `codes` holds (i, i, i, i).
__global__ void decodeTableKernel(cudaTextureObject_t codes, float4* out) {
    const uint32_t i = threadIdx.x;
    out[i] = tex2D<float4>(codes, (float(i) + 0.5f) / 256.0f, 0.5f);
}

} // namespace

cudaError_t launchFoveatedResolve(const FrameDev& fr, uint32_t view, const FoveaDev& fov, cudaStream_t st) {
    if (!fov.image || !fov.width || !fov.height || !fov.spr || !fov.rings) return cudaSuccess;
    // the reference's 16 x 8 thread groups (CUDA_GROUP_WIDTH/HEIGHT, kernel_constants.h:35-36)
    const dim3 blk(16, 8);
    const dim3 polar((fov.spr + 15) / 16, (fov.rings + 7) / 8);
    const dim3 screen((fov.width + 15) / 16, (fov.height + 7) / 8);
    polarScatterKernel<<<(fov.valid + 255) / 256, 256, 0, st>>>(fr.views, view);
    momentsKernel<<<polar, blk, 0, st>>>(fr.views, view);
    polarToScreenKernel<<<screen, blk, 0, st>>>(fr.views, view);
    const dim3 fe((fov.width + kFeW - 1) / kFeW, (fov.height + kFeH - 1) / kFeH);
    filterEnhanceKernel<<<fe, dim3(kFeW, kFeH), 0, st>>>(fr.views, view);
    return cudaGetLastError();
}

cudaError_t launchSrgbDecodeTable(cudaTextureObject_t codes, float4* out, cudaStream_t st) {
    decodeTableKernel<<<1, 256, 0, st>>>(codes, out);
    return cudaGetLastError();
}

} // namespace hvb
