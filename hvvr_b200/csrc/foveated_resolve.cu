// foveated_resolve.cu - the foveated resolve: polar sample texture -> screen image.
//
// Restates, in the reference's operation order:
//   RemapPolarFoveatedKernel          libraries/hvvr/raycaster/remap.cu:127-141
//   ComputeMoments                    libraries/hvvr/raycaster/gpu_foveated.cu:124-139, 159-172
//   FoveatedPolarToScreenSpaceKernel  gpu_foveated.cu:36-122, 141-157, 174-249
//   SeparableFilterUsingEccentricity  gpu_foveated.cu:251-294 (vertical, then horizontal pass)
//   FinishConstrastEnhancement        gpu_foveated.cu:296-333
//   the pass order of GPUCamera::foveatedPolarToScreenSpace, gpu_foveated.cu:335-375
//
// The reference reads CUDA texture objects. Here every texture is a plain array in HBM read
// by a software texture unit with the reference's texture setup (gpu_camera.cu:174-183,
// 219-227; texture.cu:283-321): normalized coordinates; wrap in azimuth and clamp in
// eccentricity on the polar textures, clamp on the screen planes; linear filtering with the
// fraction quantised to 1/256 (the texture unit's 9-bit fixed-point weights); point sampling
// for the depth; sRGB decode by sRgbToLinear (util_graphics.h:16-23) and unorm16 decode as
// v / 65535. acos, atan2, log, cos, sin and pow are evaluated in double and rounded to float,
// and the sRGB encode (linearToSRgb, util_graphics.h:26-33, then a truncating * 255,
// shading_helpers.h:193-200) is a lookup in 255 thresholds built on the host the same way, so
// the images do not depend on a float math library's last bit.
//
// Fusions that leave every value unchanged: the eccentricity and the five filter weights of a
// pixel are computed once (polar -> screen pass) and read by both filter passes; the second
// filter pass finishes the contrast enhancement itself (its sRGB round trip of the fully
// filtered value is kept); the polar -> screen pass does not write the image, which the
// contrast enhancement overwrites in the reference. A texel fetch at a pixel centre
// (texelFetch) reads the texel directly: for images up to 8192 texels wide the centre's
// filter fraction rounds to 0 or 1, so the linear fetch returns that texel exactly.
#include "dev_common.cuh"

namespace hvb {

namespace {

struct ColorTables {
    float dec[256];  // sRGB byte -> linear: sRgbToLinear(b / 255.0f)
    float thr[256];  // thr[k]: the least float whose encode is >= k (thr[0] unused)
};
__device__ ColorTables gColor;

constexpr float kPi = 3.141592653589f;        // libraries/hvvr/shared/constants_math.h:15
constexpr float kFilterDen = float(5 + 0.1);  // float(filterRadius + 0.1), gpu_foveated.cu:286

__device__ __forceinline__ void loadTables(ColorTables& t) {
    for (uint32_t k = threadIdx.x + threadIdx.y * blockDim.x; k < 256; k += blockDim.x * blockDim.y) {
        t.dec[k] = gColor.dec[k];
        t.thr[k] = gColor.thr[k];
    }
    __syncthreads();
}

__device__ __forceinline__ float dacos(float x) { return float(acos(double(x))); }
__device__ __forceinline__ float datan2(float y, float x) { return float(atan2(double(y), double(x))); }
__device__ __forceinline__ float dlog(float x) { return float(log(double(x))); }
__device__ __forceinline__ float dcos(float x) { return float(cos(double(x))); }
__device__ __forceinline__ float dsin(float x) { return float(sin(double(x))); }
__device__ __forceinline__ float dpow(float x, float y) { return float(pow(double(x), double(y))); }
// IEEE round-to-nearest division. Every division in this file goes through it: nvcc compiles a
// plain '/' by a compile-time constant to a multiply that can differ in the last bit, even under
// -prec-div=true (divisions of two constants are folded at compile time and stay as written).
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
// clamp(x, lo, hi) = min(hi, max(lo, x)) with the device min/max (NaN bounds pass x through)
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(hi, fmaxf(lo, x)); }

// byte = the largest k with thr[k] <= x (0 for NaN and x < thr[1])
__device__ __forceinline__ uint32_t encodeChannel(const ColorTables& t, float x) {
    uint32_t k = 0;
#pragma unroll
    for (uint32_t step = 128; step; step >>= 1)
        if (t.thr[k + step] <= x) k += step;
    return k;
}
// ToColor4Unorm8SRgb(vector4): sRGB rgb, linear alpha, truncating * 255
__device__ __forceinline__ uint32_t encodeSrgb(const ColorTables& t, float4 c) {
    const uint32_t a = __float2uint_rz(c.w * 255.0f);
    return encodeChannel(t, c.x) | (encodeChannel(t, c.y) << 8) | (encodeChannel(t, c.z) << 16) | (a << 24);
}
// FromColor4Unorm8SRgb / an sRGB texel as the texture unit returns it
__device__ __forceinline__ float4 decodeSrgb(const ColorTables& t, uint32_t c) {
    return make_float4(t.dec[c & 255u], t.dec[(c >> 8) & 255u], t.dec[(c >> 16) & 255u], fdiv(float(c >> 24), 255.0f));
}
__device__ __forceinline__ float4 decodeUnorm16(ushort4 v) {
    return make_float4(fdiv(float(v.x), 65535.0f), fdiv(float(v.y), 65535.0f), fdiv(float(v.z), 65535.0f),
                       fdiv(float(v.w), 65535.0f));
}
// ToColor4Unorm16 (shading_helpers.h:201-208): truncating * 65535
__device__ __forceinline__ ushort4 encodeUnorm16(float4 c) {
    return make_ushort4(uint16_t(__float2ull_rz(c.x * 65535.0f)), uint16_t(__float2ull_rz(c.y * 65535.0f)),
                        uint16_t(__float2ull_rz(c.z * 65535.0f)), uint16_t(__float2ull_rz(c.w * 65535.0f)));
}

__device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 mul4(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float4 mul4(float4 a, float4 b) { return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }

// one axis of a linear-filtered fetch: texels i0, i1 with weights w0, w1 (multiples of 1/256)
struct Axis {
    int i0, i1;
    float w0, w1;
};
__device__ __forceinline__ Axis linearAxis(float u, int n, bool wrap) {
    if (wrap) u = u - floorf(u);
    float x = u * float(n) - 0.5f;
    x = fmaxf(fminf(x, float(n)), -1.0f);
    const float fl = floorf(x);
    int i0 = int(fl);
    const int a8 = __float2int_rn((x - fl) * 256.0f);
    Axis a;
    a.w1 = float(a8) * (1.0f / 256.0f);
    a.w0 = float(256 - a8) * (1.0f / 256.0f);
    if (wrap) {
        i0 = i0 < 0 ? i0 + n : (i0 >= n ? i0 - n : i0);
        a.i0 = i0;
        a.i1 = i0 + 1 == n ? 0 : i0 + 1;
    } else {
        a.i0 = min(max(i0, 0), n - 1);
        a.i1 = min(max(i0 + 1, 0), n - 1);
    }
    return a;
}
__device__ __forceinline__ int pointAxis(float u, int n, bool wrap) {
    if (wrap) u = u - floorf(u);
    const float x = fmaxf(fminf(u * float(n), float(n)), -1.0f);
    const int i = int(floorf(x));
    if (wrap) return i < 0 ? i + n : (i >= n ? i - n : i);
    return min(max(i, 0), n - 1);
}
// ((t00 w00 + t10 w10) + t01 w01) + t11 w11
__device__ __forceinline__ float4 blend4(float4 t00, float4 t10, float4 t01, float4 t11, const Axis& ax,
                                         const Axis& ay) {
    const float w00 = ax.w0 * ay.w0, w10 = ax.w1 * ay.w0, w01 = ax.w0 * ay.w1, w11 = ax.w1 * ay.w1;
    return add4(add4(add4(mul4(t00, w00), mul4(t10, w10)), mul4(t01, w01)), mul4(t11, w11));
}
__device__ __forceinline__ float4 sampleSrgb(const ColorTables& t, const uint32_t* tex, int w, int h, bool wrapX,
                                             float u, float v) {
    const Axis ax = linearAxis(u, w, wrapX), ay = linearAxis(v, h, false);
    const uint32_t* r0 = tex + size_t(ay.i0) * w;
    const uint32_t* r1 = tex + size_t(ay.i1) * w;
    return blend4(decodeSrgb(t, r0[ax.i0]), decodeSrgb(t, r0[ax.i1]), decodeSrgb(t, r1[ax.i0]),
                  decodeSrgb(t, r1[ax.i1]), ax, ay);
}

// sampleSpaceToEyeSpace * (x, y, 1), normalized; then (theta, eccentricity)
// (getNormalizedCoord, eyeSpaceDirectionToAngularEyeCoord: gpu_foveated.cu:92-107)
__device__ __forceinline__ void pixelEyeCoord(const FoveaDev& f, uint32_t i, uint32_t j, float& theta, float& ecc) {
    const float nx = fdiv(float(i) + 0.5f, float(f.width)), ny = fdiv(float(j) + 0.5f, float(f.height));
    const float* S = f.sampleToEye;
    const F3 d = f3(S[0] * nx + S[3] * ny + S[6] * 1.0f, S[1] * nx + S[4] * ny + S[7] * 1.0f,
                    S[2] * nx + S[5] * ny + S[8] * 1.0f);
    const F3 dir = normalize3(d);
    ecc = dacos(-dir.z);
    theta = -datan2(dir.y, dir.x);
}

// EccentricityMap::applyInverse (foveated.h:106-112)
__device__ __forceinline__ float eccApplyInverse(const FoveaDev& f, float E) {
    const float i0 = E * f.eccInvW0;
    const float sDivW = f.eccS * f.eccInvW0;
    const float x = dlog((f.eccM * (i0 - sDivW)) + 1.0f) * f.eccInvLogA;
    const float i1 = x + sDivW;
    return (E < f.eccS) ? i0 : i1;
}

// RemapPolarFoveatedKernel: each sample's colour (through an sRGB decode/encode round trip)
// and view depth to its polar texel
__global__ void __launch_bounds__(256) polarScatterKernel(const ViewDev* views, uint32_t view) {
    __shared__ ColorTables t;
    loadTables(t);
    const ViewDev& V = views[view];
    const FoveaDev& f = V.fov;
    const uint32_t n = f.valid, spr = f.spr;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const uint2 tx = f.remap[s];
        const size_t o = size_t(tx.y) * spr + tx.x;
        f.polarColor[o] = encodeSrgb(t, decodeSrgb(t, V.colors[s]));
        f.polarDepth[o] = V.tmaxOut[s];
    }
}

// ComputeMoments: mean and mean square of the 3x3 window of bilinear taps at the texel corner
__global__ void __launch_bounds__(256) momentsKernel(const ViewDev* views, uint32_t view) {
    __shared__ ColorTables t;
    loadTables(t);
    const FoveaDev& f = views[view].fov;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    const int w = int(f.spr), h = int(f.rings);
    if (i >= f.spr || j >= f.rings) return;
    const float idx = fdiv(1.0f, float(w)), idy = fdiv(1.0f, float(h));
    const float cx = idx * float(i), cy = idy * float(j);
    const float offs[3] = {-1.0f, 0.0f, 1.0f};
    float4 m1 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), m2 = m1;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
#pragma unroll
        for (int y = 0; y < 3; ++y) {
            const float4 c = sampleSrgb(t, f.polarColor, w, h, true, cx + (offs[x] * idx), cy + (offs[y] * idy));
            m1 = add4(m1, c);
            m2 = add4(m2, mul4(c, c));
        }
    }
    const float wgt = 1.0f / 9.0f;
    const size_t o = size_t(j) * w + i;
    f.moments[2 * o + 0] = encodeUnorm16(mul4(m1, wgt));
    f.moments[2 * o + 1] = encodeUnorm16(mul4(m2, wgt));
}

// bicubicFast (gpu_foveated.cu:36-71): 4-tap B-spline on the polar colour texture
__device__ float4 bicubicFast(const ColorTables& t, const FoveaDev& f, float cx, float cy) {
    const int w = int(f.spr), h = int(f.rings);
    const float px = cx * float(w), py = cy * float(h);
    const float ctrx = floorf(px - 0.5f) + 0.5f, ctry = floorf(py - 0.5f) + 0.5f;
    const float idx = fdiv(1.0f, float(w)), idy = fdiv(1.0f, float(h));
    float s0[2], s1[2], t0[2], t1[2];
    const float fr[2] = {px - ctrx, py - ctry}, ctr[2] = {ctrx, ctry}, id[2] = {idx, idy};
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const float fk = fr[k], f2 = fk * fk, f3 = f2 * fk;
        const float omf = 1.0f - fk;
        const float omf2 = omf * omf, omf3 = omf2 * omf;
        const float sixth = 1.0f / 6.0f;
        const float w0 = omf3 * sixth;
        const float w1 = ((4.0f / 6.0f) + f3 * 0.5f) - f2;
        const float w3 = f3 * sixth;
        const float w2 = ((1.0f - w0) - w1) - w3;
        s0[k] = w0 + w1;
        s1[k] = w2 + w3;
        const float f0 = fdiv(w1, w0 + w1), f1 = fdiv(w3, w2 + w3);
        t0[k] = ((ctr[k] - 1.0f) + f0) * id[k];
        t1[k] = ((ctr[k] + 1.0f) + f1) * id[k];
    }
    const float4 a = sampleSrgb(t, f.polarColor, w, h, true, t0[0], t0[1]);
    const float4 b = sampleSrgb(t, f.polarColor, w, h, true, t1[0], t0[1]);
    const float4 c = sampleSrgb(t, f.polarColor, w, h, true, t0[0], t1[1]);
    const float4 d = sampleSrgb(t, f.polarColor, w, h, true, t1[0], t1[1]);
    return add4(add4(add4(mul4(mul4(a, s0[0]), s0[1]), mul4(mul4(b, s1[0]), s0[1])), mul4(mul4(c, s0[0]), s1[1])),
                mul4(mul4(d, s1[0]), s1[1]));
}

// FoveatedPolarToScreenSpaceKernel: bicubic polar lookup, temporal reprojection of the
// previous frame's result clamped to the moments' neighbourhood, eccentricity-dependent blend
__global__ void __launch_bounds__(256) polarToScreenKernel(const ViewDev* views, uint32_t view) {
    __shared__ ColorTables t;
    loadTables(t);
    const FoveaDev& f = views[view].fov;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= f.width || j >= f.height) return;
    float theta, ecc;
    pixelEyeCoord(f, i, j, theta, ecc);
    // angularEyeCoordToPolarTextureCoord
    const float cx = fdiv(theta + kPi, 2.0f * kPi);
    const float cy = (eccApplyInverse(f, ecc) + 0.5f) * f.invTexMapSize;
    const float4 newValue = bicubicFast(t, f, cx, cy);
    float4 result = newValue;
    const int pw = int(f.spr), ph = int(f.rings);
    const float tValue = f.polarDepth[size_t(pointAxis(cy, ph, false)) * pw + pointAxis(cx, pw, true)];
    if (tValue < INFINITY) {
        // angularEyeCoordToDirection(theta, eccentricity) * tValue
        const float z = -dcos(ecc);
        const float xyLength = sqrtf(1.0f - z * z);
        const F3 p = f3(dcos(-theta) * xyLength, dsin(-theta) * xyLength, z) * tValue;
        const float* M = f.eyeToSamplePrev;
        const float qx = M[0] * p.x + M[4] * p.y + M[8] * p.z + M[12] * 1.0f;
        const float qy = M[1] * p.x + M[5] * p.y + M[9] * p.z + M[13] * 1.0f;
        const float qz = M[2] * p.x + M[6] * p.y + M[10] * p.z + M[14] * 1.0f;
        const float iz = fdiv(1.0f, qz);
        const float ox = qx * iz, oy = qy * iz;
        float alpha = 0.05f;  // TemporalFilterSettings::alpha
        float4 oldValue = newValue;
        if (ox > 0 && oy > 0 && ox < 1 && oy < 1 && tValue > 0)
            oldValue = sampleSrgb(t, f.history, int(f.width), int(f.height), false, ox, oy);
        // clampToNeighborhood (stddevMultiplier 1)
        const Axis ax = linearAxis(cx, pw, true), ay = linearAxis(cy, ph, false);
        const ushort4* r0 = f.moments + 2 * size_t(ay.i0) * pw;
        const ushort4* r1 = f.moments + 2 * size_t(ay.i1) * pw;
        const float4 m1 = blend4(decodeUnorm16(r0[2 * ax.i0]), decodeUnorm16(r0[2 * ax.i1]),
                                 decodeUnorm16(r1[2 * ax.i0]), decodeUnorm16(r1[2 * ax.i1]), ax, ay);
        const float4 m2 = blend4(decodeUnorm16(r0[2 * ax.i0 + 1]), decodeUnorm16(r0[2 * ax.i1 + 1]),
                                 decodeUnorm16(r1[2 * ax.i0 + 1]), decodeUnorm16(r1[2 * ax.i1 + 1]), ax, ay);
        const float sm = 1.0f;
        const float4 sd = make_float4(sqrtf(m2.x - m1.x * m1.x), sqrtf(m2.y - m1.y * m1.y), sqrtf(m2.z - m1.z * m1.z),
                                      sqrtf(m2.w - m1.w * m1.w));
        float4 co;
        co.x = clampf(oldValue.x, m1.x - sd.x * sm, m1.x + sd.x * sm);
        co.y = clampf(oldValue.y, m1.y - sd.y * sm, m1.y + sd.y * sm);
        co.z = clampf(oldValue.z, m1.z - sd.z * sm, m1.z + sd.z * sm);
        co.w = clampf(oldValue.w, m1.w - sd.w * sm, m1.w + sd.w * sm);
        float nE = ecc * f.invMaxEcc;
        const float mn = 0.2f, mx = 0.35f;
        const float tt = clampf(fdiv(nE - mn, mx - mn), 0.0f, 1.0f);
        alpha = 0.5f + (alpha - 0.5f) * tt;
        nE = sqrtf(sqrtf(sqrtf(sqrtf(nE))));
        co.x = co.x + (oldValue.x - co.x) * nE;
        co.y = co.y + (oldValue.y - co.y) * nE;
        co.z = co.z + (oldValue.z - co.z) * nE;
        co.w = co.w + (oldValue.w - co.w) * nE;
        result = add4(mul4(newValue, alpha), mul4(co, 1.0f - alpha));
    }
    const size_t npix = size_t(f.width) * f.height, o = size_t(j) * f.width + i;
    f.result[o] = encodeSrgb(t, result);
    // eccentricity and the filter weights pow(1 - |R| / 5.1, sqrt(eccentricity)), R = 1..5
    f.ecc[o] = ecc;
    const float se = sqrtf(ecc);
#pragma unroll
    for (int r = 1; r <= 5; r++) f.ecc[r * npix + o] = dpow(1.0f - fdiv(fabsf(float(r)), kFilterDen), se);
}

// SeparableFilterUsingEccentricity over in (radius 5, clamped taps) at pixel (i, j)
template <bool Vertical>
__device__ __forceinline__ float4 eccFilter(const ColorTables& t, const FoveaDev& f, const uint32_t* in, uint32_t i,
                                            uint32_t j) {
    const size_t npix = size_t(f.width) * f.height, o = size_t(j) * f.width + i;
    float wk[6];
    wk[0] = 1.0f;  // pow(1, s)
#pragma unroll
    for (int r = 1; r <= 5; r++) wk[r] = f.ecc[r * npix + o];
    float4 vs = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float ws = 0.0f;
#pragma unroll
    for (int R = -5; R <= 5; ++R) {
        const int x = Vertical ? int(i) : min(max(int(i) + R, 0), int(f.width) - 1);
        const int y = Vertical ? min(max(int(j) + R, 0), int(f.height) - 1) : int(j);
        const float w = wk[R < 0 ? -R : R];
        vs = add4(vs, mul4(decodeSrgb(t, in[size_t(y) * f.width + x]), w));
        ws += w;
    }
    return mul4(vs, fdiv(1.0f, ws));
}

__global__ void __launch_bounds__(256) filterVerticalKernel(const ViewDev* views, uint32_t view) {
    __shared__ ColorTables t;
    loadTables(t);
    const FoveaDev& f = views[view].fov;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= f.width || j >= f.height) return;
    f.filtered[size_t(j) * f.width + i] = encodeSrgb(t, eccFilter<true>(t, f, f.result, i, j));
}

// horizontal pass, then FinishConstrastEnhancement (sigma = 8 max(0.001, t^2), f_e = 1)
__global__ void __launch_bounds__(256) filterHorizontalEnhanceKernel(const ViewDev* views, uint32_t view) {
    __shared__ ColorTables t;
    loadTables(t);
    const FoveaDev& f = views[view].fov;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= f.width || j >= f.height) return;
    const size_t o = size_t(j) * f.width + i;
    const float4 pmean = decodeSrgb(t, encodeSrgb(t, eccFilter<false>(t, f, f.filtered, i, j)));
    const float4 pix = decodeSrgb(t, f.result[o]);
    const float tt = f.ecc[o] * f.invMaxEcc;
    float sigma = 8.0f;
    sigma *= fmaxf(0.001f, clampf(tt * tt, 0.0f, 1.0f));
    const float cScale = 1.0f + sigma * 1.0f;
    float4 r;
    r.x = clampf(pmean.x + (pix.x - pmean.x) * cScale, 0.0f, 1.0f);
    r.y = clampf(pmean.y + (pix.y - pmean.y) * cScale, 0.0f, 1.0f);
    r.z = clampf(pmean.z + (pix.z - pmean.z) * cScale, 0.0f, 1.0f);
    r.w = clampf(pmean.w + (pix.w - pmean.w) * cScale, 0.0f, 1.0f);
    f.image[size_t(j) * f.imageStride + i] = encodeSrgb(t, r);
}

} // namespace

cudaError_t launchFoveatedResolve(const FrameDev& fr, uint32_t view, const FoveaDev& fov, cudaStream_t st) {
    if (!fov.image || !fov.width || !fov.height || !fov.spr || !fov.rings) return cudaSuccess;
    const dim3 blk(32, 8);
    const dim3 polar((fov.spr + 31) / 32, (fov.rings + 7) / 8);
    const dim3 screen((fov.width + 31) / 32, (fov.height + 7) / 8);
    polarScatterKernel<<<(fov.valid + 255) / 256, 256, 0, st>>>(fr.views, view);
    momentsKernel<<<polar, blk, 0, st>>>(fr.views, view);
    polarToScreenKernel<<<screen, blk, 0, st>>>(fr.views, view);
    filterVerticalKernel<<<screen, blk, 0, st>>>(fr.views, view);
    filterHorizontalEnhanceKernel<<<screen, blk, 0, st>>>(fr.views, view);
    return cudaGetLastError();
}

cudaError_t uploadColorTables(const float* decode256, const float* thresholds256, cudaStream_t st) {
    cudaError_t e = cudaMemcpyToSymbolAsync(gColor, decode256, 256 * sizeof(float), 0, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbolAsync(gColor, thresholds256, 256 * sizeof(float), offsetof(ColorTables, thr),
                                   cudaMemcpyHostToDevice, st);
}

} // namespace hvb
