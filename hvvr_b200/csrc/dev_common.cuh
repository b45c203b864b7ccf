// dev_common.cuh - device helpers shared by the kernels.
//
// Floating point: every .cu file is compiled with -fmad=false -ftz=true -prec-div=true
// -prec-sqrt=true, so a*b+c is never contracted and division/sqrt are IEEE. fmaf() is
// written out exactly where the reference issues an FMA (its AVX intrinsics, and the edge
// tests its kernel comments mark as FMA in HVVR_FP_FMA mode). -ftz matches the MXCSR
// FTZ|DAZ mode the reference runs its host traversal under.
#pragma once

#include "hvvr_internal.h"

#include <cuda_fp16.h>
#include <float.h>
#include <math.h>

namespace hvb {

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ F3 operator-(F3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ F3 operator*(F3 a, F3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
// dot/cross/normalize with the reference's association (libraries/hvvr/shared/vector_math.h:262-286)
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ F3 normalize3(F3 v) {
    float inv = 1.0f / sqrtf(dot3(v, v));
    return f3(v.x * inv, v.y * inv, v.z * inv);
}
__device__ __forceinline__ float tmaxf(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float tminf(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float satf(float x) { return x > 0.0f ? (x < 1.0f ? x : 1.0f) : 0.0f; }

// matrix4x4 * vector4(v, 1) and matrix3x3(m) * v, column-major (vector_math.h:1129-1133, 1273-1278)
__device__ __forceinline__ F3 xformPoint(const Mat4& m, F3 v) {
    return f3(m.m[0][0] * v.x + m.m[1][0] * v.y + m.m[2][0] * v.z + m.m[3][0] * 1.0f,
              m.m[0][1] * v.x + m.m[1][1] * v.y + m.m[2][1] * v.z + m.m[3][1] * 1.0f,
              m.m[0][2] * v.x + m.m[1][2] * v.y + m.m[2][2] * v.z + m.m[3][2] * 1.0f);
}
__device__ __forceinline__ F3 xformDir(const Mat4& m, F3 v) {
    return f3(m.m[0][0] * v.x + m.m[1][0] * v.y + m.m[2][0] * v.z,
              m.m[0][1] * v.x + m.m[1][1] * v.y + m.m[2][1] * v.z,
              m.m[0][2] * v.x + m.m[1][2] * v.y + m.m[2][2] * v.z);
}

// denormals-are-zero view, for the comparisons the reference makes under MXCSR.DAZ
__device__ __forceinline__ float dazf(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x7f800000u) == 0 ? __uint_as_float(u & 0x80000000u) : f;
}

__device__ __forceinline__ uint32_t laneId() { return threadIdx.x & 31u; }

#ifdef HVVR_VISIT_CLOCKS
// Profiling build only (make -C hvvr_b200/csrc visit-clocks): clock64 read once dep is available.
// The read is predicated on a test of dep, so it waits for dep's producer (the sentinel is a value
// none of the marked quantities takes in practice).
__device__ __forceinline__ long long phaseClock(uint32_t dep) {
    long long t;
    asm volatile("{ .reg .pred p; setp.ne.u32 p, %1, 0x9e3779b9; @p mov.u64 %0, %%clock64; @!p mov.u64 %0, 0; }"
                 : "=l"(t) : "r"(dep) : "memory");
    return t;
}
#endif

// ReadTexture (libraries/hvvr/raycaster/shading.h:45-47): one gradient read through a texture
// object made as the reference makes its material textures (texture.cu:234-265)
__device__ __forceinline__ float4 readTexture(cudaTextureObject_t t, float u, float v, float2 ddx, float2 ddy) {
    return tex2DGrad<float4>(t, u, v, ddx, ddy);
}

} // namespace hvb
