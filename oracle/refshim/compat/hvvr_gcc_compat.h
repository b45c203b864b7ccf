// Forced-include shim that lets the reference's MSVC-targeted sources compile with g++.
// Test infrastructure only (builds oracle/_ref); never part of the product.
//
// MSVC lets the reference overload operators on __m128/__m256 (its avx.h); GCC does not,
// because they are built-in vector types. After the intrinsic headers are parsed, the
// names are redirected to thin wrapper classes (same size and alignment) that convert
// implicitly to and from the real types, so intrinsic calls still type-check and the
// operator overloads in compat/avx.h apply.
#pragma once
#include <immintrin.h>
#include <x86intrin.h>
#include <vector_types.h>
#include <stdlib.h>
#include <stdint.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include <limits>
#include <algorithm>
#include <string>
#include <vector>

typedef __m128 hv_real_m128;
typedef __m256 hv_real_m256;
struct alignas(16) hv128 {
    hv_real_m128 v;
    hv128() = default;
    hv128(hv_real_m128 x) : v(x) {}
    operator hv_real_m128() const { return v; }
};
struct alignas(32) hv256 {
    hv_real_m256 v;
    hv256() = default;
    hv256(hv_real_m256 x) : v(x) {}
    operator hv_real_m256() const { return v; }
};
static_assert(sizeof(hv128) == 16 && sizeof(hv256) == 32, "wrapper size");
#define __m128 hv128
#define __m256 hv256

#define __forceinline inline __attribute__((always_inline))
static inline unsigned char _bittest(const long* base, long offset) {
    return (unsigned char)((((const uint32_t*)base)[offset >> 5] >> (offset & 31)) & 1u);
}
static inline unsigned char _BitScanForward(unsigned long* index, unsigned long mask) {
    if (!mask) return 0;
    *index = (unsigned long)__builtin_ctzl(mask);
    return 1;
}
static inline void* _aligned_malloc(size_t size, size_t alignment) {
    if (alignment < sizeof(void*)) alignment = sizeof(void*);
    void* p = nullptr;
    if (posix_memalign(&p, alignment, size ? size : alignment)) return nullptr;
    return p;
}
static inline void _aligned_free(void* p) { free(p); }

// CUDA builtins referenced by host-parsed device code (never executed on these paths)
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;

// Host definitions of the CUDA device intrinsics that the kernels' math headers call.
#include <texture_types.h>
static inline int __float_as_int(float f) { int i; memcpy(&i, &f, 4); return i; }
static inline float __int_as_float(int i) { float f; memcpy(&f, &i, 4); return f; }
static inline float __saturatef(float x) { return x > 0.0f ? (x < 1.0f ? x : 1.0f) : 0.0f; }
static inline int __popc(unsigned x) { return __builtin_popcount(x); }
static inline int __clz(int x) { return x ? __builtin_clz((unsigned)x) : 32; }
static inline int __ffs(int x) { return __builtin_ffs(x); }
static inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
// warp intrinsics parsed in host compiles of .cu files (the harness never runs these paths)
static inline unsigned __activemask() { return 0xffffffffu; }
static inline unsigned __ballot_sync(unsigned, int p) { return p ? 1u : 0u; }
template <class T> static inline T __shfl_sync(unsigned, T v, int, int = 32) { return v; }
template <class T> static inline T __shfl_xor_sync(unsigned, T v, int, int = 32) { return v; }
// texture reads of host-compiled shading code (ReadTexture) go to a hook the harness sets:
// hook(ctx, texture object value, {u, v, ddx.x, ddx.y, ddy.x, ddy.y}, rgba)
typedef void (*hv_texture_hook_fn)(void* ctx, uint32_t id, const float* q, float* rgba);
extern hv_texture_hook_fn hv_texture_hook;
extern void* hv_texture_hook_ctx;
template <class T> static inline T tex2DGrad(cudaTextureObject_t t, float u, float v, float2 dx, float2 dy) {
    const float q[6] = {u, v, dx.x, dx.y, dy.x, dy.y};
    float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (hv_texture_hook) hv_texture_hook(hv_texture_hook_ctx, uint32_t(t), q, o);
    T r;
    r.x = o[0];
    r.y = o[1];
    r.z = o[2];
    r.w = o[3];
    return r;
}
