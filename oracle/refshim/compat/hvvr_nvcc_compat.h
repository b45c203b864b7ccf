// Forced-include shim that lets the reference's texture sources (MSVC-targeted .cu files) compile
// with nvcc on Linux for the GPU-side texture pin (oracle/_ref/libhvvr_ref_gpu.so). Test
// infrastructure only; never part of the product.
#pragma once
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <immintrin.h>
#include <x86intrin.h>
// BMI1 lowest-bit clear (the reference's util.h), spelled out for compilers without -mbmi
static inline uint32_t hv_blsr32(uint32_t a) { return a & (a - 1u); }
static inline uint64_t hv_blsr64(uint64_t a) { return a & (a - 1u); }
#define _blsr_u32 hv_blsr32
#define _blsr_u64 hv_blsr64

#ifndef __forceinline
#define __forceinline inline __attribute__((always_inline))
#endif
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

// The reference writes 64-bit texels with surf2Dwrite(uint64_t) (gpu_foveated.cu:30); uint64_t is
// unsigned long on Linux, which CUDA's surface templates do not list, so forward it as the
// unsigned long long they accept (same bits)
#if defined(__CUDACC__)
#include <surface_indirect_functions.h>
static __device__ __forceinline__ void surf2Dwrite(unsigned long val, cudaSurfaceObject_t obj, int x, int y,
                                                   cudaSurfaceBoundaryMode mode = cudaBoundaryModeTrap) {
    surf2Dwrite((unsigned long long)val, obj, x, y, mode);
}
#endif

// vector_math.h decodes a half on the device with __half2float({bits}). Under the CUDA 9 headers
// the reference was written for, that braced list set the raw bits; under CUDA 11+ it selects
// __half's integer-value constructor (bits 0x3c00 become 15360.0), so every vertex normal would
// decode wrong. An unsigned short overload, an exact match for the braced bits, decodes them as
// bits, as the reference intends and as its host path does (_cvtsh_ss).
#if defined(__CUDACC__)
#include <cuda_fp16.h>
static __host__ __device__ __forceinline__ float hv_half2float(unsigned short bits) {
    __half_raw r;
    r.x = bits;
    return __half2float(__half(r));
}
static __host__ __device__ __forceinline__ float hv_half2float(const __half h) { return __half2float(h); }
#define __half2float hv_half2float
#endif
