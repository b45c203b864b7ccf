// Replacement for the reference's shared/avx.h under g++ (see hvvr_gcc_compat.h).
// Same helper names and lane semantics, written against the wrapper classes.
#pragma once
#include <immintrin.h>

namespace hvvr {

// ---- 128-bit
__forceinline __m128 m128(float x, float y, float z = 0, float w = 0) { return _mm_set_ps(w, z, y, x); }
__forceinline __m128 m128(float a) { return _mm_set1_ps(a); }
__forceinline __m128 m128(__m256 a) { return _mm256_castps256_ps128(a.v); }
__forceinline __m128 load_m128(const float* p) { return _mm_load_ps(p); }
__forceinline void store(float* p, __m128 a) { _mm_store_ps(p, a.v); }
__forceinline __m128 operator-(__m128 a) { return _mm_xor_ps(a.v, _mm_set1_ps(-0.0f)); }
__forceinline __m128 operator+(__m128 a, __m128 b) { return _mm_add_ps(a.v, b.v); }
__forceinline __m128 operator-(__m128 a, __m128 b) { return _mm_sub_ps(a.v, b.v); }
__forceinline __m128 operator*(__m128 a, __m128 b) { return _mm_mul_ps(a.v, b.v); }
__forceinline __m128 operator&(__m128 a, __m128 b) { return _mm_and_ps(a.v, b.v); }
__forceinline __m128 operator|(__m128 a, __m128 b) { return _mm_or_ps(a.v, b.v); }
__forceinline __m128 operator<(__m128 a, __m128 b) { return _mm_cmplt_ps(a.v, b.v); }
__forceinline __m128 operator>(__m128 a, __m128 b) { return _mm_cmpgt_ps(a.v, b.v); }
__forceinline __m128 operator<=(__m128 a, __m128 b) { return _mm_cmple_ps(a.v, b.v); }
__forceinline __m128 operator>=(__m128 a, __m128 b) { return _mm_cmpge_ps(a.v, b.v); }
__forceinline __m128 min(__m128 a, __m128 b) { return _mm_min_ps(a.v, b.v); }
__forceinline __m128 max(__m128 a, __m128 b) { return _mm_max_ps(a.v, b.v); }
__forceinline unsigned movemask(__m128 a) { return (unsigned)_mm_movemask_ps(a.v); }
template <unsigned i> __forceinline __m128 extract_m128(__m256 a) { return _mm256_extractf128_ps(a.v, i); }
template <unsigned x, unsigned y, unsigned z, unsigned w> __forceinline __m128 shuffle(__m128 a) {
    return _mm_castsi128_ps(_mm_shuffle_epi32(_mm_castps_si128(a.v), w * 64 + z * 16 + y * 4 + x));
}

// ---- 256-bit
__forceinline __m256 m256(float a, float b, float c, float d, float e, float f, float g, float h) {
    return _mm256_set_ps(h, g, f, e, d, c, b, a);
}
__forceinline __m256 m256(float a) { return _mm256_set1_ps(a); }
__forceinline __m256 load_m256(const float* p) { return _mm256_load_ps(p); }
__forceinline void store(float* p, __m256 a) { _mm256_store_ps(p, a.v); }
__forceinline __m256 operator-(__m256 a) { return _mm256_xor_ps(a.v, _mm256_set1_ps(-0.0f)); }
__forceinline __m256 operator+(__m256 a, __m256 b) { return _mm256_add_ps(a.v, b.v); }
__forceinline __m256 operator-(__m256 a, __m256 b) { return _mm256_sub_ps(a.v, b.v); }
__forceinline __m256 operator*(__m256 a, __m256 b) { return _mm256_mul_ps(a.v, b.v); }
__forceinline __m256 operator&(__m256 a, __m256 b) { return _mm256_and_ps(a.v, b.v); }
__forceinline __m256 operator|(__m256 a, __m256 b) { return _mm256_or_ps(a.v, b.v); }
__forceinline __m256 operator<(__m256 a, __m256 b) { return _mm256_cmp_ps(a.v, b.v, _CMP_LT_OQ); }
__forceinline __m256 operator>(__m256 a, __m256 b) { return _mm256_cmp_ps(a.v, b.v, _CMP_GT_OQ); }
__forceinline __m256 operator<=(__m256 a, __m256 b) { return _mm256_cmp_ps(a.v, b.v, _CMP_LE_OQ); }
__forceinline __m256 operator>=(__m256 a, __m256 b) { return _mm256_cmp_ps(a.v, b.v, _CMP_GE_OQ); }
__forceinline __m256 min(__m256 a, __m256 b) { return _mm256_min_ps(a.v, b.v); }
__forceinline __m256 max(__m256 a, __m256 b) { return _mm256_max_ps(a.v, b.v); }
__forceinline unsigned movemask(__m256 a) { return (unsigned)_mm256_movemask_ps(a.v); }
template <unsigned x, unsigned y, unsigned z, unsigned w> __forceinline __m256 shuffle(__m256 a) {
    return _mm256_castsi256_ps(_mm256_shuffle_epi32(_mm256_castps_si256(a.v), w * 64 + z * 16 + y * 4 + x));
}

} // namespace hvvr
