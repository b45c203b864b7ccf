// shade.cu - fused intersect + G-buffer compression + MSAA shade/resolve, and the remap.
//
// intersectShadeKernel<N, FMA> runs one 128-thread CTA per tile (thread = sample), like
// the reference's IntersectKernel and ResolveKernel (libraries/hvvr/raycaster/intersect.cu:298-342,
// libraries/hvvr/raycaster/resolve.cu:324-458), but as one launch: the per-subsample hit
// IDs stay in registers, are grouped into (triangle, coverage mask) pairs exactly as
// EmitGBuffer does (intersect.cu:28-89), and are shaded and resolved in the same thread
// (ShadeMSAA, resolve.cu:161-284). The G-buffer therefore never goes to HBM.
//
// The tile's triangle list is consumed in its chunks of 128 entries. Each thread tests one
// entry against the tile frustum planes, the ray-origin half space and the corner-ray
// barycentric bounds (FrustumPlanes::test, IntersectTriangleTile<false>::setup,
// TestTriangleFrustaUVW; libraries/hvvr/raycaster/prim_tests.h:18-164); survivors are compacted
// into shared memory in list order with warp ballots, and every thread then tests its
// sample's N subsamples against them in that order, so depth ties resolve as in the reference.
#include <algorithm>

#include "../../include/hvvr_c.h"
#include "dev_common.cuh"

namespace hvb {

// unit offsets for rates 1,2,4,8,16,32: rows 0-5 the spiral, rows 6-11 the rotated grid
__constant__ float2 cMsaa[12][32];
// each offset's x and y duplicated into both halves of a 64-bit pair, the operands of the packed
// tests that run one subsample against two triangles
__constant__ __align__(8) float2 cMsaaXX[12][32];
__constant__ __align__(8) float2 cMsaaYY[12][32];

namespace {

constexpr unsigned kFull = 0xffffffffu;

#ifdef HVVR_VISIT_CLOCKS
// Profiling build only (make -C hvvr_b200/csrc visit-clocks): per global tile, the SM cycles that
// thread 0 of its intersect/shade CTA spends in each phase (the CTA's barriers make thread 0's
// clock the CTA's), its chunk count and its list length, read back through hvvr_dbg_shade_clocks.
constexpr uint32_t kShadeClockTiles = 1u << 17;
enum : uint32_t {
    kScSetup, // view, frustum planes, beams, first chunk staged
    kScCull,  // per chunk: staged triangles arrive, per-triangle tile tests, survivor compaction
    kScTest,  // per chunk: depth skip and the packed subsample tests, next chunk staged
    kScShade, // hit and depth outputs, G-buffer grouping, shading, resolve
    kScPhases
};
__device__ unsigned long long gShadeClocks[kShadeClockTiles][kScPhases + 2];
#define SHADE_MARK(phase, dep)                                                                                         \
    do {                                                                                                               \
        const long long t_ = phaseClock(dep);                                                                          \
        scAcc[phase] += t_ - scLast;                                                                                   \
        scLast = t_;                                                                                                   \
    } while (0)
#else
#define SHADE_MARK(phase, dep) do { } while (0)
#endif

template <uint32_t N> struct RateIndex;
template <> struct RateIndex<1> { static constexpr int v = 0; };
template <> struct RateIndex<2> { static constexpr int v = 1; };
template <> struct RateIndex<4> { static constexpr int v = 2; };
template <> struct RateIndex<8> { static constexpr int v = 3; };
template <> struct RateIndex<16> { static constexpr int v = 4; };
template <> struct RateIndex<32> { static constexpr int v = 5; };

// Loads a pointer field of the view table where it is used. The asm is volatile so the
// compiler re-issues the (L1-resident) load instead of keeping ten 64-bit pointers live in
// registers across the tile loop, which costs two CTAs per SM of occupancy.
template <class T>
__device__ __forceinline__ T* viewPtr(T* const& field) {
    uint64_t v;
    asm volatile("ld.global.nc.u64 %0, [%1];" : "=l"(v) : "l"(&field));
    return reinterpret_cast<T*>(v);
}

struct TriGeom {
    F3 v0, e0, e1;
};
__device__ __forceinline__ TriGeom loadTri(const float4* __restrict__ tris, uint32_t i) {
    const float4 a = __ldg(tris + 3 * size_t(i) + 0);
    const float4 b = __ldg(tris + 3 * size_t(i) + 1);
    const float4 c = __ldg(tris + 3 * size_t(i) + 2);
    return TriGeom{f3(a.x, a.y, a.z), f3(a.w, b.x, b.y), f3(b.z, b.w, c.x)};
}

// per-thread scaled barycentric setup (IntersectTriangleThread ctor + GetDifferentials,
// prim_tests.h:118-134, 175-188)
struct TriThread {
    float dc, vc, wc, ddx, ddy, dvx, dvy, dwx, dwy;
};
__device__ __forceinline__ TriThread threadSetupN(F3 normal, F3 e0, F3 e1, F3 v0r, F3 c, F3 du, F3 dv) {
    TriThread r;
    r.dc = dot3(-c, normal);
    const F3 ec = cross3(-c, v0r);
    r.vc = dot3(e1, ec);
    r.wc = -dot3(e0, ec);
    r.ddx = dot3(-du, normal);
    r.ddy = dot3(-dv, normal);
    const F3 cu = cross3(-du, v0r), cv = cross3(-dv, v0r);
    r.dvx = dot3(e1, cu);
    r.dvy = dot3(e1, cv);
    r.dwx = -dot3(e0, cu);
    r.dwy = -dot3(e0, cv);
    return r;
}
// the same with normal = e0 x e1 computed here (the per-triangle part, which the tile loop
// computes once per triangle instead of once per thread)
__device__ __forceinline__ TriThread threadSetup(F3 e0, F3 e1, F3 v0r, F3 c, F3 du, F3 dv) {
    return threadSetupN(cross3(e0, e1), e0, e1, v0r, c, du, dv);
}

// Packed FP32 (sm_100 f32x2): two floats in one 64-bit register pair, each lane an ordinary IEEE
// single-precision operation (round to nearest, flush to zero like every other operation here), so
// a packed result equals the two scalar results bit for bit.
typedef unsigned long long P2;
__device__ __forceinline__ P2 pk(float lo, float hi) {
    P2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk(P2 v, float& lo, float& hi) { asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v)); }
__device__ __forceinline__ P2 fma2(P2 a, P2 b, P2 c) {
    P2 r;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
// The rounded product a*b of both lanes, written as fma(a, b, z) with z = (-0, -0): x + (-0) = x
// for every x (zeros keep their sign), so this is exactly mul.rn.ftz. The compiler contracts a
// packed mul.rn with the add that consumes it into one FMA, and it does the same to
// fma(a, b, -0) when it can see the -0 (both measured on sm_100a: the uncontracted expressions
// then round differently from their scalar forms). So z comes from constant memory that the host
// writes at run time (cNegZero2, with the offset tables), a value the compiler cannot know: the
// FMA stays a rounded product, and every product and sum below keeps its own rounding.
__constant__ P2 cNegZero2;
__device__ __forceinline__ P2 mul2(P2 a, P2 b) {
    P2 r;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(cNegZero2));
    return r;
}
__device__ __forceinline__ P2 add2(P2 a, P2 b) {
    P2 r;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ P2 sub2(P2 a, P2 b) {
    P2 r;
    asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

// exact negation of both lanes (a sign-bit flip, as the scalar unary minus)
__device__ __forceinline__ P2 neg2(P2 a) { return a ^ 0x8000000080000000ull; }

struct V2 {
    P2 x, y, z;
};
// dot3 / cross3 (same association) on two triangles at once
__device__ __forceinline__ P2 dot2(const V2& a, const V2& b) {
    return add2(add2(mul2(a.x, b.x), mul2(a.y, b.y)), mul2(a.z, b.z));
}
__device__ __forceinline__ V2 cross2(const V2& a, const V2& b) {
    return V2{sub2(mul2(a.y, b.z), mul2(a.z, b.y)), sub2(mul2(a.z, b.x), mul2(a.x, b.z)),
              sub2(mul2(a.x, b.y), mul2(a.y, b.x))};
}

// threadSetupN for two triangles j, k (lane 0 / lane 1 of every pair) against this thread's
// sample: nc, ndu, ndv are -c, -du, -dv duplicated into both lanes
struct TriPair {
    P2 dc, vc, wc, ddx, ddy, dvx, dvy, dwx, dwy;
};
__device__ __forceinline__ TriPair pairSetup(const V2& n, const V2& e0, const V2& e1, const V2& v0r, const V2& nc,
                                             const V2& ndu, const V2& ndv) {
    TriPair r;
    r.dc = dot2(nc, n);
    const V2 ec = cross2(nc, v0r);
    r.vc = dot2(e1, ec);
    r.wc = neg2(dot2(e0, ec));
    r.ddx = dot2(ndu, n);
    r.ddy = dot2(ndv, n);
    const V2 cu = cross2(ndu, v0r), cv = cross2(ndv, v0r);
    r.dvx = dot2(e1, cu);
    r.dvy = dot2(e1, cv);
    r.dwx = neg2(dot2(e0, cu));
    r.dwy = neg2(dot2(e0, cv));
    return r;
}

__device__ __forceinline__ bool signsClear(float a, float b, float c, float d) {
    return (__float_as_int(a) | __float_as_int(b) | __float_as_int(c) | __float_as_int(d)) >= 0;
}

// The depth of a hit, t / denom as the reference computes it (t times the IEEE reciprocal). Out of
// line: it runs only on a hit, and one copy of the division replaces one per unrolled subsample
// test, which keeps the pair-test loop small in the instruction cache.
__device__ __noinline__ float hitDepth(float t, float denom) { return t * (1.0f / denom); }

// IntersectTriangleThread::test (prim_tests.h:192-231) of one subsample (unit offset ax, ay
// duplicated into both lanes) against triangles j and k in that order, with the scalar test's
// operations in its order: denom, depthDelta, v, w as FMA chains (FMA) or as rounded products and
// sums (STRICT), u = (denom - v) - w, the sign-bit test and the depth update. Both depth deltas are
// formed from the depth before j; when j hits, k's is formed again from the new depth, so k sees
// exactly the depth the sequential fold gives it.
// tt holds (-t_j, -t_k) in FMA mode, (t_j, t_k) in STRICT mode.
template <bool FMA>
__device__ __forceinline__ void pairTest(const TriPair& p, P2 tt, float tj, float tk, uint32_t ij, uint32_t ik,
                                         P2 ax, P2 ay, float& depth, uint32_t& hit) {
    const P2 d2 = pk(depth, depth);
    P2 denom, dd, v, w;
    if (FMA) {
        denom = fma2(p.ddy, ay, fma2(p.ddx, ax, p.dc));
        dd = fma2(d2, denom, tt);
        v = fma2(p.dvy, ay, fma2(p.dvx, ax, p.vc));
        w = fma2(p.dwy, ay, fma2(p.dwx, ax, p.wc));
    } else {
        denom = add2(add2(p.dc, mul2(p.ddx, ax)), mul2(p.ddy, ay));
        dd = sub2(mul2(d2, denom), tt);
        v = add2(add2(p.vc, mul2(p.dvx, ax)), mul2(p.dvy, ay));
        w = add2(add2(p.wc, mul2(p.dwx, ax)), mul2(p.dwy, ay));
    }
    const P2 u = sub2(sub2(denom, v), w);
    float den0, den1, dd0, dd1, u0, u1, v0, v1, w0, w1;
    upk(denom, den0, den1);
    upk(dd, dd0, dd1);
    upk(u, u0, u1);
    upk(v, v0, v1);
    upk(w, w0, w1);
    if (signsClear(dd0, u0, v0, w0)) {
        depth = hitDepth(tj, den0);
        hit = ij;
        dd1 = FMA ? fmaf(depth, den1, -tk) : depth * den1 - tk;
    }
    if (signsClear(dd1, u1, v1, w1)) {
        depth = hitDepth(tk, den1);
        hit = ik;
    }
}

// IntersectTriangleThread::calcUVW (prim_tests.h:233-245)
template <bool FMA>
__device__ __forceinline__ F3 calcUVW(const TriThread& th, float ax, float ay) {
    float denom, v, w;
    if (FMA) {
        denom = fmaf(th.ddy, ay, fmaf(th.ddx, ax, th.dc));
        v = fmaf(th.dvy, ay, fmaf(th.dvx, ax, th.vc));
        w = fmaf(th.dwy, ay, fmaf(th.dwx, ax, th.wc));
    } else {
        denom = th.dc + th.ddx * ax + th.ddy * ay;
        v = th.vc + th.dvx * ax + th.dvy * ay;
        w = th.wc + th.dwx * ax + th.dwy * ay;
    }
    const float u = denom - v - w;
    const float inv = 1.0f / denom;
    return f3(u * inv, v * inv, w * inv);
}

// TestRayTriangle<false> barycentrics (prim_tests.h:53-82)
__device__ __forceinline__ void rayTriUVW(F3 ro, F3 rd, const TriGeom& tri, float& u, float& v, float& w) {
    const F3 n = cross3(tri.e0, tri.e1);
    const float denom = dot3(-rd, n);
    const F3 v0r = ro - tri.v0;
    const F3 e = cross3(-rd, v0r);
    v = dot3(tri.e1, e);
    w = -dot3(tri.e0, e);
    const float ood = 1.0f / denom;
    v = v * ood;
    w = w * ood;
    u = 1.0f - v - w;
}

// SimpleMaterial (material.h:15-49): textureIDsAndShadingModel holds the shading model in bits
// 0-15 and the glossiness, specular and diffuse/emissive texture ids in bits 16-31, 32-47, 48-63
constexpr uint32_t kNoTexture = 0xffffu;
struct Material {
    F3 emissive, diffuse, specular;
    float glossiness;
    uint32_t model, texGloss, texSpecular, texDiffuse;
};

__device__ __forceinline__ float pow5(float x) {
    const float x2 = x * x;
    return x2 * x2 * x;
}

// GGX_SchlickFresnel_SchlickSmithGGX + PBR_BRDF1 (libraries/hvvr/raycaster/shading_helpers.h:89-122)
__device__ F3 pbr(F3 L, F3 N, F3 V, F3 base, float roughness, F3 F0, F3 lightColor) {
    const float alpha = roughness * roughness;
    const F3 H = normalize3(L + V);
    const float alpha2 = alpha * alpha;
    const float NdotH = satf(dot3(N, H));
    const float q = (NdotH * NdotH) * (alpha2 - 1.0f) + 1.0f;
    const float D = alpha2 / (3.141592653589f * (q * q));
    const float LdotH = satf(dot3(L, H));
    const F3 F = F0 + (f3(1.0f, 1.0f, 1.0f) - F0) * pow5(1.0f - LdotH);
    const float NdotL = satf(dot3(N, L));
    const float NdotV = satf(dot3(N, V));
    const float k = alpha * 0.5f;
    const float vis = (1.0f / (NdotL * (1.0f - k) + k)) * (1.0f / (NdotV * (1.0f - k) + k));
    const F3 spec = ((F * D) * vis) * (1.0f / 4.0f);
    const float NdotL2 = satf(dot3(N, L));
    const F3 diffuse = ((base * lightColor) * (f3(1.0f, 1.0f, 1.0f) - spec)) * NdotL2;
    return diffuse + lightColor * spec;
}

// the phong branch of GGXShade (libraries/hvvr/raycaster/shading.h:127-160) once the base colour,
// F0 and roughness are known (material constants or texture reads): emissive, ambient and the
// lights, clamped at zero
__device__ F3 ggxLit(F3 emissive, F3 base, F3 F0, float roughness, F3 pos, F3 normal, F3 V, const LightEnvDev& env) {
    F3 radiance = emissive + base * f3(.15f, .15f, .165f);
    if (env.nd > 0) {
        radiance = radiance + pbr(f3(env.dir[0][0], env.dir[0][1], env.dir[0][2]), normal, V, base, roughness, F0,
                                  f3(env.dir[0][3], env.dir[0][4], env.dir[0][5]));
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (i >= env.np) break;
        const float* l = env.pt[i];
        const F3 delta = f3(l[0], l[1], l[2]) - pos;
        const float r = sqrtf(dot3(delta, delta));
        const F3 L = normalize3(delta);
        const float fd = satf((l[3] - r) * l[7]);
        radiance = radiance + pbr(L, normal, V, base, roughness, F0, f3(l[4], l[5], l[6]) * fd);
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (i >= env.ns) break;
        const float* l = env.spot[i];
        const F3 delta = f3(l[0], l[1], l[2]) - pos;
        const float r = sqrtf(dot3(delta, delta));
        const F3 L = normalize3(delta);
        const float fd = satf((l[3] - r) * l[7]);
        const F3 lit = pbr(L, normal, V, base, roughness, F0, f3(l[8], l[9], l[10]) * fd);
        const float cosA = dot3(f3(l[4], l[5], l[6]), -L);
        const float fa = satf((cosA - l[11]) * l[12]);
        radiance = radiance + lit * fa;
    }
    return f3(tmaxf(radiance.x, 0.0f), tmaxf(radiance.y, 0.0f), tmaxf(radiance.z, 0.0f));
}

// GGXShade for a material without textures (shading.h:84-161)
__device__ F3 ggxShade(const Material& m, F3 pos, F3 nrm, F3 camPos, const LightEnvDev& env) {
    const F3 normal = normalize3(nrm);
    if (m.model == 2u) return m.emissive;
    const F3 V = normalize3(camPos - pos);
    const float roughness = 1.0f - m.glossiness;
    return ggxLit(m.emissive, m.diffuse, m.specular, roughness, pos, normal, V, env);
}

// true when GGXShade reads a texture for m: the emissive id for the emissive model, else any of
// the diffuse, specular and glossiness ids
__device__ __forceinline__ bool readsTextures(const Material& m) {
    return m.model == 2u ? m.texDiffuse != kNoTexture : (m.texDiffuse & m.texSpecular & m.texGloss) != kNoTexture;
}

// ReadTexture for material texture `id` (shading.h:45-47); false (the material's constant stays)
// for no texture, and for an id that names no live texture of the scene
__device__ __forceinline__ bool materialTexture(const ViewDev& V, uint32_t id, float2 uv, float2 dx, float2 dy,
                                                float4& out) {
    if (id == kNoTexture || id >= V.textureCount) return false;
    const unsigned long long t = __ldg(viewPtr(V.textures) + id);
    if (!t) return false;
    out = readTexture(t, uv.x, uv.y, dx, dy);
    return true;
}

// ACESFilm, linearToSRgb, ToColor4Unorm8SRgb (shading_helpers.h:158-200; libraries/hvvr/shared/util_graphics.h:26-28)
__device__ __forceinline__ float aces(float x) { return satf((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f)); }
__device__ __forceinline__ float toSrgb(float x) {
    return (x <= 0.0031308f) ? (x * 12.92f) : (powf(x, (1.0f / 2.4f)) * 1.055f - .055f);
}
__device__ __forceinline__ uint32_t packColor(F3 c) {
    const uint32_t r = uint32_t(toSrgb(c.x) * 255.0f);
    const uint32_t g = uint32_t(toSrgb(c.y) * 255.0f);
    const uint32_t b = uint32_t(toSrgb(c.z) * 255.0f);
    return r | (g << 8) | (b << 16) | 0xFF000000u;
}

__device__ __forceinline__ F3 halfNormal(float4 a, float4 b) {
    const uint32_t n01 = __float_as_uint(a.w), n23 = __float_as_uint(b.x);
    return f3(__half2float(__ushort_as_half((unsigned short)(n01 & 0xffffu))),
              __half2float(__ushort_as_half((unsigned short)(n01 >> 16))),
              __half2float(__ushort_as_half((unsigned short)(n23 & 0xffffu))));
}

// ascending sort of N unique keys held in registers (odd-even transposition; N <= 32)
template <uint32_t N>
__device__ __forceinline__ void sortKeys(uint32_t (&k)[N]) {
#pragma unroll
    for (uint32_t r = 0; r < N; r++) {
#pragma unroll
        for (uint32_t i = (r & 1u); i + 1 < N; i += 2) {
            const uint32_t a = k[i], b = k[i + 1];
            k[i] = a < b ? a : b;
            k[i + 1] = a < b ? b : a;
        }
    }
}

__device__ __forceinline__ Material loadMaterial(const ViewDev& V, uint32_t index) {
    const float4* __restrict__ materials = viewPtr(V.materials);
    const float4 m0 = __ldg(materials + 4 * size_t(index) + 0);
    const float4 m1 = __ldg(materials + 4 * size_t(index) + 1);
    const float4 m2 = __ldg(materials + 4 * size_t(index) + 2);
    const float4 m3 = __ldg(materials + 4 * size_t(index) + 3);
    Material mat;
    mat.emissive = f3(m0.x, m0.y, m0.z);
    mat.diffuse = f3(m1.x, m1.y, m1.z);
    mat.specular = f3(m2.x, m2.y, m2.z);
    mat.glossiness = m3.x;
    const uint32_t code0 = __float_as_uint(m3.z), code1 = __float_as_uint(m3.w);
    mat.model = code0 & 0xffffu;
    mat.texGloss = code0 >> 16;
    mat.texSpecular = code1 & 0xffffu;
    mat.texDiffuse = code1 >> 16;
    return mat;
}

// interpolate (shading.h:18-36) of a vertex attribute pair
__device__ __forceinline__ float2 interp2(float2 t0, float2 t1, float2 t2, F3 b) {
    return make_float2((t0.x * b.x + t1.x * b.y) + t2.x * b.z, (t0.y * b.x + t1.y * b.y) + t2.y * b.z);
}

// GGXShade (shading.h:84-161) of a hit whose material reads textures. The texture coordinates and
// their screen derivatives come from the hit's barycentrics at the shading point (bc) and one
// sample step along x (bx) and y (by): dUVdX = uv(bx) - uv(bc), dUVdY = uv(by) - uv(bc)
// (ShadeMSAA, resolve.cu:230-270). Kept out of line so the untextured path's registers do not
// grow.
__device__ __noinline__ F3 shadeTextured(const ViewDev& V, uint32_t triIndex, F3 bc, F3 bx, F3 by, F3 camPos,
                                         const LightEnvDev& env) {
    const uint4 ts = __ldg(viewPtr(V.triShade) + triIndex);
    const Material m = loadMaterial(V, ts.w);
    const float4* __restrict__ verts = viewPtr(V.verts);
    const float4 a0 = __ldg(verts + 2 * size_t(ts.x)), a1 = __ldg(verts + 2 * size_t(ts.x) + 1);
    const float4 p0 = __ldg(verts + 2 * size_t(ts.y)), p1 = __ldg(verts + 2 * size_t(ts.y) + 1);
    const float4 q0 = __ldg(verts + 2 * size_t(ts.z)), q1 = __ldg(verts + 2 * size_t(ts.z) + 1);
    const F3 pos = (f3(a0.x, a0.y, a0.z) * bc.x + f3(p0.x, p0.y, p0.z) * bc.y) + f3(q0.x, q0.y, q0.z) * bc.z;
    const F3 nrm = (halfNormal(a0, a1) * bc.x + halfNormal(p0, p1) * bc.y) + halfNormal(q0, q1) * bc.z;
    const float2 t0 = make_float2(a1.y, a1.z), t1 = make_float2(p1.y, p1.z), t2 = make_float2(q1.y, q1.z);
    const float2 uv = interp2(t0, t1, t2, bc);
    const float2 uvx = interp2(t0, t1, t2, bx), uvy = interp2(t0, t1, t2, by);
    const float2 dx = make_float2(uvx.x - uv.x, uvx.y - uv.y), dy = make_float2(uvy.x - uv.x, uvy.y - uv.y);
    const F3 normal = normalize3(nrm);
    float4 tex;
    if (m.model == 2u) return materialTexture(V, m.texDiffuse, uv, dx, dy, tex) ? f3(tex.x, tex.y, tex.z) : m.emissive;
    F3 base = m.diffuse;
    if (materialTexture(V, m.texDiffuse, uv, dx, dy, tex)) base = f3(tex.x, tex.y, tex.z);
    const F3 Vd = normalize3(camPos - pos);
    F3 F0 = m.specular;
    if (materialTexture(V, m.texSpecular, uv, dx, dy, tex)) F0 = f3(tex.x, tex.y, tex.z);
    float roughness = 1.0f - m.glossiness;
    if (materialTexture(V, m.texGloss, uv, dx, dy, tex)) roughness = 1.0f - tex.x;
    return ggxLit(m.emissive, base, F0, roughness, pos, normal, Vd, env);
}

// interpolate (shading.h:18-36) the hit's vertices at barycentrics bc and GGXShade it.
// deriv(bx, by) gives the barycentrics one sample step along x and y; it runs only when the
// material reads textures.
template <class Deriv>
__device__ __forceinline__ F3 shadeHit(const ViewDev& V, uint32_t triIndex, F3 bc, F3 camPos, const LightEnvDev& env,
                                       Deriv deriv) {
    const uint4 ts = __ldg(viewPtr(V.triShade) + triIndex);
    const Material mat = loadMaterial(V, ts.w);
    // with no texture in the scene every read falls back to the constants, which is the
    // untextured path
    if (V.textureCount && readsTextures(mat)) {
        F3 bx, by;
        deriv(bx, by);
        return shadeTextured(V, triIndex, bc, bx, by, camPos, env);
    }
    const float4* __restrict__ verts = viewPtr(V.verts);
    const float4 a0 = __ldg(verts + 2 * size_t(ts.x)), a1 = __ldg(verts + 2 * size_t(ts.x) + 1);
    const float4 p0 = __ldg(verts + 2 * size_t(ts.y)), p1 = __ldg(verts + 2 * size_t(ts.y) + 1);
    const float4 q0 = __ldg(verts + 2 * size_t(ts.z)), q1 = __ldg(verts + 2 * size_t(ts.z) + 1);
    const F3 pos = (f3(a0.x, a0.y, a0.z) * bc.x + f3(p0.x, p0.y, p0.z) * bc.y) + f3(q0.x, q0.y, q0.z) * bc.z;
    const F3 nrm = (halfNormal(a0, a1) * bc.x + halfNormal(p0, p1) * bc.y) + halfNormal(q0, q1) * bc.z;
    return ggxShade(mat, pos, nrm, camPos, env);
}

// TestTriangleFrustaUVW (prim_tests.h:89-116) over the tile's four world-space corner rays:
// true when every barycentric coordinate is out of [0, 1] on the same side for all four
__device__ __forceinline__ bool uvwAllOut(const float (&ro)[4][3], const float (&rd)[4][3], const TriGeom& tri) {
    float uMin = FLT_MAX, uMax = -FLT_MAX, vMin = FLT_MAX, vMax = -FLT_MAX, wMin = FLT_MAX, wMax = -FLT_MAX;
#pragma unroll
    for (int r = 0; r < 4; r++) {
        float u, v, w;
        rayTriUVW(f3(ro[r][0], ro[r][1], ro[r][2]), f3(rd[r][0], rd[r][1], rd[r][2]), tri, u, v, w);
        uMin = tminf(uMin, u); uMax = tmaxf(uMax, u);
        vMin = tminf(vMin, v); vMax = tmaxf(vMax, v);
        wMin = tminf(wMin, w); wMax = tmaxf(wMax, w);
    }
    return uMax < 0 || uMin > 1 || vMax < 0 || vMin > 1 || wMax < 0 || wMin > 1;
}

struct ShadeSmem {
    float ro[4][3], rd[4][3]; // world corner rays
    float pl[4][4];           // frustum planes
    // the chunk's surviving triangles, one array per component (a warp reads the same entry on
    // every lane, and a pair of entries j, k loads straight into the two halves of a register
    // pair): e0, e1, camPos - v0, e0 x e1, t, |e0 x e1| (the norm as computed in float, for the
    // depth skip) and the triangle index
    float g[12][kChunk];
    float t[kChunk], nlen[kChunk];
    uint32_t idx[kChunk];
    uint32_t warpCount[4];
    uint2 list;    // the tile's TileList as thread 0 read it
    uint32_t link; // a streamed list's next chunk, as thread 0 waited for it
    // the list triangles of the chunk being culled, 48 bytes per entry (three float4 rows of the
    // triangle array), copied in by cp.async one chunk ahead; thread i writes and reads only
    // entry i, so the copy of the next chunk can start as soon as entry i has been read
    float4 stage[3 * kChunk];
};

// cp.async of 16 bytes, global to shared, cached in L2 only (the triangle rows are gathered once
// per tile; neighbouring tiles share them through L2)
__device__ __forceinline__ void cpAsync16(void* dst, const void* src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWaitAll() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// resident CTAs per SM the register allocation must allow (7 = 72 registers per thread)
// resident CTAs per SM: N <= 8 at 72 registers; N = 16 at 96 (a few spilled bytes, 5.5% faster on
// the 16xMSAA foveated frame than 4 CTAs at 107 registers without spills)
template <uint32_t N> struct MinCtas { static constexpr int v = N <= 8 ? 7 : (N == 16 ? 5 : 4); };

// Where a shade launch takes its tiles from; item i of the launch is
//   kFromOrder: order[first + i] (order == nullptr: first + i), i < count;
//   kFromReady: the tile published in ready[first + i] by the concurrent tile cull, waited for;
//   kFromList:  list[first + i], for i < *listCount (the retry list, counted on the device).
struct ShadeSource {
    const uint32_t* order;
    const uint32_t* ready;
    const uint32_t* list;
    const uint32_t* listCount;
    uint32_t first, count;
};

// Waits (one thread) until the tile cull publishes a ready slot. A wait that runs past about a
// second gives up: it sets kStatusPipelineTimeout and returns kReadyEmpty, whose kReadyRetry bit
// makes the caller skip the slot.
__device__ uint32_t waitReady(const uint32_t* slot, uint32_t* counters) {
    for (uint32_t i = 0;; i++) {
        uint32_t v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(slot) : "memory");
        if (v != kReadyEmpty) return v;
        if (i >= (1u << 20)) {
            atomicOr(&counters[1], kStatusPipelineTimeout);
            return kReadyEmpty;
        }
        __nanosleep(i < 32 ? 128 : 1024);
    }
}

// Waits (one thread) until a streamed list's chunk is linked to its successor (or marked as the
// last); gives up like waitReady, returning kNoChunk.
__device__ uint32_t waitChunkLink(const uint32_t* link, uint32_t* counters) {
    for (uint32_t i = 0;; i++) {
        uint32_t v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(link) : "memory");
        if (v != kChunkPending) return v;
        if (i >= (1u << 20)) {
            atomicOr(&counters[1], kStatusPipelineTimeout);
            return kNoChunk;
        }
        __nanosleep(i < 32 ? 128 : 1024);
    }
}

// One tile: intersect, G-buffer grouping, shading and resolve of its 128 samples. The tile's
// list (TileList, chunk links, pool entries) is read through L2 (ld.cg): in a pipelined launch
// another SM wrote it while this launch was running.
// ROW: the row of the offset tables (the rate's spiral row, or + 6 for the rotated grid), a
// compile-time constant so that the offsets stay immediate constant-bank operands
// STREAM: the tile may come from a pipelined launch, whose longest tiles stream their lists.
template <uint32_t N, bool FMA, int ROW, bool STREAM = false>
__device__ __forceinline__ void shadeTile(const FrameDev& fr, uint32_t gt, ShadeSmem& sm, LightEnvDev& env, Mat4& M) {
    const ViewDev& V = fr.views[fr.viewCount == 1 ? 0u : __ldg(fr.blockView + gt / kTilesPerBlock)];
    const uint32_t tile = gt - V.tileStart;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t sid = tile * kTileSize + tid;
    uint2 lw;
    if constexpr (STREAM) {
        // (read once, with acquire, for the whole CTA: a streamed tile's list may be completed while
        // the CTA reads it, and every thread must take the same path)
        if (tid == 0) {
            unsigned long long l;
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(l) : "l"(V.tileLists + tile) : "memory");
            sm.list = make_uint2(uint32_t(l), uint32_t(l >> 32));
        }
        __syncthreads();
        lw = sm.list;
    } else {
        lw = __ldcg(reinterpret_cast<const uint2*>(V.tileLists + tile));
    }
    const TileList L{lw.x, lw.y};
    if (L.count == 0) {
        // ClearEmptyKernel (resolve.cu:527-542)
        V.colors[sid] = 0xFF000000u;
        if (V.tmaxOut) V.tmaxOut[sid] = INFINITY;
        uint32_t* __restrict__ hitOut = V.hitIds;
        float* __restrict__ depthOut = V.depth;
        if (hitOut) {
#pragma unroll
            for (uint32_t i = 0; i < N; i++) {
                hitOut[size_t(sid) * N + i] = ~0u;
                depthOut[size_t(sid) * N + i] = INFINITY;
            }
        }
        return;
    }
#ifdef HVVR_VISIT_CLOCKS
    long long scAcc[kScPhases] = {0, 0, 0, 0};
    long long scLast = phaseClock(L.count);
    uint32_t scChunks = 0;
#endif
    const int rate = ROW;
    for (uint32_t i = tid; i < sizeof(LightEnvDev) / 4; i += kTileSize)
        reinterpret_cast<uint32_t*>(&env)[i] = reinterpret_cast<const uint32_t*>(&V.env)[i];
    if (tid < 16) reinterpret_cast<float*>(&M)[tid] = reinterpret_cast<const float*>(&V.M)[tid];
    __syncthreads();
    // world-space tile rays (the SimpleRayFrustum of transformHierarchyCameraToWorld) and
    // FrustumPlanes (prim_tests.h:22-28)
    if (tid < 8) {
        const Rays4& cr = V.tileRays[tile];
        const uint32_t i = tid & 3u;
        if (tid < 4) {
            const F3 o = xformPoint(M, f3(cr.o[i][0], cr.o[i][1], cr.o[i][2]));
            sm.ro[i][0] = o.x; sm.ro[i][1] = o.y; sm.ro[i][2] = o.z;
        } else {
            const F3 d = xformDir(M, f3(cr.d[i][0], cr.d[i][1], cr.d[i][2]));
            sm.rd[i][0] = d.x; sm.rd[i][1] = d.y; sm.rd[i][2] = d.z;
        }
    }
    __syncthreads();
    if (tid < 4) {
        const F3 d0 = f3(sm.rd[tid][0], sm.rd[tid][1], sm.rd[tid][2]);
        const F3 d1 = f3(sm.rd[(tid + 1) & 3][0], sm.rd[(tid + 1) & 3][1], sm.rd[(tid + 1) & 3][2]);
        const F3 n = cross3(d0, d1);
        sm.pl[tid][0] = n.x; sm.pl[tid][1] = n.y; sm.pl[tid][2] = n.z;
        sm.pl[tid][3] = dot3(f3(sm.ro[tid][0], sm.ro[tid][1], sm.ro[tid][2]), n);
    }
    const F3 camPos = f3(M.m[3][0], M.m[3][1], M.m[3][2]);
    // this thread's beam, rotated to world space (GetDirectionalSample3D, gpu_samples.h:78-82)
    // this thread's beam, rotated to world space (GetDirectionalSample3D, gpu_samples.h:78-82): c,
    // du, dv; loaded again after the triangle loop so that they need no registers during it
    auto beamDirs = [&](F3& c, F3& du, F3& dv) {
        const float4* __restrict__ beams = V.beams;
        const float4 b0 = __ldg(beams + 3 * size_t(sid) + 0);
        const float4 b1 = __ldg(beams + 3 * size_t(sid) + 1);
        const float4 b2 = __ldg(beams + 3 * size_t(sid) + 2);
        c = xformDir(M, f3(b0.x, b0.y, b0.z));
        du = xformDir(M, f3(b0.w, b1.x, b1.y));
        dv = xformDir(M, f3(b1.z, b1.w, b2.x));
    };
    float dirLen;
    V2 nc, ndu, ndv; // -c, -du, -dv in both lanes, for the two-triangle setup
    {
        F3 c, du, dv;
        beamDirs(c, du, dv);
        // Upper bound on |denom| / |e0 x e1| over this sample's subsamples: denom = -dir . n with
        // dir = c + ax du + ay dv and |ax|,|ay| <= 1, so |denom| <= (|c| + |du| + |dv|) |n|.
        dirLen = (sqrtf(dot3(c, c)) + sqrtf(dot3(du, du)) + sqrtf(dot3(dv, dv))) * 1.0001f;
        nc = V2{pk(-c.x, -c.x), pk(-c.y, -c.y), pk(-c.z, -c.z)};
        ndu = V2{pk(-du.x, -du.x), pk(-du.y, -du.y), pk(-du.z, -du.z)};
        ndv = V2{pk(-dv.x, -dv.x), pk(-dv.y, -dv.y), pk(-dv.z, -dv.z)};
    }
    float tmax[N];
    uint32_t hit[N];
#pragma unroll
    for (uint32_t i = 0; i < N; i++) {
        tmax[i] = FLT_MAX;
        hit[i] = ~0u;
    }
    __syncthreads();
    SHADE_MARK(kScSetup, L.first);

    // The list is consumed chunk by chunk. Entry tid of a chunk is staged into shared memory by
    // cp.async (the 48-byte triangle record that its index names) while the CTA is still testing
    // the previous chunk, so the gathers overlap the subsample tests.
    const float4* __restrict__ trisG = viewPtr(V.tris);
    auto stage = [&](uint32_t ix) {
        const float4* src = trisG + 3 * size_t(ix);
        cpAsync16(&sm.stage[3 * tid + 0], src + 0);
        cpAsync16(&sm.stage[3 * tid + 1], src + 1);
        cpAsync16(&sm.stage[3 * tid + 2], src + 2);
    };
    // A streamed list (the cull published the tile after its first chunk) is walked as its chunks
    // are linked: each chunk is taken whole (its unused entries, in the last chunk, hold
    // kNoTriangle), and the next one is staged once this one's link is set.
    const bool streamed = STREAM && L.count == kCountStreaming;
    uint32_t chunk = L.first;
    uint32_t remaining = streamed ? kChunk + 1 : L.count;
    uint32_t survivors = 0, tested = 0;
    uint32_t idx = 0;
    if (chunk < fr.poolChunks && tid < (remaining < kChunk ? remaining : kChunk)) {
        idx = __ldcg(fr.pool + size_t(chunk) * kChunk + tid);
        if (!STREAM || idx != kNoTriangle) stage(idx);
    }
    cpAsyncCommit();
    while (remaining > 0 && chunk < fr.poolChunks) {
        const uint32_t n = remaining < kChunk ? remaining : kChunk;
        uint32_t nextChunk = streamed ? kChunkPending : __ldcg(fr.chunkNext + chunk);
        bool keep = false;
        float t = 0.0f, nlen = 0.0f;
        F3 e0 = f3(0, 0, 0), e1 = f3(0, 0, 0), v0r = f3(0, 0, 0), nrm = f3(0, 0, 0);
        cpAsyncWaitAll();
        if (tid < n && (!STREAM || idx != kNoTriangle)) {
            const float4 ra = sm.stage[3 * tid + 0], rb = sm.stage[3 * tid + 1], rc = sm.stage[3 * tid + 2];
            const TriGeom tri{f3(ra.x, ra.y, ra.z), f3(ra.w, rb.x, rb.y), f3(rb.z, rb.w, rc.x)};
            // FrustumPlanes::test
            bool in = true;
#pragma unroll
            for (int p = 0; p < 4; p++) {
                const F3 dir = f3(sm.pl[p][0], sm.pl[p][1], sm.pl[p][2]);
                const float dist = sm.pl[p][3];
                const float d0 = dot3(dir, tri.v0);
                const float d1 = d0 + dot3(dir, tri.e0);
                const float d2 = d0 + dot3(dir, tri.e1);
                if (d0 > dist && d1 > dist && d2 > dist) in = false;
            }
            if (in) {
                // IntersectTriangleTile<false>::setup
                const F3 normal = cross3(tri.e0, tri.e1);
                v0r = camPos - tri.v0;
                t = dot3(v0r, normal);
                if (!(t < 0.0f)) {
                    // TestTriangleFrustaUVW != intersect_all_out
                    if (!uvwAllOut(sm.ro, sm.rd, tri)) {
                        keep = true;
                        e0 = tri.e0;
                        e1 = tri.e1;
                        nrm = normal;
                        nlen = sqrtf(dot3(normal, normal));
                    }
                }
            }
        }
        // the next chunk's index of this entry (its chunk link has arrived by now)
        const uint32_t rest = remaining - n;
        const bool more = !streamed && rest > 0 && nextChunk < fr.poolChunks;
        uint32_t idxNext = 0;
        if (more && tid < (rest < kChunk ? rest : kChunk)) idxNext = __ldcg(fr.pool + size_t(nextChunk) * kChunk + tid);
        const uint32_t bal = __ballot_sync(kFull, keep);
        if (lane == 0) sm.warpCount[warp] = __popc(bal);
        __syncthreads();
        uint32_t off = __popc(bal & ((1u << lane) - 1u));
        uint32_t total = 0;
#pragma unroll
        for (uint32_t w = 0; w < 4; w++) {
            const uint32_t cw = sm.warpCount[w];
            off += (w < warp) ? cw : 0u;
            total += cw;
        }
        if (keep) {
            sm.g[0][off] = e0.x; sm.g[1][off] = e0.y; sm.g[2][off] = e0.z;
            sm.g[3][off] = e1.x; sm.g[4][off] = e1.y; sm.g[5][off] = e1.z;
            sm.g[6][off] = v0r.x; sm.g[7][off] = v0r.y; sm.g[8][off] = v0r.z;
            sm.g[9][off] = nrm.x; sm.g[10][off] = nrm.y; sm.g[11][off] = nrm.z;
            sm.t[off] = t;
            sm.nlen[off] = nlen;
            sm.idx[off] = idx;
        }
        __syncthreads();
        SHADE_MARK(kScCull, total);
        // stage the next chunk (this thread's entry of this chunk was read above)
        if (more && tid < (rest < kChunk ? rest : kChunk)) stage(idxNext);
        cpAsyncCommit();
        // Depth skip. The test rejects a subsample when depth * denom < t (FMA mode, exactly;
        // STRICT mode with the product rounded, covered by the 1e-4 margin in dirLen). With
        // denom <= dirLen * |n| and depth <= laneT, t > laneT * dirLen * |n| rejects every
        // subsample of the lane; a triangle is skipped only when that holds for all 32 lanes, so
        // the hits are exactly those of the full loop. Misses keep laneT at FLT_MAX (no skip).
        // For |n| >= 0 the rounded product is monotone in the bound, so "for all lanes" is the
        // test against the warp's largest bound, and lane l evaluates it for survivor g + l: one
        // ballot decides 32 survivors. The bound is taken at the start of each group of 32; depths
        // only fall, so a bound taken earlier is larger and skips no triangle that could hit.
        //
        // The triangles that are not skipped are tested two at a time, in list order: j in lane 0
        // and k in lane 1 of every packed operation (pairTest). An odd one left at the end of the
        // chunk is tested as the pair (j, j): a second test of the same triangle on the same
        // subsample changes nothing (it either fails or writes the same depth and index again).
        survivors += total;
        uint32_t pend = ~0u; // a triangle waiting for its pair partner
        auto testPair = [&](uint32_t j, uint32_t k) {
            const V2 e0 = {pk(sm.g[0][j], sm.g[0][k]), pk(sm.g[1][j], sm.g[1][k]), pk(sm.g[2][j], sm.g[2][k])};
            const V2 e1 = {pk(sm.g[3][j], sm.g[3][k]), pk(sm.g[4][j], sm.g[4][k]), pk(sm.g[5][j], sm.g[5][k])};
            const V2 vr = {pk(sm.g[6][j], sm.g[6][k]), pk(sm.g[7][j], sm.g[7][k]), pk(sm.g[8][j], sm.g[8][k])};
            const V2 nn = {pk(sm.g[9][j], sm.g[9][k]), pk(sm.g[10][j], sm.g[10][k]), pk(sm.g[11][j], sm.g[11][k])};
            const float tj = sm.t[j], tk = sm.t[k];
            const uint32_t ij = sm.idx[j], ik = sm.idx[k];
            const TriPair tp = pairSetup(nn, e0, e1, vr, nc, ndu, ndv);
            const P2 tt = FMA ? pk(-tj, -tk) : pk(tj, tk);
#pragma unroll
            for (uint32_t i = 0; i < N; i++) {
                const P2 ax = *reinterpret_cast<const P2*>(&cMsaaXX[rate][i]);
                const P2 ay = *reinterpret_cast<const P2*>(&cMsaaYY[rate][i]);
                pairTest<FMA>(tp, tt, tj, tk, ij, ik, ax, ay, tmax[i], hit[i]);
            }
        };
        for (uint32_t g0 = 0; g0 < total; g0 += 32) {
            float laneT = 0.0f;
#pragma unroll
            for (uint32_t i = 0; i < N; i++) laneT = fmaxf(laneT, tmax[i]);
            const float bound = __uint_as_float(__reduce_max_sync(kFull, __float_as_uint(laneT * dirLen)));
            const uint32_t js = g0 + lane;
            const bool skip = js < total && sm.t[js] > bound * sm.nlen[js];
            uint32_t live = __ballot_sync(kFull, js < total && !skip);
            tested += __popc(live);
            while (live) {
                const uint32_t j = g0 + uint32_t(__ffs(live) - 1);
                live &= live - 1u;
                if (pend == ~0u) {
                    pend = j;
                } else {
                    testPair(pend, j);
                    pend = ~0u;
                }
            }
        }
        if (pend != ~0u) testPair(pend, pend);
        __syncthreads();
        if (STREAM && streamed) {
            if (tid == 0) sm.link = waitChunkLink(fr.chunkNext + chunk, fr.counters);
            __syncthreads();
            nextChunk = sm.link;
            if (nextChunk < fr.poolChunks) {
                idxNext = __ldcg(fr.pool + size_t(nextChunk) * kChunk + tid);
                if (idxNext != kNoTriangle) stage(idxNext);
                remaining = n + kChunk + 1; // after this chunk: a whole chunk and an unknown rest
            } else {
                remaining = n; // the list's end: the loop stops
            }
            cpAsyncCommit();
        }
        remaining -= n;
        chunk = nextChunk;
        idx = idxNext;
        SHADE_MARK(kScTest, remaining);
#ifdef HVVR_VISIT_CLOCKS
        ++scChunks;
#endif
    }

    if (tid == 0 && survivors) atomicAdd(&fr.counters[kSurvivorWord], survivors);
    if (lane == 0 && tested) atomicAdd(&fr.counters[kTestedWord], tested);
    F3 c, du, dv;
    beamDirs(c, du, dv);
    if (uint32_t* hitOut = viewPtr(V.hitIds)) {
        float* depthOut = viewPtr(V.depth);
#pragma unroll
        for (uint32_t i = 0; i < N; i++) {
            hitOut[size_t(sid) * N + i] = hit[i];
            depthOut[size_t(sid) * N + i] = hit[i] == ~0u ? INFINITY : tmax[i];
        }
    }
    // ResolveKernel's TMaxBuffer (resolve.cu:386-457): depth along the view axis of subsample 0's
    // triangle at subsample 0's position
    if (float* tmaxOut = viewPtr(V.tmaxOut)) {
        float tv = INFINITY;
        if (hit[0] != ~0u) {
            const TriGeom tri = loadTri(viewPtr(V.tris), hit[0]);
            const TriThread th = threadSetup(tri.e0, tri.e1, camPos - tri.v0, c, du, dv);
            const float2 a0 = cMsaa[rate][0];
            const F3 uvw = calcUVW<FMA>(th, a0.x, a0.y);
            const F3 p = (tri.v0 * uvw.x + (tri.v0 + tri.e0) * uvw.y) + (tri.v0 + tri.e1) * uvw.z;
            const F3 look = f3(-M.m[2][0], -M.m[2][1], -M.m[2][2]);
            tv = dot3(p - camPos, look);
        }
        tmaxOut[sid] = tv;
    }

    // G-buffer grouping (EmitGBuffer): (triangle, mask) pairs in ascending triangle order,
    // misses (~0) last; then ShadeMSAA over the groups in that order.
    uint32_t keys[N];
#pragma unroll
    for (uint32_t i = 0; i < N; i++) keys[i] = (hit[i] << 5) | i;
    bool uniform = true;
#pragma unroll
    for (uint32_t i = 1; i < N; i++) uniform = uniform && (hit[i] == hit[0]);
    if (!uniform) sortKeys<N>(keys);
    float rx = 0.0f, ry = 0.0f, rz = 0.0f;
    const uint32_t maskAll = N < 32 ? ((1u << N) - 1u) : ~0u;
    uint32_t combined = 0;
    uint32_t gi = 0;
    while (gi < N) {
        if (combined == maskAll) break;
        const uint32_t triIndex = uint32_t(int32_t(keys[gi]) >> 5);
        if (triIndex == ~0u) break;
        uint32_t sampleMask = 0;
        uint32_t gj = gi;
        if (uniform) {
            sampleMask = maskAll;
            gj = N;
        } else {
            while (gj < N && uint32_t(int32_t(keys[gj]) >> 5) == triIndex) {
                sampleMask |= 1u << (keys[gj] & 31u);
                gj++;
            }
        }
        gi = gj;
        combined |= sampleMask;
        const float pc = float(__popc(sampleMask));
        const float inv = 1.0f / pc;
        float cax = 0.0f, cay = 0.0f;
        for (uint32_t cm = sampleMask; cm;) {
            const int si = __ffs(cm) - 1;
            cm &= ~(1u << si);
            const float2 a = cMsaa[rate][si];
            cax = cax + a.x * inv;
            cay = cay + a.y * inv;
        }
        const TriGeom tri = loadTri(viewPtr(V.tris), triIndex);
        const F3 v0r = camPos - tri.v0;
        const TriThread th = threadSetup(tri.e0, tri.e1, v0r, c, du, dv);
        const F3 bc = calcUVW<FMA>(th, cax, cay);
        const F3 col = shadeHit(V, triIndex, bc, camPos, env, [&](F3& bx, F3& by) {
            bx = calcUVW<FMA>(th, cax + 1.0f, cay + 0.0f);
            by = calcUVW<FMA>(th, cax + 0.0f, cay + 1.0f);
        });
        rx = rx + col.x * pc;
        ry = ry + col.y * pc;
        rz = rz + col.z * pc;
    }
    const float sN = 1.0f / float(N);
    viewPtr(V.colors)[sid] = packColor(f3(aces(rx * sN), aces(ry * sN), aces(rz * sN)));
#ifdef HVVR_VISIT_CLOCKS
    __syncthreads();
    SHADE_MARK(kScShade, gi);
    if (tid == 0 && gt < kShadeClockTiles) {
        for (uint32_t k = 0; k < kScPhases; k++) gShadeClocks[gt][k] = uint64_t(scAcc[k]);
        gShadeClocks[gt][kScPhases] = scChunks;
        gShadeClocks[gt][kScPhases + 1] = L.count;
    }
#endif
}

// SRC selects where the launch's tiles come from (ShadeSource): kFromOrder and kFromReady run one
// tile per CTA; kFromList walks the list with a grid-stride loop.
enum : int { kFromOrder = 0, kFromReady = 1, kFromList = 2 };

template <uint32_t N, bool FMA, int SRC, int ROW>
__global__ void __launch_bounds__(kTileSize, MinCtas<N>::v) intersectShadeKernel(FrameDev fr, ShadeSource src) {
    __shared__ ShadeSmem sm;
    __shared__ LightEnvDev env;
    __shared__ Mat4 M;
    if constexpr (SRC == kFromOrder) {
        const uint32_t gt = src.order ? src.order[src.first + blockIdx.x] : src.first + blockIdx.x;
        shadeTile<N, FMA, ROW>(fr, gt, sm, env, M);
    } else if constexpr (SRC == kFromReady) {
        __shared__ uint32_t readyTile;
        if (threadIdx.x == 0) readyTile = waitReady(src.ready + src.first + blockIdx.x, fr.counters);
        __syncthreads();
        const uint32_t gt = readyTile;
        if (gt & kReadyRetry) return; // culled and shaded by the retry passes (or the wait gave up)
        shadeTile<N, FMA, ROW, true>(fr, gt, sm, env, M);
    } else {
        const uint32_t count = *src.listCount;
        for (uint32_t item = blockIdx.x; item < count; item += gridDim.x) {
            shadeTile<N, FMA, ROW>(fr, src.list[src.first + item], sm, env, M);
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------ thin lens (depth of field)
// IntersectTriangleTile<true>, IntersectTriangleThreadDoF (prim_tests.h:247-392), TileData<true>
// (tile_data.h:33-60), GetSampleUVsDoF (gpu_samples.h:84-103), and the DoF branches of
// IntersectSamples / ShadeMSAA (intersect.cu:117-168, resolve.cu:161-284). FMA selects the
// contraction the kernel comments mark (per-subsample t, denom, depth, ray origin/direction,
// cross and dot products).
__device__ __forceinline__ F3 fma3(float s, F3 a, F3 c) { return f3(fmaf(s, a.x, c.x), fmaf(s, a.y, c.y), fmaf(s, a.z, c.z)); }

template <bool FMA>
__device__ __forceinline__ void dofBary(F3 e0, F3 e1, F3 v0l, float ddx, float ddy, float dc, F3 lc2fc, F3 lu, F3 lv,
                                        float2 luv, float2 duv, float& denom, float& v, float& w) {
    if (FMA) {
        denom = fmaf(ddy, duv.y, fmaf(ddx, duv.x, dc));
        const F3 o = fma3(luv.y, lv, fma3(luv.x, lu, v0l));
        const F3 a = -fma3(duv.y, lv, fma3(duv.x, lu, lc2fc));
        const F3 e = f3(fmaf(a.y, o.z, -(a.z * o.y)), fmaf(a.z, o.x, -(a.x * o.z)), fmaf(a.x, o.y, -(a.y * o.x)));
        v = fmaf(e1.z, e.z, fmaf(e1.y, e.y, e1.x * e.x));
        w = -fmaf(e0.z, e.z, fmaf(e0.y, e.y, e0.x * e.x));
    } else {
        denom = dc + ddx * duv.x + ddy * duv.y;
        const F3 o = (v0l + lu * luv.x) + lv * luv.y;
        const F3 rd = (lc2fc + lu * duv.x) + lv * duv.y;
        const F3 e = cross3(-rd, o);
        v = dot3(e1, e);
        w = -dot3(e0, e);
    }
}

// dirUV = aaOffset * focalToLensScale - lensUV
template <bool FMA>
__device__ __forceinline__ float2 dofDirUV(float2 aa, float fx, float fy, float2 luv) {
    return FMA ? make_float2(fmaf(aa.x, fx, -luv.x), fmaf(aa.y, fy, -luv.y))
               : make_float2(aa.x * fx - luv.x, aa.y * fy - luv.y);
}

struct DofSmem {
    float ro[4][3], rd[4][3]; // world corner rays
    float pl[4][4];           // frustum planes
    float lensU[3], lensV[3], fls[2];
    uint32_t idx[kChunk];
    float tc[kChunk], tu[kChunk], tv[kChunk], ddx[kChunk], ddy[kChunk];
    float e0[3][kChunk];
    float e1[3][kChunk];
    float vl[3][kChunk];
    uint32_t warpCount[4];
};

template <uint32_t N, bool FMA>
__global__ void __launch_bounds__(kTileSize) intersectShadeDofKernel(FrameDev fr, const uint32_t* __restrict__ order,
                                                                     uint32_t first) {
    __shared__ DofSmem sm;
    __shared__ LightEnvDev env;
    __shared__ Mat4 M;
    const uint32_t gt = order ? order[first + blockIdx.x] : first + blockIdx.x;
    const ViewDev& V = fr.views[fr.viewCount == 1 ? 0u : __ldg(fr.blockView + gt / kTilesPerBlock)];
    const uint32_t tile = gt - V.tileStart;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t sid = tile * kTileSize + tid;
    const TileList L = V.tileLists[tile];
    if (L.count == 0) {
        V.colors[sid] = 0xFF000000u;
        if (uint32_t* hitOut = V.hitIds) {
#pragma unroll
            for (uint32_t i = 0; i < N; i++) {
                hitOut[size_t(sid) * N + i] = ~0u;
                V.depth[size_t(sid) * N + i] = INFINITY;
            }
        }
        return;
    }
    const int rate = RateIndex<N>::v;
    for (uint32_t i = tid; i < sizeof(LightEnvDev) / 4; i += kTileSize)
        reinterpret_cast<uint32_t*>(&env)[i] = reinterpret_cast<const uint32_t*>(&V.env)[i];
    if (tid < 16) reinterpret_cast<float*>(&M)[tid] = reinterpret_cast<const float*>(&V.M)[tid];
    __syncthreads();
    const float4* __restrict__ beams = V.beams;
    const float4 b0 = __ldg(beams + 3 * size_t(sid) + 0);
    const float4 b1 = __ldg(beams + 3 * size_t(sid) + 1);
    const float4 b2 = __ldg(beams + 3 * size_t(sid) + 2);
    const F3 c = xformDir(M, f3(b0.x, b0.y, b0.z));
    if (tid < 8) {
        const Rays4& cr = V.tileRays[tile];
        const uint32_t i = tid & 3u;
        if (tid < 4) {
            const F3 o = xformPoint(M, f3(cr.o[i][0], cr.o[i][1], cr.o[i][2]));
            sm.ro[i][0] = o.x; sm.ro[i][1] = o.y; sm.ro[i][2] = o.z;
        } else {
            const F3 d = xformDir(M, f3(cr.d[i][0], cr.d[i][1], cr.d[i][2]));
            sm.rd[i][0] = d.x; sm.rd[i][1] = d.y; sm.rd[i][2] = d.z;
        }
    }
    if (tid == kTileSize / 2) {
        // TileData<true>::load on this sample's world-space beam; the reference rotates the
        // already rotated du/dv a second time (cameraToWorldRotation * sample.du); kept
        const F3 fu = xformDir(M, xformDir(M, f3(b0.w, b1.x, b1.y)));
        const F3 fv = xformDir(M, xformDir(M, f3(b1.z, b1.w, b2.x)));
        const float uInv = 1.0f / sqrtf(dot3(fu, fu)), vInv = 1.0f / sqrtf(dot3(fv, fv));
        const float uMag = 1.0f / uInv, vMag = 1.0f / vInv;
        const F3 lu = fu * (V.lensRadius * uInv), lv = fv * (V.lensRadius * vInv);
        sm.lensU[0] = lu.x; sm.lensU[1] = lu.y; sm.lensU[2] = lu.z;
        sm.lensV[0] = lv.x; sm.lensV[1] = lv.y; sm.lensV[2] = lv.z;
        const float sc = V.focalDistance / V.lensRadius;
        sm.fls[0] = sc * uMag;
        sm.fls[1] = sc * vMag;
    }
    __syncthreads();
    if (tid < 4) {
        const F3 d0 = f3(sm.rd[tid][0], sm.rd[tid][1], sm.rd[tid][2]);
        const F3 d1 = f3(sm.rd[(tid + 1) & 3][0], sm.rd[(tid + 1) & 3][1], sm.rd[(tid + 1) & 3][2]);
        const F3 n = cross3(d0, d1);
        sm.pl[tid][0] = n.x; sm.pl[tid][1] = n.y; sm.pl[tid][2] = n.z;
        sm.pl[tid][3] = dot3(f3(sm.ro[tid][0], sm.ro[tid][1], sm.ro[tid][2]), n);
    }
    const F3 camPos = f3(M.m[3][0], M.m[3][1], M.m[3][2]);
    // IntersectSamples: lens centre to the focal point of this sample's centre ray
    const F3 centerDir = normalize3(c);
    const float zed = dot3(xformDir(M, f3(0.0f, 0.0f, -1.0f)), centerDir);
    const F3 lc2fc = centerDir * (V.focalDistance / zed);
    // GetSampleUVsDoF: table tile = the reference's occupied-tile CTA index mod 4
    const float2* __restrict__ lensPos = V.lensPos + (V.occRank[tile] & 3u) * kTileSize * N + tid;
    float tmax[N];
    uint32_t hit[N];
#pragma unroll
    for (uint32_t i = 0; i < N; i++) {
        tmax[i] = FLT_MAX;
        hit[i] = ~0u;
    }
    __syncthreads();
    const F3 lu = f3(sm.lensU[0], sm.lensU[1], sm.lensU[2]), lv = f3(sm.lensV[0], sm.lensV[1], sm.lensV[2]);
    const float flsx = sm.fls[0], flsy = sm.fls[1];

    uint32_t chunk = L.first;
    uint32_t remaining = L.count;
    uint32_t survivors = 0;
    while (remaining > 0 && chunk < fr.poolChunks) {
        const uint32_t n = remaining < kChunk ? remaining : kChunk;
        const uint32_t nextChunk = fr.chunkNext[chunk];
        bool keep = false;
        uint32_t idx = 0;
        TriGeom tri{};
        F3 v0l = f3(0, 0, 0);
        float tc = 0.0f, tu = 0.0f, tv = 0.0f, ddx = 0.0f, ddy = 0.0f;
        if (tid < n) {
            idx = fr.pool[size_t(chunk) * kChunk + tid];
            tri = loadTri(viewPtr(V.tris), idx);
            bool in = true;
#pragma unroll
            for (int p = 0; p < 4; p++) {
                const F3 dir = f3(sm.pl[p][0], sm.pl[p][1], sm.pl[p][2]);
                const float dist = sm.pl[p][3];
                const float d0 = dot3(dir, tri.v0);
                const float d1 = d0 + dot3(dir, tri.e0);
                const float d2 = d0 + dot3(dir, tri.e1);
                if (d0 > dist && d1 > dist && d2 > dist) in = false;
            }
            if (in) {
                // IntersectTriangleTile<true>::setup
                const F3 normal = cross3(tri.e0, tri.e1);
                v0l = camPos - tri.v0;
                tc = dot3(v0l, normal);
                tu = dot3(lu, normal);
                tv = dot3(lv, normal);
                const float tExtent = fabsf(tu) + fabsf(tv);
                if (!(tc + tExtent < 0.0f)) {
                    ddx = dot3(-lu, normal);
                    ddy = dot3(-lv, normal);
                    // the corner-ray test only when every lens position sees the front of the plane
                    keep = (tc - tExtent < 0.0f) || !uvwAllOut(sm.ro, sm.rd, tri);
                }
            }
        }
        const uint32_t bal = __ballot_sync(kFull, keep);
        if (lane == 0) sm.warpCount[warp] = __popc(bal);
        __syncthreads();
        uint32_t off = __popc(bal & ((1u << lane) - 1u));
        uint32_t total = 0;
#pragma unroll
        for (uint32_t w = 0; w < 4; w++) {
            const uint32_t cw = sm.warpCount[w];
            off += (w < warp) ? cw : 0u;
            total += cw;
        }
        if (keep) {
            sm.idx[off] = idx;
            sm.tc[off] = tc; sm.tu[off] = tu; sm.tv[off] = tv; sm.ddx[off] = ddx; sm.ddy[off] = ddy;
            sm.e0[0][off] = tri.e0.x; sm.e0[1][off] = tri.e0.y; sm.e0[2][off] = tri.e0.z;
            sm.e1[0][off] = tri.e1.x; sm.e1[1][off] = tri.e1.y; sm.e1[2][off] = tri.e1.z;
            sm.vl[0][off] = v0l.x; sm.vl[1][off] = v0l.y; sm.vl[2][off] = v0l.z;
        }
        survivors += total;
        __syncthreads();
        for (uint32_t j = 0; j < total; j++) {
            const F3 je0 = f3(sm.e0[0][j], sm.e0[1][j], sm.e0[2][j]);
            const F3 je1 = f3(sm.e1[0][j], sm.e1[1][j], sm.e1[2][j]);
            const F3 jvl = f3(sm.vl[0][j], sm.vl[1][j], sm.vl[2][j]);
            const float jtc = sm.tc[j], jtu = sm.tu[j], jtv = sm.tv[j], jdx = sm.ddx[j], jdy = sm.ddy[j];
            const uint32_t jidx = sm.idx[j];
            // IntersectTriangleThreadDoF ctor
            const float dc = dot3(-lc2fc, cross3(je0, je1));
#pragma unroll
            for (uint32_t i = 0; i < N; i++) {
                const float2 luv = __ldg(lensPos + i * kTileSize);
                const float2 duv = dofDirUV<FMA>(cMsaa[rate][i], flsx, flsy, luv);
                const float t = FMA ? fmaf(jtv, luv.y, fmaf(jtu, luv.x, jtc)) : jtc + jtu * luv.x + jtv * luv.y;
                float denom, v, w;
                dofBary<FMA>(je0, je1, jvl, jdx, jdy, dc, lc2fc, lu, lv, luv, duv, denom, v, w);
                const float depthDelta = FMA ? fmaf(tmax[i], denom, -t) : tmax[i] * denom - t;
                const float u = denom - v - w;
                const int test = __float_as_int(t) | __float_as_int(depthDelta) | __float_as_int(u) |
                                 __float_as_int(v) | __float_as_int(w);
                // NaN fails (a padding sample's zero beam normalises to NaN; the sign-bit test alone
                // would depend on which NaN the hardware produces)
                if (test >= 0 && u == u && depthDelta == depthDelta) {
                    tmax[i] = hitDepth(t, denom);
                    hit[i] = jidx;
                }
            }
        }
        __syncthreads();
        remaining -= n;
        chunk = nextChunk;
    }
    if (tid == 0 && survivors) atomicAdd(&fr.counters[kSurvivorWord], survivors);

    if (uint32_t* hitOut = viewPtr(V.hitIds)) {
        float* depthOut = viewPtr(V.depth);
#pragma unroll
        for (uint32_t i = 0; i < N; i++) {
            hitOut[size_t(sid) * N + i] = hit[i];
            depthOut[size_t(sid) * N + i] = hit[i] == ~0u ? INFINITY : tmax[i];
        }
    }

    // EmitGBuffer grouping, then ShadeMSAA's DoF branch: centroid lens and direction UVs
    uint32_t keys[N];
#pragma unroll
    for (uint32_t i = 0; i < N; i++) keys[i] = (hit[i] << 5) | i;
    bool uniform = true;
#pragma unroll
    for (uint32_t i = 1; i < N; i++) uniform = uniform && (hit[i] == hit[0]);
    if (!uniform) sortKeys<N>(keys);
    float rx = 0.0f, ry = 0.0f, rz = 0.0f;
    const uint32_t maskAll = N < 32 ? ((1u << N) - 1u) : ~0u;
    uint32_t combined = 0;
    uint32_t gi = 0;
    while (gi < N) {
        if (combined == maskAll) break;
        const uint32_t triIndex = uint32_t(int32_t(keys[gi]) >> 5);
        if (triIndex == ~0u) break;
        uint32_t sampleMask = 0;
        uint32_t gj = gi;
        if (uniform) {
            sampleMask = maskAll;
            gj = N;
        } else {
            while (gj < N && uint32_t(int32_t(keys[gj]) >> 5) == triIndex) {
                sampleMask |= 1u << (keys[gj] & 31u);
                gj++;
            }
        }
        gi = gj;
        combined |= sampleMask;
        const float pc = float(__popc(sampleMask));
        const float inv = 1.0f / pc;
        float clx = 0.0f, cly = 0.0f, cdx = 0.0f, cdy = 0.0f;
        for (uint32_t cm = sampleMask; cm;) {
            const int si = __ffs(cm) - 1;
            cm &= ~(1u << si);
            const float2 luv = __ldg(lensPos + uint32_t(si) * kTileSize);
            const float2 duv = dofDirUV<FMA>(cMsaa[rate][si], flsx, flsy, luv);
            clx = clx + luv.x * inv; cly = cly + luv.y * inv;
            cdx = cdx + duv.x * inv; cdy = cdy + duv.y * inv;
        }
        const TriGeom tri = loadTri(viewPtr(V.tris), triIndex);
        const F3 normal = cross3(tri.e0, tri.e1);
        const F3 v0l = camPos - tri.v0;
        const float tdx = dot3(-lu, normal), tdy = dot3(-lv, normal), tdc = dot3(-lc2fc, normal);
        // IntersectTriangleThreadDoF::calcUVW at the centroid lens position and direction duv
        auto baryAt = [&](float2 duv) {
            float denom, v, w;
            dofBary<FMA>(tri.e0, tri.e1, v0l, tdx, tdy, tdc, lc2fc, lu, lv, make_float2(clx, cly), duv, denom, v, w);
            const float u = denom - v - w;
            const float dinv = 1.0f / denom;
            return f3(u * dinv, v * dinv, w * dinv);
        };
        // the derivatives step the centroid direction by (1, 0) and (0, 1) (ShadeMSAA's DoF branch)
        const F3 col = shadeHit(V, triIndex, baryAt(make_float2(cdx, cdy)), camPos, env, [&](F3& bx, F3& by) {
            bx = baryAt(make_float2(cdx + 1.0f, cdy + 0.0f));
            by = baryAt(make_float2(cdx + 0.0f, cdy + 1.0f));
        });
        rx = rx + col.x * pc;
        ry = ry + col.y * pc;
        rz = rz + col.z * pc;
    }
    const float sN = 1.0f / float(N);
    viewPtr(V.colors)[sid] = packColor(f3(aces(rx * sN), aces(ry * sN), aces(rz * sN)));
}

template <uint32_t N>
cudaError_t launchRate(const FrameDev& fr, uint32_t pattern, bool fpStrict, bool dof, const uint32_t* order,
                       uint32_t first, uint32_t count, cudaStream_t st) {
    constexpr int S = RateIndex<N>::v, G = RateIndex<N>::v + 6; // spiral / rotated-grid offset rows
    if (dof) {
        if (fpStrict) intersectShadeDofKernel<N, false><<<count, kTileSize, 0, st>>>(fr, order, first);
        else intersectShadeDofKernel<N, true><<<count, kTileSize, 0, st>>>(fr, order, first);
    } else {
        const ShadeSource src{order, nullptr, nullptr, nullptr, first, count};
        if (fpStrict) {
            if (pattern) intersectShadeKernel<N, false, kFromOrder, G><<<count, kTileSize, 0, st>>>(fr, src);
            else intersectShadeKernel<N, false, kFromOrder, S><<<count, kTileSize, 0, st>>>(fr, src);
        } else {
            if (pattern) intersectShadeKernel<N, true, kFromOrder, G><<<count, kTileSize, 0, st>>>(fr, src);
            else intersectShadeKernel<N, true, kFromOrder, S><<<count, kTileSize, 0, st>>>(fr, src);
        }
    }
    return cudaGetLastError();
}

// The cull -> shade pipeline of one rate class (launchCullShadePipeline).
template <uint32_t N, bool FMA, int ROW>
cudaError_t launchPipelineRate(const FrameDev& fr, uint32_t first, uint32_t count, uint32_t* queues, uint32_t* pipe,
                               uint32_t warps, uint32_t stackLimit, cudaStream_t st) {
    cudaError_t e = launchTileCullMain(fr, fr.order, first, count, queues, warps, stackLimit, fr.ready, pipe, st);
    if (e != cudaSuccess) return e;
    // CTA i shades the i-th tile the cull finishes; the launch may start once every cull CTA runs
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(count);
    cfg.blockDim = dim3(kTileSize);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const ShadeSource ready{nullptr, fr.ready, nullptr, nullptr, first, count};
    if ((e = cudaLaunchKernelEx(&cfg, intersectShadeKernel<N, FMA, kFromReady, ROW>, fr, ready)) != cudaSuccess) return e;
    // tiles whose stack outgrew the main pass: culled again, then shaded by a small grid that walks
    // the retry list (its length is only known on the device)
    if ((e = launchTileCullRetryPass(fr, fr.order, first, count, queues, st)) != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t grid = std::min<uint32_t>(count, uint32_t(2 * (sms > 0 ? sms : 148)));
    const ShadeSource retried{nullptr, nullptr, fr.retry, queues + 1, first, count};
    intersectShadeKernel<N, FMA, kFromList, ROW><<<grid, kTileSize, 0, st>>>(fr, retried);
    return cudaGetLastError();
}

template <uint32_t N>
cudaError_t launchPipelineFp(const FrameDev& fr, uint32_t pattern, bool fpStrict, uint32_t first, uint32_t count,
                             uint32_t* queues, uint32_t* pipe, uint32_t warps, uint32_t stackLimit, cudaStream_t st) {
    constexpr int S = RateIndex<N>::v, G = RateIndex<N>::v + 6;
    if (pattern)
        return fpStrict ? launchPipelineRate<N, false, G>(fr, first, count, queues, pipe, warps, stackLimit, st)
                        : launchPipelineRate<N, true, G>(fr, first, count, queues, pipe, warps, stackLimit, st);
    return fpStrict ? launchPipelineRate<N, false, S>(fr, first, count, queues, pipe, warps, stackLimit, st)
                    : launchPipelineRate<N, true, S>(fr, first, count, queues, pipe, warps, stackLimit, st);
}

// RemapKernel (libraries/hvvr/raycaster/remap.cu:35-77) for split-colour 1, 2 (pentile) and 3
__global__ void remapKernel(const uint32_t* __restrict__ src, const int32_t* __restrict__ remap,
                            uint32_t* __restrict__ dst, uint32_t width, uint32_t height, uint64_t stride,
                            uint32_t split) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= width || y >= height) return;
    const size_t p = size_t(y) * width + x;
    if (split == 1) {
        const int32_t o = remap[p];
        if (o >= 0) dst[size_t(y) * stride + x] = src[o];
        return;
    }
    uint32_t cc[3] = {0, 0, 0};
    for (uint32_t ch = 0; ch < split; ch++) {
        const int32_t o = remap[p * split + ch];
        if (o >= 0) cc[ch] = src[o];
    }
    dst[size_t(y) * stride + x] = split == 2
                                      ? ((cc[1] & 0xffu) | (cc[0] & 0xff00u) | (cc[1] & 0xff0000u) | 0xff000000u)
                                      : ((cc[0] & 0xffu) | (cc[1] & 0xff00u) | (cc[2] & 0xff0000u) | 0xff000000u);
}

} // namespace

cudaError_t launchIntersectShade(const FrameDev& fr, uint32_t msaa, uint32_t pattern, bool fpStrict, bool dof,
                                 const uint32_t* order, uint32_t first, uint32_t count, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    switch (msaa) {
    case 1: return launchRate<1>(fr, pattern, fpStrict, dof, order, first, count, st);
    case 2: return launchRate<2>(fr, pattern, fpStrict, dof, order, first, count, st);
    case 4: return launchRate<4>(fr, pattern, fpStrict, dof, order, first, count, st);
    case 8: return launchRate<8>(fr, pattern, fpStrict, dof, order, first, count, st);
    case 16: return launchRate<16>(fr, pattern, fpStrict, dof, order, first, count, st);
    case 32: return launchRate<32>(fr, pattern, fpStrict, dof, order, first, count, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launchCullShadePipeline(const FrameDev& fr, uint32_t msaa, uint32_t pattern, bool fpStrict, uint32_t first,
                                    uint32_t count, uint32_t* queues, uint32_t* pipe, uint32_t warps,
                                    uint32_t stackLimit, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    if (!fr.ready) return cudaErrorInvalidValue;
    switch (msaa) {
    case 1: return launchPipelineFp<1>(fr, pattern, fpStrict, first, count, queues, pipe, warps, stackLimit, st);
    case 2: return launchPipelineFp<2>(fr, pattern, fpStrict, first, count, queues, pipe, warps, stackLimit, st);
    case 4: return launchPipelineFp<4>(fr, pattern, fpStrict, first, count, queues, pipe, warps, stackLimit, st);
    case 8: return launchPipelineFp<8>(fr, pattern, fpStrict, first, count, queues, pipe, warps, stackLimit, st);
    case 16: return launchPipelineFp<16>(fr, pattern, fpStrict, first, count, queues, pipe, warps, stackLimit, st);
    case 32: return launchPipelineFp<32>(fr, pattern, fpStrict, first, count, queues, pipe, warps, stackLimit, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launchRemap(const CameraDev& c, cudaStream_t st) {
    if (!c.image || !c.remap || c.width == 0 || c.height == 0) return cudaSuccess;
    const dim3 block(16, 8);
    const dim3 grid((c.width + 15) / 16, (c.height + 7) / 8);
    remapKernel<<<grid, block, 0, st>>>(c.colors, c.remap, c.image, c.width, c.height, c.imageStride, c.split);
    return cudaGetLastError();
}

cudaError_t uploadMsaaTable(uint32_t n, uint32_t pattern, const float* offsets, cudaStream_t st) {
    int idx = -1;
    switch (n) {
    case 1: idx = 0; break;
    case 2: idx = 1; break;
    case 4: idx = 2; break;
    case 8: idx = 3; break;
    case 16: idx = 4; break;
    case 32: idx = 5; break;
    default: return cudaErrorInvalidValue;
    }
    if (pattern > 1) return cudaErrorInvalidValue;
    idx += 6 * int(pattern);
    // the packed products' addend (-0, -0), written with every table upload (mul2)
    const unsigned long long negZero2 = 0x8000000080000000ull;
    cudaError_t ez = cudaMemcpyToSymbolAsync(cNegZero2, &negZero2, sizeof(negZero2), 0, cudaMemcpyHostToDevice, st);
    if (ez != cudaSuccess) return ez;
    cudaError_t e = cudaMemcpyToSymbolAsync(cMsaa, offsets, n * sizeof(float2), size_t(idx) * 32 * sizeof(float2),
                                            cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    // the duplicated per-axis copies (pageable host staging: the copy completes before the call returns)
    float2 xs[32], ys[32];
    for (uint32_t i = 0; i < n; i++) {
        xs[i] = make_float2(offsets[2 * i], offsets[2 * i]);
        ys[i] = make_float2(offsets[2 * i + 1], offsets[2 * i + 1]);
    }
    e = cudaMemcpyToSymbolAsync(cMsaaXX, xs, n * sizeof(float2), size_t(idx) * 32 * sizeof(float2),
                                cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbolAsync(cMsaaYY, ys, n * sizeof(float2), size_t(idx) * 32 * sizeof(float2),
                                   cudaMemcpyHostToDevice, st);
}

} // namespace hvb

#ifdef HVVR_VISIT_CLOCKS
// profiling build only: per global tile [0, tiles), kScPhases phase cycle sums of the intersect/shade
// CTA's thread 0, then its chunk count and list length
extern "C" int hvvr_dbg_shade_clocks(unsigned long long* out, uint32_t tiles) {
    if (!out || tiles > hvb::kShadeClockTiles) return HVVR_ERR_INVALID;
    return cudaMemcpyFromSymbol(out, hvb::gShadeClocks, size_t(tiles) * sizeof(hvb::gShadeClocks[0])) == cudaSuccess
               ? HVVR_OK
               : HVVR_ERR_CUDA;
}
#endif

