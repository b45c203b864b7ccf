// sample_setup.cu - the sample hierarchy built on the device: SampleData::SampleData
// (libraries/hvvr/raycaster/camera.cpp:21-64) for the perspective mapping, with naiveXYCluster
// (sample_clustering.h:17-49), BeamBatch2D (sample_hierarchy.cpp:154-190), get3DFrustumFrom2D
// (sample_hierarchy.cpp:46-123), the beams of BeamBatch::generateFrom2D (sample_hierarchy.cpp:
// 129-152) and imageLocationToSampleIndex.
//
// naiveXYCluster is four rounds of std::sort with lexicographic comparators on the sample
// position. When no two samples share a position, every round has one sorted order whatever the
// algorithm, so stable device radix sorts of (y, x) and (x, y) keys reproduce the reference's
// order exactly; the builder reports duplicate or NaN positions to the caller, which then builds
// on the host (where std::sort decides the order among equal positions). The rectangle and
// frustum arithmetic keeps the host builder's operation order (every .cu file is compiled without
// FMA contraction and with IEEE division and square root, under FTZ like the host's MXCSR).
#include "dev_common.cuh"
#include "host_objects.h"
#include "sample_setup.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <math.h>

#include <vector>

namespace hvb {
namespace {

enum : uint32_t { kKeyYX = 0, kKeyXY = 1 };
enum : uint32_t { kFlagNaN = 1, kFlagDuplicate = 2 };

// float -> uint32 with the float order (-0 and +0 equal, as the comparators treat them)
__device__ __forceinline__ uint32_t orderKey(float f) {
    uint32_t u = __float_as_uint(f);
    if (u == 0x80000000u) u = 0;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void keysKernel(const hvvr_sample* __restrict__ samples, const uint32_t* __restrict__ perm, uint32_t count,
                           uint32_t mode, unsigned long long* __restrict__ keys, uint32_t* __restrict__ flags) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    const hvvr_sample& s = samples[perm ? perm[p] : p];
    const float x = s.position.x, y = s.position.y;
    if (isnan(x) || isnan(y)) atomicOr(flags, kFlagNaN);
    const unsigned long long kx = orderKey(x), ky = orderKey(y);
    keys[p] = mode == kKeyYX ? ((ky << 32) | kx) : ((kx << 32) | ky);
}

__global__ void iotaKernel(uint32_t* __restrict__ v, uint32_t count) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < count) v[p] = p;
}

// equal neighbours in the (y, x)-sorted order: two samples at one position
__global__ void duplicateKernel(const unsigned long long* __restrict__ keys, uint32_t count, uint32_t* __restrict__ flags) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0 || p >= count) return;
    if (keys[p] == keys[p - 1]) atomicOr(flags, kFlagDuplicate);
}

struct M3 {
    F3 c0, c1, c2;
};
__device__ __forceinline__ F3 mul(const M3& m, F3 v) {
    return f3(m.c0.x * v.x + m.c1.x * v.y + m.c2.x * v.z, m.c0.y * v.x + m.c1.y * v.y + m.c2.y * v.z,
              m.c0.z * v.x + m.c1.z * v.y + m.c2.z * v.z);
}
__device__ __forceinline__ float fmin2(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmax2(float a, float b) { return a > b ? a : b; }

// get3DFrustumFrom2D (perspective branch). f = {xMin, -xMax, yMin, -yMax}.
__device__ Rays4 frustumFrom2D(const float f[4], const M3& S, float lensRadius, float focalDistance) {
    const float farPlane = -100.0f;
    const float xMin = f[0], xMax = -f[1], yMin = f[2], yMax = -f[3];
    const F3 nearP[4] = {f3(-lensRadius, -lensRadius, 0), f3(+lensRadius, -lensRadius, 0),
                         f3(+lensRadius, +lensRadius, 0), f3(-lensRadius, +lensRadius, 0)};
    const F3 rd[4] = {mul(S, f3(xMin, yMax, 1)), mul(S, f3(xMax, yMax, 1)), mul(S, f3(xMax, yMin, 1)),
                      mul(S, f3(xMin, yMin, 1))};
    F3 focus[4];
    for (int i = 0; i < 4; i++) focus[i] = rd[i] * (focalDistance / -rd[i].z);
    float fxMax = -INFINITY, fxMin = INFINITY, fyMax = -INFINITY, fyMin = INFINITY;
    for (int i = 0; i < 4; ++i) {
        for (int j = 0; j < 4; ++j) {
            const F3 pos = nearP[i];
            const F3 dir = normalize3(focus[j] - pos);
            const F3 p = pos + dir * (farPlane / dir.z);
            fxMax = fmax2(fxMax, p.x);
            fxMin = fmin2(fxMin, p.x);
            fyMax = fmax2(fyMax, p.y);
            fyMin = fmin2(fyMin, p.y);
        }
    }
    const F3 farP[4] = {f3(fxMin, fyMin, farPlane), f3(fxMax, fyMin, farPlane), f3(fxMax, fyMax, farPlane),
                        f3(fxMin, fyMax, farPlane)};
    Rays4 r;
    for (int i = 0; i < 4; i++) {
        const F3 d = normalize3(farP[i] - nearP[i]);
        r.o[i][0] = nearP[i].x;
        r.o[i][1] = nearP[i].y;
        r.o[i][2] = nearP[i].z;
        r.d[i][0] = d.x;
        r.d[i][1] = d.y;
        r.d[i][2] = d.z;
    }
    return r;
}

// BeamBatch2D per tile: the rectangle of its 128 samples padded by the major axis, in sample
// order (positions past the last sample repeat it), then the tile's frustum
__global__ void tileKernel(const hvvr_sample* __restrict__ samples, const uint32_t* __restrict__ perm, uint32_t count,
                           uint32_t tiles, M3 S, float lensRadius, float focalDistance, float4* __restrict__ rects,
                           Rays4* __restrict__ tileRays) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tiles) return;
    float tf[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
    for (uint32_t k = 0; k < kTileSize; k++) {
        const uint32_t p = min(t * kTileSize + k, count - 1);
        const hvvr_sample& s = samples[perm[p]];
        const float x = s.position.x, y = s.position.y, mj = s.major_axis_length;
        const float xs[2] = {x + mj, x - mj}, ys[2] = {y + mj, y - mj};
        for (int q = 0; q < 2; q++) {
            tf[0] = fmin2(tf[0], xs[q]);
            tf[1] = fmin2(tf[1], -xs[q]);
            tf[2] = fmin2(tf[2], ys[q]);
            tf[3] = fmin2(tf[3], -ys[q]);
        }
    }
    for (int j = 0; j < 4; j++) tf[j] = fmax2(tf[j], -INFINITY);
    rects[t] = make_float4(tf[0], tf[1], tf[2], tf[3]);
    tileRays[t] = frustumFrom2D(tf, S, lensRadius, focalDistance);
}

// a block's rectangle is the union of its tiles' in tile order
__global__ void blockKernel(const float4* __restrict__ rects, uint32_t blocks, M3 S, float lensRadius,
                            float focalDistance, Rays4* __restrict__ blockRays) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= blocks) return;
    float bf[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
    for (uint32_t t = 0; t < kTilesPerBlock; t++) {
        const float4 r = rects[b * kTilesPerBlock + t];
        bf[0] = fmin2(bf[0], r.x);
        bf[1] = fmin2(bf[1], r.y);
        bf[2] = fmin2(bf[2], r.z);
        bf[3] = fmin2(bf[3], r.w);
    }
    blockRays[b] = frustumFrom2D(bf, S, lensRadius, focalDistance);
}

// unpackSample (libraries/hvvr/raycaster/samples.cpp:144-159) and the camera-space beam
// {S (c, 1), S (major, 0), S (minor, 0)}; padding positions are zero samples
__global__ void beamsKernel(const hvvr_sample* __restrict__ samples, const uint32_t* __restrict__ perm, uint32_t count,
                            uint32_t padded, M3 S, float4* __restrict__ beams) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= padded) return;
    float cx = 0.0f, cy = 0.0f, mjx = 0.0f, mjy = 0.0f, mnx = 0.0f, mny = 0.0f;
    if (p < count) {
        const hvvr_sample& s = samples[perm[p]];
        const float ext = 0.70710678118f;
        mnx = s.minor_axis.x * ext;
        mny = s.minor_axis.y * ext;
        const float mlen = sqrtf(s.minor_axis.x * s.minor_axis.x + s.minor_axis.y * s.minor_axis.y);
        const float rescale = s.major_axis_length * ext / mlen;
        cx = s.position.x;
        cy = s.position.y;
        mjx = -mny * rescale;
        mjy = mnx * rescale;
    }
    const F3 c = mul(S, f3(cx, cy, 1.0f));
    const F3 du = mul(S, f3(mjx, mjy, 0.0f));
    const F3 dv = mul(S, f3(mnx, mny, 0.0f));
    beams[3 * size_t(p) + 0] = make_float4(c.x, c.y, c.z, du.x);
    beams[3 * size_t(p) + 1] = make_float4(du.y, du.z, dv.x, dv.y);
    beams[3 * size_t(p) + 2] = make_float4(dv.z, 0.0f, 0.0f, 0.0f);
}

// imageLocationToSampleIndex: the last sample (in cluster order) at a pixel location wins
__global__ void remapKernel(const hvvr_sample* __restrict__ samples, const uint32_t* __restrict__ perm, uint32_t count,
                            uint32_t split, uint32_t width, uint32_t height, int32_t* __restrict__ remap) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    const uint32_t i = perm[p];
    const hvvr_sample& s = samples[i];
    if (s.pixel_x < width && s.pixel_y < height) {
        const size_t idx = (size_t(s.pixel_y) * width + s.pixel_x) * split + i % split;
        atomicMax(remap + idx, int32_t(p));
    }
}

inline uint32_t grid(size_t n, uint32_t block) { return uint32_t((n + block - 1) / block); }

} // namespace

int buildSampleSetupDevice(const hvvr_sample* samples, uint32_t count, uint32_t split, const hvvr_float_rect& vp,
                           const hvvr_thin_lens& lens, uint32_t width, uint32_t height, DeviceSampleSetup& out,
                           cudaStream_t st, bool& needsHost) {
    needsHost = false;
    if (count == 0) return fail(HVVR_ERR_STATE, "camera has no samples");
    const uint32_t blocks = (count + kBlockSize - 1) / kBlockSize;
    const uint32_t tiles = blocks * kTilesPerBlock, padded = blocks * kBlockSize;
    // strata of naiveXYCluster, as the host computes them
    const size_t k = blocks;
    const size_t yStrata = (size_t)sqrt((double)k);
    const size_t xStrata = (k + yStrata - 1) / yStrata;
    const size_t blockYStrata = (size_t)sqrt((double)kTilesPerBlock);
    const size_t blockXStrata = (kTilesPerBlock + blockYStrata - 1) / blockYStrata;

    DevBuf<hvvr_sample> dSamples;
    DevBuf<unsigned long long> keys[2];
    DevBuf<uint32_t> perm[2], flags;
    TRY(dSamples.upload(samples, count, st));
    TRY(keys[0].alloc(count));
    TRY(keys[1].alloc(count));
    TRY(perm[0].alloc(count));
    TRY(perm[1].alloc(count));
    TRY(flags.alloc(1));
    CUDA_TRY(cudaMemsetAsync(flags.p, 0, 4, st));
    // sort 1 of naiveXYCluster: the whole set by (y, x)
    keysKernel<<<grid(count, 256), 256, 0, st>>>(dSamples.p, nullptr, count, kKeyYX, keys[0].p, flags.p);
    iotaKernel<<<grid(count, 256), 256, 0, st>>>(perm[0].p, count);
    size_t tempBytes = 0;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, keys[0].p, keys[1].p, perm[0].p, perm[1].p, int(count),
                                             0, 64, st));
    DevBuf<uint8_t> temp;
    TRY(temp.alloc(tempBytes));
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.p, tempBytes, keys[0].p, keys[1].p, perm[0].p, perm[1].p, int(count),
                                             0, 64, st));
    duplicateKernel<<<grid(count, 256), 256, 0, st>>>(keys[1].p, count, flags.p);
    uint32_t flag = 0;
    CUDA_TRY(cudaMemcpyAsync(&flag, flags.p, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (flag) {
        needsHost = true;
        return HVVR_OK;
    }
    // sorts 2-4: fixed-size runs of the current order, sorted within each run
    uint32_t cur = 1;  // perm[cur] holds the order
    auto round = [&](size_t run, uint32_t mode) -> int {
        std::vector<int> begins, ends;
        for (size_t lo = 0; lo < count; lo += run) {
            begins.push_back(int(lo));
            ends.push_back(int(std::min<size_t>(lo + run, count)));
        }
        DevBuf<int> dBegin, dEnd;
        TRY(dBegin.upload(begins.data(), begins.size(), st));
        TRY(dEnd.upload(ends.data(), ends.size(), st));
        keysKernel<<<grid(count, 256), 256, 0, st>>>(dSamples.p, perm[cur].p, count, mode, keys[0].p, flags.p);
        size_t bytes = 0;
        CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(nullptr, bytes, keys[0].p, keys[1].p, perm[cur].p,
                                                           perm[cur ^ 1].p, int(count), int(begins.size()),
                                                           dBegin.p, dEnd.p, st));
        TRY(temp.ensure(bytes));
        CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(temp.p, bytes, keys[0].p, keys[1].p, perm[cur].p,
                                                           perm[cur ^ 1].p, int(count), int(begins.size()),
                                                           dBegin.p, dEnd.p, st));
        cur ^= 1;
        // the offset arrays are freed on return: finish the sort first
        CUDA_TRY(cudaStreamSynchronize(st));
        return HVVR_OK;
    };
    TRY(round(kBlockSize * xStrata, kKeyXY));            // rows of blocks by (x, y)
    TRY(round(kBlockSize, kKeyYX));                       // blocks by (y, x)
    TRY(round(kTileSize * blockXStrata, kKeyXY));         // runs of tiles by (x, y)
    const uint32_t* order = perm[cur].p;

    // Camera::getSampleToCamera (libraries/hvvr/raycaster/camera.cpp:167-171)
    const M3 S{F3{vp.upper.x - vp.lower.x, 0, 0}, F3{0, vp.lower.y - vp.upper.y, 0}, F3{vp.lower.x, vp.upper.y, -1}};
    DevBuf<float4> rects;
    TRY(rects.alloc(tiles));
    TRY(out.tileRays->alloc(tiles));
    TRY(out.blockRays->alloc(blocks));
    TRY(out.beams->alloc(size_t(padded) * 3));
    TRY(out.remap->alloc(size_t(width) * height * split));
    tileKernel<<<grid(tiles, 128), 128, 0, st>>>(dSamples.p, order, count, tiles, S, lens.radius, lens.focal_distance,
                                                 rects.p, out.tileRays->p);
    blockKernel<<<grid(blocks, 64), 64, 0, st>>>(rects.p, blocks, S, lens.radius, lens.focal_distance,
                                                 out.blockRays->p);
    beamsKernel<<<grid(padded, 256), 256, 0, st>>>(dSamples.p, order, count, padded, S, out.beams->p);
    if (out.remap->n) {
        CUDA_TRY(cudaMemsetAsync(out.remap->p, 0xff, out.remap->n * sizeof(int32_t), st));
        remapKernel<<<grid(count, 256), 256, 0, st>>>(dSamples.p, order, count, split, width, height, out.remap->p);
    }
    CUDA_TRY(cudaGetLastError());
    // the scratch buffers are freed on return
    CUDA_TRY(cudaStreamSynchronize(st));
    out.blocks = blocks;
    out.tiles = tiles;
    out.padded = padded;
    out.valid = count;
    return HVVR_OK;
}

} // namespace hvb
