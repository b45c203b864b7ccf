// host_setup.h - host-side setup shared by the driver: camera matrices, the sample
// hierarchy and MSAA offsets. Computed once per sample-set change on the CPU, exactly as
// the reference does, with no floating-point contraction (built with -ffp-contract=off)
// and with MXCSR FTZ|DAZ set like the reference's worker threads.
#pragma once

#include <stdint.h>

#include <algorithm>
#include <math.h>
#include <vector>

#include "../../include/hvvr_c.h"
#include "hvvr_internal.h"

namespace hvb {

// scoped MXCSR FTZ|DAZ (libraries/hvvr/raycaster/raycaster.cpp:21-27)
struct FtzDazScope {
    unsigned saved;
    FtzDazScope();
    ~FtzDazScope();
};

// matrix4x4(const transform&) (libraries/hvvr/shared/vector_math.h:1021-1037, 1158-1161)
Mat4 transformToMatrix(const hvvr_transform& t);

// getSubsampleUnitOffset<N> with JITTER_SAMPLES=0 (libraries/hvvr/raycaster/gpu_samples.h:35-61)
void msaaOffsets(uint32_t n, float* out2n);
// the rotated-grid (n-rooks) alternative, same layout
void msaaOffsetsRotatedGrid(uint32_t n, float* out2n);
// naiveXYCluster (libraries/hvvr/raycaster/sample_clustering.h:17-49): stratified sorts into k
// blocks of kBlockSize and tiles of kTileSize; x(p), y(p) give a point's 2D position
template <class T, class X, class Y>
void naiveCluster(std::vector<T>& v, size_t k, X x, Y y) {
    const size_t yStrata = (size_t)sqrt((double)k);
    const size_t xStrata = (k + yStrata - 1) / yStrata;
    const size_t blockYStrata = (size_t)sqrt((double)kTilesPerBlock);
    const size_t blockXStrata = (kTilesPerBlock + blockYStrata - 1) / blockYStrata;
    auto byYX = [&](const T& a, const T& b) { return (y(a) < y(b)) || (y(a) == y(b) && x(a) < x(b)); };
    auto byXY = [&](const T& a, const T& b) { return (x(a) < x(b)) || (x(a) == x(b) && y(a) < y(b)); };
    const size_t n = v.size();
    std::sort(v.begin(), v.end(), byYX);
    for (size_t row = 0; row < yStrata; ++row) {
        const size_t lo = row * kBlockSize * xStrata, hi = std::min((row + 1) * kBlockSize * xStrata, n);
        if (lo < hi) std::sort(v.begin() + lo, v.begin() + hi, byXY);
    }
    for (size_t b = 0; b < k; ++b) {
        const size_t lo = b * kBlockSize, hi = std::min((b + 1) * kBlockSize, n);
        if (lo < hi) std::sort(v.begin() + lo, v.begin() + hi, byYX);
    }
    const size_t run = kTileSize * blockXStrata;
    for (size_t lo = 0; lo < n; lo += run) std::sort(v.begin() + lo, v.begin() + std::min(lo + run, n), byXY);
}

// depth-of-field lens positions for rate n: [4 tiles][n subsamples][128 samples] x 2 floats
void lensTable(uint32_t n, float* out);

struct SampleSetup {
    uint32_t blocks = 0, tiles = 0, padded = 0, valid = 0;
    std::vector<Rays4> tileRays, blockRays; // camera space
    std::vector<float> beams;               // padded * 12 (centerRay, du, dv; 3 x float4, last lane 0)
    std::vector<int32_t> remap;             // width*height*split
};

// SampleData::SampleData (libraries/hvvr/raycaster/camera.cpp:21-64) for the perspective
// and spherical-section mappings (libraries/hvvr/raycaster/sample_hierarchy.cpp:27-152)
void buildSampleSetup(const hvvr_sample* samples, uint32_t count, uint32_t split, const hvvr_float_rect& viewport,
                      const hvvr_thin_lens& lens, float fovXDeg, float fovYDeg, uint32_t width, uint32_t height,
                      SampleSetup& out);

} // namespace hvb
