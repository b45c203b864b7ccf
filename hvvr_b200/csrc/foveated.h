// foveated.h - the reference's polar foveated sample set and foveated frame transform (host).
#pragma once

#include <stdint.h>

#include <vector>

#include "../../include/hvvr_c.h"
#include "hvvr_internal.h"

namespace hvb {

struct PolarBeam {
    float c[3], du[3], dv[3]; // eye-space DirectionalBeam {centerRay, du, dv}
};

struct PolarSetup {
    uint32_t samplesPerRing = 0, ringCount = 0;
    uint32_t valid = 0, blocks = 0, tiles = 0, padded = 0;
    float eccM = 0, eccW0 = 0, eccS = 0, eccInvW0 = 0, eccInvLogA = 0, eccInvM = 0; // EccentricityMap
    float maxEccentricity = 0;                 // radians
    std::vector<PolarBeam> beams;              // [valid] clustered order
    std::vector<uint32_t> remap;               // [padded * 2] polar texel (azimuth index, ring) per sample; ~0 padding
    std::vector<Rays4> tileRays, blockRays;    // eye-space frusta; degenerate (origin at infinity) when empty
};

// polarSpaceFoveatedSetup for one camera: samples, clustering and eye-space frusta
void buildPolarFoveatedSetup(float degreeTrackingError, float maxFOVDegrees, float marSlope, float fovealMARDegrees,
                             PolarSetup& out);

// the per-frame part of renderFoveatedPolarSpaceCudaReconstruct: eyeToWorld and the four
// world-space cull planes {normal, dist} of the camera's sample bounds. Matrices column-major.
void foveatedFrame(const float cameraToWorld[16], const hvvr_vec3& eyeDir, const hvvr_float_rect& sampleBounds,
                   const hvvr_float_rect& viewport, float eyeToWorld[16], float planes[4][4]);

// the foveated resolve's matrices for a frame (render.cpp:478-486): sampleToEye =
// invert(eyeToCamera) * sampleToCamera and eyeToSamplePrevious = matrix4x4(eyePrevToSamplePrev)
// * (worldToEyePrev * eyeToWorld); then the history (worldToEyePrev, eyePrevToSamplePrev)
// becomes (invert(eyeToWorld), invert(sampleToEye)). A new camera's history is (zero,
// identity): the zero matrix sends every reprojection to NaN, so the first frame reads no
// history. Matrices column-major.
void foveatedResolveFrame(const float eyeToWorld[16], const hvvr_vec3& eyeDir, const hvvr_float_rect& viewport,
                          float worldToEyePrev[16], float eyePrevToSamplePrev[9], float sampleToEye[9],
                          float eyeToSamplePrev[16]);

} // namespace hvb
