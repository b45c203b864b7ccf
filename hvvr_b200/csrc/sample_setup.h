// sample_setup.h - the on-device sample hierarchy builder (sample_setup.cu). Not part of the
// public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/hvvr_c.h"
#include "hvvr_internal.h"

namespace hvb {

template <class T> struct DevBuf;

// where the builder writes: the camera's device buffers, sized by the builder
struct DeviceSampleSetup {
    DevBuf<Rays4>* tileRays;
    DevBuf<Rays4>* blockRays;
    DevBuf<float4>* beams;   // padded * 3
    DevBuf<int32_t>* remap;  // width * height * split
    uint32_t blocks = 0, tiles = 0, padded = 0, valid = 0;
};

// SampleData for the perspective mapping, on the device: clusters the samples, and writes the
// tile and block frusta (camera space), the beams and the image -> sample remap. needsHost is set
// (and nothing written) when two samples share a position or a position is NaN: the reference's
// std::sort then decides their order, and the caller builds on the host.
int buildSampleSetupDevice(const hvvr_sample* samples, uint32_t count, uint32_t split, const hvvr_float_rect& vp,
                           const hvvr_thin_lens& lens, uint32_t width, uint32_t height, DeviceSampleSetup& out,
                           cudaStream_t st, bool& needsHost);

} // namespace hvb
