// Link stubs (test infrastructure only): camera.cpp's Camera methods and foveated.cpp
// reference GPU-side classes that the CPU harness never constructs. Every stub counts the
// misuse and returns without side effects; the harness checks the counter stays zero.
#include "gpu_camera.h"
#include "gpu_context.h"

int hvvr_ref_stub_hits = 0;

namespace hvvr {
GPUCamera* GPUContext::getCreateCamera(const Camera*, bool& created) { hvvr_ref_stub_hits++; created = false; return nullptr; }
bool GPUCamera::bindTexture(GPUContext&, ImageResourceDescriptor) { hvvr_ref_stub_hits++; return false; }
void GPUCamera::updateConfig(RaycasterOutputFormat, int32_t*, DirectionalBeam*, ThinLens, uint32_t, uint32_t, uint32_t,
                             uint32_t, uint32_t) { hvvr_ref_stub_hits++; }
void GPUCamera::copyImageToCPU(ImageResourceDescriptor) { hvvr_ref_stub_hits++; }
void GPUCamera::setCameraJitter(vector2) { hvvr_ref_stub_hits++; }
void GPUCamera::copyImageToBoundTexture() { hvvr_ref_stub_hits++; }
void GPUCamera::registerPolarFoveatedSamples(const std::vector<vector2ui>&, float, const EccentricityMap&, uint32_t,
                                             uint32_t) { hvvr_ref_stub_hits++; }
void GPUCamera::updateEyeSpaceFoveatedSamples(BeamBatch&) { hvvr_ref_stub_hits++; }
} // namespace hvvr

// Host-memory stand-ins for the four CUDA runtime calls that GPUBuffer (gpu_buffer.h) makes in
// the host code of frusta.cu (ComputeEyeSpaceFrusta moves its samples and frusta through
// GPUBuffers). The harness has no GPU; "device" memory is host memory here.
extern "C" {
cudaError_t cudaMalloc(void** p, size_t bytes) {
    *p = malloc(bytes ? bytes : 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void* p) {
    free(p);
    return cudaSuccess;
}
cudaError_t cudaMemcpy(void* dst, const void* src, size_t bytes, enum cudaMemcpyKind) {
    if (bytes) memmove(dst, src, bytes);
    return cudaSuccess;
}
const char* cudaGetErrorString(cudaError_t) { return "host stand-in"; }
}
