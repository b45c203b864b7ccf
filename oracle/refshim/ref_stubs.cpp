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
