// facade_render.cpp - drives the C++ facade (include/hvvr.hpp) the way the reference's sample
// viewer drives its Raycaster (projects/hvvr_samples/modelviewer/modelviewer.cpp:326-383,
// libraries/hvvr/samples_shared/model_import.cpp:41-63): make a raycaster, create the scene's lights
// and models (with a model transform), create a camera, give it a render target, samples, an MSAA
// rate and a pose, render, and write the image.
//
// usage: facade_render <scene input file> <image output file>
// input (little-endian): u32 vert_count, tri_count, material_count, light_count, sample_count,
// width, height, msaa; then the ShadingVertex, PrecomputedTriangleShade, SimpleMaterial,
// LightUnion and Sample arrays; then the model transform and the camera transform (32 bytes each).
// Exit codes: 0 rendered; 2 bad input; 3 the library reported an error (printed as "hvvr::Error
// <code>: <message>").
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "hvvr.hpp"

namespace {

template <class T>
bool readArray(FILE* f, std::vector<T>& v, uint32_t n) {
    v.resize(n);
    return n == 0 || fread(v.data(), sizeof(T), n, f) == n;
}

} // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s <scene input> <image output>\n", argv[0]);
        return 2;
    }
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 2;
    uint32_t hdr[8];
    if (fread(hdr, 4, 8, f) != 8) return 2;
    const uint32_t width = hdr[5], height = hdr[6], msaa = hdr[7];
    hvvr::MeshData mesh;
    std::vector<hvvr::LightUnion> lights;
    std::vector<hvvr::Sample> samples;
    hvvr::transform modelXf, cameraXf;
    bool ok = readArray(f, mesh.verts, hdr[0]) && readArray(f, mesh.triShade, hdr[1]) &&
              readArray(f, mesh.materials, hdr[2]) && readArray(f, lights, hdr[3]) && readArray(f, samples, hdr[4]) &&
              fread(&modelXf, sizeof(modelXf), 1, f) == 1 && fread(&cameraXf, sizeof(cameraXf), 1, f) == 1;
    fclose(f);
    if (!ok) return 2;
    static_assert(sizeof(hvvr::transform) == 32, "transform layout");
    try {
        hvvr::RayCasterSpecification spec;
        auto raycaster = std::make_unique<hvvr::Raycaster>(spec);
        for (const hvvr::LightUnion& light : lights) raycaster->createLight(light);
        hvvr::Model* model = raycaster->createModel(std::move(mesh)); // topology built by the library
        model->setTransform(modelXf);
        const float aspect = float(width) / float(height);
        hvvr::Camera* camera =
            raycaster->createCamera(hvvr::FloatRect(hvvr::vector2(-aspect, -1.0f), hvvr::vector2(aspect, 1.0f)), 0.0f);
        std::vector<uint32_t> image(size_t(width) * height, 0u);
        hvvr::ImageResourceDescriptor target;
        target.memoryType = hvvr::ImageResourceDescriptor::MemoryType::CPU_MEMORY;
        target.data = image.data();
        target.width = width;
        target.height = height;
        target.stride = width;
        camera->setRenderTarget(target);
        camera->setSamples(samples.data(), uint32_t(samples.size()), 1);
        camera->setMsaa(msaa);
        camera->setCameraToWorld(cameraXf);
        if (camera->getSampleCount() != samples.size()) return 2;
        raycaster->render(0.0);
        // a viewer's per-frame calls (no effect on the image here)
        camera->advanceJitter();
        raycaster->render(1.0 / 90.0); // a second frame (scheduled by the first frame's costs)
        camera->extractImage();
        // the error model: destroying an object the raycaster does not own is reported, not fatal
        bool threw = false;
        try {
            raycaster->destroyCamera(nullptr);
        } catch (const hvvr::Error&) {
            threw = true;
        }
        if (!threw) return 2;
        FILE* o = fopen(argv[2], "wb");
        if (!o || fwrite(image.data(), 4, image.size(), o) != image.size()) return 2;
        fclose(o);
        printf("rendered %ux%u, %u samples, msaa %u\n", width, height, uint32_t(samples.size()), msaa);
    } catch (const hvvr::Error& e) {
        printf("hvvr::Error %d: %s\n", e.code(), e.what());
        return 3;
    }
    return 0;
}
