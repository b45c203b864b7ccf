/*
 * hvvr_c.h - C ABI of the B200 primary-visibility-and-shading path.
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (HVVR_OK on success). Nothing here exits the process: failures come back as a
 * status code plus a message readable through hvvr_last_error().
 *
 * Struct layouts are byte-compatible with the reference's public types so that a
 * caller holding reference data (MeshData arrays, Sample arrays, LightUnion)
 * can pass it through unchanged. Each declaration names the reference interface
 * it replaces (paths are relative to the reference project root).
 */
#ifndef HVVR_C_H
#define HVVR_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes
 * Replaces cutilSafeCall/fail()/assert, which exit the process
 * (libraries/hvvr/raycaster/cuda_util.h:18-29, libraries/hvvr/shared/debug.cpp:20-34). */
enum {
    HVVR_OK = 0,
    HVVR_ERR_INVALID = 1,   /* bad argument or unsupported configuration */
    HVVR_ERR_NOT_FOUND = 2, /* destroy of an object this raycaster does not own; a file that cannot be opened */
    HVVR_ERR_CUDA = 3,      /* a CUDA runtime call failed */
    HVVR_ERR_OOM = 4,       /* device allocation failed */
    HVVR_ERR_OVERFLOW = 5,  /* a per-frame capacity (triangle-index pool, traversal stack) was exceeded */
    HVVR_ERR_TIMEOUT = 6,   /* a bounded device-side wait gave up */
    HVVR_ERR_STATE = 7      /* call made in the wrong state (e.g. read-back before any render) */
};

/* ---------------------------------------------------------------- plain types */
typedef struct { float x, y; } hvvr_vec2;
typedef struct { float x, y, z; } hvvr_vec3;
typedef struct { float x, y, z, w; } hvvr_vec4;

/* FloatRect (libraries/hvvr/shared/graphics_types.h:27-32) */
typedef struct { hvvr_vec2 lower, upper; } hvvr_float_rect;

/* ThinLens (libraries/hvvr/shared/graphics_types.h:170-173) */
typedef struct { float radius, focal_distance; } hvvr_thin_lens;

/* transform {quaternion rotation (x,y,z,w); vector3 translation; float scale}
 * (libraries/hvvr/shared/vector_math.h:966-969) */
typedef struct { hvvr_vec4 rotation; hvvr_vec3 translation; float scale; } hvvr_transform;

/* Sample (libraries/hvvr/raycaster/samples.h:17-29), 28 bytes */
typedef struct {
    uint32_t pixel_x, pixel_y;
    hvvr_vec2 position;   /* sample-space position in [0,1]^2 */
    hvvr_vec2 minor_axis; /* ellipse minor axis */
    float major_axis_length;
} hvvr_sample;

/* ShadingVertex (libraries/hvvr/shared/graphics_types.h:83-88), 32 bytes; normal is IEEE half x4 */
typedef struct { hvvr_vec3 pos; uint16_t normal[4]; hvvr_vec2 uv; uint32_t pad0; } hvvr_shading_vertex;

/* PrecomputedTriangleShade (libraries/hvvr/shared/graphics_types.h:208-211), 16 bytes */
typedef struct { uint32_t indices[3]; uint32_t material; } hvvr_tri_shade;

/* TopologyNode (libraries/hvvr/shared/graphics_types.h:126-151), 32 bytes.
 * data[k] / data[k+1] bound leaf k's triangle range; data[1+k] is the relative
 * child offset for an internal slot k. */
typedef struct { uint32_t leaf_mask; uint32_t data[7]; } hvvr_topology_node;

/* SimpleMaterial (libraries/hvvr/raycaster/material.h:22-49), 64 bytes */
typedef struct {
    hvvr_vec4 emissive, diffuse, specular;
    float glossiness, opacity;
    uint64_t texture_ids_and_shading_model;
} hvvr_material;

/* LightUnion (libraries/hvvr/raycaster/light.h:24-59), 56 bytes */
enum { HVVR_LIGHT_NONE = 0, HVVR_LIGHT_DIRECTIONAL = 1, HVVR_LIGHT_POINT = 2, HVVR_LIGHT_SPOT = 3 };
typedef struct { hvvr_vec3 direction; hvvr_vec3 power; } hvvr_light_directional;
typedef struct { hvvr_vec3 position; float falloff_end; hvvr_vec3 color; float falloff_scale; } hvvr_light_point;
typedef struct {
    hvvr_vec3 position; float falloff_end;
    hvvr_vec3 direction; float falloff_scale;
    hvvr_vec3 color; float cos_outer_angle; float cos_angle_scale;
} hvvr_light_spot;
typedef struct {
    uint32_t type;
    union { hvvr_light_directional directional; hvvr_light_point point; hvvr_light_spot spot; } u;
} hvvr_light_union;

/* MeshData (libraries/hvvr/raycaster/model.h:26-31) as four borrowed arrays.
 * nodes may be NULL/0: the library then builds the topology itself
 * (hvvr_generate_topology) on a private copy. */
typedef struct {
    const hvvr_shading_vertex* verts; uint32_t vert_count;
    const hvvr_tri_shade* tri_shade; uint32_t tri_count;
    const hvvr_topology_node* nodes; uint32_t node_count;
    const hvvr_material* materials; uint32_t material_count;
} hvvr_mesh_data;

/* TextureFormat and TextureData (libraries/hvvr/raycaster/texture.h:16-34): the reference's
 * format values; data points at height rows of stride_elements texels of the format's size
 * (4, 4, 8, 16, 8, 4, 4 bytes). 24 bytes on LP64, byte-compatible with TextureData. */
enum {
    HVVR_TEXTURE_NONE = 0,
    HVVR_TEXTURE_RGBA8_UNORM_SRGB = 1,
    HVVR_TEXTURE_RGBA8_UNORM = 2,
    HVVR_TEXTURE_RGBA16_UNORM = 3,
    HVVR_TEXTURE_RGBA32_FLOAT = 4,
    HVVR_TEXTURE_RGBA16_FLOAT = 5,
    HVVR_TEXTURE_R11G11B10_FLOAT = 6,
    HVVR_TEXTURE_R32_FLOAT = 7
};
typedef struct {
    const uint8_t* data;
    uint32_t format;
    uint32_t width, height;
    uint32_t stride_elements;
} hvvr_texture_data;

/* ImageResourceDescriptor (libraries/hvvr/shared/graphics_types.h:56-80).
 * Only CPU_MEMORY and CUDA_MEMORY exist here (no graphics API on the target). */
enum { HVVR_PIXEL_RGBA8_SRGB = 0 };
enum { HVVR_MEMORY_CPU = 0, HVVR_MEMORY_CUDA = 1 };
typedef struct {
    uint32_t pixel_format;
    uint32_t memory_type;
    void* data;
    uint32_t width, height;
    uint64_t stride; /* in pixels */
} hvvr_image_desc;

/* RayCasterSpecification (libraries/hvvr/raycaster/raycaster_spec.h:22-50) plus
 * the device-side knobs this implementation adds. */
enum { HVVR_MODE_DEFERRED_MSAA_RESOLVE = 0, HVVR_MODE_FOVEATED_POLAR = 1 };
enum { HVVR_FP_FMA = 0, HVVR_FP_STRICT = 1 };
typedef struct {
    uint32_t mode;
    uint32_t thread_count; /* host threads for setup work; 0 = all */
    float foveated_degree_tracking_error, foveated_max_fov_degrees, foveated_mar_slope, foveated_foveal_mar_degrees;
    uint32_t output_format;
    uint32_t output_to_3d_api; /* must be 0: no graphics API here */
    /* additions */
    uint32_t fp_mode;             /* HVVR_FP_FMA (reference kernel comments) or HVVR_FP_STRICT (no FMA in edge tests) */
    uint64_t tri_index_capacity;  /* triangle-index pool shared by the raycaster's cameras, entries; 0 = default (128M as the reference) */
    int device;                   /* CUDA device ordinal */
    uint32_t sample_setup;        /* HVVR_SETUP_DEVICE (default) or HVVR_SETUP_HOST: where a camera's sample hierarchy is built */
    uint32_t bvh_build;           /* for models created without topology: HVVR_BVH_HOST (default; GenerateTopology's
                                     SAH build, the reference's triangle IDs) or HVVR_BVH_DEVICE
                                     (hvvr_generate_topology_device) */
} hvvr_spec;
enum { HVVR_BVH_HOST = 0, HVVR_BVH_DEVICE = 1 };
/* The sample hierarchy (SampleData: clustering, tile and block frusta, beams, image remap) is built
 * on the device when the samples' positions are distinct and not NaN and the spherical mapping is
 * off: the reference's clustering sorts are then order-unique and the result equals the host
 * build bit for bit. Otherwise, and with HVVR_SETUP_HOST, it is built on the host. */
enum { HVVR_SETUP_DEVICE = 0, HVVR_SETUP_HOST = 1 };

typedef struct hvvr_raycaster hvvr_raycaster;
typedef struct hvvr_camera hvvr_camera;
typedef struct hvvr_model hvvr_model;
typedef struct hvvr_light hvvr_light;
typedef struct hvvr_batch hvvr_batch;
typedef struct hvvr_texture hvvr_texture;

/* ---------------------------------------------------------------- errors */
/* Message of the last failing call on this thread (empty string if none). */
const char* hvvr_last_error(void);
/* Library/ABI version: major*10000 + minor*100 + patch. */
int hvvr_version(void);

/* ---------------------------------------------------------------- raycaster
 * Raycaster(const RayCasterSpecification&) / ~Raycaster (libraries/hvvr/raycaster/raycaster.h:44-45) */
void hvvr_spec_default(hvvr_spec* spec);
int hvvr_raycaster_create(const hvvr_spec* spec, hvvr_raycaster** out);
int hvvr_raycaster_destroy(hvvr_raycaster* rc);
/* setSceneDirty (raycaster.h:62) */
int hvvr_raycaster_set_scene_dirty(hvvr_raycaster* rc);
/* render(double) (raycaster.h:65; libraries/hvvr/raycaster/render.cpp:204-219).
 * stream: a cudaStream_t, or NULL for the raycaster's own stream. Returns after the
 * frame is enqueued; CPU_MEMORY render targets are complete on return. */
int hvvr_raycaster_render(hvvr_raycaster* rc, double elapsed_time, void* stream);
/* waits for all work the raycaster enqueued and reports any device-side status flag */
int hvvr_raycaster_synchronize(hvvr_raycaster* rc);

/* ---------------------------------------------------------------- models
 * createModel(MeshData&&) / destroyModel (raycaster.h:58-60; libraries/hvvr/raycaster/model.cpp:20-21) */
int hvvr_model_create(hvvr_raycaster* rc, const hvvr_mesh_data* mesh, hvvr_model** out);
int hvvr_model_destroy(hvvr_raycaster* rc, hvvr_model* model);
/* Model::setTransform (model.h:47; model.cpp:25-29): marks the scene dirty */
int hvvr_model_set_transform(hvvr_model* model, const hvvr_transform* xf);
/* Replace the model's vertex positions (animation) without rebuilding topology;
 * the next render refits the BVH in place on the device. count must equal the model's vertex count. */
int hvvr_model_update_vertices(hvvr_model* model, const hvvr_shading_vertex* verts, uint32_t count);
/* Device-side animation: copies count vertices from device memory over the model's vertices
 * [first, first+count) on stream (NULL: the raycaster's stream); the next render refits the
 * BVH on the device. The host copy of the mesh is not updated, so a later scene rebuild
 * (adding/removing models or lights) restores the vertices last given on the host.
 * No counterpart in the reference (its Model only has setTransform). */
int hvvr_model_update_vertices_device(hvvr_model* model, uint32_t first, uint32_t count, const void* device_verts,
                                      void* stream);

/* ---------------------------------------------------------------- lights
 * createLight(const LightUnion&) / destroyLight (raycaster.h:55-56) */
int hvvr_light_create(hvvr_raycaster* rc, const hvvr_light_union* light, hvvr_light** out);
int hvvr_light_destroy(hvvr_raycaster* rc, hvvr_light* light);

/* ---------------------------------------------------------------- textures
 * createTexture(const TextureData&) / destroyTexture (raycaster.h:51-52; libraries/hvvr/raycaster/
 * scene.cpp:28-40; texture.cu:201-272). A mipmapped CUDA array with the reference's texture object
 * (normalized coordinates, wrap/wrap addressing, linear and linear-mip filtering, anisotropy 8,
 * sRGB decode for HVVR_TEXTURE_RGBA8_UNORM_SRGB); mip levels of the 8-bit formats come from the
 * reference's generator (texture.cu:78-186), other formats use its four taps stored in their own
 * format. HVVR_TEXTURE_R11G11B10_FLOAT has no CUDA array format and is HVVR_ERR_INVALID.
 * Materials name textures by id (SimpleMaterial::textureIDsAndShadingModel, 0xffff = none): ids
 * count up from 0 per raycaster in creation order and are not reused after a destroy (the
 * reference's ids count over one process-wide atlas). Shading reads an id that names no live
 * texture as no texture. Returns after the texture is complete on the device; data is not
 * retained. Destroy waits for the device to finish the work in flight. */
int hvvr_texture_create(hvvr_raycaster* rc, const hvvr_texture_data* data, hvvr_texture** out);
int hvvr_texture_destroy(hvvr_raycaster* rc, hvvr_texture* texture);
/* Texture::getID (texture.h:44-46) */
int hvvr_texture_get_id(const hvvr_texture* texture, uint32_t* id);
/* parity read-back: mip level `level` (0 = the texels given) as rows of width * element-size
 * bytes; with data NULL only the level's size is returned */
int hvvr_texture_read_level(const hvvr_texture* texture, uint32_t level, void* data, uint64_t capacity,
                            uint32_t* width, uint32_t* height);
/* parity read-back: ReadTexture (libraries/hvvr/raycaster/shading.h:45-47), the tex2DGrad read the
 * shading makes, at count queries q[i] = {u, v, ddx.x, ddx.y, ddy.x, ddy.y}; rgba is [count][4] */
int hvvr_texture_sample(const hvvr_texture* texture, uint32_t count, const float* q, float* rgba);

/* ---------------------------------------------------------------- cameras
 * createCamera(const FloatRect&, float) / destroyCamera (raycaster.h:49-50) and the
 * Camera setters (libraries/hvvr/raycaster/camera.h:70-108) */
int hvvr_camera_create(hvvr_raycaster* rc, const hvvr_float_rect* viewport, float aperture_radius, hvvr_camera** out);
int hvvr_camera_destroy(hvvr_raycaster* rc, hvvr_camera* cam);
int hvvr_camera_set_enabled(hvvr_camera* cam, int enabled);
int hvvr_camera_set_viewport(hvvr_camera* cam, const hvvr_float_rect* viewport);
int hvvr_camera_set_lens(hvvr_camera* cam, const hvvr_thin_lens* lens);
int hvvr_camera_set_aperture(hvvr_camera* cam, float radius);
int hvvr_camera_set_focal_depth(hvvr_camera* cam, float depth);
int hvvr_camera_set_eye_dir(hvvr_camera* cam, const hvvr_vec3* eye_dir);
int hvvr_camera_set_spherical_warp(hvvr_camera* cam, float fov_x_degrees, float fov_y_degrees);
/* setRenderTarget (camera.h:87; camera.cpp:128-133) */
int hvvr_camera_set_render_target(hvvr_camera* cam, const hvvr_image_desc* target);
/* setSamples(const Sample*, count, splitColorSamples in {1,2,3}) (camera.h:88; camera.cpp:135-138) */
int hvvr_camera_set_samples(hvvr_camera* cam, const hvvr_sample* samples, uint32_t count, uint32_t split_color_samples);
/* setCameraToWorld(const transform&) (camera.h:99; camera.cpp:174-176) */
int hvvr_camera_set_camera_to_world(hvvr_camera* cam, const hvvr_transform* xf);
/* Builds the camera's sample setup now (the reference's setSamples builds SampleData at once;
 * otherwise this happens at the camera's first render) and returns when it is on the device.
 * on_host (may be NULL): 1 when the hierarchy was built on the host (see hvvr_spec.sample_setup). */
int hvvr_camera_prepare(hvvr_camera* cam, uint32_t* on_host);
/* MSAA rate in {1,2,4,8,16,32}; the reference fixes it at compile time
 * (libraries/hvvr/raycaster/raycaster_common.h:27). Default 16. */
int hvvr_camera_set_msaa(hvvr_camera* cam, uint32_t rate);
/* The subsample pattern (no counterpart in the reference, which compiles in its spiral,
 * libraries/hvvr/raycaster/gpu_samples.h:23-61): HVVR_MSAA_SPIRAL (default, the reference's) or
 * HVVR_MSAA_ROTATED_GRID, an n-rooks lattice - subsample i in column i and row (k i) mod n of an
 * n x n grid over the sample's [-1, 1]^2 unit offsets (k = 1, 3, 5, 9, 19 for n = 2, 4, 8, 16, 32),
 * scaled by 1/sqrt(2) into the unit disk; at rate 1 the sample's centre. Thin-lens cameras use the
 * spiral whatever the setting (the reference's lens table is built on it). */
enum { HVVR_MSAA_SPIRAL = 0, HVVR_MSAA_ROTATED_GRID = 1 };
int hvvr_camera_set_msaa_pattern(hvvr_camera* cam, uint32_t pattern);
/* getSampleCount (camera.h:95; camera.cpp:162-164): valid (unpadded) sample count */
int hvvr_camera_get_sample_count(const hvvr_camera* cam, uint32_t* count);

/* ---------------------------------------------------------------- parity read-back
 * Intermediate results of the last rendered frame, in sorted-sample order (the order
 * produced by the reference's naiveXYCluster, libraries/hvvr/raycaster/sample_clustering.h:17-49).
 * Sizes: tiles = blocks*64, padded samples = blocks*8192. */
enum { HVVR_CAPTURE_HITS = 1 }; /* record per-subsample hit IDs and depth during render */
int hvvr_camera_set_capture(hvvr_camera* cam, uint32_t flags);
int hvvr_camera_get_layout(const hvvr_camera* cam, uint32_t* block_count, uint32_t* tile_count,
                           uint32_t* padded_sample_count, uint32_t* msaa_rate);
/* Per-tile triangle lists (traverseTiles output, libraries/hvvr/raycaster/traverse_avx.h:412-527):
 * counts[tile_count]; indices concatenated in tile order; *total receives the total entry count.
 * Pass indices=NULL to query the total only. */
int hvvr_camera_read_tile_lists(const hvvr_camera* cam, uint32_t* counts, uint32_t* indices, uint64_t capacity,
                                uint64_t* total);
/* Block cull stacks (traverseBlocks + BlockFrame::sort, traverse_avx.h:293-410):
 * sizes[block_count]; entries[block_count*64] as {float tMin; uint32 mask; uint32 node}. */
int hvvr_camera_read_block_stacks(const hvvr_camera* cam, uint32_t* sizes, uint32_t* entries);
/* Per-subsample hit triangle IDs (~0 = miss) and parametric depth (+inf = miss) along the
 * unnormalised subsample direction; [padded_sample_count * msaa]. Needs HVVR_CAPTURE_HITS. */
int hvvr_camera_read_hits(const hvvr_camera* cam, uint32_t* tri_ids, float* depth);
/* Compressed G-buffer (EmitGBuffer, libraries/hvvr/raycaster/intersect.cu:28-89) rebuilt per sample:
 * for sample s, entries s*msaa .. s*msaa+n-1 hold (tri, mask) pairs sorted by tri, misses last.
 * n[s] is the pair count. Needs HVVR_CAPTURE_HITS. */
int hvvr_camera_read_gbuffer(const hvvr_camera* cam, uint32_t* n, uint32_t* tri, uint32_t* mask);
/* Resolved RGBA8 (sRGB) per sorted sample [padded_sample_count] (ResolveKernel output). */
int hvvr_camera_read_sample_colors(const hvvr_camera* cam, uint32_t* rgba);
/* imageLocationToSampleIndex (camera.cpp:57-63) [width*height*split] */
int hvvr_camera_read_sample_remap(const hvvr_camera* cam, int32_t* remap, uint64_t count);
/* Camera-space beams of the sorted samples, DirectionalBeam {centerRay,du,dv} x padded samples */
int hvvr_camera_read_beams(const hvvr_camera* cam, float* beams9);
/* per-frame timing of the last render, device milliseconds (CUDA events):
 * [0]=scene update/refit, [1]=block cull, [2]=tile cull, [3]=intersect+shade, [4]=remap, [5]=total */
int hvvr_camera_read_timings(const hvvr_camera* cam, float* ms6);
/* total triangle-index entries produced by the last frame's tile cull */
int hvvr_camera_read_list_total(const hvvr_camera* cam, uint64_t* total);
/* Foveated polar mode (spec.mode = HVVR_MODE_FOVEATED_POLAR): the last frame's eye-to-world
 * matrix (column-major), the four world-space tile cull planes {normal, dist}, and the view
 * depth of subsample 0 per polar sample [padded] (the reference's TMaxBuffer). */
int hvvr_camera_read_foveated_frame(const hvvr_camera* cam, float* eye_to_world16, float* cull_planes16,
                                    float* view_depth);
/* Foveated polar mode: the last frame's resolve (Raycaster::renderFoveatedPolarSpaceCudaReconstruct,
 * libraries/hvvr/raycaster/render.cpp:476-486, and GPUCamera::foveatedPolarToScreenSpace,
 * gpu_foveated.cu:335-375) - its sample-to-eye matrix [9] and eye-to-previous-sample-space
 * matrix [16] (column-major), the temporally filtered image it wrote (RGBA8 sRGB,
 * [height * width], the next frame's history) and the previous result it read
 * ([height * width]). Any pointer may be null. The final image goes to the render target. */
int hvvr_camera_read_foveated_resolve(const hvvr_camera* cam, float* sample_to_eye9, float* eye_to_sample_prev16,
                                      uint32_t* result, uint32_t* history);
/* Foveated polar mode: the last frame's polar textures [ring_count][samples_per_ring] - colour
 * (RGBA8 sRGB, RemapPolarFoveatedKernel, remap.cu:127-141), view depth, and the moments
 * (8 x uint16 per texel: first then second moment, RGBA16 unorm; ComputeMoments,
 * gpu_foveated.cu:159-172). Any pointer may be null. */
int hvvr_camera_read_polar_textures(const hvvr_camera* cam, uint32_t* color, float* depth, uint16_t* moments);
/* The per-frame matrices of a foveated camera, on the host (no device work; render.cpp:
 * 463-486): from the camera-to-world transform, gaze, sample bounds and viewport, the
 * eye-to-world matrix [16], the four tile cull planes [16], sample-to-eye [9] and
 * eye-to-previous-sample-space [16]; the history pair (world_to_eye_prev16,
 * eye_prev_to_sample_prev9) is read and then replaced by this frame's. A camera starts from
 * (zero, identity). Column-major. */
int hvvr_foveated_frame_matrices(const hvvr_transform* camera_to_world, const hvvr_vec3* eye_dir,
                                 const hvvr_float_rect* sample_bounds, const hvvr_float_rect* viewport,
                                 float* world_to_eye_prev16, float* eye_prev_to_sample_prev9, float* eye_to_world16,
                                 float* cull_planes16, float* sample_to_eye9, float* eye_to_sample_prev16);
/* BVH nodes visited per tile by the last frame's tile cull [tile_count] (the schedule of the
 * next frame is built from these) */
int hvvr_camera_read_tile_costs(const hvvr_camera* cam, uint32_t* visits);

/* ---------------------------------------------------------------- scene state read-back
 * The refit BVH (GPUSceneState::fetchUpdatedBVH, libraries/hvvr/raycaster/gpu_scene_state.cu:454-467):
 * node_count*32 floats/uints in the 128-byte BVHNode layout (libraries/hvvr/raycaster/bvh_node.h:17-36). */
int hvvr_scene_get_counts(const hvvr_raycaster* rc, uint32_t* node_count, uint32_t* tri_count, uint32_t* vert_count);
int hvvr_scene_read_nodes(hvvr_raycaster* rc, void* nodes128);
/* PrecomputedTriangleIntersect {v0, edge0, edge1} x tri_count (graphics_types.h:203-207) */
int hvvr_scene_read_triangles(hvvr_raycaster* rc, float* tris9);

/* ---------------------------------------------------------------- host utilities
 * GenerateTopology(MeshData&) (libraries/hvvr/shared/bvh.cpp:542-556): SAH BVH2 -> BVH4 -> DFS topology.
 * Reorders tri_shade and verts in place (triangle IDs everywhere are BVH-order IDs) and writes
 * node_count nodes into nodes_out (capacity >= (tri_count+1)/2 + 1). */
int hvvr_generate_topology(hvvr_shading_vertex* verts, uint32_t vert_count, hvvr_tri_shade* tri_shade,
                           uint32_t tri_count, hvvr_topology_node* nodes_out, uint32_t nodes_capacity,
                           uint32_t* node_count);
/* No counterpart in the reference (whose only build is GenerateTopology's host SAH build): a linear
 * BVH built on the GPU in milliseconds - 30-bit Morton codes of the triangle centroids, a stable
 * radix sort, the binary radix tree of the codes, leaves of at most 4 triangles, collapse to 4-wide
 * nodes (leaf slots first) and the depth-first TopologyNode layout. A different topology from
 * hvvr_generate_topology (more node visits and list entries per frame), the same rendered image up
 * to ties between coincident triangles. Reorders tri_shade in place (vertices keep their order) and
 * writes node_count nodes (capacity >= tri_count); host arrays in and out, the build runs on stream
 * of the current device and the call returns when it is done. */
int hvvr_generate_topology_device(const hvvr_shading_vertex* verts, uint32_t vert_count, hvvr_tri_shade* tri_shade,
                                  uint32_t tri_count, hvvr_topology_node* nodes_out, uint32_t nodes_capacity,
                                  uint32_t* node_count, void* stream);
/* getGridSamples(width, height) (libraries/hvvr/raycaster/samples.cpp:21-42) */
int hvvr_grid_samples(uint32_t width, uint32_t height, hvvr_sample* out);

/* ---------------------------------------------------------------- scene and sample files
 * The reference's binary scene files (model_import::loadBin / saveBin,
 * libraries/hvvr/samples_shared/model_import_bin.cpp:15-168): header {version 1, texture,
 * light and mesh counts}; per texture {TextureFormat, width, height, stride} and its texels
 * (getTextureSize, libraries/hvvr/raycaster/texture.h:56-76); the lights; per mesh {transform,
 * vertex, triangle, node and material counts} and those arrays, each record byte-compatible
 * with the types above. A loaded file owns its arrays until hvvr_scene_file_close; a short or
 * malformed file is HVVR_ERR_INVALID. Textures are handed back as bytes, in file order, for
 * hvvr_texture_create (model_import::createObjects creates them first, so their ids are the
 * file's texture indices). */
typedef struct hvvr_scene_file hvvr_scene_file;
int hvvr_scene_file_load(const char* path, hvvr_scene_file** out);
int hvvr_scene_file_counts(const hvvr_scene_file* file, uint32_t* textures, uint32_t* lights, uint32_t* meshes);
/* mesh i as borrowed arrays (valid until close) and its model transform */
int hvvr_scene_file_mesh(const hvvr_scene_file* file, uint32_t i, hvvr_mesh_data* mesh, hvvr_transform* xf);
int hvvr_scene_file_light(const hvvr_scene_file* file, uint32_t i, hvvr_light_union* light);
/* texture i: the reference's TextureFormat value, size, stride in elements and texel bytes */
int hvvr_scene_file_texture(const hvvr_scene_file* file, uint32_t i, uint32_t* format, uint32_t* width,
                            uint32_t* height, uint32_t* stride, const void** texels, uint64_t* bytes);
void hvvr_scene_file_close(hvvr_scene_file* file);
/* writes textures (stride_elements * height texels each), lights and meshes (with their
 * transforms) in the same format (saveBin) */
int hvvr_scene_file_save(const char* path, const hvvr_texture_data* textures, uint32_t texture_count,
                         const hvvr_mesh_data* meshes, const hvvr_transform* transforms, uint32_t mesh_count,
                         const hvvr_light_union* lights, uint32_t light_count);
/* sample files (loadSamples / saveSamples, libraries/hvvr/raycaster/samples.cpp:161-187):
 * {magic 0x0CD1, version 0, reserved, count} then the samples. samples == NULL: count only. */
int hvvr_samples_load(const char* path, hvvr_sample* samples, uint32_t capacity, uint32_t* count);
int hvvr_samples_save(const char* path, const hvvr_sample* samples, uint32_t count);
/* The polar foveated sample set of spec's foveated parameters (spec NULL: defaults), as the
 * reference's polarSpaceFoveatedSetup builds it: getEyeSpacePolarFoveatedSamples
 * (libraries/hvvr/raycaster/samples.cpp:44-142), generateRemapForFoveatedSamples
 * (libraries/hvvr/raycaster/foveated.cpp:19-45) and ComputeEyeSpaceFrusta (frusta.cu:26-118).
 * Host only. Layout first; then beams9[valid*9] eye-space {centerRay, du, dv} in clustered
 * order, remap2[padded*2] polar texel (azimuth, ring) per sample (~0 for padding), and the
 * eye-space tile/block frusta as {origin[4][3], dir[4][3]} (origin at infinity: no samples). */
int hvvr_polar_foveated_layout(const hvvr_spec* spec, uint32_t* samples_per_ring, uint32_t* ring_count,
                               uint32_t* valid, uint32_t* padded);
int hvvr_polar_foveated_samples(const hvvr_spec* spec, float* beams9, uint32_t* remap2, float* tile_rays24,
                                float* block_rays24);

/* ---------------------------------------------------------------- batched frames
 * No counterpart in the reference, whose render() walks the cameras of one scene one at a
 * time. A batch renders the enabled cameras of several raycasters (one scene each, all on one
 * device, all with the same fp_mode) as one frame: each stage is one launch over every view,
 * the tile cull is one persistent work queue over all tiles (longest first after the first
 * frame), and intersect/shade runs once per MSAA rate present. Per view the results are the
 * same as rendering that camera alone (same lists, hit IDs and colours). After the first
 * frame of a layout the frame is replayed from a CUDA graph (config.use_graph). Cameras keep
 * their render targets and read-backs; a camera's tile lists live in the pool of the batch
 * that rendered it last. Destroy batches before their raycasters; a batch whose raycaster
 * was destroyed returns HVVR_ERR_STATE. */
typedef struct {
    uint32_t tile_cull_warps;     /* warps per CTA of the tile-cull work queue: 1 (default), 2, 4 or 8 */
    uint32_t heavy_divisor;       /* 1/heavy_divisor of each rate's tiles (last frame's slowest) are
                                     culled and shaded on their own stream; 0 = no split */
    uint64_t tri_index_capacity;  /* triangle-list pool entries shared by all views */
    uint32_t use_graph;           /* replay frames from a CUDA graph once the layout is stable */
    float frame_ms;               /* autotune result: median device time of a frame */
    uint32_t tile_stack_entries;  /* traversal stack of the main tile-cull pass, 0 (= 256) or 8..256;
                                     tiles that need more are culled again with 4096 entries */
    uint32_t timing;              /* 1: record per-stage and per-launch events (the stage, kernel and
                                     part read-backs); they cost device time (about 0.4 ms of a 6 ms
                                     stereo frame). 0 (default): the frame's start and end only */
    uint32_t pipeline;            /* 1 (default): each part of a pinhole rate class runs its tile cull
                                     and its intersect/shade as one pipeline - a tile is shaded as soon
                                     as its list is complete, while other tiles are still being culled.
                                     0: the cull of a part finishes before its intersect/shade starts */
    uint32_t tile_cull_ctas_per_sm; /* cap on the persistent tile cull's resident CTAs per SM (0 = as many
                                     as fit): leaves room on every SM for other work (the intersect of
                                     finished tiles, another batch's launches) */
    uint32_t tile_cull_persistent; /* 1 (default): the tile cull's warps take tiles from its work queue
                                     until it is empty. 0: each warp culls one tile and its CTA exits,
                                     so the cull's CTAs are short-lived and the GPU's block scheduler
                                     can give their SM slots to work of a higher stream priority
                                     between tiles (a served throughput batch under a latency class) */
    uint32_t stream_tiles;        /* with pipeline: the first stream_tiles tiles of each rate class's
                                     first part (its longest, in last frame's order) publish their
                                     lists chunk by chunk, and their intersect/shade follows the
                                     chunks while the cull is still producing them (default 400).
                                     0: every tile is published when its list is complete. The
                                     images are the same */
} hvvr_batch_config;
void hvvr_batch_config_default(hvvr_batch_config* cfg);
int hvvr_batch_create(hvvr_raycaster* const* raycasters, uint32_t count, const hvvr_batch_config* cfg,
                      hvvr_batch** out);
/* a batch of exactly these cameras (of any raycasters on one device); a destroyed camera
 * leaves the batch */
int hvvr_batch_create_views(hvvr_camera* const* cameras, uint32_t count, const hvvr_batch_config* cfg,
                            hvvr_batch** out);
int hvvr_batch_destroy(hvvr_batch* batch);
/* scene update/refit of every raycaster, then one frame of all their enabled cameras on
 * stream (NULL: the first raycaster's stream); CPU_MEMORY targets are complete on return */
int hvvr_batch_render(hvvr_batch* batch, double elapsed_time, void* stream);
int hvvr_batch_synchronize(hvvr_batch* batch);
int hvvr_batch_get_config(const hvvr_batch* batch, hvvr_batch_config* cfg);
int hvvr_batch_set_config(hvvr_batch* batch, const hvvr_batch_config* cfg);
/* Autotuner: renders `frames` timed frames (after one warm-up) for each tile_cull_warps in
 * {1,2,4,8} x (pipeline 1 with the configured heavy_divisor, or pipeline 0 with heavy_divisor in
 * {0,16,8,4}), keeps the fastest, then sizes the pool to 1.25x the largest list total seen (at
 * least 1M entries). Writes the chosen config to *out. */
int hvvr_batch_autotune(hvvr_batch* batch, uint32_t frames, hvvr_batch_config* out);
/* device ms of the last frame: [0] total; [1] block cull, [2] first tile cull, [3] rest of
 * cull + intersect/shade, [4] remap + copies - stages are 0 unless config.timing is 1 */
int hvvr_batch_read_timings(const hvvr_batch* batch, float* ms5);
/* device ms of the last frame's launches, summed over the launches of the frame (launches on
 * different streams overlap, so the sum can exceed the frame time): [0] tile cull, [1]
 * intersect/shade, [2] block cull, [3] remap. A pipelined class counts the span of its cull and
 * shade as intersect/shade time. Needs config.timing = 1 for that frame. */
int hvvr_batch_read_kernel_times(const hvvr_batch* batch, float* ms4);
int hvvr_raycaster_read_kernel_times(const hvvr_raycaster* rc, float* ms4);
/* the configuration of the batch behind hvvr_raycaster_render (default: hvvr_batch_config_default
 * with the spec's tri_index_capacity) */
int hvvr_raycaster_get_batch_config(hvvr_raycaster* rc, hvvr_batch_config* cfg);
int hvvr_raycaster_set_batch_config(hvvr_raycaster* rc, const hvvr_batch_config* cfg);
/* The last frame's launch timeline per part: rate class r (log2 MSAA, + 6 for thin-lens views,
 * + 12 for pinhole views with the rotated-grid pattern) runs as part 2r (its slowest tiles by the
 * previous frame's cost, on a high-priority stream) and part 2r+1 (the rest).
 * ms108[3 * part + i] = tile cull start, tile cull end, intersect/shade
 * end, in ms from the frame start; -1 for parts that did not run. In a pipelined part
 * (config.pipeline) the tile cull end reads -1 (the cull and the shade overlap).
 * Needs config.timing = 1. */
int hvvr_batch_read_part_times(const hvvr_batch* batch, float* ms108);
int hvvr_raycaster_read_part_times(const hvvr_raycaster* rc, float* ms108);
/* counters of the last frame: [0] list-pool entries taken (whole chunks), [1] tiles culled
 * again with the 4096-entry stack, [2] device status bits, [3] views */
int hvvr_batch_read_stats(const hvvr_batch* batch, uint64_t* out4);
/* The last frame's counters, out[0..count): [0] triangle-list pool entries used (whole chunks),
 * [1] tiles culled again with the 4096-entry stack, [2] status bits, [3] views, [4] list entries
 * that passed the intersect's per-tile tests (frustum planes, ray-origin side, corner-ray
 * barycentrics), [5] (warp of 32 samples, passing entry) pairs whose subsample tests ran (the
 * intersect skips a pair when a depth bound proves that no subsample of the warp can hit the
 * triangle, so [5] x 32 samples x msaa is the number of subsample tests executed, at most
 * [4] x 4 warps); later indices read 0. */
int hvvr_batch_read_counters(const hvvr_batch* batch, uint64_t* out, uint32_t count);
int hvvr_raycaster_read_counters(const hvvr_raycaster* rc, uint64_t* out, uint32_t count);

/* ---------------------------------------------------------------- serving
 * No counterpart in the reference. A server owns one worker thread that renders requests as
 * they arrive over resident scenes (raycasters whose scene is uploaded and refit once, then
 * animated in place). Each request names a view template (sample set + viewport over one
 * scene, clustered once by hvvr_server_add_view), an MSAA rate, a pose and an output image.
 * Admission: a request runs on a camera instance of its template; instances are reused, and a
 * new one is made only while the device memory of all instances plus the slots' triangle-list
 * pools stays within hbm_budget_bytes (idle instances of other templates are freed to make
 * room) - otherwise the request waits. Continuous batching: up to
 * max_batch_views admitted requests form one frame batch on a free slot; `slots` batches are
 * in flight at once on their own streams, so requests that arrive while a batch runs are
 * batched into the next one and overlap with it on the device. A request's image is the same
 * alone and in any mix. While a server exists its raycasters must not be rendered, edited or
 * destroyed by other calls; destroy the server first. */
typedef struct hvvr_server hvvr_server;
typedef struct {
    uint64_t hbm_budget_bytes;    /* view buffers + list pools + framebuffers; default 120 GiB */
    uint32_t slots;               /* batches in flight (1..8, default 2) */
    uint32_t max_batch_views;     /* views per batch (default 64) */
    uint64_t slot_list_capacity;  /* triangle-list pool entries per slot (default 256M) */
    uint32_t tile_cull_warps;     /* as hvvr_batch_config (default 4) */
    uint32_t heavy_divisor;       /* as hvvr_batch_config (default 8) */
    uint32_t min_batch_views;     /* with a batch in flight, wait for this many requests (default 8) ... */
    float max_wait_ms;            /* ... or until the oldest has waited this long (default 2 ms);
                                     an idle GPU takes any request at once */
    uint32_t latency_slots;       /* slots (0..4, default 1) that render only latency-class requests
                                     (hvvr_request.priority 1), at once and on the GPU's highest stream
                                     priority; the `slots` throughput slots then run at its lowest */
    uint32_t tile_cull_ctas_per_sm; /* as hvvr_batch_config, for the throughput slots (default 0; with
                                     latency slots, a cap keeps SMs free for latency-class launches) */
    /* Every stream of the process shares the device's hardware work queues (CUDA_DEVICE_MAX_CONNECTIONS,
     * 8 by default). With fewer queues than busy streams, a latency slot's launches can wait in a
     * queue behind throughput launches whatever their stream priority: set the variable to 32 in
     * the environment before the process first uses CUDA (stereo latency class at 500 req/s,
     * p50/p99: 220/488 ms with 8 queues, 15/28 ms with 32). */
    uint32_t latency_isolation;   /* 1 (default): with latency slots, the throughput slots' frames run
                                     with a non-persistent tile cull and without the cull -> shade
                                     pipeline, so none of their CTAs holds an SM slot for longer than
                                     one tile and none waits on another: each slot a throughput CTA
                                     frees goes to the latency class's launches (highest stream
                                     priority) first. 0: throughput slots keep the batch defaults */
} hvvr_server_config;
typedef struct {
    uint32_t view;                /* from hvvr_server_add_view */
    uint32_t msaa;                /* 1,2,4,8,16,32 */
    hvvr_transform camera_to_world;
    uint32_t memory_type;         /* HVVR_MEMORY_CPU or HVVR_MEMORY_CUDA */
    void* output;                 /* width x height RGBA8 (sRGB) pixels, row stride = width; the
                                     server writes it when the request completes, so it must stay
                                     valid until hvvr_server_poll has returned the completion */
    uint64_t tag;                 /* returned with the completion */
    uint32_t priority;            /* 0: throughput class (batched); 1: latency class (e.g. the eyes of a
                                     stereo frame): dispatched ahead of the throughput class on a
                                     latency slot, never held back to fill a batch */
} hvvr_request;
typedef struct {
    uint64_t id, tag;
    int status;                   /* HVVR_OK, or the error of the batch that rendered it */
    uint32_t batch_views;         /* views in that batch */
    double submit_ms, dispatch_ms, done_ms; /* server clock (ms since creation); done = output ready */
    uint32_t priority;            /* the request's class */
} hvvr_completion;
typedef struct {
    uint64_t submitted, completed, failed, batches, queued, in_flight;
    uint64_t instances, hbm_used, hbm_peak;
    double mean_batch_views;
    uint64_t evicted;             /* idle instances freed to admit other templates */
    double batch_gpu_ms;          /* sum over batches of their device time (first launch to last copy) */
    double dispatch_host_ms;      /* sum over batches of the worker's host time to form and enqueue them */
} hvvr_server_stats;
void hvvr_server_config_default(hvvr_server_config* cfg);
int hvvr_server_create(hvvr_raycaster* const* scenes, uint32_t count, const hvvr_server_config* cfg,
                       hvvr_server** out);
int hvvr_server_destroy(hvvr_server* server);
int hvvr_server_add_view(hvvr_server* server, uint32_t scene, const hvvr_float_rect* viewport,
                         const hvvr_sample* samples, uint32_t count, uint32_t split_color_samples, uint32_t width,
                         uint32_t height, uint32_t* view_id);
/* makes idle camera instances of a view up to `count` ahead of the traffic (allocation stalls
 * the device, so a warm server admits without allocating) */
int hvvr_server_prewarm(hvvr_server* server, uint32_t view, uint32_t count);
int hvvr_server_submit(hvvr_server* server, const hvvr_request* request, uint64_t* id);
/* submits count requests at once (all checked first; none queued if one is refused), so the worker
 * sees them together and can render them in one batch: the two eyes of a stereo frame submitted as
 * one group of latency-class requests go out in one latency batch. ids[i] receives request i's id. */
int hvvr_server_submit_group(hvvr_server* server, const hvvr_request* requests, uint32_t count, uint64_t* ids);
/* moves up to capacity completions out; waits up to wait_ms for the first one */
int hvvr_server_poll(hvvr_server* server, hvvr_completion* out, uint32_t capacity, uint32_t* count, double wait_ms);
/* copies count device vertices (32 B each) now; they replace the model's vertices [first, first+count)
 * between batches, followed by a device refit of the scene */
int hvvr_server_update_vertices(hvvr_server* server, hvvr_model* model, uint32_t first, uint32_t count,
                                const void* device_verts);
int hvvr_server_get_stats(hvvr_server* server, hvvr_server_stats* out);

/* ---------------------------------------------------------------- cull without device allocation
 * No counterpart in the reference. For callers that may not call cudaMalloc: a render thread
 * with a frame deadline (an allocation can synchronise the device), a plugin whose host
 * application owns every device allocation, or code whose device memory all belongs to its own
 * pool. The caller passes device inputs and outputs; the working memory for the per-tile lists
 * is a fixed area compiled into the library (about 31 MiB, present on every GPU that loads the
 * library until the process exits), so one call handles at most 65,536 tiles and 7,864,320
 * list entries and rejects larger work with HVVR_ERR_INVALID / HVVR_ERR_OVERFLOW.
 * Calls share that area: calls whose GPU work overlaps race and must be serialised by the caller.
 * The first call on each device looks up the area's device address; make it before any stream
 * capture begins (the address stays cached until the process exits: do not cudaDeviceReset a
 * device the library uses). Every call is synchronous: it checks the inputs on the device (block
 * sizes at most 64, node indices and child offsets inside node_count; HVVR_ERR_INVALID otherwise)
 * and waits for its own work on the stream to report the status.
 * Output: counts[tile_count] and, when total <= capacity, the lists concatenated in tile order
 * in indices[] - the same lists as hvvr_camera_read_tile_lists for the same frame. */
typedef struct {
    const void* nodes;            /* device: node_count BVH nodes, 128-byte layout, refit bounds */
    uint32_t node_count;
    const void* tile_rays;        /* device: tile_count x {float origin[4][3]; float dir[4][3]}, camera space */
    uint32_t tile_count;          /* positive multiple of 64; tile t belongs to block t/64 */
    const void* block_stacks;     /* device: (tile_count/64) x 64 x {float tMin; uint32_t mask; uint32_t node} */
    const uint32_t* block_sizes;  /* device: tile_count/64 sorted block-stack sizes */
    hvvr_transform camera_to_world;
    uint32_t tile_stack_entries;  /* traversal stack of the main pass, 0 (= 256) or 8..256; tiles that
                                     need more are culled again with 4096 entries (as
                                     hvvr_batch_config.tile_stack_entries) */
} hvvr_tile_cull_args;
int hvvr_tile_cull_static(const hvvr_tile_cull_args* args, uint32_t* counts, uint32_t* indices, uint64_t capacity,
                          uint64_t* total, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HVVR_C_H */
