/*
 * hvvr_oracle.h - TEST INFRASTRUCTURE ONLY.
 *
 * Scalar CPU restatement of the reference's primary-visibility-and-shading path,
 * used as the checker for the CUDA path. Nothing in the product links, loads or
 * calls this library; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg do.
 *
 * Parity pin: tests compare this restatement against the reference's own sources
 * compiled here (oracle/refshim -> oracle/_ref) on committed seeded fixtures.
 */
#ifndef HVVR_ORACLE_H
#define HVVR_ORACLE_H

#include "../include/hvvr_c.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    /* scene: one entry per model (Raycaster::buildScene merges them) */
    uint32_t model_count;
    const hvvr_mesh_data* models;
    const hvvr_transform* model_xf;
    const hvvr_light_union* lights;
    uint32_t light_count;
    /* camera */
    hvvr_float_rect viewport;
    hvvr_thin_lens lens;
    hvvr_transform cam_xf;
    const hvvr_sample* samples;
    uint32_t sample_count;
    uint32_t split_color_samples;
    uint32_t width, height;
    uint32_t msaa;
    uint32_t fp_mode; /* HVVR_FP_FMA or HVVR_FP_STRICT */
    uint32_t threads; /* worker threads for the tile loop (0 = 1) */
    /* material textures: ids below texture_count are live; each texture read (ReadTexture,
     * RC/shading.h:45-47) calls texture_sample(ctx, id, {u, v, ddx.x, ddx.y, ddy.x, ddy.y}, rgba)
     * from any worker thread. texture_count 0: no texture is read. */
    uint32_t texture_count;
    void (*texture_sample)(void* ctx, uint32_t id, const float* q, float* rgba);
    void* texture_ctx;
    uint32_t msaa_pattern;  /* HVVR_MSAA_SPIRAL (the reference's) or HVVR_MSAA_ROTATED_GRID */
} oracle_frame_in;

/* Texture samplers for oracle_frame_in.texture_sample (and the reference harness's texture hook).
 * oracle_texture_hash: a value that depends on every bit of the id and the query, so any
 * difference in a texture coordinate or derivative shows in the colour.
 * oracle_texture_table: a table of sampled values keyed by the exact bits of (id, query); in
 * record mode it collects the queries (and reads zeros), in lookup mode it returns the values
 * set for them and counts the queries it does not hold (which read NaN). */
void oracle_texture_hash(void* ctx, uint32_t id, const float* q, float* rgba);
void oracle_texture_table(void* ctx, uint32_t id, const float* q, float* rgba);
void oracle_texture_table_reset(int record);
/* the recorded queries in a fixed order: ids [n], q [n][6]; returns n (at most capacity written) */
uint32_t oracle_texture_table_queries(uint32_t* ids, float* q, uint32_t capacity);
void oracle_texture_table_set(uint32_t n, const uint32_t* ids, const float* q, const float* rgba);
uint32_t oracle_texture_table_missing(void);

typedef struct {
    /* every pointer may be NULL to skip that output */
    uint32_t* block_sizes;     /* [blocks] */
    uint32_t* block_entries;   /* [blocks*64*3] {tMin bits, mask, node} */
    uint32_t* tile_counts;     /* [tiles] */
    uint32_t* tile_indices;    /* concatenated, capacity entries */
    uint64_t tile_capacity;
    uint64_t tile_total;       /* written */
    uint32_t* hit_ids;         /* [padded*msaa] */
    float* depth;              /* [padded*msaa] */
    double* depth64;           /* [padded*msaa] FP64 ray-triangle depth of the same hit (NaN on miss) */
    uint32_t* gb_n;            /* [padded] */
    uint32_t* gb_tri;          /* [padded*msaa] */
    uint32_t* gb_mask;         /* [padded*msaa] */
    uint32_t* colors;          /* [padded] RGBA8 */
    uint32_t* image;           /* [height*width] RGBA8 */
    int32_t* remap;            /* [height*width*split] */
    float* beams;              /* [padded*9] camera-space DirectionalBeam */
    void* nodes;               /* [node_count*128 bytes] refit BVH */
    float* tris;               /* [tri_count*9] PrecomputedTriangleIntersect */
    float* tile_rays;          /* [tiles*24] camera-space corner rays {origin[4][3], dir[4][3]} */
    uint32_t status;           /* nonzero if a capacity was exceeded */
    float* tmax;               /* [padded] view depth of subsample 0's hit (TMaxBuffer), +inf on a miss */
    float* tile_frusta;        /* [tiles*24] world-space SimpleRayFrustum {origins[4], directions[4]}
                                  (written by the reference harness) */
} oracle_frame_out;

/* The foveated path's frame: given batch-space (eye-space) beams and tile/block frusta, the
 * batch-to-world matrix (column-major 16 floats) and optional world-space cull planes
 * {normal, dist} x 4 (tiles whose frustum lies beyond one plane are culled). Scene, msaa,
 * fp_mode, lens and threads come from in; its samples, viewport and image are not used. */
typedef struct {
    const float* beams;        /* [padded*9] */
    const float* tile_rays;    /* [tiles*24] */
    const float* block_rays;   /* [blocks*24] */
    uint32_t blocks;
    const float* batch_to_world; /* 16 floats */
    const float* cull_planes;  /* 16 floats or NULL */
} oracle_beams_in;

/* sizes for a given sample count: blocks = ceil(n/8192) */
void oracle_layout(uint32_t sample_count, uint32_t* blocks, uint32_t* tiles, uint32_t* padded);
/* merged scene sizes for the given models */
void oracle_scene_counts(const oracle_frame_in* in, uint32_t* nodes, uint32_t* tris, uint32_t* verts);
/* runs the whole frame; returns 0 on success */
int oracle_render(const oracle_frame_in* in, oracle_frame_out* out);
int oracle_render_beams(const oracle_frame_in* in, const oracle_beams_in* beams, oracle_frame_out* out);
/* MSAA unit offsets for rate n (n*2 floats), the spiral pattern of the reference */
void oracle_msaa_offsets(uint32_t n, float* out);
/* the library's n-rooks ("rotated grid") MSAA pattern for rate n (n*2 floats) */
void oracle_msaa_offsets_rotated_grid(uint32_t n, float* out);
/* depth-of-field lens positions for rate n: [4 tiles][n subsamples][128 samples] x 2 floats */
void oracle_lens_table(uint32_t n, float* out);

/* Foveated resolve of one frame: the polar sample colours and view depths to the screen image
 * (RemapPolarFoveated, ComputeMoments, FoveatedPolarToScreenSpace, two eccentricity filter
 * passes and FinishConstrastEnhancement). */
typedef struct {
    float degree_tracking_error, max_fov_degrees, mar_slope, foveal_mar_degrees; /* sample pattern */
    uint32_t samples_per_ring, ring_count, valid;
    const uint32_t* colors;        /* [valid] RGBA8 per sample (clustered order) */
    const float* tmax;             /* [valid] view depth of subsample 0 */
    const uint32_t* remap;         /* [valid * 2] polar texel (azimuth index, ring) */
    uint32_t width, height;
    float sample_to_eye[9];        /* column-major */
    float eye_to_sample_prev[16];  /* column-major */
    const uint32_t* history;       /* [height * width] the previous frame's result (RGBA8 sRGB) */
    uint32_t threads;
} oracle_fov_in;
typedef struct {
    uint32_t* polar_color;         /* [ring_count * samples_per_ring] or null */
    uint16_t* moments;             /* [ring_count * samples_per_ring * 8] (m1 rgba, m2 rgba) or null */
    uint32_t* result;              /* [height * width] this frame's result (the next frame's history) */
    uint32_t* filtered;            /* [height * width] the first filter pass, or null */
    uint32_t* image;               /* [height * width] */
} oracle_fov_out;
int oracle_foveated_resolve(const oracle_fov_in* in, oracle_fov_out* out);

/* The library's device BVH build (hvvr_generate_topology_device), restated: centroids, 30-bit
 * Morton codes over the centroid bounds, a stable sort, the binary radix tree of the sorted codes,
 * leaves of at most 4 triangles, collapse to 4-wide nodes (expanding the child with the most
 * triangles, leaf slots first), depth-first layout. Writes the nodes and the triangles in leaf
 * order (vertices are not reordered); returns 0, or 1 for bad arguments / 2 when capacity is short. */
int oracle_lbvh_build(const hvvr_shading_vertex* verts, uint32_t vert_count, const hvvr_tri_shade* tris,
                      uint32_t tri_count, hvvr_tri_shade* tris_out, hvvr_topology_node* nodes_out,
                      uint32_t capacity, uint32_t* node_count);

#ifdef __cplusplus
}
#endif
#endif
