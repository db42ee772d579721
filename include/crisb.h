/*
 * crisb.h -- C ABI of the B200-native Conditional ReSTIR PT frame loop.
 *
 * This is the drop-in boundary for CrisOptix's per-frame render path.  The
 * reference exposes it as C++ classes bound to OptiX:
 *   Scene(OptixDeviceContext, instances, emitters)   include/model/Scene.h:12-24
 *   Camera(pos, viewDir, up, aspect, fov)             include/graph/Camera.h:24-79
 *   Renderer(w, h, ctx, Camera&, const Scene&)        include/graph/Renderer.h:11-21
 *   Renderer::LaunchFrame(glm::vec3* outputBuffer)    src/Renderer.cpp:209-406
 *   Renderer::GetFrameIdx()                           src/Renderer.cpp:408-411
 *   LaunchParams / RestirParams                       include/graph/LaunchParams.h:11-36,
 *                                                     include/graph/restir/RestirParams.h:11-59
 * Here the same roles are plain C entry points with plain pointers and sizes:
 * opaque handles own all device memory, every call returns a status code
 * (0 = ok, negative = error; nothing throws across the ABI), and the frame is
 * stream-ordered on the caller's CUDA stream with no host synchronisation.
 *
 * Record layouts (crisb_*_rec) are the FP32 storage layout of the device
 * buffers; the debug read-back entry points return them in this layout for
 * either storage mode.
 */
#ifndef CRISB_H
#define CRISB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define CRISB_OK 0
#define CRISB_ERR_INVALID_ARGUMENT (-1)
#define CRISB_ERR_OUT_OF_MEMORY (-2)
#define CRISB_ERR_CUDA (-3)
#define CRISB_ERR_QUEUE_OVERFLOW (-4)
#define CRISB_ERR_DEVICE_TIMEOUT (-5)
#define CRISB_ERR_NOT_SUPPORTED (-6)
#define CRISB_ERR_DEVICE_FAULT (-7)

/* ---- enums (values match the reference's enums) ------------------------ */
/* RendererType, include/graph/restir/settings.h:5-10 */
#define CRISB_RENDERER_PATH_TRACER 0
#define CRISB_RENDERER_RESTIR_PT 1
#define CRISB_RENDERER_CONDITIONAL_RESTIR 2
/* PrefixRadiusType, include/graph/restir/settings.h:15-19 */
#define CRISB_RADIUS_CONSTANT 0
#define CRISB_RADIUS_PATH_LENGTH 1
/* SpecTexUsage, include/model/Material.h:9-13 */
#define CRISB_SPEC_COLOR 0
#define CRISB_SPEC_OCC_ROUGH_METAL 1
/* reservoir / path-record storage (stands in for config.h USE_CUDA_F16) */
#define CRISB_STORAGE_FP32 0
#define CRISB_STORAGE_FP16 1

/* MAX_SPATIAL_NEIGH_COUNT, include/graph/restir/settings.h:24 */
#define CRISB_MAX_SPATIAL_NEIGH 16
/* gatherM is clamped to [1, 32] by the reference UI (src/Renderer.cpp:462) */
#define CRISB_MAX_GATHER_M 32
/* CONFIDENCE_MAX, include/graph/restir/Reservoir.h:6 */
#define CRISB_CONFIDENCE_MAX 50.0f
/* invalid hit marker in crisb_hit_rec.prim */
#define CRISB_INVALID_PRIM 0xFFFFFFFFu

/* ---- scene description ------------------------------------------------- */
/* MaterialSbtData (include/model/Material.h:15-32); its textures are in
 * crisb_scene_desc.material_textures.
 * specular is the reference's specF0 input; with spec_usage == COLOR the
 * reference replaces it by mix(diffuse, specular, 0) = diffuse
 * (shader/brdf.cu:124-138), and this library does the same. */
typedef struct crisb_material {
    float diffuse[3];
    float specular[3];
    float emission[3];
    float roughness;
    int32_t spec_usage;
    int32_t reserved;
} crisb_material;

/* A contiguous triangle range of the scene's triangle array. */
typedef struct crisb_mesh {
    uint32_t first_triangle;
    uint32_t num_triangles;
} crisb_mesh;

/* ModelInstance(model, transform) (include/model/ModelInstance.h:9).
 * transform is row-major 3x4 (object -> world).  material_override >= 0
 * replaces the mesh material for this instance (-1: keep).  Instances are
 * flattened into world-space triangles when the scene is created. */
typedef struct crisb_instance {
    uint32_t mesh;
    int32_t material_override;
    float transform[12];
} crisb_instance;

/* Emitter(mesh, transform, color) (include/model/Emitter.h:57-71): a colour
 * and a run of world-space faces in crisb_scene_desc.emitter_faces. */
typedef struct crisb_emitter {
    float color[3];
    uint32_t first_face;
    uint32_t num_faces;
} crisb_emitter;

/* Texture (src/Texture.cpp:8-75): width * height RGBA8 texels in the order
 * stbi_load(..., STBI_rgb_alpha) returns them (first row first).  Sampled as
 * the reference's texture objects are set up: normalised coordinates, wrap
 * addressing, linear filtering, texels read as c / 255. */
typedef struct crisb_texture {
    const uint8_t* rgba;
    uint32_t width;
    uint32_t height;
} crisb_texture;

typedef struct crisb_scene_desc {
    const float* positions;         /* num_vertices * 3 */
    const float* normals;           /* num_vertices * 3, or NULL (face normals) */
    uint32_t num_vertices;
    const uint32_t* indices;        /* num_triangles * 3 */
    const uint32_t* triangle_material; /* num_triangles */
    uint32_t num_triangles;
    const crisb_material* materials;
    uint32_t num_materials;
    const crisb_mesh* meshes;       /* may be NULL when num_instances == 0 */
    uint32_t num_meshes;
    const crisb_instance* instances; /* NULL/0: triangles are world space */
    uint32_t num_instances;
    const crisb_emitter* emitters;
    uint32_t num_emitters;
    const float* emitter_faces;     /* num_emitter_faces * 9 (v0,v1,v2) */
    uint32_t num_emitter_faces;
    /* Textured materials (MaterialSbtData::{diff,spec,rough}Tex,
     * include/model/Material.h:23-30; sampled in shader/brdf.cu:64-97).  All
     * may be NULL / 0: no textures. */
    const float* uvs;               /* num_vertices * 2 (Vertex::uv), or NULL */
    const crisb_texture* textures;
    uint32_t num_textures;
    const int32_t* material_textures; /* num_materials * 3: diffuse, specular,
                                         roughness texture index or -1 */
    /* Builder of the scene BVH (the OptiX GAS/IAS build of src/Scene.cpp:73-160
     * and src/Mesh.cpp:54-120): CRISB_BVH_DEVICE (0), CRISB_BVH_HOST or
     * CRISB_BVH_DEVICE_WIDE4.  Any builder gives the same hits; only
     * traversal speed differs. */
    uint32_t bvh_builder;
} crisb_scene_desc;

/* crisb_scene_desc.bvh_builder */
#define CRISB_BVH_DEVICE 0 /* on the GPU: Morton order, PLOC clustering, SAH
                              collapse into compressed 8-wide nodes (8-bit child
                              boxes on a per-node grid, 80 bytes); scenes with
                              coordinates of 1.6e7 or more, or a tree deeper than
                              the traversal stack, get CRISB_BVH_DEVICE_WIDE4 */
#define CRISB_BVH_HOST 1   /* on the host: binned SAH, collapsed into 4-wide nodes */
#define CRISB_BVH_DEVICE_WIDE4 2 /* on the GPU as CRISB_BVH_DEVICE, collapsed into
                              4-wide nodes (128 bytes) */

/* ---- camera (Camera, include/graph/Camera.h:24-79) --------------------- */
typedef struct crisb_camera {
    float pos[3];
    float view_dir[3];
    float up[3];
    float aspect;
    float fov;      /* radians, full vertical field of view */
    int32_t changed; /* Camera::HasChanged(): resets frameIdx */
} crisb_camera;

/* CameraData after Camera::GetData (src/Camera.cpp:20-32) */
typedef struct crisb_camera_data {
    float pos[3];
    float u[3];
    float v[3];
    float w[3];
} crisb_camera_data;

/* ---- parameters (RestirParams + LaunchParams knobs) --------------------- */
/* Temporal reprojection: where the temporal passes find a pixel's previous
 * reservoirs (prevPixelCoord, shader/prefix_gen_temp_reuse.cu:130-136).
 * NONE is the reference as it runs: prevPixelCoord = pixelCoord.  VECTORS is
 * the reference's commented-out form, prevPixelCoord = uvec2(pixelCoord + 0.5
 * + motionVectors[pixel]) with caller-supplied vectors
 * (crisb_set_motion_vectors; LaunchParams::motionVectors,
 * include/graph/LaunchParams.h:28), the float -> uint conversion saturating at
 * 0 as on the GPU.  REPROJECT projects the pixel's primary hit through the
 * previous frame's camera (Camera::GetData keeps prevW2V,
 * src/Camera.cpp:22): the pixel whose footprint holds it, none when it is
 * behind that camera or off screen.  In VECTORS and REPROJECT both temporal
 * passes read the previous reservoirs at prevPixelCoord (the reference's
 * prefix pass reads them at pixelCoord, prefix_gen_temp_reuse.cu:41-42,
 * which is the same pixel only under NONE). */
#define CRISB_MOTION_NONE 0
#define CRISB_MOTION_VECTORS 1
#define CRISB_MOTION_REPROJECT 2

typedef struct crisb_params {
    int32_t renderer_type;
    float nee_prob;
    int32_t max_path_len;
    int32_t enable_accum;
    float recon_min_roughness;
    float recon_min_distance;
    int32_t prefix_len;
    int32_t prefix_enable_temporal;
    int32_t prefix_enable_spatial;
    int32_t prefix_spatial_count;
    int32_t prefix_spatial_rounds;
    int32_t suffix_enable_temporal;
    int32_t suffix_enable_spatial;
    int32_t suffix_spatial_count;
    int32_t suffix_spatial_rounds;
    int32_t gather_n;
    int32_t gather_m;
    float gather_radius;
    int32_t gather_radius_type;
    int32_t window_radius; /* WINDOW_RADIUS, include/graph/restir/path_gen.h:12 */
    int32_t storage;       /* CRISB_STORAGE_* */
    int32_t motion_mode;   /* CRISB_MOTION_* (temporal reprojection) */
    uint64_t seed;         /* replaces std::random_device (src/Renderer.cpp:9-11) */
} crisb_params;

/* ---- FP32 record layouts (device storage and debug read-back) ----------- */
/* PackedInteraction (include/graph/Interaction.h:59-86) with the mesh SBT
 * pointer and instance id folded into a global triangle index. */
typedef struct crisb_hit_rec {
    uint32_t prim;      /* CRISB_INVALID_PRIM when !valid */
    float bary[2];
    float in_dir[3];
} crisb_hit_rec;

/* PrefixPath (include/graph/restir/PrefixPath.h:7-41); rng is PCG32::state
 * (the stream increment is always the default stream). */
typedef struct crisb_prefix_rec {
    uint64_t rng;
    crisb_hit_rec primary;
    crisb_hit_rec recon;
    crisb_hit_rec last;
    uint32_t flags; /* 0:8 length, 8:16 reconIdx, bit16 valid, bit17 nee */
    float f[3];
    float post_recon_f[3];
    float p;
    float path_len;
    float recon_out_dir[3];
} crisb_prefix_rec;

/* Reservoir<PrefixPath> (include/graph/restir/Reservoir.h:8-51) */
typedef struct crisb_prefix_res_rec {
    crisb_prefix_rec sample;
    float w_sum;
    float confidence;
    uint32_t pad[2];
} crisb_prefix_res_rec;

/* SuffixPath (include/graph/restir/SuffixPath.h:9-36) */
typedef struct crisb_suffix_rec {
    uint64_t rng;
    crisb_hit_rec recon;
    crisb_hit_rec last_prefix;
    uint32_t flags; /* 0:8 length, 8:16 reconIdx, bit16 valid; 24:32 loop index of the
                       suffix vertex that chose the reconnection vertex (not in the
                       reference's SuffixPath; read by the resampled-path adjoint) */
    float f[3];
    float post_recon_f[3];
    float p;
    float recon_out_dir[3];
    uint32_t pad;
} crisb_suffix_rec;

typedef struct crisb_suffix_res_rec {
    crisb_suffix_rec sample;
    float w_sum;
    float confidence;
} crisb_suffix_res_rec;

/* ---- FP16 reservoir storage (crisb_params.storage == CRISB_STORAGE_FP16) --
 * Reservoirs between passes and frames are packed: colours (f, post-recon f)
 * as IEEE binary16 RGB (round to nearest even; NaN stored as 0, magnitudes
 * saturate at 65504), barycentrics as binary16 (the reference's own F16
 * switch, include/config.h + include/util/f16.h, stores them so), directions
 * (incoming ray direction, reconOutDir) as 16+16-bit octahedral codes with
 * CRISB_OCT_ZERO for the zero vector; random states, flags, pdfs, path length,
 * weights and confidences stay 32-bit.  Canonical (per-frame working)
 * records keep the FP32 layouts above. */
typedef struct crisb_hit16_rec {
    uint32_t prim;
    uint16_t bary[2];
    uint32_t in_dir_oct;
} crisb_hit16_rec;

typedef struct crisb_prefix_res16_rec { /* 80 bytes */
    uint64_t rng;
    uint32_t flags;
    float p;
    float path_len;
    crisb_hit16_rec primary;
    crisb_hit16_rec recon;
    crisb_hit16_rec last;
    uint16_t f[3];
    uint16_t post_recon_f[3];
    uint32_t recon_out_dir_oct;
    float w_sum;
    float confidence;
} crisb_prefix_res16_rec;

typedef struct crisb_suffix_res16_rec { /* 64 bytes */
    uint64_t rng;
    uint32_t flags; /* as crisb_suffix_rec.flags */
    float p;
    crisb_hit16_rec recon;
    crisb_hit16_rec last_prefix;
    uint16_t f[3];
    uint16_t post_recon_f[3];
    uint32_t recon_out_dir_oct;
    float w_sum;
    float confidence;
} crisb_suffix_res16_rec;

#define CRISB_OCT_ZERO 0x80008000u

/* RestirGBuffer (include/graph/restir/RestirGBuffer.h:5-28) */
typedef struct crisb_gbuffer_rec {
    uint64_t rng;
    uint32_t prev_xy;  /* x | y << 16 */
    uint32_t flags;    /* bit0 primaryIntValid */
} crisb_gbuffer_rec;

/* PrefixNeighbor (include/graph/restir/PrefixAccelStruct.h:8-27) */
typedef struct crisb_neighbor_rec {
    uint32_t pixel;
    float dist;
} crisb_neighbor_rec;

/* closest-hit query result (debug / traversal tests) */
typedef struct crisb_trace_hit {
    uint32_t prim;
    float t;
    float u;
    float v;
} crisb_trace_hit;

/* per-pass device time of the last frame (ImGui panel, src/Renderer.cpp:472-485) */
typedef struct crisb_stats {
    float prefix_gen_temp_ms;
    float prefix_spatial_ms;
    float suffix_gen_temp_ms;
    float suffix_spatial_ms;
    float prefix_store_ms;
    float final_gather_ms;
    float total_ms;
    uint32_t kernel_launches;
    /* the same frame by kernel class: path traversal, shift jobs,
     * resampling (MIS / reservoir streaming, neighbour selection), and the
     * prefix-endpoint search (entries, structure build, queries) */
    float trace_ms;
    float shift_ms;
    float resample_ms;
    float search_ms;
    float shade_ms;   /* path-machine shading steps and per-pass finish kernels */
    float other_ms;
    /* rays traced in the frame (crisb_set_timing level 2 only); the shift_*
     * counts are the part traced inside shift jobs (path replays and
     * reconnection visibility) and the number of shift jobs run */
    uint64_t closest_rays;
    uint64_t shadow_rays;
    uint64_t shift_closest_rays;
    uint64_t shift_shadow_rays;
    uint64_t shift_jobs;
    /* traversal work of all rays of the frame: wide-node visits and
     * ray/triangle tests (level 2 only) */
    uint64_t node_visits;
    uint64_t tri_tests;
    /* bytes read and written by the resampling kernels for the work present
     * in the frame, at the stored size of every field they touch (level 2
     * only): prefix combine, suffix temporal combine, suffix spatial
     * selection, suffix spatial combine, final-gather combine (all rounds) */
    uint64_t resample_bytes[5];
} crisb_stats;

/* debug buffer ids for crisb_debug_read */
#define CRISB_BUF_PREFIX_RES_FRONT 0
#define CRISB_BUF_PREFIX_RES_BACK 1
#define CRISB_BUF_CANON_PREFIX 2
#define CRISB_BUF_SUFFIX_RES_FRONT 3
#define CRISB_BUF_SUFFIX_RES_BACK 4
#define CRISB_BUF_CANON_SUFFIX 5
#define CRISB_BUF_GBUFFER 6
#define CRISB_BUF_NEIGHBORS 7      /* W*H*k crisb_neighbor_rec */
#define CRISB_BUF_NEIGHBOR_COUNT 8 /* W*H uint32 (final-gather canonical query) */

typedef struct crisb_scene crisb_scene;
typedef struct crisb_renderer crisb_renderer;

/* ---- entry points -------------------------------------------------------- */
/* Library version string. */
const char* crisb_version(void);

/* Message of the last failing call on this thread. */
int crisb_last_error(char* buf, size_t len);

/* Reference defaults of Renderer::Renderer (src/Renderer.cpp:34-58);
 * reconMinDistance = 0.01 * scene_size. */
int crisb_params_default(crisb_params* out, float scene_size);

/* Camera::GetData (src/Camera.cpp:20-32). */
int crisb_camera_get_data(const crisb_camera* cam, crisb_camera_data* out);

/* Scene::Scene + BuildAccel + BuildEmitterTable (src/Scene.cpp:4-13,73-204):
 * flattens instances, builds the device BVH on the current CUDA device. */
int crisb_scene_create(const crisb_scene_desc* desc, crisb_scene** out);
int crisb_scene_destroy(crisb_scene* scene);
/* Scene::GetSceneSize (src/Scene.cpp:48-71). */
int crisb_scene_size(const crisb_scene* scene, float* out);
/* number of world-space triangles after flattening */
int crisb_scene_num_triangles(const crisb_scene* scene, uint32_t* out);

/* The scene BVH as built (a compressed build can fall back to 4-wide nodes). */
typedef struct crisb_bvh_info {
    uint32_t format;     /* CRISB_BVH_FORMAT_* */
    uint32_t on_device;  /* 1: built on the GPU */
    uint32_t num_nodes;
    uint32_t node_bytes; /* 128 (4-wide) or 80 (compressed 8-wide) */
    int32_t stack_bound; /* traversal stack entries the tree needs */
    int32_t depth;       /* collapse levels (device) or binary depth (host) */
    uint32_t inner_children; /* child slots holding a node */
    uint32_t leaf_children;  /* child slots holding triangles */
} crisb_bvh_info;
#define CRISB_BVH_FORMAT_WIDE4 0
#define CRISB_BVH_FORMAT_COMPRESSED8 1
int crisb_scene_bvh_info(const crisb_scene* scene, crisb_bvh_info* out);
/* read back flattened world-space positions (ntri*9), normals (ntri*9) and
 * materials (ntri) in original triangle order; any pointer may be NULL. */
int crisb_scene_read_triangles(const crisb_scene* scene, float* positions,
                               float* normals, uint32_t* materials);

/* Closest-hit (any_hit == 0) or occlusion (any_hit != 0) query over the
 * scene BVH for n rays given as device arrays; ray k is
 * rays[8k..8k+7] = (ox, oy, oz, tmin, dx, dy, dz, tmax).  Hits are written
 * to the device array hits (occlusion: prim = 1 occluded, 0 free). */
int crisb_trace_rays(const crisb_scene* scene, const float* rays_dev,
                     crisb_trace_hit* hits_dev, uint32_t n, int any_hit,
                     void* stream);

/* Prefix-endpoint neighbour search as one operation: the rebuild of
 * PrefixAccelStruct (src/PrefixAccelStruct.cpp:14-221) over caller-given
 * entries plus the __intersection__prefix_entry query
 * (shader/prefix_search_hit.cu:9-73) for a batch of points.
 * entries_dev: n_entries float4 (x, y, z, radius) in device memory, 16-byte
 * aligned; an entry with radius < 0 (or non-finite) is absent.
 * queries_dev: n_queries float triples.  For query q, out_dev[q*k .. q*k+k)
 * receives the k nearest entries j with |p_j - q| <= radius_j, ordered by
 * (distance, entry index), unused slots zeroed; count_dev[q] their number.
 * k in [1, 31].  out_dev and count_dev must be 4-byte aligned.
 * Scratch comes from the stream-ordered allocator (cudaMallocAsync /
 * cudaFreeAsync on `stream`); the call is asynchronous.  A query that hits
 * the traversal's visit cap or stack depth keeps the neighbours found so far
 * and marks the search error word, which crisb_endpoint_search_status reads
 * (the reference's OptiX query has no such cap and reports nothing). */
int crisb_endpoint_search(const float* entries_dev, uint32_t n_entries,
                          const float* queries_dev, uint32_t n_queries,
                          uint32_t k, crisb_neighbor_rec* out_dev,
                          uint32_t* count_dev, void* stream);

/* Reads and clears the error word of crisb_endpoint_search and
 * crisb_endpoint_search_noalloc for the current CUDA context: synchronises
 * `stream`, then returns CRISB_OK when no query stopped early since the last
 * read, else CRISB_ERR_DEVICE_FAULT (message via crisb_last_error).  Calls no
 * allocator.  The renderer's own searches report through
 * crisb_check_device_errors instead. */
int crisb_endpoint_search_status(void* stream);

/* Test hook: caps the node visits of each standalone search query at
 * max_visits (0 restores the default cap of 2^21).  Process-wide. */
int crisb_endpoint_search_set_visit_cap(uint32_t max_visits);

/* Largest n_entries crisb_endpoint_search_noalloc accepts. */
#define CRISB_NOALLOC_MAX_ENTRIES 32768u

/* The same search as crisb_endpoint_search for callers that must not
 * allocate device memory while they run -- for example an engine that
 * reserves its whole device-memory budget at start-up and forbids allocation
 * during a frame (an allocation can synchronise the device and its latency
 * is unbounded), or a plugin host that gives its plugins no allocator.  It
 * has no counterpart in the reference.  It calls no allocator: its scratch is
 * one static 8 MiB device array in the library, held by every GPU that loads
 * the library until the process exits.  n_entries above
 * CRISB_NOALLOC_MAX_ENTRIES returns CRISB_ERR_INVALID_ARGUMENT.  All calls
 * share that array (it keeps the last call's contents; each call clears what
 * it needs), so calls that overlap on the GPU -- on different streams, or
 * from different host threads -- race and corrupt each other's results:
 * serialise them.  The first call in each CUDA context looks up the array's
 * device address there (cudaGetSymbolAddress) and keeps it for that context
 * (keyed by the context's id, so a context made after cudaDeviceReset, or a
 * caller's own context, does its own lookup); make that first call before
 * any stream capture. */
int crisb_endpoint_search_noalloc(const float* entries_dev, uint32_t n_entries,
                                  const float* queries_dev, uint32_t n_queries,
                                  uint32_t k, crisb_neighbor_rec* out_dev,
                                  uint32_t* count_dev, void* stream);

/* Renderer::Renderer (src/Renderer.cpp:13-200). */
int crisb_renderer_create(const crisb_scene* scene, uint32_t width,
                          uint32_t height, const crisb_params* params,
                          crisb_renderer** out);
int crisb_renderer_destroy(crisb_renderer* r);
int crisb_renderer_set_params(crisb_renderer* r, const crisb_params* params);
int crisb_renderer_get_params(const crisb_renderer* r, crisb_params* out);

/* Renderer::LaunchFrame (src/Renderer.cpp:209-406): one frame of the pass
 * chain on `stream` (a cudaStream_t, NULL = legacy default stream).
 * out_rgb_dev is a caller-owned device buffer of width*height*3 floats,
 * row-major, y down; written in place (blended when enable_accum). */
int crisb_render_frame(crisb_renderer* r, const crisb_camera* cam,
                       float* out_rgb_dev, void* stream);

/* Capacity of the shift machines' job records, in jobs per pixel (default
 * 2; at most the pass's job slots, 2 x max(k, spatial neighbours)).  A pass
 * whose jobs exceed it runs the rest with their rays traced in place: results
 * do not depend on the capacity, only speed and memory do (96 bytes per job
 * of capacity).  Synchronises the device; call between frames.  No
 * counterpart in the reference (its OptiX launches trace in place). */
int crisb_set_job_capacity(crisb_renderer* r, uint32_t jobs_per_pixel);
int crisb_get_job_capacity(const crisb_renderer* r, uint32_t* jobs_per_pixel);

/* Renderer::GetFrameIdx (src/Renderer.cpp:408-411). */
/* Scene material and emitter tables after creation (for parameter updates of
 * inverse rendering; counts must equal those given at creation).  Renderers
 * and adjoint contexts of the scene see the new values from their next call. */
int crisb_scene_get_materials(const crisb_scene* scene, crisb_material* out, uint32_t n);
int crisb_scene_set_materials(crisb_scene* scene, const crisb_material* mats, uint32_t n);
int crisb_scene_set_emitter_colors(crisb_scene* scene, const float* rgb, uint32_t n);

/* Path-replay adjoint (inverse rendering: materials' albedo, roughness and
 * emission, emitters' colour).  The estimator is the path tracer
 * (TraceCompletePath, include/graph/restir/path_gen.h:389-472) with frozen
 * sampling: random decisions, sampled directions and sampling pdfs use the
 * material table copied when the context is made (or at
 * crisb_adjoint_refreeze), BRDF values, emissions and emitter colours use the
 * scene's current tables.  At the frozen parameters it equals the path tracer
 * sample for sample, and it is smooth in the parameters.
 * crisb_adjoint_forward writes one sample per pixel (seed from params.seed and
 * `frame`) into out_rgb_dev (W*H*3 floats).  crisb_adjoint_backward replays the
 * same paths and ADDS dLoss/dparameter, given d_image_dev = dLoss/dimage
 * (W*H*3), into d_materials_dev (7 floats per material: diffuse rgb,
 * roughness, emission rgb) and d_emitters_dev (3 floats per emitter: colour).
 * max_path_len must be <= 16.  No counterpart in the reference, which has no
 * differentiable renderer. */
typedef struct crisb_adjoint crisb_adjoint;
int crisb_adjoint_create(crisb_scene* scene, uint32_t width, uint32_t height, const crisb_params* params,
                         crisb_adjoint** out);
int crisb_adjoint_destroy(crisb_adjoint* a);
int crisb_adjoint_refreeze(crisb_adjoint* a);
int crisb_adjoint_forward(crisb_adjoint* a, const crisb_camera* cam, uint64_t frame, float* out_rgb_dev,
                          void* stream);
int crisb_adjoint_backward(crisb_adjoint* a, const crisb_camera* cam, uint64_t frame, const float* d_image_dev,
                           float* d_materials_dev, float* d_emitters_dev, void* stream);

/* Path-replay adjoint of the resampled estimator: each pixel's selected
 * resampled paths re-traced from their stored seeds.  The estimator is the
 * final gather of the frame `r` rendered last
 * (FinalGatherCanon, shader/final_gather.cu:69-188): per pixel the canonical
 * path and each valid neighbour's suffix shifted onto the canonical prefix,
 * combined with pairwise MIS.  Frozen at the material and emitter tables that
 * frame was rendered with: random decisions, sampled directions, sampling
 * pdfs, path and shift validity, neighbour lists, MIS weights, the
 * neighbours' unbiased contribution weights and the reconnection Jacobians.
 * Evaluated at the scene's current tables: every BRDF value along the paths,
 * emitter colours and emissions.  Each factor is re-traced from stored state
 * (the gather's canonical prefix and suffix, each neighbour sample's seed), no
 * tape.  At the frame's tables it equals the frame's gather value; for any
 * tables it is unbiased for the expected image at those tables as far as the
 * frame's estimator is, so its gradient is an unbiased gradient estimate.
 * crisb_restir_adjoint_enable(r, 1) must precede the frame (each frame then
 * copies the tables it uses: 48 bytes per material, 20 per emitter).
 * crisb_restir_adjoint_forward writes the estimator at the current tables into
 * out_rgb_dev (W*H*3 floats, before any accumulation blend);
 * crisb_restir_adjoint_backward ADDS dLoss/dparameter at the frame's tables,
 * given d_image_dev = dLoss/dimage (W*H*3), into d_materials_dev (7 floats per
 * material: diffuse rgb, roughness, emission rgb) and d_emitters_dev (3 floats
 * per emitter: colour).  Both read the frame's buffers: run them on the
 * frame's stream (or after it) and before the next frame (a
 * crisb_renderer_set_params, crisb_set_job_capacity or crisb_autotune_ex that
 * reallocates the renderer's buffers also ends the frame's adjoint: they
 * return CRISB_ERR_INVALID_ARGUMENT until another frame); the first call
 * allocates width*height*k*16 bytes of scratch (k = gather_m - 1).  Requires
 * CRISB_RENDERER_CONDITIONAL_RESTIR, gather_n 1, FP32 storage, an untextured
 * scene and max_path_len <= 16.  No counterpart in the reference, which has no
 * differentiable renderer. */
int crisb_restir_adjoint_enable(crisb_renderer* r, int on);
int crisb_restir_adjoint_forward(crisb_renderer* r, float* out_rgb_dev, void* stream);
int crisb_restir_adjoint_backward(crisb_renderer* r, const float* d_image_dev, float* d_materials_dev,
                                  float* d_emitters_dev, void* stream);

/* Batched views (many cameras of uneven resolution).  A
 * batch holds renderers of one device -- one per view, each with its own
 * resolution, parameters and storage -- and crisb_batch_render runs one frame
 * of every view as parallel branches of a single CUDA graph launched on
 * `stream`: cams[k] and outs[k] (W*H*3 floats on the device) belong to
 * renderers[k].  Each view's results are those of crisb_render_frame on the
 * same renderer.  The renderers must not be used on other streams while a
 * batch frame runs, and per-kernel timing must be off.  No counterpart in the
 * reference, which renders one view per Renderer::LaunchFrame
 * (src/Renderer.cpp:209-406). */
typedef struct crisb_batch crisb_batch;
int crisb_batch_create(crisb_renderer* const* renderers, uint32_t n, crisb_batch** out);
int crisb_batch_destroy(crisb_batch* b);
int crisb_batch_render(crisb_batch* b, const crisb_camera* cams, float* const* outs, void* stream);

/* ToneMapping (src/kernel/tonemap.cu:7-39, called from src/main.cpp:127): the
 * sRGB transfer curve per channel, clamped to [0, 1] and truncated to 8 bits,
 * from num_pixels float RGB triples to num_pixels byte triples, both on the
 * device, stream-ordered.  The reference then draws the bytes with OpenGL;
 * here the caller keeps them (crisoptix_b200.image writes PNG files).
 * num_pixels = 0 is a no-op (the pointers may then be null). */
int crisb_tonemap_srgb8(const float* rgb_dev, uint8_t* srgb_dev, uint32_t num_pixels, void* stream);

/* Per-pixel motion vectors for CRISB_MOTION_VECTORS: width * height float
 * pairs on the device, read during each crisb_render_frame (NULL clears). */
int crisb_set_motion_vectors(crisb_renderer* r, const float* motion_dev);

/* Tone-map every frame of `r` into srgb_dev (width * height * 3 bytes on the
 * device; NULL stops it): the same kernel as crisb_tonemap_srgb8, run as the
 * last kernel of each crisb_render_frame / crisb_batch_render frame on the
 * frame's stream (inside the frame's CUDA graph).  This is the reference's
 * frame loop, LaunchFrame then ToneMapping (src/main.cpp:122-127). */
int crisb_set_srgb_output(crisb_renderer* r, uint8_t* srgb_dev);

/* The step table crisb_tonemap_srgb8 searches (host memory, no GPU needed):
 * thresholds[k] (k = 1..255) is the smallest float c >= 0 whose byte is at
 * least k, thresholds[0] = 0; *c_max is the largest float with a finite
 * 12.92 c.  A channel's byte is the count of k >= 1 with thresholds[k] <= c
 * for 0 <= c <= c_max, and 0 otherwise (negative, NaN, larger). */
int crisb_srgb8_thresholds(float* thresholds /* 256 */, float* c_max);

/* Launch shape of the traversal kernels: blocks per block resident at once
 * (default 8; results do not depend on it).  crisb_autotune renders `frames`
 * frames of `cam` for each candidate (1, 2, 4, 8, 16) on a scratch renderer of
 * the same scene, size and parameters -- the given renderer's state is left
 * alone -- and keeps the fastest, returned in *chosen.  No counterpart in the
 * reference. */
int crisb_set_trace_grid(crisb_renderer* r, uint32_t blocks_per_resident_block);
int crisb_autotune(crisb_renderer* r, const crisb_camera* cam, uint32_t frames, uint32_t* chosen);

/* Threads per block of the traversal kernels: 64, 128 (default) or 256; each
 * size keeps the same register budget.  Results do not depend on it. */
int crisb_set_trace_block(crisb_renderer* r, uint32_t threads);

/* Launch settings chosen by crisb_autotune_ex, and the frame time they gave. */
typedef struct crisb_tuning {
    uint32_t trace_block;    /* threads per traversal block */
    uint32_t trace_grid;     /* traversal blocks per resident block */
    uint32_t jobs_per_pixel; /* shift-machine job capacity (crisb_set_job_capacity) */
    float frame_ms;          /* the fastest candidate's frame time */
} crisb_tuning;

/* Coordinate descent over the launch settings on a scratch renderer of the
 * same scene, size and parameters (the given renderer's frames are left
 * alone): traversal block size (64, 128, 256), traversal grid (1, 2, 4, 8, 16
 * x the resident blocks), then the job capacity (1, 2, 4, 8 jobs per pixel
 * or every slot: the smallest within 1% of the fastest, as capacity costs
 * memory).  Each candidate renders `frames` frames of `cam`, interleaved with
 * the others.  The choices are applied to the renderer and returned in *out
 * (may be NULL).  Results do not depend on any of them.  No counterpart in
 * the reference. */
int crisb_autotune_ex(crisb_renderer* r, const crisb_camera* cam, uint32_t frames, crisb_tuning* out);

/* The spatial-neighbour count of suffix spatial reuse (suffix_spatial_count,
 * the reference's ImGui knob in src/Renderer.cpp:413-470) picked for a frame
 * budget: candidates 1, 2, 3, 4, 5, 6, 8, 10, 12, 16 in turn, each on a
 * scratch renderer of the same scene, size, parameters and launch settings
 * (4 warm-up frames, then `frames` timed frames of `cam`), until one's mean
 * frame time exceeds budget_ms; the largest count within the budget (the
 * cheapest when none fits) is set on `r` through crisb_renderer_set_params
 * and returned in *chosen, its frame time in *chosen_ms (either may be
 * NULL).  Unlike the launch settings this changes the estimator: more
 * neighbours give lower variance per frame for more time.  Conditional ReSTIR
 * with suffix spatial reuse on only.  No counterpart in the reference. */
int crisb_autotune_spatial(crisb_renderer* r, const crisb_camera* cam, uint32_t frames, float budget_ms,
                           uint32_t* chosen, float* chosen_ms);

/* Frames run as one CUDA graph of the pass chain by default (captured, updated in
 * place and launched on the caller's stream); 0 launches the kernels directly.
 * Frames with per-kernel timing on (crisb_set_timing) always launch directly.
 * Results are identical either way.  No counterpart in the reference, whose
 * LaunchFrame synchronises the device between passes (src/Renderer.cpp:253-405). */
int crisb_set_graph(crisb_renderer* r, int enable);

int crisb_frame_index(const crisb_renderer* r, uint64_t* out);
/* per-frame random value the last frame used (params.random) */
int crisb_frame_random(const crisb_renderer* r, uint32_t* out);

/* Per-pass CUDA-event timing: 0 off, 1 events on the stream, 2 events plus
 * ray counters (atomics in the traversal, for statistics runs). */
int crisb_set_timing(crisb_renderer* r, int enable);
/* Per-pass times of the last frame; synchronises on its stop event. */
int crisb_get_stats(crisb_renderer* r, crisb_stats* out);

/* Device error word (traversal stack overflow, kNN overflow, ...); reading
 * synchronises the renderer's last stream.  Returns CRISB_OK or the error. */
int crisb_check_device_errors(crisb_renderer* r);

/* Copy an internal buffer (CRISB_BUF_*) to host memory in the FP32 record
 * layout.  bytes must equal the buffer size; synchronises the device. */
int crisb_debug_read(crisb_renderer* r, int buffer_id, void* host_dst,
                     size_t bytes);
/* Size in bytes of an internal buffer in the FP32 record layout. */
int crisb_debug_size(const crisb_renderer* r, int buffer_id, size_t* out);

/* sizeof of every public struct, in declaration order (material, mesh,
 * instance, emitter, scene_desc, camera, camera_data, params, hit_rec,
 * prefix_rec, prefix_res_rec, suffix_rec, suffix_res_rec, gbuffer_rec,
 * neighbor_rec, trace_hit, stats) -- lets bindings check their layouts.
 * Writes up to n values; returns the number of structs. */
int crisb_abi_sizes(uint32_t* out, uint32_t n);

/* Test hook: evaluates the library's device implementation of one unit-level
 * function of the reference on n packed records in device memory (record
 * layouts and function ids as in the project's oracle/kat.h: SampleTEA64,
 * PCG32 seeding and draws, GetLuminance, the two pairwise MIS weights,
 * SelectSpatialNeighbor, CalcReconnectionJacobian, Reservoir::Update +
 * FinalizeGRIS, D_GGX / V_SmithJointGGX / FresnelSchlick, SpawnCameraRay),
 * so tests can hold them to known answers of the reference's own code.
 * PCG32 records outside the default stream are answered with all words set
 * (the library's generator runs the default stream only, as the reference
 * uses it).  Asynchronous on `stream`. */
int crisb_selftest_kat(int fn, const void* in_dev, uint32_t n, void* out_dev,
                       void* stream);

/* Test hook: the library's radix sort of the prefix-endpoint keys on its own
 * (the per-frame structure rebuild uses it, replacing the OptiX GAS rebuild of
 * src/PrefixAccelStruct.cpp:66-221): out_dev = in_dev's n keys sorted stably
 * by their high 32 bits; temp_dev holds crisb_selftest_sort_temp_bytes(n)
 * bytes.  Asynchronous on `stream`. */
int crisb_selftest_sort(const uint64_t* in_dev, uint64_t* out_dev, uint32_t n,
                        void* temp_dev, size_t temp_bytes, void* stream);
size_t crisb_selftest_sort_temp_bytes(uint32_t n);

#ifdef __cplusplus
}
#endif

#endif /* CRISB_H */
