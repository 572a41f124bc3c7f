/*
 * hpt.h - C ABI of the B200 wavefront path tracer (libhpt.so).
 *
 * The library replaces the OpenCL host driver and kernels of hpTracing:
 *   hp::TraceRunner::TraceRunner(std::unique_ptr<hp::KDTree>&)  src/hp/trace_runner.h:51
 *   hp::TraceRunner::run(...)                                    src/hp/trace_runner.h:53-65
 *   the eleven __kernel functions of                              src/hp/cl_src/kernel.cl
 * and keeps the reference's data formats at the boundary: the 48-byte
 * KDTreeNodeHeader array plus the [count, ids...] leaf list that
 * KDTree::getData() emits (src/hp/scene/kdtree.cpp:248-292), the 96-byte
 * Material record (src/hp/cl_src/types.h.cl:19-34), cl_float3 points and
 * normals padded to 16 bytes, cl_float2 texcoords, cl_int4 triangles
 * (v0, v1, v2, material) and the 256-entry cl_int4 light table
 * (src/hp/scene/base.cpp:160-198).
 *
 * Conventions
 *  - Every entry point returns hpt_status; nothing throws across the ABI.
 *    hpt_last_error() gives a message for the calling thread's last error.
 *  - Host buffers are caller-owned; device memory belongs to the handle
 *    that allocated it and is released by the matching *_destroy call.
 *  - A scene handle owns one CUDA stream; calls on one handle are
 *    serialised by an internal mutex, so a handle may be shared by threads.
 *  - No call falls back to the CPU: without a usable CUDA device every
 *    GPU entry point returns HPT_ERR_CUDA.
 */
#ifndef HPT_H
#define HPT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HPT_VERSION 1000

typedef enum hpt_status {
  HPT_OK = 0,
  HPT_ERR_INVALID_ARGUMENT = 1, /* a NULL pointer, a negative size, ...   */
  HPT_ERR_INVALID_SCENE = 2,    /* buffers that fail validation           */
  HPT_ERR_CUDA = 3,             /* CUDA runtime error or no device        */
  HPT_ERR_OUT_OF_MEMORY = 4,    /* device or admission budget exhausted  */
  HPT_ERR_TRAVERSAL_LIMIT = 5,  /* a bounded device loop hit its cap      */
  HPT_ERR_NOT_FOUND = 6,        /* unknown request / job id               */
  HPT_ERR_IO = 7,               /* file could not be read or parsed       */
  HPT_ERR_CANCELLED = 8,        /* request cancelled or timed out         */
  HPT_ERR_BUSY = 9,             /* request still running                  */
  HPT_ERR_UNSUPPORTED = 10      /* e.g. a texture format we cannot decode */
} hpt_status;

/* ---------------------------------------------------------------------- */
/* Reference record layouts (byte-compatible with src/hp/cl_src/types.h)   */
/* ---------------------------------------------------------------------- */

/* KDTreeNodeHeader, src/hp/cl_src/types.h.cl:36-43 (48 bytes). */
typedef struct hpt_ref_node {
  float box_start[4]; /* cl_float3: x, y, z, pad */
  float box_end[4];
  int32_t child;      /* first child (= own index + 1) or -1 for a leaf   */
  int32_t parent;     /* -1 at the root                                   */
  int32_t sibling;    /* right sibling, set on left children only         */
  int32_t data;       /* offset of [count, ids...] in the leaf list, or -1 */
} hpt_ref_node;

/* Material, src/hp/cl_src/types.h.cl:19-34 (96 bytes). */
typedef struct hpt_ref_material {
  float emission[4];
  float ambient[4];
  float diffuse[4];
  float specular[4];
  float optical_density;
  float dissolve;
  float shininess;
  int32_t diffuse_texture_id;
  int32_t ambient_texture_id;
  float specular_possibility; /* cumulative branch probabilities, */
  float refract_possibility;  /* src/hp/scene/base.cpp:85-93      */
  float diffuse_possibility;
} hpt_ref_material;

/* ---------------------------------------------------------------------- */
/* Errors                                                                  */
/* ---------------------------------------------------------------------- */

const char* hpt_status_string(hpt_status s);
/* Message of the calling thread's most recent failing call ("" if none). */
const char* hpt_last_error(void);
int hpt_version(void);
/* Number of visible CUDA devices (0 when none); never fails. */
int hpt_device_count(void);

/* ---------------------------------------------------------------------- */
/* Host-side producers: OBJ/MTL scene, synthetic scenes, SAH KD-tree      */
/* ---------------------------------------------------------------------- */

typedef struct hpt_mesh hpt_mesh;

/* Views into a mesh's arrays (owned by the mesh). Layouts as in hp::Scene,
 * src/hp/scene/base.h:30-40. */
typedef struct hpt_mesh_arrays {
  const float* points;      int32_t num_points;    /* float4 per vertex   */
  const float* normals;     int32_t num_normals;   /* float4, by vertex id */
  const float* texcoords;   int32_t num_texcoords; /* float2, by vertex id */
  const int32_t* triangles; int32_t num_triangles; /* int4 (v0,v1,v2,mat)  */
  const hpt_ref_material* materials; int32_t num_materials;
  const int32_t* lights;    int32_t num_lights;    /* int4, 256 or 0       */
  const uint8_t* texture_data;                     /* RGBA8 layers          */
  int32_t num_textures;
  const int32_t* texture_dims;                     /* (w, h) per texture    */
  int64_t texture_bytes;
} hpt_mesh_arrays;

/* Loads a Wavefront OBJ (+ MTL) the way hp::Scene::Scene does
 * (src/hp/scene/base.cpp:37-158, parser semantics of the vendored
 * tinyobjloader src/objloader/tiny_obj_loader.cpp:278-723), including the
 * material branch probabilities and the 256-entry light table.
 * Textures: binary/ASCII PPM (P6/P3) are decoded; texture_size > 0
 * resamples (nearest) every texture to texture_size x texture_size (512
 * is the reference's behaviour, base.cpp:31-32, 101-102), 0 keeps each
 * texture at its own size (hpt_mesh_arrays.texture_dims lists them).
 * Other formats return HPT_ERR_UNSUPPORTED unless ignore_textures != 0,
 * in which case every texture becomes a 1x1 mid-grey layer. */
hpt_status hpt_mesh_load_obj(const char* filename, const char* mtl_basepath,
                             int32_t texture_size, int32_t ignore_textures,
                             hpt_mesh** out);

/* Seeded synthetic scenes (no reference counterpart; stand-ins for scenes
 * the reference renders from files):
 *   0 box room (~36 triangles)           1 room + 64 UV spheres (~61k)
 *   2 heightfield + 16 columns (~2.4M)   3 scaled variant of family
 *     `family` with about `target_triangles` triangles (batch jobs).
 * detail scales texture resolution and tessellation (1.0 = nominal). */
typedef struct hpt_gen_params {
  int32_t family;            /* for config 3: 0, 1 or 2                  */
  int32_t target_triangles;  /* for config 3                             */
  int32_t texture_size;      /* 0 = nominal (1024 for 1, 2048 for 2)      */
  int32_t heightfield_n;     /* 0 = nominal 1024 vertices per side        */
  int32_t reserved[4];
} hpt_gen_params;
hpt_status hpt_mesh_generate(int32_t config, uint64_t seed,
                             const hpt_gen_params* params, hpt_mesh** out);

/* Builds a mesh from caller arrays (copied). Material probabilities are
 * recomputed from Ks/Kd/d when recompute_probabilities != 0, and the light
 * table is rebuilt from emissive triangles. */
hpt_status hpt_mesh_create(const hpt_mesh_arrays* arrays,
                           int32_t recompute_probabilities, hpt_mesh** out);
hpt_status hpt_mesh_view(const hpt_mesh* mesh, hpt_mesh_arrays* out);
void hpt_mesh_destroy(hpt_mesh* mesh);

/* Branch probabilities of one material, src/hp/scene/base.cpp:85-93. */
hpt_status hpt_material_probabilities(hpt_ref_material* material);

/* Light table, src/hp/scene/base.cpp:160-198: lights_out receives up to
 * 256 int4 entries; *num_lights is 256, or 0 without emissive triangles. */
hpt_status hpt_light_table(const float* points4, int32_t num_points,
                           const int32_t* triangles4, int32_t num_triangles,
                           const hpt_ref_material* materials,
                           int32_t num_materials, int32_t* lights_out,
                           int32_t* num_lights);

typedef struct hpt_kdtree hpt_kdtree;

/* SAH KD-tree: KDTree::KDTree + KDTree::getData
 * (src/hp/scene/kdtree.cpp:235-246, 248-292), bit-identical output.
 * num_threads <= 0 uses all host cores (the result does not depend on it). */
hpt_status hpt_kdtree_build(const float* points4, int32_t num_points,
                            const int32_t* triangles4, int32_t num_triangles,
                            int32_t num_threads, hpt_kdtree** out);
hpt_status hpt_kdtree_view(const hpt_kdtree* tree, const hpt_ref_node** nodes,
                           int32_t* num_nodes, const int32_t** leaf_data,
                           int32_t* num_leaf_data);
void hpt_kdtree_destroy(hpt_kdtree* tree);

/* ---------------------------------------------------------------------- */
/* Device-resident scene (replaces the TraceRunner constructor uploads,    */
/* src/hp/trace_runner.cpp:41-108)                                         */
/* ---------------------------------------------------------------------- */

typedef struct hpt_scene hpt_scene;

typedef struct hpt_scene_desc {
  const float* points;       int32_t num_points;     /* float4 (x,y,z,pad) */
  const float* normals;      int32_t num_normals;    /* 0 or num_points     */
  const float* texcoords;    int32_t num_texcoords;  /* 0 or num_points     */
  const int32_t* triangles;  int32_t num_triangles;  /* int4                */
  const hpt_ref_node* nodes; int32_t num_nodes;
  const int32_t* leaf_data;  int32_t num_leaf_data;
  const hpt_ref_material* materials; int32_t num_materials;
  const int32_t* lights;     int32_t num_lights;     /* int4               */
  const uint8_t* texture_data;                       /* RGBA8 layers        */
  int32_t num_textures;
  const int32_t* texture_dims; /* (w, h) per layer; NULL = 512 x 512 each */
  int32_t device;              /* CUDA device ordinal                     */
} hpt_scene_desc;

typedef struct hpt_scene_info {
  int32_t num_triangles;
  int32_t num_ref_nodes;
  int32_t num_device_nodes;   /* 8-byte traversal nodes                  */
  int32_t num_leaves;
  int32_t num_leaf_triangles; /* triangle references in leaf order       */
  int32_t max_depth;
  int64_t device_bytes;       /* HBM held by the scene                   */
} hpt_scene_info;

/* Validates every buffer (index ranges, pre-order and rope invariants,
 * finite coordinates) before anything is uploaded. */
hpt_status hpt_scene_create(const hpt_scene_desc* desc, hpt_scene** out);
hpt_status hpt_scene_info_get(const hpt_scene* scene, hpt_scene_info* out);
void hpt_scene_destroy(hpt_scene* scene);

/* ---------------------------------------------------------------------- */
/* Render (replaces TraceRunner::run, src/hp/trace_runner.cpp:116-356)     */
/* ---------------------------------------------------------------------- */

typedef struct hpt_camera {
  float view_p[3];    /* eye position                                    */
  float top_dir[3];   /* "up"; the view direction is cross(top, right)   */
  float right_dir[3];
  float width;        /* image-plane extent along right_dir              */
  float height;       /* extent along top_dir; < 0 selects the           */
                      /* equirectangular panorama (x shift = right_dir.x) */
} hpt_camera;

typedef struct hpt_render_params {
  int32_t sample_x, sample_y;           /* output image size (pixels)    */
  int32_t supersample_x, supersample_y; /* rays per pixel per axis       */
  float background[3];
  int32_t sample;          /* samples per ray (spp), >= 1                */
  int32_t depth;           /* shading passes per sample, >= 1            */
  int32_t disable_diffuse;
  float brightness;
  uint64_t seed;           /* counter-based RNG key                      */
  int32_t first_sample;    /* index of this render's first sample, >= 0 */
                           /* (0 for a whole frame). Renders of samples  */
                           /* [f, f + sample) of one frame trace the     */
                           /* paths one render of all its samples would; */
                           /* their accumulators add up to its (spp     */
                           /* split over GPUs, one reduction).           */
} hpt_render_params;

typedef struct hpt_render_stats {
  int64_t primary_rays;       /* primary intersect queries               */
  int64_t intersect_queries;  /* all intersect queries incl. primary     */
  int64_t shade_calls;        /* hits shaded                             */
  int64_t paths;              /* (primary hit, sample) paths traced      */
  int32_t iterations;         /* wavefront iterations                    */
  int32_t error_flags;        /* device status word (0 = ok)             */
  float ms_total;             /* CUDA-event time of the whole render     */
  float ms_primary;
  float ms_shade;             /* sum over iterations (profile only, else  */
  float ms_intersect;         /* -1; ms_loop covers both)                 */
  float ms_resolve;
  float ms_loop;              /* all wavefront iterations                */
  int64_t nodes_visited;      /* inner nodes descended, all queries      */
  int64_t leaves_visited;
  int64_t triangle_tests;     /* Moller-Trumbore tests run               */
  int64_t triangle_repeats;   /* leaf references skipped as already tested */
} hpt_render_stats;

/* rgba_out: sample_x * sample_y * 4 bytes, layout of get_image
 * (src/hp/cl_src/kernel.cl:615-652, alpha 0). accum_out (nullable):
 * sample_x*supersample_x * sample_y*supersample_y * 3 floats, the
 * per-ray radiance sums before the resolve. */
hpt_status hpt_render(hpt_scene* scene, const hpt_camera* camera,
                      const hpt_render_params* params, uint8_t* rgba_out,
                      float* accum_out);
/* Statistics of the last hpt_render / batch / server call on the scene. */
hpt_status hpt_render_stats_get(const hpt_scene* scene, hpt_render_stats* out);

/* Engine tuning knobs (defaults come from the autotuner cache when set). */
typedef struct hpt_tuning {
  int32_t capacity;          /* paths in flight (wavefront size); a run's */
                             /* queues hold at most its rays x spp paths; */
                             /* default 2^24 (208 B per path)             */
  int32_t isect_block;       /* threads per intersect block (128 / 256)   */
  int32_t shade_block;       /* threads per shade block                   */
  int32_t refill_chunk;      /* lanes idle before a warp refills          */
  int32_t smem_nodes;        /* top-of-tree nodes staged in shared memory */
  int32_t use_graph;         /* capture the bounce loop in a CUDA graph   */
  int32_t profile;           /* time each stage with CUDA events          */
  int32_t isect_min_blocks;  /* register budget: blocks per SM to fit     */
  int32_t trav_steps;        /* 0: one leaf per lane per round; n > 0:    */
                             /* n traversal steps (descent step, leaf     */
                             /* set-up, triangle test or leaf exit) per   */
                             /* lane between refills                      */
  int32_t max_steps;         /* traversal steps one ray may take before   */
                             /* the walk gives up and the render returns  */
                             /* HPT_ERR_TRAVERSAL_LIMIT; 0 = the scene's  */
                             /* cap, 8 x (nodes + leaf references) +      */
                             /* 100000. Larger values are clamped to it.  */
  int32_t shade_min_blocks;  /* register budget of the shading kernel:    */
                             /* 3 or 4 blocks of 256 threads per SM; 0 =  */
                             /* the natural allocation (2 blocks). The    */
                             /* default is 4                              */
} hpt_tuning;
hpt_status hpt_tuning_get(const hpt_scene* scene, hpt_tuning* out);
hpt_status hpt_tuning_set(hpt_scene* scene, const hpt_tuning* in);

/* ---------------------------------------------------------------------- */
/* Stage entry points (one per reference kernel; host arrays in and out).  */
/* Used for per-stage parity and by hosts that run their own loop.         */
/* ---------------------------------------------------------------------- */

/* set_viewdirs / set_viewdirs_vr (src/hp/cl_src/kernel.cl:559-613) with the
 * host arguments of src/hp/trace_runner.cpp:131-150. Writes
 * nx*ny rays, nx = sample_x*supersample_x, ny = sample_y*supersample_y,
 * index = nx*y + x: origin (3 floats) and direction (3 floats). */
hpt_status hpt_raygen(const hpt_camera* camera, int32_t sample_x,
                      int32_t sample_y, int32_t supersample_x,
                      int32_t supersample_y, float* origins,
                      float* directions);

/* kdtree_intersect (src/hp/cl_src/kernel.cl:111-208): closest hit per ray.
 * tri_out: triangle id or -1; t_out: hit distance; u_out, v_out: the
 * Moller-Trumbore coordinates of the winning test (0 on a miss).
 * Differences from the reference: no 512-leaf gather cap (a ray whose line
 * pierces more leaves keeps its true closest hit); a ray aimed exactly at a
 * vertex or edge may report another triangle meeting there at the same t;
 * a zero direction vector is a miss (the reference reports t = +inf). */
hpt_status hpt_intersect(hpt_scene* scene, int32_t n, const float* origins,
                         const float* directions, int32_t* tri_out,
                         float* t_out, float* u_out, float* v_out);

/* s1_run (src/hp/cl_src/kernel.cl:258-409) for n hits. seeds: the 48-bit
 * LCG state each element draws from (updated in place). Outputs:
 *   contrib  3n  radiance added to the ray's accumulator
 *   branch   n   -1 terminated, 0 refract, 1 specular, 2 diffuse, 3 light
 *   hit_p    3n  intersect_p;  normal 3n (not normalised, as reference)
 *   strength 3n  strength after the branch factor
 *   param    n   shininess (specular) or optical density (refract)   */
hpt_status hpt_shade(hpt_scene* scene, int32_t n, const float* origins,
                     const float* directions, const float* strengths,
                     const int32_t* tris, const float* ts, uint64_t* seeds,
                     int32_t disable_diffuse, float* contrib,
                     int32_t* branch, float* hit_p, float* normal,
                     float* strength_out, float* param);

/* s2_refract_run / s2_specular_run / s2_diffuse_run / s2_light_run
 * (src/hp/cl_src/kernel.cl:413-557): next ray of each element.
 * alive_out: 1 if the ray continues (appended to S0), else 0. */
hpt_status hpt_next_dir(hpt_scene* scene, int32_t n, const int32_t* branch,
                        const float* directions, const float* hit_p,
                        const float* normal, const float* strengths,
                        const float* param, uint64_t* seeds,
                        float* origins_out, float* directions_out,
                        float* strength_out, int32_t* alive_out);

/* Stable stream compaction (warp ballot + block scan): out receives the
 * indices i with flags[i] != 0 in increasing order, *count their number.
 * Replaces the atomic_inc appends of kernel.cl (e.g. :188-189). */
hpt_status hpt_compact(const uint32_t* flags, int32_t n, int32_t* out,
                       int32_t* count);

/* No counterpart in the reference. hpt_compact on DEVICE buffers that
 * allocates nothing: for callers that must not allocate device memory
 * mid-stream - cudaMalloc/cudaFree synchronise the whole device, which
 * would stall a stream-ordered pipeline, and a caller that has divided a
 * fixed memory budget among its buffers has none left to give. flags,
 * out and count are device pointers; the work is enqueued on `stream`
 * (a cudaStream_t, NULL = legacy default stream) and the call returns
 * without waiting: *count is valid once the stream reaches that point.
 * The scratch (tile counts, superblock totals, one mask bit per flag:
 * 4.1 MiB) is fixed static device arrays, so n is limited to
 * HPT_COMPACT_NOALLOC_MAX_N flags (larger n: HPT_ERR_INVALID_ARGUMENT,
 * nothing enqueued). The first call on each device looks up those arrays'
 * addresses (set-up, with the device current). Every call shares the one
 * set of arrays: calls whose
 * work overlaps on the GPU (different streams, or host threads) race on it
 * and must be serialised by the caller. Each call overwrites (or zeroes,
 * with cudaMemsetAsync on `stream`) every scratch entry it reads, so no
 * state carries over between calls. The addresses are cached per device:
 * after cudaDeviceReset this entry point must not be called again in the
 * same process. */
#define HPT_COMPACT_NOALLOC_MAX_N (8192 * 4096)
hpt_status hpt_compact_noalloc(const uint32_t* flags, int32_t n,
                               int32_t* out, int32_t* count, void* stream);

/* get_image (src/hp/cl_src/kernel.cl:615-652) over a float accumulator of
 * (sample_x*ssx) x (sample_y*ssy) rays. */
hpt_status hpt_resolve(const float* accum, int32_t sample_x,
                       int32_t sample_y, int32_t supersample_x,
                       int32_t supersample_y, int32_t sample,
                       float brightness, uint8_t* rgba_out);

/* ---------------------------------------------------------------------- */
/* Batching: many jobs in one persistent wavefront (no reference           */
/* counterpart; the reference renders one job per TraceRunner::run call)   */
/* ---------------------------------------------------------------------- */

typedef struct hpt_batch hpt_batch;
hpt_status hpt_batch_create(int32_t device, hpt_batch** out);
/* Queues one job; outputs are written by hpt_batch_run. */
hpt_status hpt_batch_add(hpt_batch* batch, hpt_scene* scene,
                         const hpt_camera* camera,
                         const hpt_render_params* params, uint8_t* rgba_out,
                         float* accum_out, int32_t* job_id);
hpt_status hpt_batch_run(hpt_batch* batch);
hpt_status hpt_batch_stats_get(const hpt_batch* batch, hpt_render_stats* out);
hpt_status hpt_batch_tuning_set(hpt_batch* batch, const hpt_tuning* in);
void hpt_batch_destroy(hpt_batch* batch);

/* ---------------------------------------------------------------------- */
/* Serving: continuous batching of render requests against resident scenes */
/* (no reference counterpart; replaces the GLUT re-render loop of          */
/* src/hptracing.cpp:124-211)                                              */
/* ---------------------------------------------------------------------- */

typedef struct hpt_server hpt_server;

typedef struct hpt_server_config {
  int32_t device;
  int32_t max_jobs;           /* concurrent requests on the GPU           */
  int64_t memory_budget;      /* bytes of per-request device state; mapped */
                              /* at creation and kept for the server      */
  int32_t capacity;           /* paths in flight shared by all requests   */
  int32_t progressive;        /* stream partial accumulations             */
  /* Requests with more paths (rays x spp) than `capacity` keep together at
   * most this percentage of `capacity` in flight, so they cannot crowd out
   * the smaller requests admitted after them (0 or 100 = no cap). */
  int32_t large_inflight_pct;
  /* Wavefront iterations kept queued on the device ahead of the host's
   * slot read-backs (0 = 1; at most 7). */
  int32_t pipeline_depth;
  /* Keep each request's float accumulator for hpt_server_poll's accum_out
   * (costs 12 bytes per ray of device memory and copy-back). */
  int32_t keep_accum;
  /* Overload policy (0 = off). Requests with at most `capacity` paths
   * (rays x spp) are latency-bound: they are granted wavefront capacity
   * first-come first-served ahead of larger ones. Each is admitted when it
   * is predicted to finish within deadline_ms of its submission behind the
   * latency-bound work already admitted (per-scene service times learned
   * from finished requests), waits while it is not, and is shed as soon as
   * it could not finish in time even on an idle wavefront (poll returns
   * HPT_ERR_CANCELLED; hpt_server_shed counts them). Larger requests are
   * never shed. */
  int32_t deadline_ms;
} hpt_server_config;

typedef struct hpt_request_info {
  int32_t state;              /* 0 queued, 1 running, 2 done, 3 failed, 4 cancelled */
  int32_t samples_done;       /* completed samples per ray (progressive)  */
  double submit_ms;           /* host clock, ms since server start        */
  double admit_ms;
  double done_ms;
  int64_t intersect_queries;
  /* Completion the overload policy predicted when it admitted the request
   * (deadline_ms > 0 and a latency-bound request), else -1. */
  double due_ms;
} hpt_request_info;

hpt_status hpt_server_create(const hpt_server_config* config,
                             hpt_server** out);
hpt_status hpt_server_add_scene(hpt_server* server, hpt_scene* scene,
                                int32_t* scene_slot);
/* Copies camera and params; the request runs as soon as it is admitted. */
hpt_status hpt_server_submit(hpt_server* server, int32_t scene_slot,
                             const hpt_camera* camera,
                             const hpt_render_params* params,
                             uint64_t* request_id);
/* Advances the device work (admission, wavefront iterations, completions);
 * returns after at most max_iterations wavefront iterations. */
hpt_status hpt_server_pump(hpt_server* server, int32_t max_iterations);
/* Status of a request; when done, copies the image (and accumulator) out
 * and releases the request. When progressive and running, copies the
 * current partial image if rgba_out is not NULL. */
hpt_status hpt_server_poll(hpt_server* server, uint64_t request_id,
                           hpt_request_info* info, uint8_t* rgba_out,
                           float* accum_out);
hpt_status hpt_server_cancel(hpt_server* server, uint64_t request_id);
/* Ids of requests that finished (done, cancelled or failed) since the
 * previous call, oldest first; at most max_ids, *count of them. Lets a host
 * poll only finished requests. */
hpt_status hpt_server_drain_completed(hpt_server* server, uint64_t* ids,
                                      int32_t max_ids, int32_t* count);
/* Requests queued + running. */
int32_t hpt_server_pending(const hpt_server* server);
/* Requests shed by the overload policy (deadline_ms) since creation. */
int64_t hpt_server_shed(const hpt_server* server);
/* Cumulative device counters of the server's wavefront (intersect queries
 * including primary rays, shade calls, iterations, traversal work); `paths`
 * holds the number of completed requests. */
hpt_status hpt_server_stats_get(hpt_server* server, hpt_render_stats* out);
void hpt_server_destroy(hpt_server* server);

/* ---------------------------------------------------------------------- */
/* Autotuner (no reference counterpart)                                     */
/* ---------------------------------------------------------------------- */

/* Times candidate tunings on a short render of (camera, params), stores
 * the best in the scene and, when cache_path is not NULL, in a text cache
 * keyed by device name and scene shape; a cache hit skips the search. */
hpt_status hpt_autotune(hpt_scene* scene, const hpt_camera* camera,
                        const hpt_render_params* params,
                        const char* cache_path, hpt_tuning* best);

#ifdef __cplusplus
}
#endif

#endif /* HPT_H */
