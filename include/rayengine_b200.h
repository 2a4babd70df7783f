/*
 * rayengine_b200.h -- C ABI of the B200-native RayEngine ray-query path.
 *
 * Plain C types only (no CUDA or torch types): device buffers are passed as
 * raw pointers to device memory, streams as an opaque `void*` holding a
 * cudaStream_t (NULL = legacy default stream).  Every entry point returns a
 * re_status; nothing calls exit().  The last error message of the calling
 * thread is available from re_last_error().
 *
 * Reference interface each entry replaces (hadalhw17/RayEngine, paths
 * relative to its repository root, "RE/" = RayEngine/src/):
 *
 *   re_scene_create / re_scene_create_packed
 *       RKDTreeCPU::RKDTreeCPU + RKDThreeGPU::RKDThreeGPU + RTScene
 *       init_triangles + copy_memory
 *       (RE/Primitives/KDTree.cpp:117-173, RE/Primitives/KDThreeGPU.cpp:9-54,
 *        RE/World/RTScene.cpp:210-285, RE/cuda-src/cuda_memory_functions.cuh:58-211)
 *   re_scene_destroy          free of the copy_memory buffers (no reference free)
 *   re_trace_primary          trace_primary_rays kernel launch in cuda_render_frame
 *                             (RE/cuda-src/renderer.cu:390-410, :705-709)
 *   re_trace_rays             trace_scene / trace_shadow on caller rays
 *                             (RE/cuda-src/ray_functions.cuh:366-396)
 *   re_render_ao              primary + shade()/trace_shadow shadow ray + hemisphere
 *                             rays of trace_secondary_shadow_rays
 *                             (RE/cuda-src/material_functions.cuh:99-119,
 *                              RE/cuda-src/renderer.cu:537-613)
 *   re_perlin_permutation     RPerlinNoise::RPerlinNoise (RE/World/PerlinNoise.h:16-52)
 *   re_noise_fbm              eval / terrain fBm (RE/cuda-src/sdf_functions.cuh:84-206)
 *   re_heightfield            generate_noise bake kernel (RE/cuda-src/renderer.cu:106-126,
 *                             :813-836) producing a height grid
 *   re_sdf_trace              render_sphere_trace's march
 *                             (RE/cuda-src/renderer.cu:143-235,
 *                              RE/cuda-src/sphere_tracing.cuh:183-216)
 */
#ifndef RAYENGINE_B200_H
#define RAYENGINE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RE_API __attribute__((visibility("default")))
/* 2: re_nsdf_trace_params gained the cone tracer's fields and root_tol;
 *    re_tuning.ray_lanes accepts 32 (the warp-cooperative walk) */
#define RE_ABI_VERSION 2

typedef enum re_status {
  RE_OK = 0,
  RE_ERR_INVALID_ARG = 1,   /* null pointer, zero size, bad flag           */
  RE_ERR_CUDA = 2,          /* a CUDA runtime call or launch failed        */
  RE_ERR_OUT_OF_MEMORY = 3, /* device or host allocation failed            */
  RE_ERR_LIMIT = 4,         /* a size exceeds a documented maximum         */
  RE_ERR_NO_DEVICE = 5,     /* no CUDA device / library built without one  */
  RE_ERR_INTERNAL = 6
} re_status;

/* Same field order and size (88 bytes) as the reference's RCamera
 * (RE/Primitives/Camera.h:7-16).  generate_ray reads campos, view, camdown,
 * fov (full angles in degrees) and focial_distance. */
typedef struct re_camera {
  float campos[3], camdir[3], camright[3], camdown[3], lookat[3], view[3];
  float fov[2];
  float focial_distance, apertude_radius;
} re_camera;

/* Closest-hit record, 16 bytes: triangle index in the caller's face order
 * (-1 = miss), ray parameter t (1e20 on a miss) and barycentrics u, v. */
typedef struct re_hit {
  int32_t id;
  float t, u, v;
} re_hit;

/* A ray, 32 bytes: origin, maximum t, unit direction, caller tag. */
typedef struct re_ray {
  float o[3];
  float tmax;
  float d[3];
  uint32_t tag;
} re_ray;

/* kd-tree build parameters (defaults from re_kd_params_default). */
typedef struct re_kd_params {
  uint32_t max_depth;      /* 40 (<= 64)                          */
  uint32_t leaf_size;      /* 2: nodes above this size are split  */
  float cost_traversal;    /* SAH cost of one inner-node step (1) */
  float cost_intersect;    /* SAH cost of one triangle test (2)   */
  float empty_bonus;       /* SAH discount for an empty child (0.1) */
  uint32_t bfs_levels;     /* top levels laid out breadth-first   */
  uint32_t threads;        /* host build threads, 0 = all         */
  uint32_t max_leaf_visits;/* per-ray traversal bound (16384); a ray that
                              reaches it stops and is reported: see
                              re_scene_truncated and the AO mask bit 6
                              (the reference stops at 50 leaves without
                              a report, ray_functions.cuh:284)           */
} re_kd_params;

typedef struct re_scene re_scene;

/* Launch tuning of a scene (see re_autotune_ao, re_autotune_primary). */
typedef struct re_tuning {
  uint32_t stage_nodes;      /* top nodes staged in shared memory per block (<= 8192) */
  uint32_t queue_kind_major; /* secondary-ray queue: 0 pixel-major, 1 kind-major,
                                2 shadow rays first, then each pixel's AO rays    */
  uint32_t refill_min;       /* idle lanes before a warp claims new secondary rays, 1..32 */
  uint32_t ray_refill_min;   /* the same for primary and caller rays (re_trace_primary,
                                re_count_primary, re_trace_rays), 1..32; 32 (default):
                                each lane runs its ray to the end, no refill */
  uint32_t ray_lanes;        /* lanes per primary ray in re_trace_primary: 1 (default; 0
                                reads as 1), 2, 4 or 8.  Above 1 the lanes of a ray split
                                each leaf's triangle tests (same hits); it shortens the
                                longest walks of frames too small to fill the GPU.  32:
                                one ray per lane, and the warp tests the triangles of all
                                its lanes' leaves together (finished lanes help; same
                                hits) */
} re_tuning;

typedef struct re_scene_stats {
  uint32_t num_tris, num_nodes, num_leaves, num_refs;
  uint32_t max_depth, max_leaf_size, bfs_nodes, pad;
  float bmin[3], bmax[3];
  double build_seconds;
  uint64_t device_bytes;
} re_scene_stats;

/* Trace flags. */
#define RE_TRACE_TWO_SIDED 0u /* KDTree.cpp:909-949 test (default) */
#define RE_TRACE_ONE_SIDED 1u /* ray_functions.cuh:174-223 test     */
#define RE_TRACE_ANY_HIT 2u   /* stop at the first hit (shadow)     */

RE_API int re_abi_version(void);
RE_API const char* re_status_string(re_status s);
RE_API const char* re_last_error(void);
RE_API void re_kd_params_default(re_kd_params* p);

/* Indexed mesh: verts = num_verts x 3 floats, faces = num_faces x 3 indices.
 * Builds the SAH kd-tree with ropes on the host, flattens it and uploads it
 * to the current device.  The mesh arrays are read only during the call. */
RE_API re_status re_scene_create(const float* verts, uint32_t num_verts,
                                 const uint32_t* faces, uint32_t num_faces,
                                 const re_kd_params* params, re_scene** out);
/* The reference's packed triangles (RTScene.cpp:239-241): per triangle
 * 12 floats {v0.xyz,0, e1.xyz,0, e2.xyz,0} with e = v - v0. */
RE_API re_status re_scene_create_packed(const float* tris, uint32_t num_tris,
                                        const re_kd_params* params,
                                        re_scene** out);
/* Host-only build of the same tree (no device upload): stats and export
 * work, trace calls return RE_ERR_NO_DEVICE.  Lets a caller without a GPU
 * inspect or serialise the tree. */
RE_API re_status re_scene_build_host(const float* tris, uint32_t num_tris,
                                     const re_kd_params* params, re_scene** out);
RE_API re_status re_scene_stats_get(const re_scene* s, re_scene_stats* out);
/* Copies the flattened host arrays (for checking): nodes 2 words each,
 * leaves 16 words each, triangle references 12 words each.  Any pointer may
 * be NULL; sizes come from re_scene_stats. */
RE_API re_status re_scene_export(const re_scene* s, uint32_t* nodes,
                                 uint32_t* leaves, float* tris);
/* The entry table (for checking): *res = cells per face side; when out is
 * not NULL it receives 6 * res * res start nodes, entry (k, side, i, j) at
 * ((k * 2 + side) * res + i) * res + j for the face of axis k (side 0: -k,
 * 1: +k), cell i along the face's lower other axis and j along the higher.
 * Each is the deepest node whose region holds the cell grown by 1e-4 x the
 * scene box's largest extent; primary and caller rays that enter the box
 * through a cell start their first descent there (the counting calls start
 * at the root). */
RE_API re_status re_scene_export_entry(const re_scene* s, uint32_t* out, uint32_t* res);
RE_API re_status re_scene_destroy(re_scene* s);

/* Primary rays for every pixel of a w x h image (row-major, d_out has w*h
 * entries).  flags: RE_TRACE_TWO_SIDED or RE_TRACE_ONE_SIDED. */
RE_API re_status re_trace_primary(re_scene* s, const re_camera* cam,
                                  uint32_t w, uint32_t h, uint32_t flags,
                                  re_hit* d_out, void* stream);
/* Caller rays (device array of n re_ray). */
RE_API re_status re_trace_rays(re_scene* s, const re_ray* d_rays, uint32_t n,
                               uint32_t flags, re_hit* d_out, void* stream);

/* Rays of the last trace call on this scene that stopped at the leaf-visit
 * cap (re_kd_params.max_leaf_visits), copied to *d_count (device memory) on
 * `stream`.  Counted by re_trace_primary, re_count_primary, re_trace_rays,
 * re_render_ao (both passes: the count covers the frame), re_render_frame;
 * each of those calls clears it first.  Per ray: re_count_primary's status
 * word (1 = stopped at the cap) and the AO mask bit 6.  Replaces the
 * reference's silent cut-off (stackless_kdtree_traversal's
 * `limit < 50`, ray_functions.cuh:284). */
RE_API re_status re_scene_truncated(const re_scene* s, uint32_t* d_count, void* stream);

/* Per-pixel work counters of a primary-ray pass (device array of w*h
 * uint4: inner-node steps, leaf visits, triangle tests, status).  Used to
 * compute the algorithmic bytes of a pass. */
RE_API re_status re_count_primary(re_scene* s, const re_camera* cam,
                                  uint32_t w, uint32_t h, uint32_t flags,
                                  uint32_t* d_counts, void* stream);

/* Primary + shadow + ambient-occlusion frame.
 *   d_primary: w*h re_hit (closest hit, two-sided)
 *   d_mask:    w*h uint32, bit0 primary hit, bit1 shadow ray unoccluded,
 *              bits 2..5 AO ray j unoccluded, bit6 one of the pixel's rays
 *              stopped at the leaf-visit cap (its result covers only the
 *              leaves it reached).
 * Secondary rays start at hit + n * bias (n = geometric normal facing the
 * ray); the shadow ray goes along light_dir without bound, the four
 * cosine-weighted AO rays are ao_length long.  The secondary-ray queue is
 * owned by the scene and grown on demand (5 rays per pixel). */
typedef struct re_ao_params {
  float light_dir[3]; /* unit vector */
  float ao_length;
  float bias;
  uint32_t seed;
} re_ao_params;
RE_API re_status re_render_ao(re_scene* s, const re_camera* cam, uint32_t w,
                              uint32_t h, const re_ao_params* p,
                              re_hit* d_primary, uint32_t* d_mask,
                              uint32_t* d_num_secondary, void* stream);
/* The two passes of re_render_ao as separate calls (same results), so a
 * caller can time or overlap them: the primary pass writes d_primary and
 * d_mask and fills the scene's secondary-ray queue, the secondary pass
 * traces that queue into d_mask. */
RE_API re_status re_render_ao_primary(re_scene* s, const re_camera* cam,
                                      uint32_t w, uint32_t h,
                                      const re_ao_params* p, re_hit* d_primary,
                                      uint32_t* d_mask, void* stream);
RE_API re_status re_render_ao_secondary(re_scene* s, uint32_t* d_mask,
                                        uint32_t* d_num_secondary,
                                        void* stream);
/* re_render_ao without any device allocation during the call.
 *
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory while they render: an engine that reserves all device memory at
 * start-up through its own pool, or a frame loop that cannot afford
 * cudaMalloc's implicit synchronisation or an out-of-memory failure in the
 * middle of a frame.  re_render_ao grows its secondary-ray queue with
 * cudaMalloc on first use; this entry point instead keeps the queue in a
 * fixed array inside the library (RE_NOALLOC_SCRATCH_BYTES on every GPU that
 * loads the library, held until the process exits).  Inputs, outputs and the
 * scene are the caller's, exactly as for re_render_ao, and the results are
 * identical.
 *   - w * h must not exceed RE_NOALLOC_MAX_PIXELS (5 secondary rays of 32
 *     bytes per pixel); larger images return RE_ERR_LIMIT without launching.
 *   - Every call looks up the array's device address on the current device
 *     (cudaGetSymbolAddress, which allocates nothing), so the entry point
 *     stays valid after a device reset; the first call on a device may also
 *     load the library's device code, so make that first call before any
 *     stream capture.
 *   - Every call on a device shares the one array: calls that overlap on the
 *     GPU (other streams, other threads) race and must be serialised by the
 *     caller. */
#define RE_NOALLOC_MAX_PIXELS 419430u
#define RE_NOALLOC_SCRATCH_BYTES (256u + 160u * RE_NOALLOC_MAX_PIXELS)
RE_API re_status re_render_ao_noalloc(re_scene* s, const re_camera* cam,
                                      uint32_t w, uint32_t h,
                                      const re_ao_params* p, re_hit* d_primary,
                                      uint32_t* d_mask,
                                      uint32_t* d_num_secondary, void* stream);
/* Autotuner: times the AO frame for each combination of shared-memory
 * staging depth, queue layout and refill threshold (one warm-up and three
 * timed frames each, CUDA events on `stream`), keeps the fastest on the
 * scene and returns it with its frame time.  Allocates temporary output
 * buffers: call at set-up, not in a frame loop. */
RE_API re_status re_autotune_ao(re_scene* s, const re_camera* cam, uint32_t w,
                                uint32_t h, const re_ao_params* p,
                                re_tuning* best, float* best_ms, void* stream);
/* Autotuner of the primary pass: times re_trace_primary(flags) for each
 * combination of staging depth, ray_refill_min and ray_lanes and keeps the
 * fastest (other fields unchanged).  Each timed pass follows a write of twice
 * the L2 size (a frame whose tree is not cached).  Set-up time only: it
 * allocates that scratch and its own output. */
RE_API re_status re_autotune_primary(re_scene* s, const re_camera* cam, uint32_t w,
                                     uint32_t h, uint32_t flags, re_tuning* best,
                                     float* best_ms, void* stream);
RE_API re_status re_scene_get_tuning(const re_scene* s, re_tuning* out);
RE_API re_status re_scene_set_tuning(re_scene* s, const re_tuning* t);
/* Work counters of the same frame (device array of 8 uint64): primary
 * inner-node steps, leaf visits, triangle tests, rays; then the same four
 * for the secondary rays.  Used for the algorithmic bytes of each pass. */
RE_API re_status re_render_ao_counts(re_scene* s, const re_camera* cam,
                                     uint32_t w, uint32_t h,
                                     const re_ao_params* p, uint64_t* d_totals,
                                     void* stream);

/* ---- noise -------------------------------------------------------- */
/* RPerlinNoise(seed).permutationTable: 512 entries (256 duplicated). */
RE_API re_status re_perlin_permutation(uint32_t seed, uint32_t* out512);

typedef struct re_fbm_params {
  uint32_t seed;     /* permutation table seed (RPerlinNoise default 2016) */
  uint32_t octaves;
  float lacunarity;  /* 2.0 */
  float gain;        /* 0.5 */
  float scale;       /* input scale applied before octave 0 */
  float amplitude;   /* output scale */
} re_fbm_params;
/* d_pts: n x 3 floats; d_out[i] = amplitude * fbm(scale * p_i). */
RE_API re_status re_noise_fbm(const re_fbm_params* p, const float* d_pts,
                              uint32_t n, float* d_out, void* stream);
/* Height grid of (cells+1)^2 vertices over [lo,hi]^2 (x fastest), written as
 * xyz floats with y = amplitude * fbm(x, 0, z) (lacunarity/gain from p). */
RE_API re_status re_heightfield(const re_fbm_params* p, uint32_t cells,
                                float lo, float hi, float* d_verts,
                                void* stream);
/* Host helpers that generate the synthetic scenes. */
RE_API re_status re_gen_soup(uint64_t seed, uint32_t n, float* verts);
RE_API re_status re_gen_grid_faces(uint32_t cells, uint32_t* faces);

/* ---- exact-SDF sphere tracing ---------------------------------------- */
typedef struct re_sdf_params {
  uint32_t seed;       /* permutation table seed                     */
  uint32_t octaves;    /* 8                                         */
  float scale;         /* 0.25: d(p) = p.y - amplitude*fbm(scale*p) */
  float amplitude;     /* 3                                         */
  float step_factor;   /* 0.6                                       */
  float eps;           /* 1e-4                                      */
  float tmax;          /* 200                                       */
  uint32_t max_steps;  /* 512                                       */
} re_sdf_params;

/* 32 bytes per pixel: hit position, unit normal (central differences),
 * number of field evaluations of the march, status (1 hit, 0 left the
 * [0,tmax] range, 2 step bound reached). */
typedef struct re_sdf_hit {
  float pos[3];
  float normal[3];
  uint32_t steps;
  uint32_t status;
} re_sdf_hit;

RE_API re_status re_sdf_trace(const re_sdf_params* p, const re_camera* cam,
                              uint32_t w, uint32_t h, re_sdf_hit* d_out,
                              void* stream);

/* ---- shaded SDF terrain frame ----------------------------------------
 * The reference's live render path: with `sphere_tracing` defined
 * (RE/RayEngine/RayEngine.h:22) cuda_render_frame (renderer.cu:702-738)
 * runs render_sphere_trace (renderer.cu:143-285): march, shade
 * (paint_surface and the soft-shadowed light of sphere_trace_shadow,
 * sphere_tracing.cuh:246-273,322-360,408-477), atmosphere sky for misses
 * (compute_incident_light, material_functions.cuh:296-344), fog, gamma,
 * vignetting, rgbaFloatToInt (cuda_helper_functions.h:61-68).  Here the
 * terrain is the exact field of re_sdf_params, traced by re_sdf_trace.
 * Output: W x H packed RGBA8 (R in the low byte, alpha 255). */
#define RE_SDF_SHADE 1u      /* soft shadow + light terms (the reference's should_shade) */
#define RE_SDF_FOG 2u        /* apply_fog (SceneSettings::enable_fog)                  */
#define RE_SDF_GAMMA 4u      /* colour^(1/2.2) (RenderingSettings::gamma)               */
#define RE_SDF_VIGNETTING 8u /* RenderingSettings::vignetting                           */

typedef struct re_sdf_shade_params {
  float light_pos[2];       /* SceneSettings::light_pos (x, y): the light is at (x, y, x) */
  float light_intensity;    /* colour (0.86,0.80,0.45) * I / (4 pi |light|^2)           */
  float soft_shadow_k;      /* penumbra factor, SceneSettings::soft_shadow_k (32)       */
  float shadow_tmin;        /* shadow march start along the light direction (> 0)      */
  float shadow_tmax;        /* shadow march end                                         */
  uint32_t shadow_max_steps;/* field evaluations per shadow ray (<= 4096)              */
  float sun_dir[3];         /* atmosphere sun direction, unit length                   */
  float max_y;              /* terrain volume top: ocean below 0.2 max_y, snow above 0.8 */
  float fog_density;        /* SceneSettings::fog_deisity (RE_SDF_FOG)                 */
  float vignetting_k;       /* RenderingSettings::vignetting_k (RE_SDF_VIGNETTING)     */
  uint32_t flags;           /* RE_SDF_*                                                 */
} re_sdf_shade_params;

RE_API void re_sdf_shade_params_default(re_sdf_shade_params* s);
/* The shading pass alone over a hit record from re_sdf_trace (or
 * re_nsdf_trace); d_evals (device, may be NULL) accumulates the shadow
 * rays' field evaluations.  Two kernels: the soft-shadow march of the lit
 * hits, whose shadow factors d_rgba holds in between, then the paint of
 * every pixel into d_rgba. */
RE_API re_status re_sdf_shade(const re_sdf_params* field, const re_sdf_shade_params* shade,
                              const re_camera* cam, uint32_t w, uint32_t h,
                              const re_sdf_hit* d_hits, uint32_t* d_rgba,
                              uint64_t* d_evals, void* stream);
/* Trace (into the caller's w*h d_hits) and shade one frame. */
RE_API re_status re_render_sdf_frame(const re_sdf_params* field,
                                     const re_sdf_shade_params* shade,
                                     const re_camera* cam, uint32_t w, uint32_t h,
                                     re_sdf_hit* d_hits, uint32_t* d_rgba, void* stream);
/* State for cuda_render_frame() in the reference's shipped mode, the
 * counterpart of initialize_volume_render (sphere_tracing.cuh:617-755): the
 * next cuda_render_frame calls render this terrain until re_frame_bind binds
 * a mesh scene again.  animate_sun != 0 moves the sun after every frame as
 * Craze does (renderer.cu:287-298). */
RE_API re_status re_sdf_frame_bind(const re_sdf_params* field,
                                   const re_sdf_shade_params* shade,
                                   const re_camera* cam, int animate_sun);
/* The frame's elementary functions over device arrays (fn 0: e^x, 1: ln x,
 * 2: x^y), for checking them against CUDA's. */
RE_API re_status re_fmath(uint32_t fn, const float* d_x, const float* d_y, uint32_t n,
                          float* d_out, void* stream);

/* ---- neural SDF surrogate ------------------------------------------
 * No counterpart in the reference (it has no learned component): a
 * Fourier-feature MLP (3 -> 128 features -> 4 x 64 softplus -> 1) that
 * stands in for the terrain density d(p) = p.y - amp*fbm(scale*p) while
 * sphere tracing, with the exact field finishing every ray.  Trained on the
 * device by hand-written forward/backward/Adam kernels; evaluated with BF16
 * operands on the tensor cores (tcgen05, FP32 accumulation in tensor
 * memory). */
typedef struct re_nsdf re_nsdf;

typedef struct re_nsdf_config {
  float box_min[3], box_max[3]; /* input box, mapped to [-1, 1]^3          */
  float f0;                     /* lowest feature frequency (cycles/unit)   */
  uint32_t seed;                /* weight initialisation and sampling seed  */
} re_nsdf_config;

/* flags of re_nsdf_trace_params */
#define RE_NSDF_EXACT_ONLY 1u /* skip the network: the exact phase from t = 0 */

typedef struct re_nsdf_trace_params {
  float lipschitz;      /* bound on the network's gradient norm           */
  float safety;         /* step = safety * distance / lipschitz            */
  float switch_dist;    /* hand over to the exact field below this         */
  float min_step;       /* smallest network step                           */
  uint32_t max_network_steps; /* 0 = 256; with cones: passes per cone      */
                              /* (a tile that reaches it starts its exact  */
                              /* phase where its cone is)                  */
  uint32_t max_exact_steps;   /* exact evaluations per ray; 0 = max_steps  */
  uint32_t root_steps;  /* regula-falsi steps on a bracketed crossing; 0=4 */
  float relax;          /* exact steps may grow along the secant up to     */
                        /* relax x step_factor * d; <= 1: the plain rule   */
  uint32_t flags;       /* RE_NSDF_EXACT_ONLY                              */
  uint32_t cone_tile;   /* > 0 (<= 256): the network marches cones of      */
                        /* cone_tile x cone_tile pixel tiles instead of    */
                        /* single rays, and every pixel's exact phase      */
                        /* starts where its tile's cone stopped; 0: the    */
                        /* per-ray network march and hand-over queue       */
  uint32_t cone_coarse; /* 0, or a multiple of cone_tile (<= 1024): a      */
                        /* first cone level over tiles of this size        */
  uint32_t normal_taps; /* 0 or 6: central differences; 4: tetrahedral;   */
                        /* 1: the exact field's analytic gradient, in a   */
                        /* second pass over the hits                      */
  uint32_t cone_lanes;  /* 0 or 1, 2, 4, 8, 16: lanes per cone; above 1   */
                        /* evaluate successive guessed steps in one pass   */
  float root_tol;       /* > 0: the root search ends when its next secant  */
                        /* point moves less than this (scene units)        */
} re_nsdf_trace_params;

RE_API uint32_t re_nsdf_num_params(void);
/* Axis-aligned box of the view frustum [0, tmax] with y clamped. */
RE_API re_status re_nsdf_box_for_camera(const re_camera* cam, uint32_t w,
                                        uint32_t h, float tmax, float y_lo,
                                        float y_hi, float* box_min,
                                        float* box_max);
RE_API re_status re_nsdf_create(const re_nsdf_config* cfg, re_nsdf** out);
RE_API re_status re_nsdf_destroy(re_nsdf* s);
/* Parameters as FP32 (re_nsdf_num_params values): W1 [64][128], b1, W2,
 * b2, W3, b3, W4, b4 ([64][64] and 64 each), w5 [64], b5. */
RE_API re_status re_nsdf_get_params(const re_nsdf* s, float* host);
RE_API re_status re_nsdf_set_params(re_nsdf* s, const float* host);
/* Training data: num_points float4 {x, y, z, label}, half uniform in the
 * box and half within N(0, 0.02) of exact-traced camera hits; label = the
 * exact field's first-order distance d / |grad d| clipped to [-4, 4]. */
RE_API re_status re_nsdf_generate(re_nsdf* s, const re_sdf_params* field,
                                  const re_camera* cam, uint32_t w, uint32_t h,
                                  uint32_t num_points, uint32_t seed,
                                  void* stream);
RE_API re_status re_nsdf_get_data(const re_nsdf* s, float* host_xyzl,
                                  uint32_t max_points);
/* `steps` Adam steps (L1 loss) on batches of `batch` points sampled from the
 * generated data; batch must be a multiple of 512.  loss_out (host, steps
 * floats) may be NULL.  Synchronises the stream. */
RE_API re_status re_nsdf_train(re_nsdf* s, uint32_t steps, uint32_t batch,
                               float lr, float* loss_out, void* stream);
/* Gradient of the mean L1 loss of n points (device float4 {x,y,z,label},
 * n a multiple of 512) w.r.t. the parameters (device, re_nsdf_num_params
 * floats) and the predictions (device, n floats, may be NULL). */
RE_API re_status re_nsdf_loss_grad(re_nsdf* s, const float* d_xyzl, uint32_t n,
                                   float* d_grad, float* d_pred, void* stream);
/* Network distance of n points (device, 3 floats each): tensor cores. */
RE_API re_status re_nsdf_eval(re_nsdf* s, const float* d_pts, uint32_t n,
                              float* d_out, void* stream);
/* The same with the training arithmetic (SIMT FP32, BF16-rounded). */
RE_API re_status re_nsdf_eval_reference(re_nsdf* s, const float* d_pts,
                                        uint32_t n, float* d_out, void* stream);
/* Gradient-norm bound: the `quantile` (0 < q <= 1; 1 = the largest) of
 * the forward-difference gradient norms at `samples` training points. */
RE_API re_status re_nsdf_lipschitz(re_nsdf* s, uint32_t samples, float h,
                                   float quantile, float* out, void* stream);
/* Neural march inside the network's box, then the exact phase: the exact
 * tracer's steps from the hand-over point, a bracketed crossing refined by
 * regula falsi, the exact tracer's central-difference normal (or the
 * reference's tetrahedral one).  With cone_tile > 0 the network phase
 * marches one cone per pixel tile (the network distance less the cone's
 * radius bounds the step of every ray of the tile) and each pixel's exact
 * phase starts at its tile's stop.  Output as re_sdf_trace (steps =
 * network steps + exact evaluations). */
RE_API re_status re_nsdf_trace(re_nsdf* s, const re_sdf_params* field,
                               const re_nsdf_trace_params* tp,
                               const re_camera* cam, uint32_t w, uint32_t h,
                               re_sdf_hit* d_out, void* stream);
/* The two phases of re_nsdf_trace as separate calls on the same stream
 * (network march into the hand-over queue, then the exact phase), for
 * timing each and for callers that interleave other work. */
RE_API re_status re_nsdf_trace_network(re_nsdf* s, const re_sdf_params* field,
                                       const re_nsdf_trace_params* tp,
                                       const re_camera* cam, uint32_t w,
                                       uint32_t h, re_sdf_hit* d_out,
                                       void* stream);
RE_API re_status re_nsdf_trace_exact(re_nsdf* s, const re_sdf_params* field,
                                     const re_nsdf_trace_params* tp,
                                     const re_camera* cam, uint32_t w, uint32_t h,
                                     re_sdf_hit* d_out, void* stream);
/* Of the last trace: rays handed to the exact phase through the queue of
 * the per-ray network march (0 with cone_tile > 0, where every pixel runs
 * the exact phase from its tile's stop), the device error flag
 * (1 = a tensor-core wait reached its bound) and, when evals is not NULL,
 * four totals: network evaluations of rays, exact-field evaluations of the
 * march / bracket / root steps, exact normal taps, network rows computed
 * (rays and idle rows of the 128-row tiles). */
RE_API re_status re_nsdf_trace_status(re_nsdf* s, uint32_t* num_refined,
                                      int* error, uint64_t* evals);
/* Checkpoint: parameters, Adam moments and step count. */
RE_API re_status re_nsdf_save(const re_nsdf* s, const char* path);
RE_API re_status re_nsdf_load(re_nsdf* s, const char* path);

/* ---- instanced scenes --------------------------------------------------
 * Replaces the reference's per-object ray transform and closest-hit loop
 * (ray_functions.cuh:236-267,377-396; objects in RTScene.cpp:40-62): each
 * instance is a built scene seen through a yaw rotation and a location,
 * object-space ray d' = normalize(Ry d), o' = Ry o + location. */
typedef struct re_instance {
  const re_scene* mesh;
  float yaw;              /* radians, about +y                              */
  float location[3];
} re_instance;
/* Primary rays against all instances: re_hit per pixel and the index of
 * the instance hit (-1 for none); one-sided with RE_TRACE_ONE_SIDED. */
RE_API re_status re_trace_instances(const re_instance* instances, uint32_t n,
                                    const re_camera* cam, uint32_t w, uint32_t h,
                                    uint32_t flags, re_hit* d_out, int32_t* d_instance,
                                    void* stream);
/* cos and sin of a yaw exactly as re_trace_instances computes them. */
RE_API void re_instance_trig(float yaw, float* c, float* s);

/* ---- voxel SDF ----------------------------------------------------------
 * Replaces the reference's voxel-SDF path: the bake kernel generate_noise
 * (renderer.cu:106-126), the .rsdf file (Grid.cpp:23-64, save_map
 * renderer.cu:839-870) and get_distance's LOW / MEDIUM / HIGH sampling
 * (sdf_functions.cuh:394-419).  A grid is dim[0] x dim[1] x dim[2] voxels
 * of 2 floats {distance, material}, x fastest; voxel (i, j, k) holds the
 * field at origin + (i, j, k) * spacing; lookups clamp to the edge. */
#define RE_VOXEL_LOW 0u    /* nearest voxel                                  */
#define RE_VOXEL_MEDIUM 1u /* trilinear                                      */
#define RE_VOXEL_HIGH 2u   /* tricubic B-spline over 4 x 4 x 4 voxels        */
typedef struct re_voxel_grid {
  uint32_t dim[3];
  float spacing[3];
  float origin[3];
} re_voxel_grid;
/* d_grid: 2 * voxels floats; distance = the field's density, material 0. */
RE_API re_status re_voxel_bake(const re_sdf_params* field, const re_voxel_grid* g,
                               float* d_grid, void* stream);
RE_API re_status re_voxel_sample(const float* d_grid, const re_voxel_grid* g,
                                 uint32_t quality, const float* d_pts, uint32_t n,
                                 float* d_out, void* stream);
/* Sphere tracing inside the grid's box with march's step_factor, eps, tmax
 * and max_steps; output as re_sdf_trace (normal: central differences with
 * half the smallest spacing). */
RE_API re_status re_voxel_trace(const float* d_grid, const re_voxel_grid* g,
                                uint32_t quality, const re_sdf_params* march,
                                const re_camera* cam, uint32_t w, uint32_t h,
                                re_sdf_hit* d_out, void* stream);
/* Brush edits of a grid (insert_sphere_to_texture, renderer.cu:31-92) at a
 * world-space centre: sphere add (smooth union with k = smooth, the
 * reference uses 0.1) / subtract, cube add / subtract (half-extents). */
#define RE_BRUSH_SPHERE_ADD 0u
#define RE_BRUSH_SPHERE_SUBTRACT 1u
#define RE_BRUSH_CUBE_ADD 2u
#define RE_BRUSH_CUBE_SUBTRACT 3u
typedef struct re_voxel_brush_params {
  uint32_t type;
  float center[3];
  float extent[3];        /* sphere: radius in extent[0]                    */
  float material;
  float smooth;
} re_voxel_brush_params;
RE_API re_status re_voxel_brush(float* d_grid, const re_voxel_grid* g,
                                const re_voxel_brush_params* b, void* stream);
/* .rsdf files: int32 dim[3], float spacing[3], {distance, material} per
 * voxel, x fastest.  re_voxel_load fills g (origin 0) and, when host_grid
 * is not NULL, up to capacity_voxels voxels. */
RE_API re_status re_voxel_save(const char* path, const re_voxel_grid* g,
                               const float* host_grid);
RE_API re_status re_voxel_load(const char* path, re_voxel_grid* g, float* host_grid,
                               uint64_t capacity_voxels);

/* ---- mesh ingestion (host) ---------------------------------------------
 * Replaces RStaticMesh::LoadFromFile (RE/Objects/RStaticMesh.cpp:68-128,
 * PLY through rply) and WavefrontOBJ::loadObjFromFile
 * (RayEngine/includes/ObjFileReader.h:65-180).  PLY: ascii or binary, any
 * numeric property types, vertex x/y/z and face vertex_indices; faces with
 * more corners are fan-triangulated unless RE_MESH_FIRST_TRIANGLE (the
 * reference's reader keeps the first three corners).  OBJ: v and f with
 * p, p/t, p//n, p/t/n corners; one vertex per distinct corner in order of
 * first use, quads split as the reference does, larger polygons fanned. */
#define RE_MESH_FIRST_TRIANGLE 1u
typedef struct re_mesh re_mesh;
RE_API re_status re_mesh_load(const char* path, uint32_t flags, re_mesh** out);
RE_API re_status re_mesh_info(const re_mesh* m, uint32_t* num_verts,
                              uint32_t* num_faces);
/* verts: 3 floats per vertex; faces: 3 indices per triangle. */
RE_API re_status re_mesh_copy(const re_mesh* m, float* verts, uint32_t* faces);
RE_API re_status re_mesh_destroy(re_mesh* m);

/* ---- shaded frame (the reference's render call) ----------------------
 * Replaces cuda_render_frame (renderer.cu:702-738) with its per-pixel
 * shading (trace_secondary_rays :435-492, phong_light / shade
 * material_functions.cuh:69-119, illuminate cuda_helper_functions.h:90-102)
 * and rgbaFloatToInt (cuda_helper_functions.h:61-68): primary closest hits,
 * Phong with one shadow ray per point light, a sky gradient for misses,
 * packed RGBA8 (R in the low byte, alpha 255) in a W x H device buffer. */
typedef struct re_light {
  float pos[3];
  float intensity;        /* the reference's scene uses 20000               */
} re_light;

typedef struct re_shade_params {
  float albedo[3];        /* material colour, the base of every hit         */
  float sky_zenith[3];    /* miss colour = lerp(horizon, zenith, max(d.y,0))*/
  float sky_horizon[3];
  uint32_t flags;         /* RE_TRACE_ONE_SIDED for the primary rays        */
} re_shade_params;

RE_API re_status re_render_frame(re_scene* s, const re_camera* cam,
                                 const re_light* lights, uint32_t num_lights,
                                 const re_shade_params* sp, uint32_t w, uint32_t h,
                                 uint32_t* d_rgba, void* stream);
/* State for cuda_render_frame(), which keeps the reference's signature
 * (scene, camera and lights are globals there); animate_light != 0 moves
 * light 0 after every frame as the reference's Craze kernel does. */
RE_API re_status re_frame_bind(re_scene* s, const re_camera* cam,
                               const re_light* lights, uint32_t num_lights,
                               const re_shade_params* sp, int animate_light);

/* ---- batched wavefront path tracing ----------------------------------
 * No single counterpart in the reference, which renders one scene per
 * frame (cuda_render_frame, renderer.cu:702-738; bounce rays in
 * trace_secondary_rays, renderer.cu:435-492).  Many scenes of uneven size
 * (rope kd-tree meshes and exact-SDF terrains, each with its own camera and
 * resolution) are path traced (1 sample per pixel, Lambertian bounces) by
 * one persistent kernel launch that pulls rays from per-bounce queues.
 * Radiance of pixel i of scene s is out[offset(s) + i]: albedo^b * sky(d)
 * for a path that leaves the scene at bounce b with direction d, sky(d) =
 * 0.5 (1 + d.y); 0 for a path still on a surface after max_depth rays. */
#define RE_BATCH_MESH 0u
#define RE_BATCH_TERRAIN 1u
typedef struct re_batch re_batch;

typedef struct re_batch_scene {
  uint32_t kind;          /* RE_BATCH_MESH or RE_BATCH_TERRAIN              */
  const re_scene* mesh;   /* MESH: a built scene, used in place (must       */
                          /* outlive the batch); two-sided triangles        */
  re_sdf_params field;    /* TERRAIN: the exact field and its march         */
  re_camera camera;
  uint32_t width, height;
  float albedo;           /* Lambertian reflectance in [0, 1]               */
} re_batch_scene;

typedef struct re_path_params {
  uint32_t max_depth;     /* rays per path, the primary included (4); <= 8  */
  uint32_t seed;          /* bounce directions: hash(seed, pixel, bounce)   */
  float mesh_bias;        /* bounce origin offset along a mesh normal       */
} re_path_params;

typedef struct re_batch_tuning {
  uint32_t block_threads; /* 32..256, multiple of 32 (256)                  */
  uint32_t refill_min;    /* idle lanes a warp waits for before claiming    */
  uint32_t stage_nodes;   /* top nodes per mesh scene in shared memory      */
  uint32_t steps_per_trip;/* leaves / field evaluations a lane advances     */
                          /* between the warp's refills (0 = 1; 8)          */
} re_batch_tuning;

RE_API re_status re_batch_create(const re_batch_scene* scenes, uint32_t num_scenes,
                                 const re_path_params* pp, re_batch** out);
RE_API re_status re_batch_destroy(re_batch* b);
/* Total pixels of the batch and each scene's first pixel (num_scenes
 * values; offsets may be NULL). */
RE_API re_status re_batch_pixels(const re_batch* b, uint64_t* total,
                                 uint64_t* offsets);
/* One frame, one launch.  d_radiance: total pixels floats; d_primary (may
 * be NULL): the primary ray's hit per pixel (mesh: id, t, u, v; terrain:
 * id 0 on a hit, -1 otherwise, t). */
RE_API re_status re_batch_render(re_batch* b, float* d_radiance, re_hit* d_primary,
                                 void* stream);
/* The same frame from a CUDA graph captured on the first call (and again
 * when the buffers, the stream or the tuning change), then replayed. */
RE_API re_status re_batch_render_graph(re_batch* b, float* d_radiance,
                                       re_hit* d_primary, void* stream);
/* Rays traced in the last frame: rays[2 * bounce + kind] (bounce 0: all
 * primary rays under kind 0), 2 * max_depth values; error = 1 if a wait
 * bound was reached (rays dropped). */
RE_API re_status re_batch_stats_get(re_batch* b, uint64_t* rays, int* error);
/* Bounds of the persistent kernel's waits: polls of one queue slot's flag
 * before a claim is dropped, and trips of the kernel's loop (0 = the
 * defaults, 2^22 each).  Reaching either sets the frame's error flag
 * (re_batch_stats_get) and the kernel returns instead of waiting on.  Lower
 * them only to exercise that error path (tests); the next frame after the
 * defaults are restored is complete again.  No reference counterpart. */
RE_API re_status re_batch_set_wait_bounds(re_batch* b, uint32_t pending_polls,
                                          uint32_t loop_trips);
/* One frame with work counters: totals[0..3] = inner-node visits, leaf
 * visits, triangle tests, terrain field evaluations (host array). */
RE_API re_status re_batch_counts(re_batch* b, float* d_radiance, void* stream,
                                 uint64_t* totals);
RE_API re_status re_batch_get_tuning(const re_batch* b, re_batch_tuning* out);
RE_API re_status re_batch_set_tuning(re_batch* b, const re_batch_tuning* t);
/* Times one frame per candidate (block size x refill threshold x staged
 * nodes x steps per trip) and keeps the fastest. */
RE_API re_status re_batch_autotune(re_batch* b, float* d_radiance, void* stream,
                                   re_batch_tuning* out, float* best_ms);

/* ---- measurement ---------------------------------------------------------
 * L2 read bandwidth (16-byte L2-only loads over an L2-resident buffer of
 * `bytes`, 1-64 MB, read `passes` times in one launch), in GB/s: the
 * denominator of the traversal kernels' L2 roofline.  No reference
 * counterpart. */
RE_API re_status re_measure_l2_read(size_t bytes, uint32_t passes, float* gbs, void* stream);
/* FP32 fused multiply-add rate (8 independent chains of `iters` FMAs per
 * thread, 8 blocks of 256 threads per SM, `iters` in [1024, 2^20]), in
 * 10^12 FMAs per second: the denominator of the SIMT field kernels'
 * roofline.  No reference counterpart. */
RE_API re_status re_measure_fp32_fma(uint32_t iters, float* tops, void* stream);

#ifdef __cplusplus
}
/* The reference's render call, same C++ signature (renderer.cu:701):
 * renders the state bound by re_sdf_frame_bind (the reference's shipped
 * SDF mode) or re_frame_bind (its kd-tree mode), whichever was bound last,
 * into `output` (device, W x H RGBA8) and waits; errors go to
 * re_last_error(), which the call empties on entry (so an empty message
 * after it means success). */
void cuda_render_frame(unsigned int* output, const unsigned int& width,
                       const unsigned int& heigth);
#endif
#endif
