/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle.
 *
 * A plain-C restatement of RayEngine's ray-query hot path, used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.
 * Nothing in the product (rayengine_b200/) links, loads or calls it.
 *
 * Parity pin: the Perlin permutation table and the as-shipped kd-tree (a
 * single leaf => brute-force Moller-Trumbore in index order) are checked
 * against the reference's own host code compiled from its sources
 * (oracle/_ref/libre_ref.so, recipe oracle/Makefile.ref) and against the
 * golden fixtures under tests/golden/ generated from it.
 *
 * Floating point: compiled with -ffp-contract=off.  Every fused multiply-add
 * is an explicit fmaf(), every division and square root is IEEE, so the CUDA
 * kernels (built with -fmad=false and the same explicit fmaf calls) produce
 * bit-identical results.
 */
#ifndef RE_ORACLE_H
#define RE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float x, y, z; } of3;

/* --- camera (RayEngine/src/cuda-src/ray_functions.cuh:14-55) ------------ */
typedef struct {
  float campos[3], view[3], camdown[3];
  float fov[2];
  float focal;
} o_camera;

/* per-frame constants the reference recomputes per pixel */
typedef struct {
  float campos[3], middle[3], horizontal[3], vertical[3];
  float focal;
} o_camera_basis;

void o_camera_setup(const o_camera* cam, o_camera_basis* out);
void o_generate_ray(const o_camera_basis* b, uint32_t w, uint32_t h,
                    uint32_t x, uint32_t y, float o[3], float d[3]);

/* --- ray/box and ray/triangle ------------------------------------------ */
/* ray_functions.cuh:62-92 */
int o_ray_box(const float bmin[3], const float bmax[3], const float o[3],
              const float d[3], float* t_near, float* t_far);
/* mode 0: two-sided (KDTree.cpp:909-949, |a|<1e-5, t>1e-5)
 * mode 1: one-sided (ray_functions.cuh:174-223, a<1e-4 rejected, t>1e-4) */
int o_ray_tri(const float o[3], const float d[3], const float v0[3],
              const float e1[3], const float e2[3], int mode, float* t,
              float* u, float* v);

typedef struct { int32_t id; float t, u, v; } o_hit;

/* Reference as shipped: RKDTreeCPU with MAX_DEPTH=1 is one leaf holding every
 * triangle, so stackless_kdtree_traversal (ray_functions.cuh:231-360) is a
 * root-box test followed by an index-order MT loop keeping t < t_exit.
 * tris: n x 12 floats {v0.xyz,_, e1.xyz,_, e2.xyz,_}. */
void o_trace_bruteforce(const float* tris, int32_t n, const float bmin[3],
                        const float bmax[3], const float o[3], const float d[3],
                        int mode, o_hit* out);

/* --- the project's flattened kd-tree (same layout the kernels read) ---- */
typedef struct {
  const float* nodes;      /* 2 x 32-bit per node: split, meta            */
  const float* leaves;     /* 16 x 32-bit per leaf                        */
  const float* tris;       /* 12 floats per reference, leaf order         */
  float bmin[3], bmax[3];  /* root box                                    */
} o_kdtree;

typedef struct {
  uint32_t inner_visits, leaf_visits, tri_tests, status;
} o_counts;

/* The reference's rope traversal restated over the project's tree, with the
 * exit face taken from the slab test (not the reference's 1e-4 proximity test).
 * anyhit != 0: stop at the first hit with t < tmax (shadow/AO rays). */
void o_trace_kd(const o_kdtree* kd, const float o[3], const float d[3],
                float tmax, int mode, int anyhit, uint32_t max_leaf_visits,
                o_hit* out, o_counts* cnt);
/* the same, starting in leaf node `start` when the origin lies in its region
 * (0 = root), and reporting the node of the leaf holding the best hit */
void o_trace_kd_ex(const o_kdtree* kd, const float o[3], const float d[3],
                   float tmax, int mode, int anyhit, uint32_t max_leaf_visits,
                   uint32_t start, o_hit* out, o_counts* cnt, uint32_t* out_leaf);

/* --- Perlin / fBm (sdf_functions.cuh:26-135, PerlinNoise.h:16-52) ------ */
void o_perlin_permutation(uint32_t seed, uint32_t perm[512]);
float o_perlin(const uint32_t perm[512], float x, float y, float z);
float o_fbm(const uint32_t perm[512], float x, float y, float z, int octaves,
            float lacunarity, float gain);
/* heightfield: y = amp * fbm(x, 0, z) */
float o_height(const uint32_t perm[512], float x, float z, int octaves,
               float amp);
/* volumetric terrain d(p) = p.y - amp * fbm(scale * p) */
float o_terrain_density(const uint32_t perm[512], const float p[3], int octaves,
                        float scale, float amp);

/* --- scene generators -------------------------------------------------- */
uint64_t o_mt64_next(uint64_t* state /* 312 + 1 words */);
void o_gen_soup(uint64_t seed, int32_t n, float* verts /* n*9 */);
/* grid of (cells+1)^2 vertices over [lo,hi]^2, 2*cells^2 triangles */
void o_gen_heightfield(const uint32_t perm[512], int32_t cells, float lo,
                       float hi, int octaves, float amp, float* verts,
                       uint32_t* faces);

/* --- exact-SDF sphere tracer (sphere_tracing.cuh:183-216) --------------- */
typedef struct {
  float pos[3], normal[3];
  uint32_t steps, status; /* status: 1 hit, 0 miss, 2 step cap */
  float t, pad;
} o_sdf_hit;

void o_sdf_trace(const uint32_t perm[512], const float o[3], const float d[3],
                 int octaves, float scale, float amp, float step_factor,
                 float eps, float tmax, uint32_t max_steps, o_sdf_hit* out);

/* --- shaded SDF terrain frame (oracle_sdf_frame.c) ---------------------- */
typedef struct {
  uint32_t octaves;
  float scale, amp, step_factor, eps, tmax;
  uint32_t max_steps;
} o_sdf_field;

/* same field order as re_sdf_shade_params */
typedef struct {
  float light_pos[2];
  float light_intensity, soft_shadow_k, shadow_tmin, shadow_tmax;
  uint32_t shadow_max_steps;
  float sun_dir[3];
  float max_y, fog_density, vignetting_k;
  uint32_t flags; /* 1 shade, 2 fog, 4 gamma, 8 vignetting */
} o_sdf_shade;

float o_fm_exp(float x);
float o_fm_log(float x);
float o_fm_pow(float x, float y);
uint32_t o_sdf_shade_pixel(const uint32_t perm[512], const o_sdf_field* f, const o_sdf_shade* s,
                           const float o[3], const float d[3], const o_sdf_hit* hit, float u,
                           float v, uint32_t* evals);

/* --- deterministic sampling shared with the kernels -------------------- */
uint32_t o_hash_u32(uint32_t a, uint32_t b, uint32_t c);
void o_sincos_2pi(float u, float* s, float* c);
void o_secondary_rays(const float hitp[3], const float n[3], uint32_t seed,
                      uint32_t pixel, const float light_dir[3], float bias,
                      float o_out[5][3], float d_out[5][3], float tmax_out[5]);

/* --- batched path tracing (one pixel of the wavefront renderer) -------- */
typedef struct {
  uint32_t kind;              /* 0 mesh, 1 terrain                         */
  const float* tris;          /* mesh: n x 12 floats in triangle-id order  */
  int32_t ntris;
  float bmin[3], bmax[3];     /* mesh: root box of the scene               */
  const uint32_t* perm;       /* terrain                                   */
  int octaves;
  float scale, amp, step_factor, eps, tmax;
  uint32_t max_steps;
  o_camera cam;
  uint32_t w, h;
  float albedo;
} o_path_scene;
/* returns the number of rays the path traced */
uint32_t o_path_pixel(const o_path_scene* s, uint32_t gpix, uint32_t local_pix, uint32_t depth,
                      uint32_t seed, float mesh_bias, float* radiance, o_hit* primary);
/* --- shaded frame: one pixel, packed RGBA8 ------------------------------ */
uint32_t o_frame_pixel(const float* tris, int32_t n, const float bmin[3], const float bmax[3],
                       const o_camera_basis* cb, uint32_t w, uint32_t h, uint32_t x, uint32_t y,
                       int mode, const float* light_pos, const float* light_int,
                       uint32_t num_lights, const float albedo[3], const float zenith[3],
                       const float horizon[3]);
/* --- voxel SDF (grid lookups, voxel sphere tracer) --------------------- */
typedef struct {
  const float* v;   /* 2 floats per voxel {distance, material}, x fastest */
  int dim[3];
  float spacing[3], origin[3];
} o_voxel;
float o_voxel_sample(const o_voxel* g, uint32_t quality, const float p[3]);
void o_voxel_trace_pixel(const o_voxel* g, uint32_t quality, float step_factor, float eps,
                         float tmax, uint32_t max_steps, const o_camera_basis* cb, uint32_t w,
                         uint32_t h, uint32_t pix, o_sdf_hit* out);
/* --- instances and voxel brush ------------------------------------------ */
void o_trace_instances_pixel(const float* const* tris, const int32_t* ntris, const float* bmin,
                             const float* bmax, const float* cs, const float* loc, int32_t n,
                             const float o[3], const float d[3], int mode, o_hit* out,
                             int32_t* inst);
void o_voxel_brush(float* v, const int dim[3], const float spacing[3], const float origin[3],
                   uint32_t type, const float c[3], const float e[3], float mat, float k);
/* --- SAH kd-tree for the reference arm (oracle_kdbuild.c) -------------- */
/* Pre-order nodes: axis 0..2 (inner: children left/right, split plane) or
 * 3 (leaf: triangles index[first .. first + count)). */
typedef struct {
  int32_t axis;
  float split;
  int32_t left, right, first, count;
} o_kdb_node;

typedef struct {
  o_kdb_node* nodes;
  int32_t n_nodes;
  int32_t* index;
  int64_t n_index;
  float bmin[3], bmax[3];
} o_kdb_tree;

/* Binned SAH (32 planes per axis) over an indexed mesh; 0 on success. */
int o_kdb_build(const float* verts, int32_t nv, const uint32_t* faces, int32_t nf,
                int max_depth, int leaf_size, float ci, float ct, float empty_bonus,
                o_kdb_tree* out);
void o_kdb_free(o_kdb_tree* t);

#ifdef __cplusplus
}
#endif
#endif
