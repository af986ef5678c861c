/*
 * clay_oracle.h - CPU restatement of clay-engine's fluid hot path. TEST INFRASTRUCTURE.
 *
 * This library is the checker, never the product: only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark load it. It restates, in plain C++ compiled with
 * -ffp-contract=off, the WGSL that TypeGPU generates from the reference's 'use gpu'
 * closures, in the reference's operation order, in two precisions:
 *   - f32 ("port"): every operation rounded to binary32 in reference order, host-derived
 *     constants computed in binary64 and rounded once (as the reference's JS does);
 *   - f64 ("truth"): the same algorithm with every operation in binary64, used only to
 *     report the error of f32 results.
 * Each function names the reference file:line it follows. Where WGSL leaves precision to the
 * implementation (pow, normalize, texture filtering, f32->f16 rounding) the choice made
 * here is stated beside the function and is shared with the CUDA path.
 */
#ifndef CLAY_ORACLE_H
#define CLAY_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* An SdfVolume as data: f16 distance/material planes of all levels (x fastest). */
typedef struct orc_volume {
  int32_t res;
  int32_t mips;
  double origin[3];
  double world_size;
  double band;
  double gradient_voxels;
  const uint16_t* dist;
  const uint16_t* mat;
} orc_volume;

/* A collider: unionField over up to 8 volumeFields, each optionally offsetField-moved. */
typedef struct orc_field {
  int32_t n;
  int32_t pad;
  orc_volume vol[8];
  double offset[8][3];
} orc_field;

/* FluidSim construction options after `??` defaults (fluid.ts:141-160). */
typedef struct orc_fluid_cfg {
  uint32_t capacity;
  uint32_t bucket;
  double spacing;
  double h;
  double radius;
  double surface_radius;
  double material;
  int32_t bake_res;
  int32_t bake_mips;
  double bake_band;
  double origin[3];
  double world_size;
  int32_t substeps;
  int32_t pad;
} orc_fluid_cfg;

/* FluidParams (fluid.ts:28-51), 80 bytes. */
typedef struct orc_params {
  float gravity[3];
  float dt;
  float emit_pos[3];
  float emit_radius;
  float emit_vel[3];
  float max_speed;
  float stiffness;
  float viscosity;
  float damping;
  uint32_t count;
  uint32_t emit_base;
  uint32_t emit_count;
  uint32_t emit_seed;
  float contact_depth;
} orc_params;

/* FluidParticle (fluid.ts:20-26) in f32 (48 B) and its f64 twin (96 B). */
typedef struct orc_particle {
  float pos[3], density, vel[3], pressure, nvel[3], pad;
} orc_particle;
typedef struct orc_particle_d {
  double pos[3], density, vel[3], pressure, nvel[3], pad;
} orc_particle_d;

/* Derived constants of a FluidSim (fluid.ts:143-266), in f64 as the host computes them. */
typedef struct orc_fluid_derived {
  double h, poly6, spiky_grad, mass, rest_density;
  int32_t grid_res;
  int32_t pad;
  double grid_origin[3];
  double wall_lo[3], wall_hi[3];
} orc_fluid_derived;

/* A ParticleCloud (splat.ts:15-38) as arrays. live_mode: 0 all, 1 i < a, 2 a <= i < a+b. */
typedef struct orc_cloud {
  uint32_t capacity;
  uint32_t pos_stride;   /* floats between records */
  const float* pos;
  uint32_t live_mode;
  uint32_t live_a;
  uint32_t live_b;
  uint32_t nrm_stride;   /* floats */
  const float* nrm;      /* NULL: no normalAt */
  const float* quat;     /* NULL or xyzw */
} orc_cloud;

/* SplatField options after defaults (splat.ts:147-153) and its current origin. */
typedef struct orc_splat_cfg {
  int32_t res;
  int32_t mips;
  double band;
  double radius;
  double world_size;
  double material;
  double origin[3];
} orc_splat_cfg;

/* ---- math/gpu.ts ---- */
float orc_hash1(uint32_t seed);                          /* gpu.ts:103-112 */
void orc_hash3(uint32_t seed, float out[3]);             /* gpu.ts:114-117 */

/* ---- field/volume.ts ---- */
/* Mip-chain rule and refusal (volume.ts:140-160). Returns levels, or -1 with `err` set. */
int32_t orc_volume_mip_levels(int32_t resolution, int32_t requested, char* err, int32_t errlen);
int64_t orc_volume_total_voxels(int32_t res, int32_t mips);

/* ---- trace/field.ts: collider sample(p,0) and normal(p) ---- */
void orc_field_query_f32(const orc_field* f, const float p[3], float sample_xy[2], float nrm[3]);
void orc_field_query_f64(const orc_field* f, const double p[3], double sample_xy[2], double nrm[3]);

/* ---- sim/fluid.ts ---- */
void orc_fluid_derive(const orc_fluid_cfg* cfg, orc_fluid_derived* out);   /* :143-266 */
double orc_rest_density(double spacing, double h);                         /* :168-182 */
/* cellIndex of every particle i < count, or 0xffffffff when !inGrid (:253-266,318-322). */
void orc_fluid_cells(const orc_fluid_cfg* cfg, const orc_particle* parts, uint32_t count,
                     uint32_t* keys);
void orc_fluid_emit(const orc_fluid_cfg* cfg, const orc_params* prm, orc_particle* parts); /* :268-291 */
/* One substep: clearGrid, insert, density, forces, integrate (:293-491). Buckets keep the
 * first `bucket` particles of each cell in ascending index order. Contacts: every particle
 * that reaches the append is listed in `contact_ids` (ascending, up to `max_ids`), `count`
 * is the reference's atomic counter value, and `points` holds the first 32 in index order.
 * `threads` > 1 runs the independent per-particle passes with OpenMP. */
void orc_fluid_substep_f32(const orc_fluid_cfg* cfg, const orc_params* prm, const orc_field* world,
                           orc_particle* parts, uint32_t* contact_count, float* contact_points,
                           uint32_t* contact_ids, uint32_t max_ids, int32_t threads);
void orc_fluid_substep_f64(const orc_fluid_cfg* cfg, const orc_params* prm, const orc_field* world,
                           orc_particle_d* parts, int32_t threads);
/* Density/pressure pass only (:333-368), in f64, from an f32 state: out[2*i] = density,
 * out[2*i+1] = pressure. */
void orc_fluid_density_f64(const orc_fluid_cfg* cfg, const orc_params* prm,
                           const orc_particle* parts, double* out, int32_t threads);

/* ---- sim/splat.ts ---- */
/* The u32 key grid after clear + every splat[m] (:200-256). `keys` holds total voxels. */
void orc_splat_keys(const orc_splat_cfg* cfg, const orc_cloud* cloud, uint32_t* keys,
                    int32_t threads);
/* The fixed-point key of splat.ts:108-110,247 and its inverse of :272. */
uint32_t orc_splat_encode(float sd, float band_world);
float orc_splat_decode(uint32_t key);
/* resolve[m] (:258-276): key -> f32 -> f16 (round to nearest even), material -> f16. */
void orc_splat_resolve(const orc_splat_cfg* cfg, const uint32_t* keys, uint16_t* dist_f16,
                       uint16_t* mat_f16);
/* Unquantised f64 value of every voxel: clamp(min sd / bandWorld, -1, 1), or 1 when no
 * particle reaches it. For the error report only. */
void orc_splat_values_f64(const orc_splat_cfg* cfg, const orc_cloud* cloud, double* vals,
                          int32_t threads);

/* ---- field/builder.ts + brush.ts: collider fixtures ---- */
typedef struct orc_brush {
  float pos[3], scale, rot[4], size[3], radius, material, blend, bound, mask;
  uint32_t kind, op, slot, pad;
} orc_brush;
/* SdfBuilder.rebuild (builder.ts:76-142) into f16 planes of all levels. */
void orc_build_brushes(const orc_volume* vol_shape, const orc_brush* brushes, int32_t n,
                       uint16_t* dist_f16, uint16_t* mat_f16, int32_t threads);
/* BrushSet.evalBrush (brush.ts:475-480) at points, f32 (for the brush known answers). */
void orc_eval_brush(const orc_brush* b, const float* pts, int32_t n, float* out);

/* f32 <-> f16 (round to nearest even) helpers shared by the tests. */
uint16_t orc_f32_to_f16(float f);
float orc_f16_to_f32(uint16_t h);

/* ---- trace/field.ts: sample(p, mip) and field(p, mip), level capped (f32) ---- */
void orc_field_query_mip_f32(const orc_field* f, const float p[3], int mip, float sample_xy[2], float field_xy[2]);
/* the same over n points (xyz triples), OpenMP over points: the CPU leg of the sampling measurement */
void orc_field_query_mip_batch(const orc_field* f, const float* pts, int64_t n, int mip, float* sample_xy,
                               float* field_xy, int threads);

/* ---- sim/extract.ts: SurfaceExtractor.extract (f32) ---- */
typedef struct orc_extract_cfg {
  int32_t res, body, base, capacity, quad_cap, has_motion;
  float origin[3];
  float cell;
  float vel[3];
  uint32_t preserve;
  int32_t offset_by_motion; /* the field's leaves follow the motion centre (offsetField) */
  int32_t pad;
} orc_extract_cfg;
/* motion: 8 floats (centre, pad, velocity, pad), in/out, NULL without motion; particles and
 * bodies: 96- and 64-byte records; indices: quad_cap * 6; draw_args[4]; counters[2];
 * id_grid: res^3 (scratch, left holding the biased ids). */
void orc_extract(const orc_extract_cfg* cfg, const orc_field* f, float* motion, unsigned char* particles,
                 unsigned char* bodies, uint32_t* indices, uint32_t* draw_args, uint32_t* counters, uint32_t* id_grid);

/* ---- sim/pbd.ts: ClaySolver.step (f32) ---- */
typedef struct orc_solve_cfg {
  float gravity[3];
  float h;
  float radius, friction, damping, max_speed;
  float push[3];
  uint32_t push_body;
  float kick[3];
  int32_t capacity, max_bodies, rot_iters, substeps, kicking;
} orc_solve_cfg;
void orc_solver_step(const orc_solve_cfg* cfg, const orc_field* world, unsigned char* particles, unsigned char* bodies,
                     int body_count);
/* the sin/cos shared with the CUDA path: sc = (sin x, cos x) */
void orc_sincos_f32(float x, float sc[2]);

#ifdef __cplusplus
}
#endif
#endif
