/*
 * clay_fluid.h - C ABI of the B200-native fluid hot path of clay-engine.
 *
 * The path is one frame of `FluidSim.step` (lib/src/sim/fluid.ts:536-558): emission,
 * `substeps` x (grid build, density/pressure, XSPH + pressure forces, integrate with
 * collision against a `TracedField`), followed by `SplatField.bake`
 * (lib/src/sim/splat.ts:296-304). Every entry point below replaces one member of the
 * reference's `FluidSim` / `SplatField` / `SdfVolume` / `ParticleCloud` surface; the
 * comment on each names the reference interface (file:line) it stands in for.
 *
 * Conventions
 *  - Every function returns 0 on success or a negative CLAY_E* code; the message of the
 *    last failure on the calling thread is `clay_last_error()`. Where the reference throws
 *    an `Error`, the same condition returns CLAY_EINVAL with the reference's message text.
 *  - Real-valued options are `double`: the reference's options are JavaScript numbers
 *    (binary64) and its host-side derivations (voxel size, rest density, wall box) are done
 *    in binary64 before they are rounded once to f32 for the device.
 *  - Work is enqueued on the caller's CUDA stream (`void* stream` is a `cudaStream_t`,
 *    NULL = the legacy default stream) and never blocks, which is what "records into a
 *    caller-owned compute pass" means in the reference. Readbacks are asynchronous copies
 *    into caller memory; synchronise the stream before reading them.
 *  - The library owns all device memory it allocates; `*_destroy` frees it. The caller owns
 *    streams and host buffers.
 */
#ifndef CLAY_FLUID_H
#define CLAY_FLUID_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CLAY_OK 0
#define CLAY_EINVAL (-1)   /* bad argument / option (reference: constructor throws) */
#define CLAY_ECUDA (-2)    /* a CUDA runtime call failed */
#define CLAY_ENOMEM (-3)   /* device allocation failed or the HBM budget is exceeded */
#define CLAY_ESTATE (-4)   /* call not valid in the object's current state */
#define CLAY_ETIMEOUT (-5) /* a bounded device-side wait gave up */

/* Thread-local message of the last failing call on this thread ("" if none). */
const char* clay_last_error(void);
/* Library version string. */
const char* clay_version(void);

/* ------------------------------------------------------------------------------------
 * Context: binds a CUDA device. Replaces the `TgpuRoot` every reference constructor takes
 * (fluid.ts:140, splat.ts:147, volume.ts:139).
 * ---------------------------------------------------------------------------------- */
typedef struct clay_ctx clay_ctx;
int clay_ctx_create(int device, clay_ctx** out);
void clay_ctx_destroy(clay_ctx* ctx);
/* Bytes of device memory currently allocated by objects of this context. */
int clay_ctx_bytes_in_use(const clay_ctx* ctx, uint64_t* out);

/* ------------------------------------------------------------------------------------
 * SdfVolume (lib/src/field/volume.ts:36-62 options, :139-314 class).
 *
 * Device layout: per mip level m (resolution R_m = resolution >> m) one f16 plane of
 * band-normalised distance (`.r` of the reference's rgba16float texel) and one f16 plane of
 * material (`.g`), each x-fastest then y then z, levels concatenated. The constant `.b`/`.a`
 * channels (0, 1) are not stored.
 * ---------------------------------------------------------------------------------- */
typedef struct clay_volume clay_volume;

enum {
  CLAY_VOL_RESOLUTION = 1u << 0,
  CLAY_VOL_WORLD_SIZE = 1u << 1,
  CLAY_VOL_ORIGIN = 1u << 2,
  CLAY_VOL_MIP_LEVELS = 1u << 3,
  CLAY_VOL_BAND = 1u << 4,
  CLAY_VOL_GRADIENT_VOXELS = 1u << 5,
};

/* `SdfVolumeOptions` (volume.ts:36-62). A field whose bit is clear in `set` takes the
 * reference default (`??` at volume.ts:140-154,299). */
typedef struct clay_volume_opts {
  uint32_t set;
  int32_t resolution;      /* ?? 128 */
  double world_size;       /* ?? 16 */
  double origin[3];        /* ?? [0,0,0] */
  int32_t mip_levels;      /* ?? derived from resolution (volume.ts:148-151) */
  double band;             /* ?? 4 */
  double gradient_voxels;  /* ?? 1 */
} clay_volume_opts;

/* Read-only description of a volume (the reference's public fields). */
typedef struct clay_volume_info {
  int32_t resolution;
  int32_t mip_levels;
  double world_size;
  double voxel_size;       /* mip 0 */
  double band;
  double origin[3];
  int32_t tile_res_per_mip[16];
  int64_t level_offset[16]; /* voxel offset of each level inside the concatenated planes */
  int64_t total_voxels;
  int32_t total_cells;      /* tile records, volume.ts:172-179 */
} clay_volume_info;

/* new SdfVolume(root, options) (volume.ts:139). Errors with the reference's message when
 * the resolution cannot carry the mip chain (volume.ts:156-160). */
int clay_volume_create(clay_ctx* ctx, const clay_volume_opts* opts, clay_volume** out);
void clay_volume_destroy(clay_volume* vol);
int clay_volume_get_info(const clay_volume* vol, clay_volume_info* out);
/* SdfVolume.setOrigin (volume.ts:327-334). */
int clay_volume_set_origin(clay_volume* vol, double x, double y, double z);
/* voxelSizeAt (volume.ts:336-338). */
double clay_volume_voxel_size_at(const clay_volume* vol, int mip);
/* Device views of the f16 distance and material planes (all levels). */
int clay_volume_device_planes(clay_volume* vol, void** dist_f16, void** material_f16);
/* Host <-> device copies of whole planes (all levels, `total_voxels` halves each). Either
 * pointer may be NULL to skip that plane. Asynchronous on `stream`. */
int clay_volume_upload(clay_volume* vol, const uint16_t* dist_f16, const uint16_t* material_f16,
                       void* stream);
int clay_volume_download(const clay_volume* vol, uint16_t* dist_f16, uint16_t* material_f16,
                         void* stream);
/* The reference's texel layout: one level as interleaved rgba16float (r=dist, g=material,
 * b=0, a=1), 4 halves per voxel, written into host memory. */
int clay_volume_download_rgba16f(const clay_volume* vol, int mip, uint16_t* rgba, void* stream);

/* One brush record, laid out exactly as the reference's `Brush` struct (brush.ts:52-78,
 * 80 bytes). Produced on the host by the reference's `BrushSet.make` rule. */
typedef struct clay_brush {
  float pos[3];
  float scale;
  float rot[4];   /* xyzw */
  float size[3];
  float radius;
  float material;
  float blend;
  float bound;
  float mask;
  uint32_t kind;
  uint32_t op;
  uint32_t slot;
  uint32_t pad;
} clay_brush;

/* SdfBuilder.setBrushes + rebuild (lib/src/field/builder.ts:147-172): folds the brush list,
 * in order, into every mip level of the volume on the device. Brushes beyond 256 are
 * dropped as in builder.ts:148-153. */
int clay_volume_build_brushes(clay_volume* vol, const clay_brush* brushes, int count, void* stream);

/* ------------------------------------------------------------------------------------
 * TracedField as a collider (lib/src/trace/field.ts:20-73). Only what the fluid reads:
 * `sample(p, 0).x` and `normal(p)`.
 * ---------------------------------------------------------------------------------- */
typedef struct clay_field clay_field;
/* volumeField(volume) (trace/field.ts:102-180). */
int clay_field_from_volume(clay_volume* vol, clay_field** out);
/* unionField(a, b) (trace/field.ts:246-315). At most 8 volume leaves in total. */
int clay_field_union(const clay_field* a, const clay_field* b, clay_field** out);
/* offsetField(field, offset) (trace/field.ts:396-429) with a host-set translation. */
int clay_field_offset(const clay_field* f, double dx, double dy, double dz, clay_field** out);
int clay_field_set_offset(clay_field* f, double dx, double dy, double dz);
void clay_field_destroy(clay_field* f);
/* Evaluates the collider at `n` points on the device (test/debug hook): writes
 * `sample(p,0)` as (x,y) pairs into `sample_xy` and `normal(p)` as xyz triples into `nrm`.
 * All pointers are host memory; the call synchronises `stream`. */
int clay_field_query(const clay_field* f, const float* points_xyz, int n, float* sample_xy,
                     float* nrm, void* stream);
/* TracedField.sample(p, mip) and field(p, mip) (trace/field.ts:135-150, 264-293, 396-415)
 * at n host points, the level capped at each volume's top level (:117-124): per point the
 * (distance, raw) and (distance, material) pairs. Test and tool hook (allocates). */
int clay_field_query_mip(const clay_field* f, const float* pts, int n, int mip, float* sample_xy, float* field_xy,
                         void* stream);
/* The same with every pointer in device memory, asynchronous on `stream`, allocating nothing:
 * sampling by a device-side consumer of the baked volume (the reference's tracer samples the
 * same way from its shaders). */
int clay_field_query_mip_device(const clay_field* f, const float* pts, int n, int mip, float* sample_xy,
                                float* field_xy, void* stream);
/* bandWorld(mip) and voxelWorld(mip) of the field (trace/field.ts:151-155, 294-305): the
 * smallest band and the largest voxel over the union's volumes, each at its capped level. */
int clay_field_band_voxel(const clay_field* f, int mip, float* band_world, float* voxel_world);

/* ------------------------------------------------------------------------------------
 * ParticleCloud (lib/src/sim/splat.ts:15-38) and bodyCloud (splat.ts:47-72).
 * ---------------------------------------------------------------------------------- */
enum {
  CLAY_LIVE_ALL = 0,    /* liveAt(i) = true */
  CLAY_LIVE_COUNT = 1,  /* liveAt(i) = i < *live_count                 (fluid.ts:221-224) */
  CLAY_LIVE_RANGE = 2,  /* liveAt(i) = first <= i < first + count       (splat.ts:56-60) */
};

typedef struct clay_cloud_desc {
  uint32_t capacity;            /* the dispatch bound */
  const void* positions;        /* device: float[3] at the start of each record */
  uint32_t position_stride;     /* bytes between records */
  uint32_t live_mode;           /* CLAY_LIVE_* */
  const uint32_t* live_count;   /* device u32, CLAY_LIVE_COUNT */
  const uint32_t* live_first;   /* device u32, CLAY_LIVE_RANGE */
  const uint32_t* live_range_count; /* device u32, CLAY_LIVE_RANGE */
  const void* normals;          /* device float[3] per record, or NULL: no normalAt */
  uint32_t normal_stride;       /* bytes */
  const float* rotation;        /* device xyzw quaternion applied to normals, or NULL */
} clay_cloud_desc;

/* ------------------------------------------------------------------------------------
 * SplatField (lib/src/sim/splat.ts:74-106 options, :136-309 class).
 * ---------------------------------------------------------------------------------- */
typedef struct clay_splat clay_splat;

enum {
  CLAY_SPLAT_MATERIAL = 1u << 0,
  CLAY_SPLAT_RESOLUTION = 1u << 1,
  CLAY_SPLAT_MIP_LEVELS = 1u << 2,
  CLAY_SPLAT_BAND = 1u << 3,
  CLAY_SPLAT_ORIGIN = 1u << 4,
  CLAY_SPLAT_WORLD_SIZE = 1u << 5,
};

typedef struct clay_splat_opts {
  uint32_t set;
  double radius;          /* required */
  double material;        /* ?? 0 */
  int32_t resolution;     /* ?? 64 */
  int32_t mip_levels;     /* ?? max(1, log2(res / 8) | 0) (splat.ts:149) */
  double band;            /* ?? 2 */
  double origin[3];       /* ?? [-12,-4,-12] */
  double world_size;      /* ?? 24 */
} clay_splat_opts;

/* new SplatField(root, cloud, options) (splat.ts:147). */
int clay_splat_create(clay_ctx* ctx, const clay_cloud_desc* cloud, const clay_splat_opts* opts,
                      clay_splat** out);
void clay_splat_destroy(clay_splat* s);
/* SplatField.setCenter (splat.ts:284-287). */
int clay_splat_set_center(clay_splat* s, double x, double y, double z);
/* SplatField.bake (splat.ts:296-304). */
int clay_splat_bake(clay_splat* s, void* stream);
/* Measurement hook, no counterpart in the reference: the (particle, voxel) pairs a bake of
 * the cloud as it is now lowers (sd < bandWorld, splat.ts:246), over every level.
 * Allocates a small temporary and synchronises `stream`. */
int clay_splat_census(clay_splat* s, void* stream, uint64_t* pairs_out);
/* A SplatField bake that allocates no device memory. No counterpart in the reference: it
 * is for callers that may not allocate once running - a per-frame tick where cudaMalloc or
 * cudaFree would synchronise the device and stall the frame, or a plugin host that gives
 * the library only buffers allocated up front. The caller passes the cloud and the output
 * planes (`dist_out_f16`, and `material_out_f16` or NULL; total-voxel halves each, levels
 * concatenated as in an SdfVolume); options as clay_splat_create, origin taken from
 * `opts` (default [-12,-4,-12]). Output is bit for bit that of clay_splat_bake.
 * Limit: at most CLAY_STATIC_BAKE_MAX_VOXELS voxels over all levels (e.g. 96^3 with 3
 * levels); larger bakes are refused with CLAY_EINVAL. The key scratch is one fixed
 * file-scope device array (4 MiB, held by every GPU that loads the library until exit)
 * shared by every call: each call clears it before use, and calls that overlap on the GPU
 * race on it, so order them. The first call on each device also looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream capture. */
#define CLAY_STATIC_BAKE_MAX_VOXELS 1048576
int clay_splat_bake_static(const clay_cloud_desc* cloud, const clay_splat_opts* opts, void* dist_out_f16,
                           void* material_out_f16, void* stream);
/* SplatField.volume / .field. The returned objects are owned by the splat. */
clay_volume* clay_splat_volume(clay_splat* s);
clay_field* clay_splat_field(clay_splat* s);
/* Test hook: during the next bakes, copy each voxel's 16-bit key (the u32 the reference
 * `atomicMin`s, splat.ts:247-249) into `keys_device` (total_voxels u32) as the resolve pass
 * computes it. NULL turns it off. */
int clay_splat_capture_keys(clay_splat* s, uint32_t* keys_device);

/* ------------------------------------------------------------------------------------
 * FluidSim (lib/src/sim/fluid.ts:60-91 options, :111-582 class).
 * ---------------------------------------------------------------------------------- */
typedef struct clay_fluid clay_fluid;

enum {
  CLAY_FLUID_CAPACITY = 1u << 0,
  CLAY_FLUID_SPACING = 1u << 1,
  CLAY_FLUID_SMOOTHING = 1u << 2,
  CLAY_FLUID_BUCKET = 1u << 3,
  CLAY_FLUID_RADIUS = 1u << 4,
  CLAY_FLUID_SURFACE_RADIUS = 1u << 5,
  CLAY_FLUID_MATERIAL = 1u << 6,
  CLAY_FLUID_BAKE_RESOLUTION = 1u << 7,
  CLAY_FLUID_BAKE_MIP_LEVELS = 1u << 8,
  CLAY_FLUID_BAKE_BAND = 1u << 9,
  CLAY_FLUID_ORIGIN = 1u << 10,
  CLAY_FLUID_WORLD_SIZE = 1u << 11,
  CLAY_FLUID_SUBSTEPS = 1u << 12,
  CLAY_FLUID_GRAVITY = 1u << 13,
  CLAY_FLUID_STIFFNESS = 1u << 14,
  CLAY_FLUID_VISCOSITY = 1u << 15,
  CLAY_FLUID_DAMPING = 1u << 16,
  CLAY_FLUID_MAX_SPEED = 1u << 17,
};

/* `FluidSimOptions` (fluid.ts:60-91); unset fields take the `??` defaults of
 * fluid.ts:141-160,184-203. */
typedef struct clay_fluid_opts {
  uint32_t set;
  int64_t capacity;        /* ?? 8192; at most 2^26 (the neighbour list is addressed in 32-bit words) */
  double spacing;          /* ?? 0.45 */
  double smoothing;        /* ?? spacing * 2.2 */
  int32_t bucket;          /* ?? 64 */
  double radius;           /* ?? spacing * 0.5 */
  double surface_radius;   /* ?? spacing * 1.1 */
  double material;         /* ?? 0 */
  int32_t bake_resolution; /* ?? 64 */
  int32_t bake_mip_levels; /* ?? max(1, log2(bakeRes / 8) | 0) */
  double bake_band;        /* ?? 2 */
  double origin[3];        /* ?? [-12,-4,-12] */
  double world_size;       /* ?? 24 */
  int32_t substeps;        /* ?? 3 */
  double gravity[3];       /* ?? [0,-9.81,0] */
  double stiffness;        /* ?? 220 */
  double viscosity;        /* ?? 0.4 */
  double damping;          /* ?? 0.995 */
  double max_speed;        /* ?? 15 */
} clay_fluid_opts;

/* `FluidParams` (fluid.ts:28-51): the 80-byte per-frame uniform, WGSL layout. */
typedef struct clay_fluid_params {
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
} clay_fluid_params;

/* Fields `configure` may patch (fluid.ts:528: everything except the emission cursor). */
enum {
  CLAY_P_GRAVITY = 1u << 0,
  CLAY_P_DT = 1u << 1,
  CLAY_P_EMIT_POS = 1u << 2,
  CLAY_P_EMIT_RADIUS = 1u << 3,
  CLAY_P_EMIT_VEL = 1u << 4,
  CLAY_P_MAX_SPEED = 1u << 5,
  CLAY_P_STIFFNESS = 1u << 6,
  CLAY_P_VISCOSITY = 1u << 7,
  CLAY_P_DAMPING = 1u << 8,
  CLAY_P_CONTACT_DEPTH = 1u << 9,
};

/* One `FluidParticle` record (fluid.ts:20-26): WGSL layout, 48-byte stride. */
typedef struct clay_fluid_particle {
  float pos[3];
  float density;
  float vel[3];
  float pressure;
  float nvel[3];
  float pad;
} clay_fluid_particle;

/* `ContactList` (fluid.ts:55-58): WGSL layout (points start at byte 16). */
typedef struct clay_contact_list {
  uint32_t count;
  uint32_t pad[3];
  float points[32][4];
} clay_contact_list;

/* Arithmetic of the SPH passes. REFERENCE follows the reference's operation order with no
 * fused multiply-add and plain f32 sums, and reproduces the f32 CPU restatement bit for
 * bit. FAST (the default) lets the compiler contract multiply-adds and accumulates density
 * with compensated (Kahan-Neumaier) summation. The bake is exact in both modes. */
enum { CLAY_MODE_FAST = 0, CLAY_MODE_REFERENCE = 1 };

/* new FluidSim(root, world, options) (fluid.ts:140). `world` may be NULL (no collider). */
int clay_fluid_create(clay_ctx* ctx, const clay_field* world, const clay_fluid_opts* opts,
                      clay_fluid** out);
void clay_fluid_destroy(clay_fluid* sim);
int clay_fluid_set_mode(clay_fluid* sim, int mode);
/* FluidSim.spawn (fluid.ts:511-525). `spread` NULL = the reference default
 * `spacing * cbrt(max(n,1)) * 0.62`. */
int clay_fluid_spawn(clay_fluid* sim, int64_t n, const double pos[3], const double vel[3],
                     const double* spread);
/* FluidSim.configure (fluid.ts:528-530). `mask` = CLAY_P_* bits naming patched fields. */
int clay_fluid_configure(clay_fluid* sim, const clay_fluid_params* patch, uint32_t mask);
/* FluidSim.step (fluid.ts:536-558): emit, substeps, bake, enqueued on `stream`. */
int clay_fluid_step(clay_fluid* sim, void* stream);
/* FluidSim.particleCount (fluid.ts:496-498). */
int64_t clay_fluid_particle_count(const clay_fluid* sim);
/* The host copy of the uniform as the next step will write it (`frozen`, fluid.ts:185-203). */
int clay_fluid_get_params(const clay_fluid* sim, clay_fluid_params* out);
/* FluidSim.readContacts (fluid.ts:565-569): copies the raw ContactList into `host_out`
 * asynchronously; n = min(count, 32) once the stream has completed. */
int clay_fluid_read_contacts_async(clay_fluid* sim, clay_contact_list* host_out, void* stream);
/* FluidSim.particles (fluid.ts:116): device pointer to `capacity` FluidParticle records. */
int clay_fluid_particles_device(clay_fluid* sim, clay_fluid_particle** ptr, uint32_t* stride);
/* Test hook: writes `count` records into slots [0, count) and sets the live count and the
 * emission cursor to `count` (the reference can only emit jittered balls). Asynchronous. */
int clay_fluid_upload(clay_fluid* sim, const clay_fluid_particle* host, int64_t count, void* stream);
int clay_fluid_download(const clay_fluid* sim, clay_fluid_particle* host, int64_t count, void* stream);
/* Test hook: the reference's `cellIndex` (fluid.ts:258-262) of each of the first
 * particleCount particles, or 0xffffffff for a particle outside the grid (fluid.ts:319-321).
 * Host output; synchronises `stream`. */
int clay_fluid_cell_indices(clay_fluid* sim, uint32_t* host_out, void* stream);
/* Measurement hook, no counterpart in the reference: the algorithmic work of the frame the
 * last clay_fluid_step did, counted with the reference's own arithmetic. `candidates` are
 * the neighbours the density pass tests (fluid.ts:346-364) and `accepted` those within the
 * smoothing length (self included, :357-361), both over the cell order of the LAST substep
 * (multiply by the substeps for a frame); `splat_pairs` are the (particle, voxel) pairs of
 * the surface bake with sd < bandWorld (splat.ts:246: the reference's atomicMin count), over
 * every level. Allocates a small temporary and synchronises `stream`. */
typedef struct clay_census {
  uint64_t particles;
  uint64_t candidates;
  uint64_t accepted;
  uint64_t splat_pairs;
} clay_census;
int clay_fluid_census(clay_fluid* sim, void* stream, clay_census* out);
/* FluidSim.surface / .field (fluid.ts:119-120); owned by the sim. */
clay_splat* clay_fluid_surface(clay_fluid* sim);
clay_field* clay_fluid_field(clay_fluid* sim);
/* Derived constants, for tests: h, rest density, grid resolution, grid origin. */
typedef struct clay_fluid_info {
  int64_t capacity;
  int32_t substeps;
  int32_t bucket;
  int32_t grid_res;
  double smoothing;
  double rest_density;
  double grid_origin[3];
  double spacing;
  double radius;
  uint64_t device_bytes;
} clay_fluid_info;
int clay_fluid_get_info(const clay_fluid* sim, clay_fluid_info* out);

/* ------------------------------------------------------------------------------------
 * Batched stepping (no reference counterpart: the reference steps one FluidSim per
 * `FluidSim.step`). Independent scenes of uneven size advance one frame each per launch:
 * every pass of the frame runs once for all scenes, and the whole frame is captured into
 * one CUDA graph.
 * ---------------------------------------------------------------------------------- */
typedef struct clay_batch clay_batch;
int clay_batch_create(clay_ctx* ctx, clay_fluid* const* sims, int n, clay_batch** out);
void clay_batch_destroy(clay_batch* b);
/* Extra clouds baked in the same launch (e.g. clay-body shells), before the fluid steps. */
int clay_batch_add_splat(clay_batch* b, clay_splat* s);
/* Tile shapes: threads per block of the particle passes and particles per block. */
typedef struct clay_batch_tuning {
  int32_t sph_block;     /* threads per block of the particle passes: 64..256, multiple of 32 */
  int32_t splat_block;   /* threads per block of the splat pass: 64..512 */
  int32_t use_graph;     /* 1: capture the frame into a CUDA graph */
} clay_batch_tuning;
int clay_batch_set_tuning(clay_batch* b, const clay_batch_tuning* t);
int clay_batch_get_tuning(const clay_batch* b, clay_batch_tuning* t);
/* Per scene-size bucket block sizes of the particle passes (the autotuner's output): a scene
 * whose capacity is below upper[i] uses blocks[i] threads per block; larger scenes use the
 * batch's sph_block. upper[] increasing; blocks[] multiples of 32 in 64..256. */
int clay_batch_set_bucket_blocks(clay_batch* b, const int64_t* upper, const int32_t* blocks, int n);
/* The autotuner's full output, per scene-size bucket: bucket i < n holds the scenes whose
 * capacity is below upper[i] (and not below upper[i-1]); bucket n the rest, so `t` has n + 1
 * entries. Every choice gives the same results (reference mode bit for bit): they only move
 * time between the passes' strategies. */
typedef struct clay_bucket_tuning {
  int32_t sph_block;          /* threads per block of the particle passes, 64..256, multiple of 32 */
  int32_t density_variant;    /* 0: one loop (default); 1: distance tests, then the accepted
                                  neighbours; 2: one loop over neighbours staged in shared memory */
  int32_t splat_tile_ratio;   /* sphere blocks take the tile walk up to this many times their pairs (6) */
  int32_t splat_walk_weight;  /* blocks take the block walk up to this many times their pairs (3) */
  int32_t forces_split;       /* 1: the forces pass without the integrate, then the integrate as a
                                  launch of its own; 0: one fused pass (default) */
} clay_bucket_tuning;
int clay_batch_set_bucket_tuning(clay_batch* b, const int64_t* upper, const clay_bucket_tuning* t, int n);
/* No counterpart in the reference: split the scenes into `lanes` (1..8, default 1) groups of
 * about equal particle counts, each stepped as its own chain of launches on its own stream
 * inside the frame, so the groups' passes run side by side on the GPU. Same results. */
int clay_batch_set_lanes(clay_batch* b, int lanes);
/* One frame for every scene: host bookkeeping of each sim (as clay_fluid_step), then the
 * batched passes (or the captured graph) on `stream`. */
int clay_batch_step(clay_batch* b, void* stream);
/* One frame for a subset of the batch's scenes (indices, each at most once): the other
 * scenes keep their state. Work tables are sized from the listed scenes' live counts and
 * uploaded with their uniforms in one copy; no graph. The batch's extra clouds are not baked.
 * This is the launch of the continuous-batching server. */
int clay_batch_step_subset(clay_batch* b, const int32_t* scenes, int n, void* stream);
/* The ContactList of every scene, in batch order, copied into `host_out` (n records)
 * asynchronously: one gather launch and one device-to-host copy. */
int clay_batch_read_contacts_async(clay_batch* b, clay_contact_list* host_out, void* stream);
/* One frame of the batch without the graph, each kernel bracketed by CUDA events on
 * `stream`; per kernel (summed over substeps) its total milliseconds and launch count. */
typedef struct clay_phase_time {
  char name[32];
  float ms;
  int32_t launches;
} clay_phase_time;
int clay_batch_profile(clay_batch* b, void* stream, clay_phase_time* out, int cap, int* n_out);
/* Kernel launches one clay_batch_step enqueues (graph nodes count as launches). */
int clay_batch_launches_per_step(const clay_batch* b, int64_t* out);

/* ------------------------------------------------------------------------------------
 * SurfaceExtractor (lib/src/sim/extract.ts:84-484): naive surface nets of a field's zero
 * level set on a res^3 lattice, written into a caller-owned ParticleSet: one 96-byte
 * Particle record (particles.ts:18-34) per dual vertex in the slice [base, base+capacity),
 * a quad index list (6 indices per quad, extract.ts:330-350), and the body record's first,
 * count, rest centre of mass, centre of mass and rotation (64-byte Body, particles.ts:52-68)
 * plus indirect draw arguments (extract.ts:395-436). Particle and quad slots come in lattice
 * order (the reference's atomics leave the order unspecified).
 * ---------------------------------------------------------------------------------- */
typedef struct clay_extractor clay_extractor;
#define CLAY_EXTRACT_RESOLUTION (1u << 0)
typedef struct clay_extractor_opts {
  uint32_t set;        /* CLAY_EXTRACT_RESOLUTION: `resolution` given, else 32 (extract.ts:99) */
  int32_t resolution;  /* lattice cells per axis */
  int32_t body;        /* body index in the set */
  int32_t base;        /* first particle of this body's slice */
  int32_t capacity;    /* particles the extractor may emit */
  int32_t pad;
  /* optional ExtractMotion (extract.ts:30-45): 8 device floats (centre xyz, pad, velocity
   * xyz, pad), owned by the caller; the region is then relative to its centre, emitted
   * particles take its velocity, and preserveMotion refreshes it from the live body */
  float* motion;
} clay_extractor_opts;
/* `particles` (set_capacity records) and `bodies` (max_bodies records): device memory,
 * 16-byte aligned, owned by the caller. The field must outlive the extractor. Refuses a
 * slice past the set's capacity with the reference's message (extract.ts:101-103). */
int clay_extractor_create(clay_ctx* ctx, const clay_field* field, void* particles, int64_t set_capacity, void* bodies,
                          int32_t max_bodies, const clay_extractor_opts* opts, clay_extractor** out);
void clay_extractor_destroy(clay_extractor* x);
/* setRegion (extract.ts:451-463): cell = size / resolution; with motion, origin is relative
 * to the motion's centre and preserve_motion snapshots the body's current centre and mean
 * velocity into it at the next extraction. */
int clay_extractor_set_region(clay_extractor* x, const double origin[3], double size, const double vel[3],
                              int preserve_motion);
/* extract (extract.ts:469-475): reset, cells, quads, finish, on `stream`. The eight passes
 * run as one CUDA graph that the first call captures (on a private stream) and later calls
 * replay; every pass reads the region and motion from device memory, so setRegion between
 * calls needs no new graph. */
int clay_extractor_extract(clay_extractor* x, void* stream);
/* Device views: the quad index list (quad_capacity * 6 u32) and the 4 draw arguments. */
int clay_extractor_views(clay_extractor* x, uint32_t** indices, uint32_t** draw_args, int64_t* quad_capacity);
/* The extraction's dual-vertex and quad counts before the capacity clamps (SimCounters). */
int clay_extractor_read_counts_async(clay_extractor* x, uint32_t* host_counts, void* stream);
/* The quad index list (quad_capacity * 6 u32) and the 4 draw arguments, into host memory. */
int clay_extractor_read_indices_async(clay_extractor* x, uint32_t* host_indices, uint32_t* host_draw_args, void* stream);
/* offsetField(field, () => offset) with the offset read from device memory at every sample
 * (trace/field.ts:396-429), e.g. an ExtractMotion's centre, so a body-local field follows
 * the centre an extraction computes on the GPU. `device_offset`: 3 floats that must outlive
 * the field. */
int clay_field_offset_device(const clay_field* f, const float* device_offset, clay_field** out);

/* ------------------------------------------------------------------------------------
 * ClaySolver (lib/src/sim/pbd.ts:78-424): shape-matched bodies of a ParticleSet colliding
 * against a field. Per step: the one-shot kick, then `substeps` x (BDF2 predict with world
 * collision and positional friction, per-body shape match with the polar rotation of
 * math/gpu.ts:55-77, pull and projection with plasticity, velocity finalize). Particles and
 * bodies are the caller's device buffers (96- and 64-byte records, particles.ts:18-68).
 * ---------------------------------------------------------------------------------- */
typedef struct clay_solver clay_solver;
#define CLAY_SOLVER_GRAVITY (1u << 0)
#define CLAY_SOLVER_DT (1u << 1)
#define CLAY_SOLVER_SUBSTEPS (1u << 2)
#define CLAY_SOLVER_RADIUS (1u << 3)
#define CLAY_SOLVER_FRICTION (1u << 4)
#define CLAY_SOLVER_DAMPING (1u << 5)
#define CLAY_SOLVER_MAX_SPEED (1u << 6)
#define CLAY_SOLVER_ROTATION_ITERATIONS (1u << 7)
/* ClaySolverOptions (pbd.ts:44-55); unset options take the reference's defaults: gravity
 * (0,-9.81,0), dt 1/60, substeps 2, radius 0.1, friction 0.35, damping 0.995, maxSpeed 40,
 * rotationIterations 2 (pbd.ts:101-118). */
typedef struct clay_solver_opts {
  uint32_t set;
  int32_t substeps;
  double gravity[3];
  double dt;
  double radius;
  double friction;
  double damping;
  double max_speed;
  int32_t rotation_iterations;
  int32_t pad;
} clay_solver_opts;
int clay_solver_create(clay_ctx* ctx, const clay_field* world, void* particles, int64_t capacity, void* bodies,
                       int32_t max_bodies, const clay_solver_opts* opts, clay_solver** out);
void clay_solver_destroy(clay_solver* s);
/* setForce (pbd.ts:376-398): a uniform acceleration of one body for the next steps and a
 * one-shot velocity change (`impulse`, may be NULL) applied once by the next step. */
int clay_solver_set_force(clay_solver* s, uint32_t body, const double accel[3], const double impulse[3]);
/* step (pbd.ts:396-416) over the set's first `body_count` bodies, on `stream`. The substeps'
 * passes run as one CUDA graph, captured (on a private stream) at the first step and again
 * when `body_count` changes; the impulse of set_force is a separate launch before it. */
int clay_solver_step(clay_solver* s, int32_t body_count, void* stream);

/* ------------------------------------------------------------------------------------
 * Continuous-batching server (no reference counterpart: the reference steps the scenes of
 * one game). Serves requests "advance scene i by k frames" (each frame: FluidSim.step with
 * its bake) over many registered scenes. Each frame it launches one clay_batch_step_subset
 * over the scenes with a request in progress; requests arriving while frames run join at the
 * next frame boundary; up to `depth` frames are in flight. Scenes become resident (their
 * FluidSim created) when a request needs them, within a device-byte budget: idle scenes are
 * evicted least-recently-used first, keeping their particle state on the host, and get it
 * back on return. Colliders stay owned by the caller and must outlive the server.
 * One host thread per server; all device work goes to the server's stream.
 * ---------------------------------------------------------------------------------- */
typedef struct clay_server clay_server;
typedef struct clay_server_opts {
  uint64_t budget_bytes; /* device bytes the resident scenes may hold; 0: no limit */
  int32_t depth;         /* frames in flight, 1..8; 0: 2 */
  int32_t max_batch;     /* scenes stepped per frame; 0: every scene with a request */
  int32_t mode;          /* CLAY_MODE_FAST or CLAY_MODE_REFERENCE */
  int32_t sph_block;     /* threads per block of the particle passes; 0: the batch default */
} clay_server_opts;
int clay_server_create(clay_ctx* ctx, const clay_server_opts* opts, void* stream, clay_server** out);
/* Waits for the frames in flight, then frees every resident scene. */
void clay_server_destroy(clay_server* s);
/* Registers a scene (not resident until a request needs it): its FluidSim options, the
 * collider it collides with (may be NULL) and its initial particles (copied; count <= the
 * capacity). Its id is returned in `scene_out` (0, 1, 2, ... in registration order). */
int clay_server_add_scene(clay_server* s, const clay_field* world, const clay_fluid_opts* opts,
                          const clay_fluid_particle* particles, int64_t count, int32_t* scene_out);
/* Queues `frames` (>= 1) frames of `scene`, arriving now (the host's steady clock). A scene's
 * requests run one after another in submission order. */
int clay_server_submit(clay_server* s, int32_t scene, int32_t frames, int64_t* ticket_out);
/* One scheduling step, without waiting on the device: retire completed frames, admit scenes
 * that have requests, launch at most one frame. `launched` (may be NULL): 1 if it did. */
int clay_server_pump(clay_server* s, int32_t* launched);
/* Waits until the oldest frame in flight completes (and retires it), or `timeout_ms` passes
 * (< 0: no limit). Returns at once when nothing is in flight. */
int clay_server_wait(clay_server* s, double timeout_ms);
/* Pumps, waiting on the oldest frame when nothing can launch, until every submitted request
 * is done. CLAY_ENOMEM when a waiting scene can never fit the budget. */
int clay_server_drain(clay_server* s);
/* done = 1 once the ticket's last frame has completed on the device; latency_ms = that
 * completion minus the submission, on one clock (a CUDA event tied to the host clock). */
int clay_server_poll(const clay_server* s, int64_t ticket, int32_t* done, double* latency_ms);
typedef struct clay_server_stats {
  int64_t submitted;
  int64_t completed;
  int64_t frames;        /* batched launches */
  int64_t scene_frames;  /* scenes stepped, summed over frames */
  int64_t particle_steps;
  int64_t admissions;
  int64_t evictions;
  uint64_t resident_bytes;
  int32_t resident_scenes;
  int32_t inflight;
} clay_server_stats;
int clay_server_get_stats(const clay_server* s, clay_server_stats* out);
/* The scene's FluidSim while it is resident, else NULL (valid until the next pump). An
 * eviction keeps the particle records and their count only: a spawn made through this
 * view that is still pending, and the sim's emission seed, do not survive it. */
int clay_server_scene_sim(clay_server* s, int32_t scene, clay_fluid** sim_out);
/* The scene's particle state after all its submitted frames: waits for them, then copies
 * from the device (resident) or the host snapshot (evicted). `n_out`: live particles. */
int clay_server_download(clay_server* s, int32_t scene, clay_fluid_particle* host, int64_t cap, int64_t* n_out);
/* Device bytes a FluidSim with these options allocates (what the server budgets with). */
int clay_fluid_estimate_bytes(const clay_fluid_opts* opts, uint64_t* out);

/* ------------------------------------------------------------------------------------
 * Number of library kernel launches enqueued by this process so far (all objects).
 * ---------------------------------------------------------------------------------- */
uint64_t clay_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* CLAY_FLUID_H */
