// clay_device.cuh - device-side data layout and kernels of the fluid hot path.
//
// Included by two translation units: kern_ref.cu (compiled with -fmad=false: every f32
// expression rounds exactly as written, which is what makes the bake, the cell build and
// the reference-mode SPH passes reproduce the f32 CPU restatement bit for bit) and
// kern_fast.cu (multiply-adds contracted; compensated density sums) for the fast-mode
// neighbour passes. Kernels take a table of scenes and a table of work items, so the same
// code runs one scene per launch (the plain path) or every scene of a batch in one launch.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace clay {

constexpr uint32_t kSentinel = 0xffffffffu;
constexpr int kMaxLeaves = 8;
constexpr int kMaxParts = 64;
constexpr int kMaxMips = 8;
constexpr uint32_t kMaxNbr = 64;  // neighbour-list slots per particle
// Largest scene: the neighbour list is addressed in 32-bit words, slot-major (slot j of particle
// k at word (j / 4) * 4 * capacity + j % 4), so every such offset must stay below 2^32.
constexpr int64_t kMaxCapacity = int64_t{1} << 26;
static_assert((kMaxNbr / 4) * 4 * static_cast<uint64_t>(kMaxCapacity) <= (uint64_t{1} << 32), "list offsets");
constexpr int kSplatWarps = 8;  // warps per block of the splat pass
constexpr int kSplatItems = 2048;  // compacted (brick, slice) items of the sphere block walk
constexpr int kSplatStencil = 2048;  // voxel offsets of the own-box walk's stencil (8 KB of shared memory)
constexpr int kSplatAccVoxels = 4096;   // shared-memory minimum tile of the splat pass (spheres)
constexpr int kSplatSubtiles = 8;       // sub-boxes of that tile a sphere block's union box may take
constexpr int kSplatAccVoxelsDiscs = 4096;  // the same for oriented-disc clouds
// the tile walk decodes items (< tile voxels x warps) by multiplication, exact below 2^16
static_assert(kSplatAccVoxels <= 4096 && kSplatAccVoxels * kSplatWarps <= 65536, "item decode range");

// FluidParticle (fluid.ts:20-26): (pos, density), (vel, pressure), (nvel, pad).
struct __align__(16) ParticleDev {
  float4 a, b, c;
};

// FluidParams (fluid.ts:28-51), WGSL uniform layout, 80 bytes.
struct __align__(16) ParamsDev {
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
};
static_assert(sizeof(ParamsDev) == 80, "FluidParams layout");

// ContactList (fluid.ts:55-58).
struct __align__(16) ContactsDev {
  uint32_t count;
  uint32_t pad[3];
  float4 points[32];
};

// The f32 VolumeParams uniform of an SdfVolume (volume.ts:10-23,220-230), plus the
// gradient stencil and the plane pointers. Written by the host whenever it changes.
struct __align__(16) VolParamsDev {
  float origin[3];
  float voxel;
  float center[3];
  float extent;
  float half;
  float band;
  float grad_h;
  int32_t res;
  int32_t mips;
  int32_t pad_;
  const __half* dist;  // level 0 plane; level m follows at the sum of the finer levels' sizes
  const __half* mat;
};

// One leaf of a collider: volumeField(volume), optionally offsetField-moved by a constant
// and, outermost, by an offset read on the device (an extractor's GPU-side motion centre).
struct LeafDev {
  const VolParamsDev* vp;
  float offset[3];
  int32_t has_offset;
  const float* dyn_offset;
};

// The point in a leaf's own frame: offsetField subtracts its offset (trace/field.ts:396-429),
// the outermost one first.
__device__ __forceinline__ void leaf_point(const LeafDev& lf, float px, float py, float pz, float& qx, float& qy, float& qz) {
  qx = px;
  qy = py;
  qz = pz;
  if (lf.dyn_offset) {
    qx = qx - lf.dyn_offset[0];
    qy = qy - lf.dyn_offset[1];
    qz = qz - lf.dyn_offset[2];
  }
  if (lf.has_offset) {
    qx = qx - lf.offset[0];
    qy = qy - lf.offset[1];
    qz = qz - lf.offset[2];
  }
}
struct __align__(16) FieldDev {
  int32_t n;
  int32_t pad[3];
  LeafDev leaf[kMaxLeaves];
};

// Per-scene cell-build state. `lo`/`hi_inv` accumulate the bounding box of occupied cells
// (both with atomicMin; hi is stored complemented); the derived box is written once per
// substep by the count pass and read by the later passes.
struct __align__(16) GridState {
  uint32_t lo[3];
  uint32_t hi_inv[3];
  uint32_t overflow;
  uint32_t L;  // bbox cells; local index L is the out-of-grid bucket
  int32_t x0, y0, z0;
  uint32_t bx, by, bz;
  uint32_t part_sum[kMaxParts];
};

// One FluidSim as the kernels see it. Constants are the f32 literals of fluid.ts,
// computed in binary64 on the host and rounded once.
struct __align__(16) SceneDev {
  ParticleDev* parts;
  ParamsDev* prm;
  ContactsDev* contacts;
  GridState* gs;
  uint32_t* key;
  uint32_t* rank;
  uint32_t* tmp;
  uint32_t* sorted_id;
  float4* spos;
  float4* svel;
  float4* sdp;  // density, pressure, 1/density (the reference's per-pair `1 / other.density`), neighbours
  // what the forces pass reads of a neighbour, in two 16-byte records: spx = position and
  // 1/density (written by the density pass), svel = velocity and pressure (.w written by it)
  float4* spx;
  uint4* nbr;  // accepted neighbours of the density pass, 4 per entry, slot-major: nbr[(j / 4) * capacity + k]
  uint32_t* counts;
  uint32_t* cell_start;
  const FieldDev* world;
  float h, h2, inv_h, h6, mass, mass_poly6, spiky, rest, rest_floor, radius;
  float gorig[3], wlo[3], whi[3];
  int32_t G;
  uint32_t capacity, bucket, parts_scan;
  int32_t substeps;
  int32_t pad_[3];
};

// A ParticleCloud plus the SplatField it bakes into (splat.ts:136-276).
struct __align__(16) SplatDev {
  const char* pos;
  const char* nrm;
  const float* quat;
  const uint32_t* order;  // optional iteration order (the fluid's cell order)
  const uint32_t* live_count;
  const uint32_t* live_first;
  const uint32_t* live_range_count;
  uint32_t* keys;
  __half* dist_out;
  uint32_t* key_capture;
  const VolParamsDev* vp;
  uint32_t pos_stride, nrm_stride, capacity, live_mode;
  int32_t mips;
  float radius;
  int32_t r[kMaxMips];
  long long off[kMaxMips];
  float voxel[kMaxMips], bw[kMaxMips], reach[kMaxMips], inv_voxel[kMaxMips];
  long long total;
  // Strategy thresholds of the splat (every strategy gives the same keys): a sphere block takes
  // the register-blocked tile walk while its union box holds at most tile_ratio times the pairs
  // of the particles' own boxes; the block walk is taken while its pairs (x2 for discs) are at
  // most walk_weight times those of the own boxes.
  uint32_t tile_ratio, walk_weight;
};
constexpr uint32_t kSplatTileRatio = 6, kSplatWalkWeight = 3;

// A unit of work of one launch: object index (scene or splat), sub-index (mip level or
// scan part), first element, element count.
struct Work {
  uint32_t obj, sub, first, n;
};

// A SurfaceExtractor (extract.ts:84-484) as the kernels see it: the field, the caller's
// ParticleSet (96-byte Particle and 64-byte Body records), the scratch of one extraction,
// the region uniform and the optional GPU-side motion (centre xyz, pad, velocity xyz, pad).
struct __align__(16) ExtractDev {
  const FieldDev* field;
  unsigned char* particles;
  unsigned char* bodies;
  float* motion;
  uint32_t* id_grid;   // res^3, +1 biased particle index, 0: no dual vertex
  float4* rec;         // res^3 x 2: (vertex, material), (normal, has-vertex)
  uint32_t* blk;       // per block of 256 cells: vertex count, then its exclusive offset
  uint32_t* qblk;      // per block of 256 lattice points: quad count, then offset
  unsigned char* qmask;  // res^3: the edges (x, y, z bits) whose quad is emitted
  uint32_t* indices;   // quad_cap x 6
  uint32_t* draw_args; // vertexCount, instanceCount, firstVertex, firstInstance
  uint32_t* counters;  // vertex cells, quads (before the capacity clamps)
  float origin[3];
  float cell;
  float vel[3];
  uint32_t preserve;
  int32_t res, body, base, capacity, quad_cap, has_motion, nblocks, pad_;
};
constexpr int kExtractThreads = 256;  // cells (lattice points) per block of the grid passes

// A ClaySolver (sim/pbd.ts:78-424) as the kernels see it: the caller's ParticleSet records,
// the world field and the SolveParams uniform (pbd.ts:12-41).
struct __align__(16) SolveDev {
  unsigned char* particles;
  unsigned char* bodies;
  const FieldDev* world;
  float gravity[3];
  float h;  // substep length
  float radius, friction, damping, max_speed;
  float push[3];
  uint32_t push_body;
  float kick[3];
  int32_t capacity, max_bodies, rot_iters, pad_;
};
constexpr int kSolveThreads = 64;    // particle passes (pbd.ts:10)
constexpr int kSolveReduce = 256;    // threads per body in the match pass (pbd.ts:8)
constexpr uint32_t kBodyKinematic = 1u, kBodyWeightless = 2u;  // BodyFlags (particles.ts:38-43)

// The brush record (brush.ts:52-78), 80 bytes.
struct BrushDev {
  float pos[3];
  float scale;
  float rot[4];
  float size[3];
  float radius;
  float material;
  float blend;
  float bound;
  float mask;
  uint32_t kind, op, slot, pad;
};
static_assert(sizeof(BrushDev) == 80, "Brush layout");

struct BuildLevelDev {
  __half* dist;
  __half* mat;
  int32_t R, tiles;
  float ox, oy, oz, voxel, tile_size, tile_half, bw, empty;
};

}  // namespace clay

#ifdef CLAY_DEFINE_KERNELS
// =======================================================================================
// Device code. Only translation units that define CLAY_DEFINE_KERNELS compile it.
namespace clay {

__device__ __forceinline__ int f2i(float f) {
  // Saturating conversion, NaN -> 0 (WGSL value conversion).
  return __float2int_rz(f);
}
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return (ax * bx + ay * by) + az * bz;
}
__device__ __forceinline__ float len3(float x, float y, float z) { return sqrtf(dot3(x, y, z, x, y, z)); }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// hash1 (math/gpu.ts:103-112).
__device__ __forceinline__ float hash1(uint32_t x) {
  x = x ^ (x >> 16);
  x = x * 0x7feb352du;
  x = x ^ (x >> 15);
  x = x * 0x846ca68bu;
  x = x ^ (x >> 16);
  return static_cast<float>(x & 0xffffffu) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ uint32_t work_count(const SceneDev& S) { return min(S.prm->count, S.capacity); }

// ---------------------------------------------------------------------------------------
// Collider: volumeField.sample(p, 0) / normal(p) (trace/field.ts:102-180, volume.ts:262-313)
// with a software trilinear filter of exact f32 weights.
struct Vol {
  float ox, oy, oz, voxel, cx, cy, cz, extent, half, band, grad_h;
  int res;
  const __half* dist;
};

__device__ __forceinline__ Vol load_vol(const VolParamsDev* vp) {
  Vol v;
  v.ox = vp->origin[0];
  v.oy = vp->origin[1];
  v.oz = vp->origin[2];
  v.voxel = vp->voxel;
  v.cx = vp->center[0];
  v.cy = vp->center[1];
  v.cz = vp->center[2];
  v.extent = vp->extent;
  v.half = vp->half;
  v.band = vp->band;
  v.grad_h = vp->grad_h;
  v.res = vp->res;
  v.dist = vp->dist;
  return v;
}

__device__ __forceinline__ float sd_box(float px, float py, float pz, float b) {
  float qx = fabsf(px) - b, qy = fabsf(py) - b, qz = fabsf(pz) - b;
  float mx = fmaxf(qx, 0.0f), my = fmaxf(qy, 0.0f), mz = fmaxf(qz, 0.0f);
  return len3(mx, my, mz) + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.0f);
}

__device__ __forceinline__ float texel(const Vol& v, int x, int y, int z) {
  size_t idx = static_cast<size_t>(x) + static_cast<size_t>(v.res) * (static_cast<size_t>(y) + static_cast<size_t>(v.res) * z);
  return __half2float(__ldg(v.dist + idx));
}

__device__ __forceinline__ void tri_axis(float u, int R, int& i0, int& i1, float& fr) {
  float t = u * static_cast<float>(R) - 0.5f;
  float fl = floorf(t);
  fr = t - fl;
  int ii = f2i(fl);
  i0 = min(max(ii, 0), R - 1);
  int jj = ii == 2147483647 ? ii : ii + 1;
  i1 = min(max(jj, 0), R - 1);
}

__device__ __forceinline__ float lerpf(float a, float b, float f) { return a + (b - a) * f; }

__device__ __forceinline__ float trilinear(const Vol& v, float px, float py, float pz) {
  float ux = __fdiv_rn(px - v.ox, v.extent);
  float uy = __fdiv_rn(py - v.oy, v.extent);
  float uz = __fdiv_rn(pz - v.oz, v.extent);
  int x0, x1, y0, y1, z0, z1;
  float fx, fy, fz;
  tri_axis(ux, v.res, x0, x1, fx);
  tri_axis(uy, v.res, y0, y1, fy);
  tri_axis(uz, v.res, z0, z1, fz);
  float c00 = lerpf(texel(v, x0, y0, z0), texel(v, x1, y0, z0), fx);
  float c10 = lerpf(texel(v, x0, y1, z0), texel(v, x1, y1, z0), fx);
  float c01 = lerpf(texel(v, x0, y0, z1), texel(v, x1, y0, z1), fx);
  float c11 = lerpf(texel(v, x0, y1, z1), texel(v, x1, y1, z1), fx);
  float c0 = lerpf(c00, c10, fy);
  float c1 = lerpf(c01, c11, fy);
  return lerpf(c0, c1, fz);
}

__device__ __forceinline__ void vol_sample(const Vol& v, float px, float py, float pz, float& sx, float& sy) {
  float dbox = sd_box(px - v.cx, py - v.cy, pz - v.cz, v.half);
  if (dbox > 0.0f) {
    sx = dbox;
    sy = 1.0f;
    return;
  }
  float raw = trilinear(v, px, py, pz);
  float bw = v.band * v.voxel * 1.0f;
  sx = raw * bw;
  sy = raw;
}

__device__ __forceinline__ float vol_dist(const Vol& v, float px, float py, float pz) {
  float dbox = sd_box(px - v.cx, py - v.cy, pz - v.cz, v.half);
  if (dbox > 0.0f) return dbox;
  return trilinear(v, px, py, pz) * (v.band * v.voxel * 1.0f);
}

__device__ __forceinline__ void vol_normal(const Vol& v, float px, float py, float pz, float& nx, float& ny, float& nz) {
  float h = v.grad_h;
  float gx = vol_dist(v, px + h, py, pz) - vol_dist(v, px - h, py, pz);
  float gy = vol_dist(v, px, py + h, pz) - vol_dist(v, px, py - h, pz);
  float gz = vol_dist(v, px, py, pz + h) - vol_dist(v, px, py, pz - h);
  float len = len3(gx, gy, gz);
  if (len > 1e-8f) {
    float inv = __frcp_rn(len);
    nx = gx * inv;
    ny = gy * inv;
    nz = gz * inv;
  } else {
    nx = 0.0f;
    ny = 1.0f;
    nz = 0.0f;
  }
}

// unionField: the pair of the nearer child, the later child on ties.
__device__ __forceinline__ int field_pick(const FieldDev* f, float px, float py, float pz, float& sx, float& sy) {
  int best = -1;
  float bx = 0.0f, by = 0.0f;
  int n = f->n;
  for (int i = 0; i < n; i++) {
    const LeafDev& lf = f->leaf[i];
    Vol v = load_vol(lf.vp);
    float qx, qy, qz;
    leaf_point(lf, px, py, pz, qx, qy, qz);
    float s0, s1;
    vol_sample(v, qx, qy, qz, s0, s1);
    if (best < 0 || !(bx < s0)) {
      best = i;
      bx = s0;
      by = s1;
    }
  }
  sx = bx;
  sy = by;
  return best;
}

__device__ __forceinline__ void field_normal(const FieldDev* f, int child, float px, float py, float pz, float& nx, float& ny,
                                             float& nz) {
  const LeafDev& lf = f->leaf[child];
  Vol v = load_vol(lf.vp);
  float qx, qy, qz;
  leaf_point(lf, px, py, pz, qx, qy, qz);
  vol_normal(v, qx, qy, qz, nx, ny, nz);
}

// field(p, 0).y of the child `field_pick` chose at p (trace/field.ts:147-150,288-293,
// volume.ts:288-296): the material channel, trilinear like the distance, 0 outside the box.
__device__ __forceinline__ float field_material(const FieldDev* f, int child, float px, float py, float pz) {
  if (child < 0) return 0.0f;
  const LeafDev& lf = f->leaf[child];
  Vol v = load_vol(lf.vp);
  float qx, qy, qz;
  leaf_point(lf, px, py, pz, qx, qy, qz);
  if (sd_box(qx - v.cx, qy - v.cy, qz - v.cz, v.half) > 0.0f) return 0.0f;
  v.dist = lf.vp->mat;
  return trilinear(v, qx, qy, qz);
}

// Level m of a volume, capped at its top level (trace/field.ts:117-124): the plane offset,
// the side, and bandWorld(m) = band * voxelSize * exp2(m) (volume.ts:269-272).
__device__ __forceinline__ int vol_level(const VolParamsDev* vp, int mip, size_t& off, int& R, float& bw) {
  const int m = min(max(mip, 0), vp->mips - 1);
  off = 0;
  for (int l = 0; l < m; l++) {
    const size_t r = static_cast<size_t>(vp->res >> l);
    off += r * r * r;
  }
  R = vp->res >> m;
  bw = (vp->band * vp->voxel) * ldexpf(1.0f, m);  // exp2 of an integer level: exactly 2^m
  return m;
}

// volumeField.sample(p, mip) (trace/field.ts:135-146) and field(p, mip) (:147-150,
// volume.ts:288-296) of one leaf: (dBox, 1) / (dBox, 0) outside the box, else
// (raw * bandWorld, raw) / (raw * bandWorld, material) from level m's texels.
__device__ __forceinline__ void leaf_sample_mip(const LeafDev& lf, float px, float py, float pz, int mip, float& sx,
                                                float& sy, float& fy) {
  Vol v = load_vol(lf.vp);
  float qx, qy, qz;
  leaf_point(lf, px, py, pz, qx, qy, qz);
  const float dbox = sd_box(qx - v.cx, qy - v.cy, qz - v.cz, v.half);
  if (dbox > 0.0f) {
    sx = dbox;
    sy = 1.0f;
    fy = 0.0f;
    return;
  }
  size_t off;
  int R;
  float bw;
  vol_level(lf.vp, mip, off, R, bw);
  v.res = R;
  v.dist = lf.vp->dist + off;
  const float raw = trilinear(v, qx, qy, qz);
  v.dist = lf.vp->mat + off;
  fy = trilinear(v, qx, qy, qz);
  sx = raw * bw;
  sy = raw;
}

// unionField.sample / field (trace/field.ts:264-293): the pair of the nearer child (the
// later one on ties); both pick the same child, their x being the same distance.
__device__ __forceinline__ void field_sample_mip(const FieldDev* f, float px, float py, float pz, int mip, float& sx,
                                                 float& sy, float& fx, float& fy) {
  int best = -1;
  float bx = 0.0f, by = 0.0f, bf = 0.0f;
  for (int i = 0; i < f->n; i++) {
    float a, b, c;
    leaf_sample_mip(f->leaf[i], px, py, pz, mip, a, b, c);
    if (best < 0 || !(bx < a)) {
      best = i;
      bx = a;
      by = b;
      bf = c;
    }
  }
  sx = bx;
  sy = by;
  fx = bx;
  fy = bf;
}

// ---------------------------------------------------------------------------------------
// Work-item decoding: `work` == nullptr means "one object, blocks tile [0, n)".
__device__ __forceinline__ Work get_work(const Work* work) {
  if (work) return work[blockIdx.x];
  Work w;
  w.obj = 0;
  w.sub = blockIdx.y;
  w.first = blockIdx.x * blockDim.x;
  w.n = blockDim.x;
  return w;
}

// The same work, the blocks taken in reverse order: a pass that reads what the previous pass
// wrote (in forward block order) starts on the part written last, which is still in L2.
__device__ __forceinline__ Work get_work_reversed(const Work* work) {
  const uint32_t b = gridDim.x - 1u - blockIdx.x;
  if (work) return work[b];
  Work w;
  w.obj = 0;
  w.sub = blockIdx.y;
  w.first = b * blockDim.x;
  w.n = blockDim.x;
  return w;
}

// cellOf (fluid.ts:253-257).
__device__ __forceinline__ void cell_of(const SceneDev& S, float px, float py, float pz, int& cx, int& cy, int& cz) {
  cx = f2i(floorf((px - S.gorig[0]) * S.inv_h));
  cy = f2i(floorf((py - S.gorig[1]) * S.inv_h));
  cz = f2i(floorf((pz - S.gorig[2]) * S.inv_h));
}

struct BoxInfo {
  int x0, y0, z0;
  uint32_t bx, by, bz, L;
};

__device__ __forceinline__ BoxInfo box_from_acc(const GridState* gs) {
  BoxInfo b;
  uint32_t lx = gs->lo[0], ly = gs->lo[1], lz = gs->lo[2];
  if (lx == 0xffffffffu) {  // no particle in the grid
    b.x0 = b.y0 = b.z0 = 0;
    b.bx = b.by = b.bz = 0;
    b.L = 0;
    return b;
  }
  uint32_t hx = ~gs->hi_inv[0], hy = ~gs->hi_inv[1], hz = ~gs->hi_inv[2];
  b.x0 = static_cast<int>(lx);
  b.y0 = static_cast<int>(ly);
  b.z0 = static_cast<int>(lz);
  b.bx = hx - lx + 1;
  b.by = hy - ly + 1;
  b.bz = hz - lz + 1;
  b.L = b.bx * b.by * b.bz;
  return b;
}

__device__ __forceinline__ BoxInfo box_from_state(const GridState* gs) {
  BoxInfo b;
  b.x0 = gs->x0;
  b.y0 = gs->y0;
  b.z0 = gs->z0;
  b.bx = gs->bx;
  b.by = gs->by;
  b.bz = gs->bz;
  b.L = gs->L;
  return b;
}

__device__ __forceinline__ uint32_t local_of(const BoxInfo& b, uint32_t key) {
  if (key == kSentinel) return b.L;
  int x = static_cast<int>(key & 1023u), y = static_cast<int>((key >> 10) & 1023u), z = static_cast<int>(key >> 20);
  return static_cast<uint32_t>(x - b.x0) + b.bx * (static_cast<uint32_t>(y - b.y0) + b.by * static_cast<uint32_t>(z - b.z0));
}

#ifndef CLAY_ONLY_NEIGHBOUR_PASSES
// ---------------------------------------------------------------------------------------
// emit (fluid.ts:268-291). pow(r.x, 1/3) is taken in binary64 and rounded to f32;
// normalize(v) = v / length(v).
__global__ void k_emit(const SceneDev* __restrict__ scenes, const Work* __restrict__ work) {
  Work w = get_work(work);
  const SceneDev& S = scenes[w.obj];
  const ParamsDev& P = *S.prm;
  for (uint32_t i = w.first + threadIdx.x; i < P.emit_count; i += (work ? w.n : gridDim.x * blockDim.x)) {
    uint32_t slot = (P.emit_base + i) % S.capacity;
    uint32_t seed = P.emit_seed * 9781u + i;
    float r0 = hash1(seed * 3u + 0u), r1 = hash1(seed * 3u + 1u), r2 = hash1(seed * 3u + 2u);
    float dx = (r0 * 2.0f - 1.0f) + 1e-4f, dy = (r1 * 2.0f - 1.0f) + 1e-4f, dz = (r2 * 2.0f - 1.0f) + 1e-4f;
    float len = len3(dx, dy, dz);
    float ux = __fdiv_rn(dx, len), uy = __fdiv_rn(dy, len), uz = __fdiv_rn(dz, len);
    const float third = 0.333333343267440796f;  // f32(1/3)
    float pw = static_cast<float>(pow(static_cast<double>(r0), static_cast<double>(third)));
    float s = P.emit_radius * pw;
    ParticleDev q;
    q.a = make_float4(P.emit_pos[0] + ux * s, P.emit_pos[1] + uy * s, P.emit_pos[2] + uz * s, 0.0f);
    q.b = make_float4(P.emit_vel[0], P.emit_vel[1], P.emit_vel[2], 0.0f);
    q.c = make_float4(P.emit_vel[0], P.emit_vel[1], P.emit_vel[2], 0.0f);
    S.parts[slot] = q;
    if (!work) break;
  }
}

// ---------------------------------------------------------------------------------------
// Cell build, pass 1: the cell of every live particle (packed x|y<<10|z<<20, or the
// sentinel when !inGrid, fluid.ts:318-322) and the bounding box of occupied cells. The
// first block of a scene also clears the contact counter (fluid.ts:302-304) and the
// bucket-overflow flag.
__global__ void k_cell_key(const SceneDev* __restrict__ scenes, const Work* __restrict__ work, int substep) {
  Work w = get_work(work);
  const SceneDev& S = scenes[w.obj];
  if (substep >= S.substeps) return;
  uint32_t count = work_count(S);
  uint32_t i = w.first + threadIdx.x;
  if (w.first == 0 && threadIdx.x == 0) {
    S.contacts->count = 0u;
    S.gs->overflow = 0u;
  }
  uint32_t lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu};
  uint32_t hinv[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu};
  if (i < count && threadIdx.x < w.n) {
    float4 p = S.parts[i].a;
    int cx, cy, cz;
    cell_of(S, p.x, p.y, p.z, cx, cy, cz);
    bool in = cx >= 0 && cy >= 0 && cz >= 0 && cx < S.G && cy < S.G && cz < S.G;
    uint32_t key = kSentinel;
    if (in) {
      key = static_cast<uint32_t>(cx) | (static_cast<uint32_t>(cy) << 10) | (static_cast<uint32_t>(cz) << 20);
      lo[0] = cx;
      lo[1] = cy;
      lo[2] = cz;
      hinv[0] = ~static_cast<uint32_t>(cx);
      hinv[1] = ~static_cast<uint32_t>(cy);
      hinv[2] = ~static_cast<uint32_t>(cz);
    }
    S.key[i] = key;
  }
  // warp then block reduction of the box
#pragma unroll
  for (int k = 0; k < 3; k++) {
    lo[k] = __reduce_min_sync(0xffffffffu, lo[k]);
    hinv[k] = __reduce_min_sync(0xffffffffu, hinv[k]);
  }
  __shared__ uint32_t s_box[6];
  if (threadIdx.x < 6) s_box[threadIdx.x] = 0xffffffffu;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      if (lo[k] != 0xffffffffu) atomicMin(&s_box[k], lo[k]);
      if (hinv[k] != 0xffffffffu) atomicMin(&s_box[3 + k], hinv[k]);
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    if (s_box[threadIdx.x] != 0xffffffffu) atomicMin(&S.gs->lo[threadIdx.x], s_box[threadIdx.x]);
  } else if (threadIdx.x < 6) {
    if (s_box[threadIdx.x] != 0xffffffffu) atomicMin(&S.gs->hi_inv[threadIdx.x - 3], s_box[threadIdx.x]);
  }
}

// Cell build, pass 2: per-cell counts with warp-aggregated atomics; every particle keeps
// its provisional slot. The scene's first block publishes the box for the later passes.
__global__ void k_cell_count(const SceneDev* __restrict__ scenes, const Work* __restrict__ work, int substep) {
  Work w = get_work(work);
  const SceneDev& S = scenes[w.obj];
  if (substep >= S.substeps) return;
  uint32_t count = work_count(S);
  BoxInfo b = box_from_acc(S.gs);
  if (w.first == 0 && threadIdx.x == 0) {
    GridState* g = S.gs;
    g->x0 = b.x0;
    g->y0 = b.y0;
    g->z0 = b.z0;
    g->bx = b.bx;
    g->by = b.by;
    g->bz = b.bz;
    g->L = b.L;
  }
  uint32_t i = w.first + threadIdx.x;
  bool act = i < count && threadIdx.x < w.n;
  uint32_t l = 0xffffffffu;
  if (act) {
    l = local_of(b, S.key[i]);
    S.key[i] = l;
  }
  // warp-aggregated increment: one atomic per distinct cell per warp
  uint32_t peers = __match_any_sync(0xffffffffu, l);
  if (act) {
    int leader = __ffs(peers) - 1;
    uint32_t lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if (static_cast<int>(lane) == leader) base = atomicAdd(&S.counts[l], static_cast<uint32_t>(__popc(peers)));
    base = __shfl_sync(peers, base, leader);
    uint32_t rank = base + __popc(peers & ((1u << lane) - 1u));
    S.rank[i] = rank;
    if (l != b.L && base + __popc(peers) > S.bucket) S.gs->overflow = 1u;
  }
}

// Cell build, pass 3a: partial sums of the counts of [0, L] split into `parts_scan`
// parts. Part 0 also resets the box accumulators for the next substep.
__global__ void k_scan_partial(const SceneDev* __restrict__ scenes, const Work* __restrict__ work, int substep) {
  Work w = get_work(work);
  const SceneDev& S = scenes[w.obj];
  if (substep >= S.substeps) return;
  if (work_count(S) == 0) return;
  GridState* gs = S.gs;
  uint32_t n = gs->L + 1;
  uint32_t P = S.parts_scan;
  uint32_t per = (n + P - 1) / P;
  uint32_t beg = min(w.sub * per, n), end = min(beg + per, n);
  uint32_t s = 0;
  for (uint32_t c = beg + threadIdx.x; c < end; c += blockDim.x) s += S.counts[c];
  s = __reduce_add_sync(0xffffffffu, s);
  __shared__ uint32_t red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0u;
    v = __reduce_add_sync(0xffffffffu, v);
    if (threadIdx.x == 0) gs->part_sum[w.sub] = v;
  }
  if (w.sub == 0 && threadIdx.x < 6) {
    if (threadIdx.x < 3) gs->lo[threadIdx.x] = 0xffffffffu;
    else gs->hi_inv[threadIdx.x - 3] = 0xffffffffu;
  }
}

// Cell build, pass 3b: exclusive scan into cell_start[0 .. L+1], counts cleared behind.
__global__ void k_scan_final(const SceneDev* __restrict__ scenes, const Work* __restrict__ work, int substep) {
  Work w = get_work(work);
  const SceneDev& S = scenes[w.obj];
  if (substep >= S.substeps) return;
  if (work_count(S) == 0) return;
  const GridState* gs = S.gs;
  uint32_t n = gs->L + 1;
  uint32_t P = S.parts_scan;
  uint32_t per = (n + P - 1) / P;
  uint32_t beg = min(w.sub * per, n), end = min(beg + per, n);
  __shared__ uint32_t s_off;
  __shared__ uint32_t s_warp[32];
  if (threadIdx.x == 0) {
    uint32_t o = 0;
    for (uint32_t q = 0; q < w.sub; q++) o += gs->part_sum[q];
    s_off = o;
  }
  __syncthreads();
  uint32_t run = s_off;
  const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (uint32_t c0 = beg; c0 < end; c0 += blockDim.x) {
    uint32_t c = c0 + threadIdx.x;
    uint32_t v = c < end ? S.counts[c] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= static_cast<uint32_t>(o)) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
      uint32_t t = lane < nw ? s_warp[lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= static_cast<uint32_t>(o)) t += y;
      }
      s_warp[lane] = t;
    }
    __syncthreads();
    uint32_t before = (wid > 0 ? s_warp[wid - 1] : 0u) + x - v;
    if (c < end) {
      S.cell_start[c] = run + before;
      S.counts[c] = 0u;
    }
    uint32_t tot = s_warp[nw - 1];
    __syncthreads();
    run += tot;
  }
  if (end == n && beg < end && threadIdx.x == 0) S.cell_start[n] = run;
  if (n == 0 && threadIdx.x == 0 && w.sub == 0) S.cell_start[0] = 0;
}

// Cell build, pass 4: provisional placement.
__global__ void k_cell_scatter(const SceneDev* __restrict__ scenes, const Work* __restrict__ work, int substep) {
  Work w = get_work(work);
  const SceneDev& S = scenes[w.obj];
  if (substep >= S.substeps) return;
  uint32_t count = work_count(S);
  uint32_t i = w.first + threadIdx.x;
  if (i >= count || threadIdx.x >= w.n) return;
  S.tmp[S.cell_start[S.key[i]] + S.rank[i]] = i;
}

// Cell build, pass 5: deterministic order inside each cell (ascending particle index, so
// a full cell keeps its `bucket` lowest indices, fluid.ts:323-329) and the gather of the
// particle state into cell order.
__global__ void k_cell_order(const SceneDev* __restrict__ scenes, const Work* __restrict__ work, int substep) {
  Work w = get_work(work);
  const SceneDev& S = scenes[w.obj];
  if (substep >= S.substeps) return;
  uint32_t count = work_count(S);
  uint32_t k = w.first + threadIdx.x;
  if (k >= count || threadIdx.x >= w.n) return;
  uint32_t id = S.tmp[k];
  // the record is gathered before the rank loop, so its load overlaps the loop
  const float4 pa = S.parts[id].a, pb = S.parts[id].b;
  uint32_t l = S.key[id];
  uint32_t s = S.cell_start[l], e = S.cell_start[l + 1];
  uint32_t r = 0;
  for (uint32_t q = s; q < e; q++) r += (S.tmp[q] < id) ? 1u : 0u;
  uint32_t f = s + r;
  S.sorted_id[f] = id;
  S.spos[f] = pa;
  S.svel[f] = pb;
}

#endif  // CLAY_ONLY_NEIGHBOUR_PASSES

// ---------------------------------------------------------------------------------------
// Neighbour iteration over the 27 cells (fluid.ts:346-364) in the reference's order: dz,
// dy, dx ascending, then ascending index inside a cell. Cells along x are adjacent in the
// cell order, so each (dy, dz) row is one contiguous range unless some cell of the scene
// holds more than `bucket` particles.
template <class F>
__device__ __forceinline__ void for_neighbours(const SceneDev& S, const BoxInfo& b, bool overflow, int cx, int cy, int cz,
                                               F&& f) {
  const int G = S.G;
  cx = min(max(cx, -2), G + 1);
  cy = min(max(cy, -2), G + 1);
  cz = min(max(cz, -2), G + 1);
  const int x1b = b.x0 + static_cast<int>(b.bx) - 1;
  const int y1b = b.y0 + static_cast<int>(b.by) - 1;
  const int z1b = b.z0 + static_cast<int>(b.bz) - 1;
  if (b.L == 0) return;
  int xl = max(cx - 1, b.x0), xh = min(cx + 1, x1b);
  if (xl > xh) return;
  for (int dz = -1; dz <= 1; dz++) {
    int z = cz + dz;
    if (z < b.z0 || z > z1b) continue;
    for (int dy = -1; dy <= 1; dy++) {
      int y = cy + dy;
      if (y < b.y0 || y > y1b) continue;
      uint32_t row = b.bx * (static_cast<uint32_t>(y - b.y0) + b.by * static_cast<uint32_t>(z - b.z0));
      uint32_t l0 = row + static_cast<uint32_t>(xl - b.x0);
      uint32_t l1 = row + static_cast<uint32_t>(xh - b.x0);
      if (!overflow) {
        uint32_t s = __ldg(S.cell_start + l0), e = __ldg(S.cell_start + l1 + 1);
        for (uint32_t q = s; q < e; q++) f(q);
      } else {
        for (uint32_t l = l0; l <= l1; l++) {
          uint32_t s = __ldg(S.cell_start + l), e = __ldg(S.cell_start + l + 1);
          uint32_t n = min(e - s, S.bucket);
          for (uint32_t q = s; q < s + n; q++) f(q);
        }
      }
    }
  }
}

// The same 27 cells as contiguous ranges of the cell order, in the reference's visiting
// order: f(s, e) once per (dz, dy) row of cells (or per cell, capped at `bucket`, when some
// cell of the scene overflowed).
template <class F>
__device__ __forceinline__ void for_neighbour_ranges(const SceneDev& S, const BoxInfo& b, bool overflow, int cx, int cy,
                                                     int cz, F&& f) {
  const int G = S.G;
  cx = min(max(cx, -2), G + 1);
  cy = min(max(cy, -2), G + 1);
  cz = min(max(cz, -2), G + 1);
  const int x1b = b.x0 + static_cast<int>(b.bx) - 1;
  const int y1b = b.y0 + static_cast<int>(b.by) - 1;
  const int z1b = b.z0 + static_cast<int>(b.bz) - 1;
  if (b.L == 0) return;
  int xl = max(cx - 1, b.x0), xh = min(cx + 1, x1b);
  if (xl > xh) return;
  for (int dz = -1; dz <= 1; dz++) {
    int z = cz + dz;
    if (z < b.z0 || z > z1b) continue;
    for (int dy = -1; dy <= 1; dy++) {
      int y = cy + dy;
      if (y < b.y0 || y > y1b) continue;
      uint32_t row = b.bx * (static_cast<uint32_t>(y - b.y0) + b.by * static_cast<uint32_t>(z - b.z0));
      uint32_t l0 = row + static_cast<uint32_t>(xl - b.x0);
      uint32_t l1 = row + static_cast<uint32_t>(xh - b.x0);
      const int r = (dz + 1) * 3 + (dy + 1);
      if (!overflow) {
        f(__ldg(S.cell_start + l0), __ldg(S.cell_start + l1 + 1), r);
      } else {
        for (uint32_t l = l0; l <= l1; l++) {
          uint32_t s = __ldg(S.cell_start + l), e = __ldg(S.cell_start + l + 1);
          f(s, s + min(e - s, S.bucket), r);
        }
      }
    }
  }
}

// The local cell index (the cell build's order key) of a position: L, the out-of-grid bucket,
// outside the grid (fluid.ts:318-322), else its place in the box of occupied cells.
__device__ __forceinline__ uint32_t local_cell(const SceneDev& S, const BoxInfo& b, float4 p) {
  int cx, cy, cz;
  cell_of(S, p.x, p.y, p.z, cx, cy, cz);
  if (cx < 0 || cy < 0 || cz < 0 || cx >= S.G || cy >= S.G || cz >= S.G) return b.L;
  return static_cast<uint32_t>(cx - b.x0) + b.bx * (static_cast<uint32_t>(cy - b.y0) + b.by * static_cast<uint32_t>(cz - b.z0));
}

constexpr int kDensityStage = 3040;  // staged neighbour positions per block (47.5 KB, under the 48 KB static limit)

// density (fluid.ts:333-368). kFast accumulates with Kahan compensation.
//
// Three variants, which visit, sum and list the neighbours in the same order:
//  - kVariant 0: one loop, the accept work inside the distance-test loop;
//  - kVariant 1: the candidates of a range 32 at a time in two phases: the distance test of
//    every candidate, which leaves a bit mask of the accepted ones, then the accepted ones
//    alone, in ascending order (the reference's visiting order), each re-read from cache. A
//    warp's lanes accept at different candidates, so running the accept work inside the test
//    loop keeps most lanes idle through it; in the second phase every lane with a pending
//    neighbour works;
//  - kVariant 2: variant 0 reading the candidates from shared memory. The block's particles
//    are consecutive in the cell order, so their cells span a run [l0, l1] of local cell
//    indices, and the neighbour row (dz, dy) of any of them lies in the cells
//    [l0 + off - 1, l1 + off + 1], off = bx * (dy + by * dz): nine ranges of the cell-ordered
//    positions, copied into shared memory once per block when they fit (else the block reads
//    through the cache as variant 0 does).
template <bool kFast, int kVariant>
__global__ void __launch_bounds__(256, 5) k_density(const SceneDev* __restrict__ scenes, const Work* __restrict__ work, int substep) {
  Work w = get_work_reversed(work);
  const SceneDev& S = scenes[w.obj];
  if (substep >= S.substeps) return;
  uint32_t count = work_count(S);
  uint32_t k = w.first + threadIdx.x;
  const BoxInfo b = box_from_state(S.gs);
  const bool overflow = S.gs->overflow != 0u;
  [[maybe_unused]] float4* s_pos = nullptr;
  [[maybe_unused]] uint32_t* s_q0 = nullptr;  // first staged particle of each row range
  [[maybe_unused]] uint32_t* s_sb = nullptr;  // its place in s_pos
  [[maybe_unused]] bool staged = false;
  if constexpr (kVariant == 2) {
    __shared__ float4 st_pos[kDensityStage];
    __shared__ uint32_t st_q0[9], st_sb[9], st_n[9];
    __shared__ int st_ok;
    s_pos = st_pos;
    s_q0 = st_q0;
    s_sb = st_sb;
    const uint32_t last = min(count, w.first + w.n);  // one past the block's last particle
    if (w.first >= last) return;  // the whole block is past the live count
    if (threadIdx.x < 32) {
      const uint32_t lane = threadIdx.x;
      uint32_t n = 0, q0 = 0;
      // a particle outside the grid (sorted last, local cell L) still reads the grid's edge
      // rows around its clamped cell, which the ranges below do not cover: such a block reads
      // through the cache
      const uint32_t l1u = b.L > 0 ? local_cell(S, b, S.spos[last - 1]) : 0u;
      const bool fits = b.L > 0 && l1u < b.L;
      if (lane < 9 && fits) {
        const int l0 = static_cast<int>(local_cell(S, b, S.spos[w.first]));
        const int l1 = static_cast<int>(l1u);
        const int dz = static_cast<int>(lane) / 3 - 1, dy = static_cast<int>(lane) % 3 - 1;
        const int off = static_cast<int>(b.bx) * (dy + static_cast<int>(b.by) * dz);
        const int lo = max(l0 + off - 1, 0), hi = min(l1 + off + 1, static_cast<int>(b.L) - 1);
        if (lo <= hi) {
          q0 = S.cell_start[lo];
          n = S.cell_start[hi + 1] - q0;
        }
      }
      uint32_t incl = n;
#pragma unroll
      for (int o = 1; o < 16; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= static_cast<uint32_t>(o)) incl += y;
      }
      if (lane < 9) {
        st_q0[lane] = q0;
        st_sb[lane] = incl - n;
        st_n[lane] = n;
      }
      const uint32_t total = __shfl_sync(0xffffffffu, incl, 8);
      if (lane == 0) st_ok = fits && total <= static_cast<uint32_t>(kDensityStage);
    }
    __syncthreads();
    staged = st_ok != 0;
    if (staged) {
      for (int r = 0; r < 9; r++) {
        const uint32_t n = st_n[r], q0 = st_q0[r], sb = st_sb[r];
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) st_pos[sb + i] = __ldg(S.spos + q0 + i);
      }
      __syncthreads();
    }
  }
  if (k >= count || threadIdx.x >= w.n) return;
  const float4 me = S.spos[k];
  int cx, cy, cz;
  cell_of(S, me.x, me.y, me.z, cx, cy, cz);
  const float h2 = S.h2, mp6 = S.mass_poly6;
  float rho = 0.0f, comp = 0.0f;
  const float4* __restrict__ spos = S.spos;
  // The accepted neighbours, in visiting order, for the forces pass: entry j of particle k is
  // word j % 4 of nbr[(j / 4) * capacity + k], so the forces pass reads 4 at a time and a
  // warp's lanes at one slot as contiguous lines.
  uint32_t* __restrict__ nl = reinterpret_cast<uint32_t*>(S.nbr + k);
  const uint32_t stride = 4u * S.capacity;
  uint32_t cnt = 0;
  // one accepted neighbour q at squared length r2, in visiting order
  auto accept = [&](uint32_t q, float r2) {
    if (cnt < kMaxNbr) nl[(cnt >> 2) * stride + (cnt & 3u)] = q;
    cnt++;
    // variant 1 recomputes the length: fast mode may contract it differently from the test,
    // and a pair at the boundary then adds a term of order (h^2 * 1e-7)^3, not a missing one
    const float wv = kVariant == 1 ? fmaxf(h2 - r2, 0.0f) : h2 - r2;
    // fast mode sums (h^2 - r^2)^3 and scales the sum by mass * poly6 once at the end; the
    // reference mode scales every term, as the reference does
    const float term = kFast ? (wv * wv) * wv : mp6 * ((wv * wv) * wv);
    if (kFast) {
      // Kahan: explicit round-to-nearest operations so nothing is contracted into an FMA
      // (every term is positive, so the running sum bounds each term after the first)
      const float y = __fsub_rn(term, comp);
      const float t = __fadd_rn(rho, y);
      comp = __fsub_rn(__fsub_rn(t, rho), y);
      rho = t;
    } else {
      rho = rho + term;
    }
  };
  if constexpr (kVariant == 0) {
    for_neighbours(S, b, overflow, cx, cy, cz, [&](uint32_t q) {
      const float4 o = __ldg(spos + q);
      const float dx = me.x - o.x, dy = me.y - o.y, dz = me.z - o.z;
      const float r2 = (dx * dx + dy * dy) + dz * dz;
      if (r2 < h2) accept(q, r2);
    });
  } else if constexpr (kVariant == 2) {
    for_neighbour_ranges(S, b, overflow, cx, cy, cz, [&](uint32_t s, uint32_t e, int r) {
      // the row's candidates [s, e) lie inside staged range r (see above): candidate q sits
      // at s_pos[q - q0 + sb], computed modulo 2^32 as q + shift
      const uint32_t shift = staged ? s_sb[r] - s_q0[r] : 0u;
      for (uint32_t q = s; q < e; q++) {
        const float4 o = staged ? s_pos[q + shift] : __ldg(spos + q);
        const float dx = me.x - o.x, dy = me.y - o.y, dz = me.z - o.z;
        const float r2 = (dx * dx + dy * dy) + dz * dz;
        if (r2 < h2) accept(q, r2);
      }
    });
  } else for_neighbour_ranges(S, b, overflow, cx, cy, cz, [&](uint32_t s, uint32_t e, int) {
    for (uint32_t base = s; base < e; base += 32u) {
      const uint32_t n = min(32u, e - base);
      uint32_t m = 0;
      for (uint32_t i = 0; i < n; i++) {
        const float4 o = __ldg(spos + base + i);
        const float dx = me.x - o.x, dy = me.y - o.y, dz = me.z - o.z;
        const float r2 = (dx * dx + dy * dy) + dz * dz;
        m |= (r2 < h2 ? 1u : 0u) << i;
      }
      while (m) {
        const uint32_t q = base + static_cast<uint32_t>(__ffs(m) - 1);
        m &= m - 1u;
        const float4 o = __ldg(spos + q);
        const float dx = me.x - o.x, dy = me.y - o.y, dz = me.z - o.z;
        accept(q, (dx * dx + dy * dy) + dz * dz);
      }
    }
  });
  if (kFast) rho = mp6 * __fsub_rn(rho, comp);
  const float stiff = S.prm->stiffness;
  const float dens = fmaxf(rho, S.rest_floor);
  const float pres = fmaxf(stiff * (rho - S.rest), 0.0f), inv = __frcp_rn(dens);
  S.sdp[k] = make_float4(dens, pres, inv, __uint_as_float(cnt));
  // the neighbour view of this particle for the forces pass (svel is not read in this pass);
  // fast mode stores p / rho beside the velocity, so that the forces pass forms a neighbour's
  // (p_i + p_j) / rho_j as one multiply-add, p_i * (1 / rho_j) + p_j / rho_j
  S.spx[k] = make_float4(me.x, me.y, me.z, inv);
  S.svel[k].w = kFast ? pres * inv : pres;
}

// integrate (fluid.ts:449-491) of cell-ordered particle k: advance with the new velocity, collide
// with the world field (push out along its normal, drop the inward velocity, record a contact),
// clamp to the bake volume's walls, and write the particle's record.
__device__ __forceinline__ void integrate_particle(const SceneDev& S, const ParamsDev& P, uint32_t k, const float4 me,
                                                   const float4 mdp, float vx, float vy, float vz) {
  const float nvx = vx, nvy = vy, nvz = vz;
  float px = me.x + vx * P.dt, py = me.y + vy * P.dt, pz = me.z + vz * P.dt;
  const FieldDev* world = S.world;
  if (world && world->n > 0) {
    float sx, sy;
    int child = field_pick(world, px, py, pz, sx, sy);
    float dw = sx;
    if (dw < S.radius) {
      float nx, ny, nz;
      field_normal(world, child, px, py, pz, nx, ny, nz);
      float push = S.radius - dw;
      px = px + nx * push;
      py = py + ny * push;
      pz = pz + nz * push;
      float vn = fminf(dot3(vx, vy, vz, nx, ny, nz), 0.0f);
      vx = vx - nx * vn;
      vy = vy - ny * vn;
      vz = vz - nz * vn;
      if (dw < P.contact_depth) {
        uint32_t slot = atomicAdd(&S.contacts->count, 1u);
        if (slot < 32u) S.contacts->points[slot] = make_float4(px, py, pz, len3(vx, vy, vz));
      }
    }
  }
  float clx = clampf(px, S.wlo[0], S.whi[0]), cly = clampf(py, S.wlo[1], S.whi[1]), clz = clampf(pz, S.wlo[2], S.whi[2]);
  ParticleDev out;
  out.a = make_float4(clx, cly, clz, mdp.x);
  out.b = make_float4(clx == px ? vx : 0.0f, cly == py ? vy : 0.0f, clz == pz ? vz : 0.0f, mdp.y);
  out.c = make_float4(nvx, nvy, nvz, 0.0f);
  S.parts[S.sorted_id[k]] = out;
}

// forces (fluid.ts:370-439) fused with integrate (fluid.ts:449-491). The neighbour pass
// reads only the cell-ordered copies made by the cell build, and writes only the particle
// records, so no neighbour can observe a half-updated particle.
//
// kSplit leaves the integrate to k_integrate, a launch of its own: without the collider
// sampling the neighbour loop needs fewer registers, and five blocks fit an SM instead of four.
template <bool kFast, bool kSplit>
__global__ void __launch_bounds__(256, kSplit ? 5 : 4) k_forces_integrate(const SceneDev* __restrict__ scenes,
                                                                          const Work* __restrict__ work, int substep) {
  Work w = get_work(work);
  const SceneDev& S = scenes[w.obj];
  if (substep >= S.substeps) return;
  uint32_t count = work_count(S);
  uint32_t k = w.first + threadIdx.x;
  if (k >= count || threadIdx.x >= w.n) return;
  const BoxInfo b = box_from_state(S.gs);
  const bool overflow = S.gs->overflow != 0u;
  const ParamsDev& P = *S.prm;
  const float4 me = S.spos[k];
  const float4 mv = S.svel[k];
  const float4 mdp = S.sdp[k];
  int cx, cy, cz;
  cell_of(S, me.x, me.y, me.z, cx, cy, cz);
  const float h2 = S.h2, h = S.h, mass = S.mass, spiky = S.spiky;
  const float mp = mdp.y;
  float fx = 0.0f, fy = 0.0f, fz = 0.0f;
  float vsx = mv.x * S.h6, vsy = mv.y * S.h6, vsz = mv.z * S.h6;
  float wsum = S.h6;
  const float4* __restrict__ spx = S.spx;
  const float4* __restrict__ svel = S.svel;
  // Fast mode forms the pressure factor mass * (p_i + p_j) / 2 / rho_j * spiky * (h - r)^2 / r
  // with the constants folded into one and (p_i + p_j) / rho_j = p_i * (1 / rho_j) + p_j / rho_j
  // (the density pass stored p_j / rho_j), rounding differently from the reference's order.
  const float half_mass_spiky = (mass * 0.5f) * spiky;
  // one neighbour q: o = position and 1/density, ov = velocity and pressure (p / rho in fast mode)
  auto accum = [&](uint32_t q, const float4 o, const float4 ov) {
    if (q == k) return;
    float dx = me.x - o.x, dy = me.y - o.y, dz = me.z - o.z;
    float r2 = (dx * dx + dy * dy) + dz * dz;
    if (r2 >= h2) return;
    const float inv = o.w;
    float w0 = h2 - r2;
    float wv = (w0 * w0) * w0;
    vsx = vsx + ov.x * wv;
    vsy = vsy + ov.y * wv;
    vsz = vsz + ov.z * wv;
    wsum = wsum + wv;
    // fast mode: hardware reciprocal square root; reference mode: IEEE sqrt and 1/r
    const float irs = kFast ? rsqrtf(r2) : 0.0f;
    const float r = kFast ? r2 * irs : __fsqrt_rn(r2);
    if (r > 1e-6f) {
      float hr = h - r;
      float s = kFast ? half_mass_spiky * fmaf(mp, inv, ov.w) * (hr * hr) : mass * (mp + ov.w) * 0.5f * inv * spiky * (hr * hr);
      float ir = kFast ? irs : __frcp_rn(r);
      fx = fx - (dx * ir) * s;
      fy = fy - (dy * ir) * s;
      fz = fz - (dz * ir) * s;
    }
  };
  // Fast mode, a neighbour from the list: the density pass accepted it (r^2 < h^2, up to how
  // each pass contracts the length: a pair on the boundary adds a term of order
  // (h^2 * 1e-7)^3), and the particle itself is on its own list at r = 0, where its XSPH
  // term is the (h^2)^3 the reference starts the sums with and no pressure force applies. So
  // the list loop tests neither q == k nor r^2 < h^2.
  auto accum_listed = [&](const float4 o, const float4 ov) {
    const float dx = me.x - o.x, dy = me.y - o.y, dz = me.z - o.z;
    const float r2 = (dx * dx + dy * dy) + dz * dz;
    const float w0 = h2 - r2;
    const float wv = (w0 * w0) * w0;
    vsx = vsx + ov.x * wv;
    vsy = vsy + ov.y * wv;
    vsz = vsz + ov.z * wv;
    wsum = wsum + wv;
    if (r2 > 1e-12f) {  // r > 1e-6
      const float irs = rsqrtf(r2);
      const float hr = h - r2 * irs;
      const float t = half_mass_spiky * fmaf(mp, o.w, ov.w) * ((hr * hr) * irs);
      fx = fx - dx * t;
      fy = fy - dy * t;
      fz = fz - dz * t;
    }
  };
  auto pair = [&](uint32_t q) {
    if (q == k) return;
    const float4 o = __ldg(spx + q);
    float dx = me.x - o.x, dy = me.y - o.y, dz = me.z - o.z;
    if ((dx * dx + dy * dy) + dz * dz >= h2) return;
    accum(q, o, __ldg(svel + q));
  };
  // The density pass of this substep stored the neighbours it accepted, in the same visiting
  // order, with the same squared lengths: the list replaces the scan of the 27 cells, and
  // every load of a group of kForceLoads neighbours is issued before any of them is used (a
  // list entry is a neighbour, so nothing waits on the distance test). A particle with more
  // than kMaxNbr neighbours scans the cells again.
  constexpr int kForceLoads = 2;
  const uint32_t cnt = __float_as_uint(mdp.w);
  if (cnt <= kMaxNbr) {
    const uint4* __restrict__ nl = S.nbr + k;
    const uint32_t stride = S.capacity;
    if (kFast) {  // the particle's own entry brings its term
      vsx = 0.0f;
      vsy = 0.0f;
      vsz = 0.0f;
      wsum = 0.0f;
    }
    // the entries of slot j / 4 below `lim` (entries past the count hold no index); the full
    // slots pass lim = 4, which needs no test once the lambda is inlined
    auto slot = [&](uint32_t j, uint32_t lim) {
      const uint4 e = __ldg(nl + (j / 4u) * stride);
      const uint32_t qa[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
      for (int g = 0; g < 4; g += kForceLoads) {
        float4 o[kForceLoads], v[kForceLoads];
#pragma unroll
        for (int u = 0; u < kForceLoads; u++) {
          if (static_cast<uint32_t>(g + u) < lim) {
            o[u] = __ldg(spx + qa[g + u]);
            v[u] = __ldg(svel + qa[g + u]);
          }
        }
#pragma unroll
        for (int u = 0; u < kForceLoads; u++) {
          if (static_cast<uint32_t>(g + u) < lim) {
            if (kFast) accum_listed(o[u], v[u]);
            else accum(qa[g + u], o[u], v[u]);
          }
        }
      }
    };
    // the list's slots come from DRAM (the whole batch's lists do not fit in L2): ask for all of
    // them at once, so that each slot's load waits on L2 rather than on DRAM
    for (uint32_t p = 0; p < cnt; p += 4)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(nl + (p / 4u) * stride));
    uint32_t j = 0;
    for (; j + 4u <= cnt; j += 4) slot(j, 4u);
    if (j < cnt) slot(j, cnt - j);
  } else {
    for_neighbours(S, b, overflow, cx, cy, cz, pair);
  }
  float id = mdp.z;
  float ax = fx * id + P.gravity[0], ay = fy * id + P.gravity[1], az = fz * id + P.gravity[2];
  float t = clampf(P.viscosity, 0.0f, 1.0f);
  float iw = __frcp_rn(wsum);
  float mx = vsx * iw, my = vsy * iw, mz = vsz * iw;
  float omt = 1.0f - t;
  float vx = mv.x * omt + mx * t, vy = mv.y * omt + my * t, vz = mv.z * omt + mz * t;
  vx = (vx + ax * P.dt) * P.damping;
  vy = (vy + ay * P.dt) * P.damping;
  vz = (vz + az * P.dt) * P.damping;
  float speed = len3(vx, vy, vz);
  if (speed > P.max_speed) {
    float sc = __fdiv_rn(P.max_speed, speed);
    vx = vx * sc;
    vy = vy * sc;
    vz = vz * sc;
  }
  if constexpr (kSplit) {
    // the integrate pass runs as its own launch: the new velocity waits in the first entry of
    // this particle's neighbour list, which no other particle reads
    reinterpret_cast<float4*>(S.nbr)[k] = make_float4(vx, vy, vz, 0.0f);
  } else {
    integrate_particle(S, P, k, me, mdp, vx, vy, vz);
  }
}

// The integrate half of a split forces pass (see k_forces_integrate), compiled with the same
// contraction rule as the fused pass of its mode.
template <bool kFast>
__global__ void __launch_bounds__(256) k_integrate(const SceneDev* __restrict__ scenes, const Work* __restrict__ work,
                                                    int substep) {
  Work w = get_work(work);
  const SceneDev& S = scenes[w.obj];
  if (substep >= S.substeps) return;
  uint32_t count = work_count(S);
  uint32_t k = w.first + threadIdx.x;
  if (k >= count || threadIdx.x >= w.n) return;
  const float4 v = reinterpret_cast<const float4*>(S.nbr)[k];
  integrate_particle(S, *S.prm, k, S.spos[k], S.sdp[k], v.x, v.y, v.z);
}

// ---------------------------------------------------------------------------------------
// SplatField bake (splat.ts:200-276).
//
// One warp takes 32 consecutive particles of the cloud (in cell order for the fluid) and
// the union U of their voxel boxes (splat.ts:238-243). When U is compact it walks U with
// one voxel per lane and takes, per voxel, the minimum of every particle's contribution
// before a single atomicMin; otherwise it walks each particle's own box. Both give the
// reference's result exactly: the key is a monotone function of the distance, so the
// atomicMin of keys equals the key of the minimum distance, and a voxel outside a
// particle's box is at least half a voxel beyond its reach, so it can never pass
// `sd < bandWorld` (splat.ts:246). For spheres the minimum is taken over squared lengths:
// sqrt and the subtraction of the radius are both monotone in f32.

// The key grid holds, per voxel, the smallest distance lowered into it so far as an
// order-preserving integer of its f32 bits (negative values flipped whole, positive ones with
// the sign bit set): kNoHit until a particle reaches the voxel. The reference's key is a
// monotone function of the distance, so the key of the smallest distance, taken once per
// voxel by the resolve pass, equals the smallest of the keys the reference's atomicMin keeps;
// the splat passes never divide.
constexpr uint32_t kNoHit = 0xffffffffu;
__device__ __forceinline__ uint32_t sd_bits(float sd) {
  const uint32_t u = __float_as_uint(sd);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float bits_sd(uint32_t u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u); }

__device__ __forceinline__ uint32_t enc_key(float sd, float bw) {
  float v = clampf(__fdiv_rn(sd, bw), -1.0f, 1.0f);
  return static_cast<uint32_t>((v + 1.0f) * 32767.5f);
}

__device__ __forceinline__ bool cloud_live(const SplatDev& D, uint32_t idx, uint32_t& i) {
  if (D.order) {
    uint32_t n = min(*D.live_count, D.capacity);
    if (idx >= n) return false;
    i = D.order[idx];
    return i < D.capacity;
  }
  if (idx >= D.capacity) return false;
  i = idx;
  if (D.live_mode == 1) return idx < *D.live_count;
  if (D.live_mode == 2) {
    uint32_t f = *D.live_first;
    return idx >= f && idx < f + *D.live_range_count;
  }
  return true;
}


// Walks a bx*by*bz box in x-fastest order with one voxel per lane, 32 at a time, keeping the
// lane's (x, y, z) incrementally: the integer divisions happen once per box, not per voxel.
struct BoxWalk {
  int x, y, z;       // current voxel (relative to the box corner)
  int sx, sy, sz;    // the step of 32 voxels decomposed in the box
  int bx, by;
  __device__ __forceinline__ void init(uint32_t lane, uint32_t bxn, uint32_t byn) {
    bx = static_cast<int>(bxn);
    by = static_cast<int>(byn);
    const uint32_t bxy = bxn * byn;
    x = static_cast<int>(lane % bxn);
    y = static_cast<int>((lane / bxn) % byn);
    z = static_cast<int>(lane / bxy);
    sx = static_cast<int>(32u % bxn);
    sy = static_cast<int>((32u / bxn) % byn);
    sz = static_cast<int>(32u / bxy);
  }
  __device__ __forceinline__ void next() {
    x += sx;
    y += sy;
    z += sz;
    if (x >= bx) {
      x -= bx;
      y++;
    }
    if (y >= by) {
      y -= by;
      z++;
    }
  }
};

// One block of the splat pass: level w.sub, cloud indices [w.first, w.first + w.n). The
// volume origin (ox, oy, oz) is the f32 uniform of the baked volume.
//
// Two strategies, chosen per block from the particles' voxel boxes:
//  - block walk: when the union U of the block's boxes is compact (a cell-ordered fluid),
//    each thread owns 4 voxels of U along x and takes the minimum over every live particle
//    of the block, read as broadcasts from shared memory; one atomicMin per voxel per block.
//    dy*dy and dz*dz are computed once per particle and row, so the squared length keeps the
//    reference's rounding order (dx*dx + dy*dy) + dz*dz.
//  - warp walk: otherwise each warp works on its 32 particles, walking their union box with a
//    voxel per lane when that is compact, or each particle's own box.
__device__ __forceinline__ void splat_block(const SplatDev& D, const Work w, float ox, float oy, float oz,
                                            uint32_t acc_cap) {
  const int m = static_cast<int>(w.sub);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __shared__ float4 s_p[kSplatWarps][32];
  __shared__ float4 s_n[kSplatWarps][32];
  __shared__ int4 s_lo[kSplatWarps][32];
  __shared__ int4 s_hi[kSplatWarps][32];
  __shared__ float4 s_cp[32 * kSplatWarps];
  __shared__ float4 s_cn[32 * kSplatWarps];
  __shared__ int s_box[6];
  __shared__ float s_wb[kSplatWarps][6];  // bounding box of each warp's live particle positions
  __shared__ unsigned long long s_cost;
  __shared__ uint32_t s_woff[kSplatWarps];
  __shared__ uint32_t s_nlive;
  const uint32_t idx = w.first + threadIdx.x;
  const bool has_n = D.nrm != nullptr;
  const float voxel = D.voxel[m], bw = D.bw[m], reach = D.reach[m], inv_voxel = D.inv_voxel[m], radius = D.radius;
  const int R = D.r[m];
  const int last = R - 1;
  const long long off = D.off[m];
  uint32_t i = 0;
  bool live = (threadIdx.x < w.n) && cloud_live(D, idx, i);
  float px = 0, py = 0, pz = 0, nx = 0, ny = 0, nz = 0;
  int lx = 0, ly = 0, lz = 0, hx = -1, hy = -1, hz = -1;
  if (live) {
    const float* pp = reinterpret_cast<const float*>(D.pos + static_cast<size_t>(i) * D.pos_stride);
    px = pp[0] - ox;
    py = pp[1] - oy;
    pz = pp[2] - oz;
    if (has_n) {
      const float* nn = reinterpret_cast<const float*>(D.nrm + static_cast<size_t>(i) * D.nrm_stride);
      nx = nn[0];
      ny = nn[1];
      nz = nn[2];
      if (D.quat) {  // quatRotate (math/gpu.ts:21-25)
        float qx = D.quat[0], qy = D.quat[1], qz = D.quat[2], qw = D.quat[3];
        float tx = (qy * nz - qz * ny) * 2.0f, ty = (qz * nx - qx * nz) * 2.0f, tz = (qx * ny - qy * nx) * 2.0f;
        float rx = (nx + tx * qw) + (qy * tz - qz * ty);
        float ry = (ny + ty * qw) + (qz * tx - qx * tz);
        float rz = (nz + tz * qw) + (qx * ty - qy * tx);
        nx = rx;
        ny = ry;
        nz = rz;
      }
    }
    lx = max(f2i(floorf((px - reach) * inv_voxel)), 0);
    ly = max(f2i(floorf((py - reach) * inv_voxel)), 0);
    lz = max(f2i(floorf((pz - reach) * inv_voxel)), 0);
    hx = min(f2i(floorf((px + reach) * inv_voxel)), last);
    hy = min(f2i(floorf((py + reach) * inv_voxel)), last);
    hz = min(f2i(floorf((pz + reach) * inv_voxel)), last);
    if (lx > hx || ly > hy || lz > hz) live = false;
  }
  s_p[wid][lane] = make_float4(px, py, pz, 0.0f);
  s_n[wid][lane] = make_float4(nx, ny, nz, 0.0f);
  s_lo[wid][lane] = make_int4(lx, ly, lz, 0);
  s_hi[wid][lane] = make_int4(hx, hy, hz, 0);
  if (threadIdx.x < 6) s_box[threadIdx.x] = threadIdx.x < 3 ? 0x7fffffff : -1;
  if (threadIdx.x == 0) s_cost = 0ull;
  __syncthreads();
  // warp then block union box, live counts and the sum of the particles' own box sizes
  const uint32_t active = __ballot_sync(0xffffffffu, live);
  int ulx = __reduce_min_sync(0xffffffffu, live ? lx : 0x7fffffff);
  int uly = __reduce_min_sync(0xffffffffu, live ? ly : 0x7fffffff);
  int ulz = __reduce_min_sync(0xffffffffu, live ? lz : 0x7fffffff);
  int uhx = __reduce_max_sync(0xffffffffu, live ? hx : -1);
  int uhy = __reduce_max_sync(0xffffffffu, live ? hy : -1);
  int uhz = __reduce_max_sync(0xffffffffu, live ? hz : -1);
  const uint32_t own = live ? static_cast<uint32_t>((hx - lx + 1) * (hy - ly + 1) * (hz - lz + 1)) : 0u;
  const uint32_t cost_ind = __reduce_add_sync(0xffffffffu, (own + 31u) >> 5);
  const uint32_t wsum = __reduce_add_sync(0xffffffffu, own);
  {
    // the warp's particle bounding box (+inf / -inf when it has no live particle)
    float a0 = live ? px : __int_as_float(0x7f800000), a1 = live ? py : __int_as_float(0x7f800000),
          a2 = live ? pz : __int_as_float(0x7f800000);
    float b0 = live ? px : -__int_as_float(0x7f800000), b1 = live ? py : -__int_as_float(0x7f800000),
          b2 = live ? pz : -__int_as_float(0x7f800000);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a0 = fminf(a0, __shfl_xor_sync(0xffffffffu, a0, o));
      a1 = fminf(a1, __shfl_xor_sync(0xffffffffu, a1, o));
      a2 = fminf(a2, __shfl_xor_sync(0xffffffffu, a2, o));
      b0 = fmaxf(b0, __shfl_xor_sync(0xffffffffu, b0, o));
      b1 = fmaxf(b1, __shfl_xor_sync(0xffffffffu, b1, o));
      b2 = fmaxf(b2, __shfl_xor_sync(0xffffffffu, b2, o));
    }
    if (lane == 0) {
      s_wb[wid][0] = a0;
      s_wb[wid][1] = a1;
      s_wb[wid][2] = a2;
      s_wb[wid][3] = b0;
      s_wb[wid][4] = b1;
      s_wb[wid][5] = b2;
    }
  }
  if (lane == 0) {
    if (active) {
      atomicMin(&s_box[0], ulx);
      atomicMin(&s_box[1], uly);
      atomicMin(&s_box[2], ulz);
      atomicMax(&s_box[3], uhx);
      atomicMax(&s_box[4], uhy);
      atomicMax(&s_box[5], uhz);
    }
    atomicAdd(&s_cost, static_cast<unsigned long long>(wsum));
    s_woff[wid] = __popc(active);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t o = 0;
    for (int k = 0; k < kSplatWarps; k++) {
      uint32_t c = s_woff[k];
      s_woff[k] = o;
      o += c;
    }
    s_nlive = o;
  }
  __syncthreads();
  if (live) {
    uint32_t slot = s_woff[wid] + __popc(active & ((1u << lane) - 1u));
    s_cp[slot] = make_float4(px, py, pz, 0.0f);
    if (has_n) s_cn[slot] = make_float4(nx, ny, nz, 0.0f);
  }
  __syncthreads();
  const uint32_t nlive = s_nlive;
  if (nlive == 0) return;
  uint32_t* __restrict__ keys = D.keys + off;
  {
    const int bx0 = s_box[0], by0 = s_box[1], bz0 = s_box[2];
    const uint64_t bnx = static_cast<uint64_t>(s_box[3] - bx0 + 1), bny = static_cast<uint64_t>(s_box[4] - by0 + 1),
                   bnz = static_cast<uint64_t>(s_box[5] - bz0 + 1);
    const uint64_t bnu = bnx * bny * bnz;
    // pair evaluations of the block walk against those of each particle's own box, weighted by
    // their relative cost (the block walk's pair is ~3x cheaper for spheres, ~1.5x for discs)
    const uint64_t lhs = bnu * nlive * (has_n ? 2ull : 1ull);
    const uint64_t rhs = s_cost * D.walk_weight;
    // Spheres: register-blocked tile walk. A work item is a brick of 4 x 2 x 2 voxels against
    // a slice of the block's particles; the squared lengths share dx*dx, dy*dy, dz*dz and
    // dx*dx + dy*dy across the brick (the reference's rounding order is kept), minima go to the
    // shared tile as float bits (non-negative floats order like their bit patterns), and the
    // tile is turned into keys at the end. A union box larger than the tile (a block whose
    // particles cross from one layer of cells to the next, or a splash) is walked as sub-boxes
    // of at most acc_cap voxels, one after another through the same tile: every brick still
    // meets only the slices within reach of it, and a voxel's minimum is the same.
    const bool tile_fits = bnu <= acc_cap;
    const bool subtiled = !tile_fits && bnu <= static_cast<uint64_t>(kSplatSubtiles) * acc_cap && bnx * 4u <= acc_cap;
    if (!has_n && ((tile_fits && bnu * nlive <= s_cost * D.tile_ratio) || subtiled)) {
      extern __shared__ uint32_t s_tile[];
      // slices of ~32 consecutive (cell-ordered, so spatially close) particles, each with its
      // own bounding box: a brick out of reach of a slice's box skips that slice
      const uint32_t nsl = max(1u, (nlive + 31u) >> 5);  // <= kSplatWarps
      const uint32_t per = (nlive + nsl - 1u) / nsl;
      __shared__ float s_sb[kSplatWarps][6];
      // with every particle of the block live, slice k is warp k and its box is the warp's
      const bool warp_slices = nlive == 32u * kSplatWarps;
      if (static_cast<uint32_t>(wid) < nsl) {
        if (warp_slices) {
          if (lane < 6) s_sb[wid][lane] = s_wb[wid][lane];
        } else {
          const uint32_t j0 = static_cast<uint32_t>(wid) * per, j1 = min(nlive, j0 + per);
          float a0 = __int_as_float(0x7f800000), a1 = a0, a2 = a0, b0 = -a0, b1 = -a0, b2 = -a0;
          for (uint32_t j = j0 + lane; j < j1; j += 32) {
            const float4 q = s_cp[j];
            a0 = fminf(a0, q.x);
            a1 = fminf(a1, q.y);
            a2 = fminf(a2, q.z);
            b0 = fmaxf(b0, q.x);
            b1 = fmaxf(b1, q.y);
            b2 = fmaxf(b2, q.z);
          }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            a0 = fminf(a0, __shfl_xor_sync(0xffffffffu, a0, o));
            a1 = fminf(a1, __shfl_xor_sync(0xffffffffu, a1, o));
            a2 = fminf(a2, __shfl_xor_sync(0xffffffffu, a2, o));
            b0 = fmaxf(b0, __shfl_xor_sync(0xffffffffu, b0, o));
            b1 = fmaxf(b1, __shfl_xor_sync(0xffffffffu, b1, o));
            b2 = fmaxf(b2, __shfl_xor_sync(0xffffffffu, b2, o));
          }
          if (lane == 0) {
            s_sb[wid][0] = a0;
            s_sb[wid][1] = a1;
            s_sb[wid][2] = a2;
            s_sb[wid][3] = b0;
            s_sb[wid][4] = b1;
            s_sb[wid][5] = b2;
          }
        }
      }
      const float cull = reach * 1.0001f + 1e-5f;
      const float cull2 = cull * cull;
      __shared__ uint16_t s_items[kSplatItems];
      __shared__ uint32_t s_nitems;
      auto divm = [](uint32_t x, uint64_t m) { return static_cast<uint32_t>((static_cast<uint64_t>(x) * m) >> 32); };
      // Sub-boxes: the full x extent (at most acc_cap / 4 voxels, checked above) times an even
      // number of rows and of layers, so that bricks never straddle two sub-boxes and each
      // sub-box holds at most acc_cap voxels.
      // The sub-box being walked lives in shared memory (its first row and layer in the union
      // box, and the rows and layers per sub-box), so that no loop state stays in registers
      // through the walk.
      __shared__ uint32_t s_subbox[4];
      if (threadIdx.x == 0) {
        const uint32_t fx = static_cast<uint32_t>(bnx), fy = static_cast<uint32_t>(bny), fz = static_cast<uint32_t>(bnz);
        const uint32_t sub_y = tile_fits ? fy : min(fy, max(2u, (acc_cap / (2u * fx)) & ~1u));
        s_subbox[0] = 0u;
        s_subbox[1] = 0u;
        s_subbox[2] = sub_y;
        s_subbox[3] = tile_fits ? fz : min(fz, max(2u, (acc_cap / (fx * sub_y)) & ~1u));
      }
      for (;;) {
        __syncthreads();  // the previous sub-box's write-out has read the tile; the next one is published
        const uint32_t oy = s_subbox[0], oz = s_subbox[1];
        const uint32_t ux = static_cast<uint32_t>(s_box[3] - s_box[0] + 1);
        const uint32_t fy = static_cast<uint32_t>(s_box[4] - s_box[1] + 1), fz = static_cast<uint32_t>(s_box[5] - s_box[2] + 1);
        if (oz >= fz) break;
        const int bx0 = s_box[0], by0 = s_box[1] + static_cast<int>(oy), bz0 = s_box[2] + static_cast<int>(oz);
        const uint32_t uy = min(s_subbox[2], fy - oy), uz = min(s_subbox[3], fz - oz);
        const uint32_t nbu = ux * uy * uz;
        for (uint32_t v = threadIdx.x; v < nbu; v += blockDim.x) s_tile[v] = 0x7f800000u;
        const uint32_t ngx = (ux + 3u) >> 2, ngy = (uy + 1u) >> 1, ngz = (uz + 1u) >> 1;
        const uint32_t ngroups = ngx * ngy * ngz;
        if (threadIdx.x == 0) s_nitems = 0u;
        __syncthreads();
        const uint32_t nall = ngroups * nsl;
        // Item decode by multiplication: for x < 2^16 and 1 <= d < 2^15, floor(x * ceil(2^32 / d)
        // / 2^32) == x / d (the excess x * (ceil - 2^32 / d) / 2^32 stays below 2^-16 < 1 / d).
        // Items number below ngroups * nsl <= 4096 * 8 and tile voxels below 4096, so every
        // operand is in range.
        const uint64_t m_groups = static_cast<uint64_t>(0xffffffffu / ngroups) + 1u;
        const uint64_t m_gx = static_cast<uint64_t>(0xffffffffu / ngx) + 1u;
        const uint64_t m_gy = static_cast<uint64_t>(0xffffffffu / ngy) + 1u;
        const uint64_t m_ux = static_cast<uint64_t>(0xffffffffu / ux) + 1u;
        const uint64_t m_uy = static_cast<uint64_t>(0xffffffffu / uy) + 1u;
        auto brick_of = [&](uint32_t it, uint32_t& sl, uint32_t& lx0, uint32_t& ly0, uint32_t& lz0) {
          sl = divm(it, m_groups);
          const uint32_t g = it - sl * ngroups;
          const uint32_t rest = divm(g, m_gx);
          lx0 = (g - rest * ngx) * 4u;  // brick corner in the union box
          const uint32_t rz = divm(rest, m_gy);
          ly0 = (rest - rz * ngy) * 2u;
          lz0 = rz * 2u;
        };
        // a brick farther than the reach from a slice's bounding box: nothing to lower
        auto culled = [&](uint32_t sl, uint32_t lx0, uint32_t ly0, uint32_t lz0) {
          const float* sb = s_sb[sl];
          const float x0f = (static_cast<float>(bx0 + static_cast<int>(lx0)) + 0.5f) * voxel;
          const float y0f = (static_cast<float>(by0 + static_cast<int>(ly0)) + 0.5f) * voxel;
          const float z0f = (static_cast<float>(bz0 + static_cast<int>(lz0)) + 0.5f) * voxel;
          const float x1f = (static_cast<float>(bx0 + static_cast<int>(lx0) + 3) + 0.5f) * voxel;
          const float y1f = (static_cast<float>(by0 + static_cast<int>(ly0) + 1) + 0.5f) * voxel;
          const float z1f = (static_cast<float>(bz0 + static_cast<int>(lz0) + 1) + 0.5f) * voxel;
          const float ex = fmaxf(fmaxf(sb[0] - x1f, x0f - sb[3]), 0.0f);
          const float ey = fmaxf(fmaxf(sb[1] - y1f, y0f - sb[4]), 0.0f);
          const float ez = fmaxf(fmaxf(sb[2] - z1f, z0f - sb[5]), 0.0f);
          return ex * ex + ey * ey + ez * ez > cull2;
        };
        // the (brick, slice) items that survive the cull, compacted so that lanes stay busy
        const bool compact = nall <= static_cast<uint32_t>(kSplatItems);
        if (compact) {
          // One thread per row of bricks along x (a slice, a row and a layer of bricks): the
          // y and z parts of the cull are formed once per row, then each brick of the row takes
          // the same test as culled() (the same operations, so the same survivors). The row's
          // survivors are counted, placed after the warp's earlier rows by a warp scan and one
          // atomic per warp, and written (the items' order does not change any minimum).
          const uint32_t nyz = ngy * ngz, nrows = nyz * nsl;
          const uint64_t m_yz = static_cast<uint64_t>(0xffffffffu / nyz) + 1u;
          for (uint32_t base = 0; base < nrows; base += blockDim.x) {
            const uint32_t r = base + threadIdx.x;
            uint32_t sl = 0, gyz = 0, keep = 0;
            float ey2 = 0.0f, ez2 = 0.0f;
            const float* sb = s_sb[0];
            auto row_keeps = [&](uint32_t gx) {
              const float x0f = (static_cast<float>(bx0 + static_cast<int>(gx * 4u)) + 0.5f) * voxel;
              const float x1f = (static_cast<float>(bx0 + static_cast<int>(gx * 4u) + 3) + 0.5f) * voxel;
              const float ex = fmaxf(fmaxf(sb[0] - x1f, x0f - sb[3]), 0.0f);
              return !(ex * ex + ey2 + ez2 > cull2);
            };
            if (r < nrows) {
              sl = divm(r, m_yz);
              gyz = r - sl * nyz;
              const uint32_t gz = divm(gyz, m_gy), gy = gyz - gz * ngy;
              sb = s_sb[sl];
              const float y0f = (static_cast<float>(by0 + static_cast<int>(gy * 2u)) + 0.5f) * voxel;
              const float z0f = (static_cast<float>(bz0 + static_cast<int>(gz * 2u)) + 0.5f) * voxel;
              const float y1f = (static_cast<float>(by0 + static_cast<int>(gy * 2u) + 1) + 0.5f) * voxel;
              const float z1f = (static_cast<float>(bz0 + static_cast<int>(gz * 2u) + 1) + 0.5f) * voxel;
              const float ey = fmaxf(fmaxf(sb[1] - y1f, y0f - sb[4]), 0.0f);
              const float ez = fmaxf(fmaxf(sb[2] - z1f, z0f - sb[5]), 0.0f);
              ey2 = ey * ey;
              ez2 = ez * ez;
              for (uint32_t gx = 0; gx < ngx; gx++) keep += row_keeps(gx) ? 1u : 0u;
            }
            uint32_t incl = keep;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
              const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
              if (lane >= static_cast<uint32_t>(o)) incl += y;
            }
            uint32_t o = 0;
            if (lane == 31 && incl) o = atomicAdd(&s_nitems, incl);
            o = __shfl_sync(0xffffffffu, o, 31) + incl - keep;
            if (keep) {
              const uint32_t it0 = sl * ngroups + ngx * gyz;
              for (uint32_t gx = 0; gx < ngx; gx++)
                if (row_keeps(gx)) s_items[o++] = static_cast<uint16_t>(it0 + gx);
            }
          }
          __syncthreads();
        }
        const uint32_t nwork = compact ? s_nitems : nall;
        // Work units: the items of the last partial round are split into their slices' two halves,
        // so that round's threads carry half an item each rather than some a whole one and the
        // rest none; the block waits for its slowest thread at the barrier below. A voxel's
        // minimum is the same over the halves as over the whole slice.
        const uint32_t full = (nwork / blockDim.x) * blockDim.x;
        const uint32_t rest = nwork - full;
        const bool split = rest > 0 && 2u * rest <= blockDim.x;
        const uint32_t nunits = split ? full + 2u * rest : nwork;
        for (uint32_t u = threadIdx.x; u < nunits; u += blockDim.x) {
          const bool half_unit = split && u >= full;
          const uint32_t i = half_unit ? full + ((u - full) >> 1) : u;
          const uint32_t it = compact ? static_cast<uint32_t>(s_items[i]) : i;
          uint32_t sl, lx0, ly0, lz0;
          brick_of(it, sl, lx0, ly0, lz0);
          if (!compact && culled(sl, lx0, ly0, lz0)) continue;
          const int x0 = bx0 + static_cast<int>(lx0), y0 = by0 + static_cast<int>(ly0), z0 = bz0 + static_cast<int>(lz0);
          // voxel centres (x + 0.5) * voxel: one conversion per axis, since float(x0) + (k + 0.5)
          // equals float(x0 + k) + 0.5 exactly for grid coordinates (integers far below 2^23)
          float cx[4], cy[2], cz[2];
          const float fx0 = static_cast<float>(x0), fy0 = static_cast<float>(y0), fz0 = static_cast<float>(z0);
#pragma unroll
          for (int k = 0; k < 4; k++) cx[k] = (fx0 + (static_cast<float>(k) + 0.5f)) * voxel;
#pragma unroll
          for (int k = 0; k < 2; k++) {
            cy[k] = (fy0 + (static_cast<float>(k) + 0.5f)) * voxel;
            cz[k] = (fz0 + (static_cast<float>(k) + 0.5f)) * voxel;
          }
          // Minima of squared lengths as float bits (non-negative floats order like their bit
          // patterns), two particles per step: the squared lengths keep the reference's rounding
          // order (dx*dx + dy*dy) + dz*dz, and one three-input minimum folds both particles into
          // a voxel's running minimum.
          uint32_t b[16];
#pragma unroll
          for (int k = 0; k < 16; k++) b[k] = 0x7f800000u;
          // the 16 squared lengths of one particle, indexed xx + 4 * yy + 8 * zz
          auto lengths = [&](const float4 q, uint32_t (&u)[16]) {
            float dx2[4], dy2[2], dz2[2];
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const float d = cx[k] - q.x;
              dx2[k] = d * d;
            }
#pragma unroll
            for (int k = 0; k < 2; k++) {
              const float dy = cy[k] - q.y, dz = cz[k] - q.z;
              dy2[k] = dy * dy;
              dz2[k] = dz * dz;
            }
#pragma unroll
            for (int yy = 0; yy < 2; yy++)
#pragma unroll
              for (int xx = 0; xx < 4; xx++) {
                const float t = dx2[xx] + dy2[yy];
#pragma unroll
                for (int zz = 0; zz < 2; zz++) u[xx + 4 * yy + 8 * zz] = __float_as_uint(t + dz2[zz]);
              }
          };
          uint32_t j1 = min(nlive, (sl + 1u) * per);
          uint32_t j = sl * per;
          if (half_unit) {  // this unit's half of the slice
            const uint32_t mid = j + ((j1 - min(j, j1)) >> 1);
            if ((u - full) & 1u) j = mid;
            else j1 = mid;
          }
          for (; j + 1u < j1; j += 2u) {
            uint32_t ua[16], ub[16];
            lengths(s_cp[j], ua);
            lengths(s_cp[j + 1u], ub);
#pragma unroll
            for (int k = 0; k < 16; k++) b[k] = __vimin3_u32(b[k], ua[k], ub[k]);
          }
          if (j < j1) {
            uint32_t ua[16];
            lengths(s_cp[j], ua);
#pragma unroll
            for (int k = 0; k < 16; k++) b[k] = min(b[k], ua[k]);
          }
#pragma unroll
          for (int zz = 0; zz < 2; zz++)
#pragma unroll
            for (int yy = 0; yy < 2; yy++)
#pragma unroll
              for (int xx = 0; xx < 4; xx++) {
                const uint32_t lx = lx0 + xx, ly = ly0 + yy, lz = lz0 + zz;
                const uint32_t v = b[xx + 4 * yy + 8 * zz];
                if (lx < ux && ly < uy && lz < uz && v < 0x7f800000u) atomicMin(&s_tile[lx + ux * (ly + uy * lz)], v);
              }
        }
        __syncthreads();
        for (uint32_t v = threadIdx.x; v < nbu; v += blockDim.x) {
          const uint32_t bits = s_tile[v];
          if (bits == 0x7f800000u) continue;
          const float sd = __fsqrt_rn(__uint_as_float(bits)) - radius;
          if (sd < bw) {
            const uint32_t vy = divm(v, m_ux), vz = divm(vy, m_uy);  // v < 4096: decode by multiplication
            const int x = bx0 + static_cast<int>(v - vy * ux), y = by0 + static_cast<int>(vy - vz * uy), z = bz0 + static_cast<int>(vz);
            atomicMin(keys + (static_cast<long long>(x) + static_cast<long long>(R) * (y + static_cast<long long>(R) * z)),
                      sd_bits(sd));
          }
        }
        if (threadIdx.x == 0) {  // the next sub-box: along y, then along z
          const uint32_t ny = s_subbox[0] + s_subbox[2];
          const bool wrap = ny >= static_cast<uint32_t>(s_box[4] - s_box[1] + 1);
          s_subbox[0] = wrap ? 0u : ny;
          s_subbox[1] = wrap ? s_subbox[1] + s_subbox[3] : s_subbox[1];
        }
      }
      return;
    }
    if (bnu < (1ull << 30) && lhs <= rhs) {
      const uint32_t ngx = static_cast<uint32_t>((bnx + 3) >> 2);
      const uint32_t ngroups = ngx * static_cast<uint32_t>(bny * bnz);
      const int bhx = s_box[3];
      // the block's particle bounding box from its warps' boxes
      float pbx0 = s_wb[0][0], pby0 = s_wb[0][1], pbz0 = s_wb[0][2], pbx1 = s_wb[0][3], pby1 = s_wb[0][4], pbz1 = s_wb[0][5];
      for (int k = 1; k < kSplatWarps; k++) {
        pbx0 = fminf(pbx0, s_wb[k][0]);
        pby0 = fminf(pby0, s_wb[k][1]);
        pbz0 = fminf(pbz0, s_wb[k][2]);
        pbx1 = fmaxf(pbx1, s_wb[k][3]);
        pby1 = fmaxf(pby1, s_wb[k][4]);
        pbz1 = fmaxf(pbz1, s_wb[k][5]);
      }
      // A group of voxels farther than the reach from the particles' bounding box cannot be
      // lowered by any of them (sd >= bandWorld): skipped. The 1e-4 margin covers f32 rounding.
      const float cull = reach * 1.0001f + 1e-5f;
      const float cull2 = cull * cull;
      for (uint32_t g = threadIdx.x; g < ngroups; g += blockDim.x) {
        const uint32_t gx = g % ngx, rest = g / ngx;
        const int y = by0 + static_cast<int>(rest % static_cast<uint32_t>(bny));
        const int z = bz0 + static_cast<int>(rest / static_cast<uint32_t>(bny));
        const int x0 = bx0 + static_cast<int>(gx * 4);
        {
          const float gx0 = (static_cast<float>(x0) + 0.5f) * voxel, gx1 = (static_cast<float>(x0 + 3) + 0.5f) * voxel;
          const float gy = (static_cast<float>(y) + 0.5f) * voxel, gz = (static_cast<float>(z) + 0.5f) * voxel;
          const float ex = fmaxf(fmaxf(pbx0 - gx1, gx0 - pbx1), 0.0f);
          const float ey = fmaxf(fmaxf(pby0 - gy, gy - pby1), 0.0f);
          const float ez = fmaxf(fmaxf(pbz0 - gz, gz - pbz1), 0.0f);
          if (ex * ex + ey * ey + ez * ez > cull2) continue;
        }
        float cx[4], b[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          cx[k] = (static_cast<float>(x0 + k) + 0.5f) * voxel;
          b[k] = __int_as_float(0x7f800000);
        }
        const float cy = (static_cast<float>(y) + 0.5f) * voxel;
        const float cz = (static_cast<float>(z) + 0.5f) * voxel;
        if (!has_n) {
#pragma unroll 4
          for (uint32_t j = 0; j < nlive; j++) {
            const float4 q = s_cp[j];
            const float dy = cy - q.y, dz = cz - q.z;
            const float dy2 = dy * dy, dz2 = dz * dz;
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const float dx = cx[k] - q.x;
              float t = dx * dx;
              t = t + dy2;
              t = t + dz2;
              b[k] = fminf(b[k], t);
            }
          }
#pragma unroll
          for (int k = 0; k < 4; k++) b[k] = __fsqrt_rn(b[k]) - radius;
        } else {
          // b starts at bandWorld: only values below it are ever written. A pair is skipped
          // when it provably cannot lower b: its plane term is already >= b, or its squared
          // length is beyond (b + radius)^2 (with a 1e-5 margin over f32 rounding).
#pragma unroll
          for (int k = 0; k < 4; k++) b[k] = bw;
          for (uint32_t j = 0; j < nlive; j++) {
            const float4 q = s_cp[j];
            const float4 nn = s_cn[j];
            const float dy = cy - q.y, dz = cz - q.z;
            const float dy2 = dy * dy, dz2 = dz * dz;
            const float dyn = dy * nn.y, dzn = dz * nn.z;
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const float dx = cx[k] - q.x;
              float pl = dx * nn.x;
              pl = pl + dyn;
              pl = pl + dzn;
              if (pl < b[k]) {
                float t = dx * dx;
                t = t + dy2;
                t = t + dz2;
                const float thr = b[k] + radius;
                if (thr > 0.0f && t < thr * thr * 1.00001f) b[k] = fminf(b[k], fmaxf(pl, __fsqrt_rn(t) - radius));
              }
            }
          }
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
          if (x0 + k <= bhx && b[k] < bw)
            atomicMin(keys + (static_cast<long long>(x0 + k) + static_cast<long long>(R) * (y + static_cast<long long>(R) * z)),
                      sd_bits(b[k]));
        }
      }
      return;
    }
  }
  // Warp walks. When the block's union box fits in shared memory the minima are taken there
  // first (shared-memory atomicMin of the distance as an order-preserving integer, so the key,
  // a division, is taken once per voxel) and written out with one global atomicMin per touched
  // voxel; otherwise every hit goes to the key grid directly. The key is monotone in the
  // distance, so the key of the minimum is the minimum of the keys.
  extern __shared__ uint32_t s_acc[];  // acc_cap voxels of dynamic shared memory
  const int ax0 = s_box[0], ay0 = s_box[1], az0 = s_box[2];
  const uint32_t anx = static_cast<uint32_t>(s_box[3] - ax0 + 1), any = static_cast<uint32_t>(s_box[4] - ay0 + 1),
                 anz = static_cast<uint32_t>(s_box[5] - az0 + 1);
  const uint64_t an = static_cast<uint64_t>(anx) * any * anz;
  const bool use_acc = an <= static_cast<uint64_t>(acc_cap);
  if (use_acc) {
    for (uint32_t v = threadIdx.x; v < static_cast<uint32_t>(an); v += blockDim.x) s_acc[v] = kNoHit;
    __syncthreads();
  }
  auto emit = [&](int x, int y, int z, float sd) {  // sd < bandWorld
    if (use_acc) {
      uint32_t a = static_cast<uint32_t>(x - ax0) + anx * (static_cast<uint32_t>(y - ay0) + any * static_cast<uint32_t>(z - az0));
      atomicMin(&s_acc[a], sd_bits(sd));
    } else {
      atomicMin(keys + (static_cast<long long>(x) + static_cast<long long>(R) * (y + static_cast<long long>(R) * z)),
                sd_bits(sd));
    }
  };
  const float reach2_hi = (bw + radius) * (bw + radius) * 1.00001f;
  // The own-box walk visits a stencil instead of a particle's whole box: the voxel offsets,
  // relative to the voxel holding the particle, that lie within the reach of some point of
  // one octant of that voxel (mirrored per axis to the particle's octant). Every voxel the
  // particle can lower (squared length below reach2_hi, i.e. within the reach to 1e-5) is in
  // it: the octant is widened by 0.02 voxel and the reach by 0.02 voxel, far above the f32
  // rounding of the particle's voxel coordinates. With a band of 4 voxels it holds about half
  // of the box's voxels, so lanes spend fewer steps outside the reach. Offsets are packed in
  // 4 bits per axis; a reach beyond 6 voxels keeps the box walk.
  __shared__ uint32_t s_st[kSplatStencil];
  __shared__ uint32_t s_nst;
  __shared__ float2 s_dt[kSplatWarps][3][16];  // per warp: the current particle's per-axis terms
  const float rv = reach * inv_voxel;
  const int sn = static_cast<int>(ceilf(rv)) + 1;  // candidate offsets in [-sn, sn]
  bool use_st = rv > 0.0f && sn <= 7;
  if (use_st) {
    if (threadIdx.x == 0) s_nst = 0u;
    __syncthreads();
    const uint32_t side = static_cast<uint32_t>(2 * sn + 1), cand = side * side * side;
    const float lim = (rv + 0.02f) * (rv + 0.02f);
    auto gap = [](int o) {  // distance from the centre at offset o to the widened octant [-0.02, 0.52]
      const float f = static_cast<float>(o);
      return f > 0.52f ? f - 0.52f : (f < -0.02f ? -0.02f - f : 0.0f);
    };
    for (uint32_t c0 = 0; c0 < cand; c0 += blockDim.x) {
      const uint32_t c = c0 + threadIdx.x;
      bool keep = false;
      uint32_t e = 0;
      if (c < cand) {
        const int ox = static_cast<int>(c % side) - sn, oy = static_cast<int>((c / side) % side) - sn,
                  oz = static_cast<int>(c / (side * side)) - sn;
        const float gx = gap(ox), gy = gap(oy), gz = gap(oz);
        keep = gx * gx + gy * gy + gz * gz < lim;
        e = static_cast<uint32_t>(ox + 8) | (static_cast<uint32_t>(oy + 8) << 4) | (static_cast<uint32_t>(oz + 8) << 8);
      }
      const uint32_t m = __ballot_sync(0xffffffffu, keep);
      uint32_t o = 0;
      if (lane == 0 && m) o = atomicAdd(&s_nst, static_cast<uint32_t>(__popc(m)));
      o = __shfl_sync(0xffffffffu, o, 0);
      const uint32_t pos = o + __popc(m & ((1u << lane) - 1u));
      if (keep && pos < static_cast<uint32_t>(kSplatStencil)) s_st[pos] = e;
    }
    __syncthreads();
    use_st = s_nst <= static_cast<uint32_t>(kSplatStencil);
  }
  if (active != 0u) {
    const uint32_t nux = static_cast<uint32_t>(uhx - ulx + 1), nuy = static_cast<uint32_t>(uhy - uly + 1),
                   nuz = static_cast<uint32_t>(uhz - ulz + 1);
    const uint64_t nu64 = static_cast<uint64_t>(nux) * nuy * nuz;
    const uint32_t nact = __popc(active);
    // union walk when its lane-steps (each over every particle of the warp) cost less than the
    // particles' own walks: a union step per particle costs about half an own-walk step for
    // discs, a third for spheres (no plane term, no square root until the end)
    const uint64_t own_steps = use_st ? static_cast<uint64_t>(nact) * ((s_nst + 31u) >> 5) : cost_ind;
    if (nu64 < (1ull << 31) && ((nu64 + 31) >> 5) * nact <= (has_n ? 2ull : 3ull) * own_steps) {
      const uint32_t nu = static_cast<uint32_t>(nu64);
      BoxWalk bw_;
      bw_.init(lane, nux, nuy);
      for (uint32_t v0 = 0; v0 < nu; v0 += 32, bw_.next()) {
        uint32_t v = v0 + lane;
        int x = ulx + bw_.x;
        int y = uly + bw_.y;
        int z = ulz + (v < nu ? bw_.z : 0);
        float cxf = (static_cast<float>(x) + 0.5f) * voxel;
        float cyf = (static_cast<float>(y) + 0.5f) * voxel;
        float czf = (static_cast<float>(z) + 0.5f) * voxel;
        float best = __int_as_float(0x7f800000);
        uint32_t rem = active;
        if (!has_n) {
          while (rem) {
            int j = __ffs(rem) - 1;
            rem &= rem - 1;
            float4 q = s_p[wid][j];
            float dx = cxf - q.x, dy = cyf - q.y, dz = czf - q.z;
            float d2 = (dx * dx + dy * dy) + dz * dz;
            best = fminf(best, d2);
          }
          best = __fsqrt_rn(best) - radius;
        } else {
          best = bw;  // as in the block walk: skip pairs that cannot lower best
          while (rem) {
            int j = __ffs(rem) - 1;
            rem &= rem - 1;
            float4 q = s_p[wid][j];
            float4 nn = s_n[wid][j];
            float dx = cxf - q.x, dy = cyf - q.y, dz = czf - q.z;
            float pl = dot3(dx, dy, dz, nn.x, nn.y, nn.z);
            if (pl < best) {
              float t = (dx * dx + dy * dy) + dz * dz;
              const float thr = best + radius;
              if (thr > 0.0f && t < thr * thr * 1.00001f) best = fminf(best, fmaxf(pl, __fsqrt_rn(t) - radius));
            }
          }
        }
        if (v < nu && best < bw) emit(x, y, z, best);
      }
    } else {
      uint32_t rem = active;
      while (rem) {
        int j = __ffs(rem) - 1;
        rem &= rem - 1;
        float4 q = s_p[wid][j];
        float4 nn = s_n[wid][j];
        int4 lo = s_lo[wid][j], hi = s_hi[wid][j];
        auto visit = [&](int x, int y, int z) {
          float dx = (static_cast<float>(x) + 0.5f) * voxel - q.x;
          float dy = (static_cast<float>(y) + 0.5f) * voxel - q.y;
          float dz = (static_cast<float>(z) + 0.5f) * voxel - q.z;
          // a voxel whose plane term or squared length already puts it at or beyond the band
          // cannot pass sd < bandWorld: skip its square root
          float pl = has_n ? dot3(dx, dy, dz, nn.x, nn.y, nn.z) : -__int_as_float(0x7f800000);
          if (pl >= bw) return;
          float t = (dx * dx + dy * dy) + dz * dz;
          if (t >= reach2_hi) return;
          float sd = fmaxf(pl, __fsqrt_rn(t) - radius);
          if (sd < bw) emit(x, y, z, sd);
        };
        if (use_st) {
          const float fx = q.x * inv_voxel, fy = q.y * inv_voxel, fz = q.z * inv_voxel;
          const float flx = floorf(fx), fly = floorf(fy), flz = floorf(fz);
          const int cxv = f2i(flx), cyv = f2i(fly), czv = f2i(flz);
          const int sx = fx - flx >= 0.5f ? 1 : -1, sy = fy - fly >= 0.5f ? 1 : -1, sz = fz - flz >= 0.5f ? 1 : -1;
          // Per axis, the voxel offsets the stencil can reach, indexed by the stencil's own 4-bit
          // field i (offset i - 8, mirrored to the particle's octant), as (d * n, d * d) with
          // d = centre - particle: the same operations visit() does per voxel, done once per
          // particle; a voxel then adds them as (dx*nx + dy*ny) + dz*nz and (dx*dx + dy*dy) +
          // dz*dz, the reference's rounding order. Which offsets land inside the particle's box
          // is kept as bits (ballots): x in the low half of vxy, y in the high half, z in vz.
          bool in_box;
          {
            const int axis = lane >= 16 ? 1 : 0, i = static_cast<int>(lane & 15u);
            const int c = (axis ? cyv : cxv) + (axis ? sy : sx) * (i - 8);
            const float d = (static_cast<float>(c) + 0.5f) * voxel - (axis ? q.y : q.x);
            s_dt[wid][axis][i] = make_float2(d * (axis ? nn.y : nn.x), d * d);
            in_box = axis ? (c >= lo.y && c <= hi.y) : (c >= lo.x && c <= hi.x);
          }
          const uint32_t vxy = __ballot_sync(0xffffffffu, in_box);
          {
            const int i = static_cast<int>(lane & 15u), c = czv + sz * (i - 8);
            if (lane < 16) {
              const float d = (static_cast<float>(c) + 0.5f) * voxel - q.z;
              s_dt[wid][2][i] = make_float2(d * nn.z, d * d);
            }
            in_box = lane < 16 && c >= lo.z && c <= hi.z;
          }
          const uint32_t vz = __ballot_sync(0xffffffffu, in_box);
          __syncwarp();
          const uint32_t ns = s_nst;
          // A stencil wholly inside the volume needs no box test: a voxel outside the
          // particle's box is at least half a voxel beyond its reach, which the length test
          // below rejects. Only where the volume clips the box does the box decide.
          const bool inside = cxv - sn >= 0 && cxv + sn <= last && cyv - sn >= 0 && cyv + sn <= last &&
                              czv - sn >= 0 && czv + sn <= last;
          // the voxel of stencil field (ex, ey, ez) as a linear index: in the shared minimum
          // tile when the block's union box fits it, else in the level's key grid
          const int asy = sy * static_cast<int>(anx), asz = sz * static_cast<int>(anx * any);
          const int abase = (cxv - ax0) + static_cast<int>(anx) * ((cyv - ay0) + static_cast<int>(any) * (czv - az0));
          const int gsy = sy * R, gsz = sz * R * R;
          const long long gbase = static_cast<long long>(cxv) + static_cast<long long>(R) * (cyv + static_cast<long long>(R) * czv);
          for (uint32_t v = lane; v < ns; v += 32) {
            const uint32_t e = s_st[v];
            const uint32_t ex = e & 15u, ey = (e >> 4) & 15u, ez = (e >> 8) & 15u;
            if (!inside && !((vxy >> ex) & (vxy >> (16u + ey)) & (vz >> ez) & 1u)) continue;
            const float2 tx = s_dt[wid][0][ex], ty = s_dt[wid][1][ey], tz = s_dt[wid][2][ez];
            const float pl = has_n ? (tx.x + ty.x) + tz.x : -__int_as_float(0x7f800000);
            if (pl >= bw) continue;
            const float t = (tx.y + ty.y) + tz.y;
            if (t >= reach2_hi) continue;
            const float sd = fmaxf(pl, __fsqrt_rn(t) - radius);
            if (sd < bw) {
              const int rx = static_cast<int>(ex) - 8, ry = static_cast<int>(ey) - 8, rz = static_cast<int>(ez) - 8;
              if (use_acc) atomicMin(&s_acc[abase + sx * rx + asy * ry + asz * rz], sd_bits(sd));
              else atomicMin(keys + (gbase + (sx * rx + gsy * ry + gsz * rz)), sd_bits(sd));
            }
          }
          __syncwarp();  // the tables are rewritten for the next particle
          continue;
        }
        uint32_t bxn = static_cast<uint32_t>(hi.x - lo.x + 1), byn = static_cast<uint32_t>(hi.y - lo.y + 1),
                 bzn = static_cast<uint32_t>(hi.z - lo.z + 1);
        uint32_t nb = bxn * byn * bzn;
        BoxWalk bw_;
        bw_.init(lane, bxn, byn);
        for (uint32_t v = lane; v < nb; v += 32, bw_.next()) visit(lo.x + bw_.x, lo.y + bw_.y, lo.z + bw_.z);
      }
    }
  }
  if (use_acc) {
    __syncthreads();
    for (uint32_t v = threadIdx.x; v < static_cast<uint32_t>(an); v += blockDim.x) {
      const uint32_t u = s_acc[v];
      if (u != kNoHit) {
        int x = ax0 + static_cast<int>(v % anx);
        int y = ay0 + static_cast<int>((v / anx) % any);
        int z = az0 + static_cast<int>(v / (anx * any));
        atomicMin(keys + (static_cast<long long>(x) + static_cast<long long>(R) * (y + static_cast<long long>(R) * z)), u);
      }
    }
  }
}

// resolve[m] (splat.ts:258-276): the voxel's key, u32((clamp(sd / bandWorld, -1, 1) + 1) *
// 32767.5) of its smallest distance (65535 where no particle reached it), then
// v = f32(key) * (1/32767.5) - 1 stored as f16 (round to nearest even). The grid is reset to
// kNoHit behind the read, which is the clear of the next bake (splat.ts:200-210).
__device__ __forceinline__ void resolve_block(const SplatDev& D, const Work w) {
  const long long base = static_cast<long long>(w.first) * 4;
  const long long v0 = base + static_cast<long long>(threadIdx.x) * 4;
  const float inv = 3.0518043793392844e-05f;  // f32(1/32767.5)
  if (v0 >= D.total) return;
  // the level of these voxels (level sizes are multiples of 4, so four share one)
  int m = 0;
  while (m + 1 < D.mips && v0 >= D.off[m + 1]) m++;
  const float bw = D.bw[m];
  auto key_of = [&](uint32_t u) { return u == kNoHit ? 65535u : enc_key(bits_sd(u), bw); };
  if (v0 + 3 < D.total) {
    const uint4 u4 = *reinterpret_cast<const uint4*>(D.keys + v0);
    const uint4 k4 = make_uint4(key_of(u4.x), key_of(u4.y), key_of(u4.z), key_of(u4.w));
    if (D.key_capture) *reinterpret_cast<uint4*>(D.key_capture + v0) = k4;
    // most voxels of a bake volume are reached by no particle and hold kNoHit already
    if ((u4.x & u4.y & u4.z & u4.w) != kNoHit)
      *reinterpret_cast<uint4*>(D.keys + v0) = make_uint4(kNoHit, kNoHit, kNoHit, kNoHit);
    __half2 a = __halves2half2(__float2half_rn(static_cast<float>(k4.x) * inv - 1.0f),
                               __float2half_rn(static_cast<float>(k4.y) * inv - 1.0f));
    __half2 b = __halves2half2(__float2half_rn(static_cast<float>(k4.z) * inv - 1.0f),
                               __float2half_rn(static_cast<float>(k4.w) * inv - 1.0f));
    __half2* out = reinterpret_cast<__half2*>(D.dist_out + v0);
    out[0] = a;
    out[1] = b;
  } else {
    for (long long v = v0; v < D.total && v < v0 + 4; v++) {
      const uint32_t key = key_of(D.keys[v]);
      if (D.key_capture) D.key_capture[v] = key;
      D.keys[v] = kNoHit;
      D.dist_out[v] = __float2half_rn(static_cast<float>(key) * inv - 1.0f);
    }
  }
}

#ifndef CLAY_ONLY_NEIGHBOUR_PASSES
__global__ void __launch_bounds__(32 * kSplatWarps, 4) k_splat(const SplatDev* __restrict__ splats, const Work* __restrict__ work,
                                                             uint32_t acc_cap) {
  const Work w = get_work_reversed(work);
  const SplatDev& D = splats[w.obj];
  splat_block(D, w, D.vp->origin[0], D.vp->origin[1], D.vp->origin[2], acc_cap);
}

__global__ void k_resolve(const SplatDev* __restrict__ splats, const Work* __restrict__ work) {
  const Work w = get_work(work);
  resolve_block(splats[w.obj], w);
}

// ---------------------------------------------------------------------------------------
// SdfBuilder.rebuild (builder.ts:87-142) with the brush fold of brush.ts:239-372.
__device__ __forceinline__ float sd_box3(float px, float py, float pz, float bx, float by, float bz) {
  float qx = fabsf(px) - bx, qy = fabsf(py) - by, qz = fabsf(pz) - bz;
  float mx = fmaxf(qx, 0.0f), my = fmaxf(qy, 0.0f), mz = fmaxf(qz, 0.0f);
  return len3(mx, my, mz) + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.0f);
}

__device__ float eval_local(uint32_t kind, float px, float py, float pz, float sx, float sy, float sz, float radius) {
  switch (kind) {
    case 0:
      return len3(px, py, pz) - sx;
    case 1:
      return sd_box3(px, py, pz, sx, sy, sz);
    case 2: {
      float qx = fabsf(px) - (sx - radius), qy = fabsf(py) - (sy - radius), qz = fabsf(pz) - (sz - radius);
      float mx = fmaxf(qx, 0.0f), my = fmaxf(qy, 0.0f), mz = fmaxf(qz, 0.0f);
      return len3(mx, my, mz) + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.0f) - radius;
    }
    case 3: {
      float pax = px, pay = py - (-sy), paz = pz;
      float bay = sy - (-sy);
      float h = clampf(__fdiv_rn(dot3(pax, pay, paz, 0.0f, bay, 0.0f), dot3(0.0f, bay, 0.0f, 0.0f, bay, 0.0f)), 0.0f, 1.0f);
      return len3(pax - 0.0f * h, pay - bay * h, paz - 0.0f * h) - radius;
    }
    case 4: {
      float qx = sqrtf(px * px + pz * pz) - sx;
      return sqrtf(qx * qx + py * py) - radius;
    }
    case 5: {
      float dx = sqrtf(px * px + pz * pz) - sx;
      float dy = fabsf(py) - sy;
      float mx = fmaxf(dx, 0.0f), my = fmaxf(dy, 0.0f);
      return fminf(fmaxf(dx, dy), 0.0f) + sqrtf(mx * mx + my * my);
    }
    case 6:
      return py - radius;
    case 7: {
      float ax = fabsf(px) - sx, ay = fabsf(py) - sy, az = fabsf(pz) - sz;
      float qx = fabsf(ax + radius) - radius, qy = fabsf(ay + radius) - radius, qz = fabsf(az + radius) - radius;
      auto term = [](float a, float b, float c) {
        return len3(fmaxf(a, 0.0f), fmaxf(b, 0.0f), fmaxf(c, 0.0f)) + fminf(fmaxf(a, fmaxf(b, c)), 0.0f);
      };
      return fminf(fminf(term(ax, qy, qz), term(qx, ay, qz)), term(qx, qy, az));
    }
    case 9: {
      float qx = sqrtf(px * px + pz * pz), qy = py;
      float k1x = sz, k1y = sy, k2x = sz - sx, k2y = 2.0f * sy;
      float cax = qx - fminf(qx, qy < 0.0f ? sx : sz);
      float cay = fabsf(qy) - sy;
      float num = (k1x - qx) * k2x + (k1y - qy) * k2y;
      float den = fmaxf(k2x * k2x + k2y * k2y, 1e-20f);
      float t = clampf(__fdiv_rn(num, den), 0.0f, 1.0f);
      float cbx = qx - k1x + k2x * t, cby = qy - k1y + k2y * t;
      float sg = (cbx < 0.0f && cay < 0.0f) ? -1.0f : 1.0f;
      return sg * sqrtf(fminf(cax * cax + cay * cay, cbx * cbx + cby * cby));
    }
    case 10: {
      float ax = fabsf(px), ay = fabsf(py), az = fabsf(pz);
      float m = ax + ay + az - sx;
      float qx, qy, qz;
      if (3.0f * ax < m) {
        qx = ax; qy = ay; qz = az;
      } else if (3.0f * ay < m) {
        qx = ay; qy = az; qz = ax;
      } else if (3.0f * az < m) {
        qx = az; qy = ax; qz = ay;
      } else {
        return m * 0.57735026918962584f;
      }
      float k = clampf(0.5f * (qz - qy + sx), 0.0f, sx);
      return len3(qx, qy - sx + k, qz - k);
    }
    case 11: {
      float m = fmaxf(fmaxf(-px - py - pz, -px + py + pz), fmaxf(px - py + pz, px + py - pz)) * 0.57735026918962584f;
      return m - __fdiv_rn(sx, 3.0f);
    }
    case 12: {
      const float phi = 1.6180339887498949f;
      float qx = fabsf(px), qy = fabsf(py), qz = fabsf(pz);
      float m = fmaxf(fmaxf(phi * qy + qz, qx + phi * qz), phi * qx + qy) * 0.52573111211913359f;
      return m - sx * 0.79465447229176612f;
    }
    case 13: {
      const float phi = 1.6180339887498949f, iphi = 0.61803398874989485f;
      float qx = fabsf(px), qy = fabsf(py), qz = fabsf(pz);
      float m = fmaxf(fmaxf(qx + qy + qz, qy * phi + qz * iphi), fmaxf(qx * iphi + qz * phi, qx * phi + qy * iphi)) *
                0.57735026918962584f;
      return m - sx * 0.79465447229176612f;
    }
    default:
      return 1e9f;
  }
}

__device__ __forceinline__ float smoothstepf(float e0, float e1, float x) {
  float t = clampf(__fdiv_rn(x - e0, e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

__device__ __forceinline__ void apply_brush(float& ax, float& ay, const BrushDev& b, float px, float py, float pz) {
  float inv_scale = __frcp_rn(fmaxf(b.scale, 1e-5f));
  float qx = -b.rot[0], qy = -b.rot[1], qz = -b.rot[2], qw = b.rot[3];
  float vx = px - b.pos[0], vy = py - b.pos[1], vz = pz - b.pos[2];
  float tx = (qy * vz - qz * vy) * 2.0f, ty = (qz * vx - qx * vz) * 2.0f, tz = (qx * vy - qy * vx) * 2.0f;
  float lx = ((vx + tx * qw) + (qy * tz - qz * ty)) * inv_scale;
  float ly = ((vy + ty * qw) + (qz * tx - qx * tz)) * inv_scale;
  float lz = ((vz + tz * qw) + (qx * ty - qy * tx)) * inv_scale;
  float dist = eval_local(b.kind, lx, ly, lz, b.size[0], b.size[1], b.size[2], b.radius) * b.scale;
  float keep = b.mask >= 0.0f ? 1.0f - smoothstepf(0.25f, 0.75f, fabsf(ay - b.mask)) : 1.0f;
  if (b.op == 0u) {
    float kk = fmaxf(b.blend, 1e-6f);
    float h = clampf(0.5f + __fdiv_rn(0.5f * (ax - dist), kk), 0.0f, 1.0f);
    float rx = (ax * (1.0f - h) + dist * h) - kk * h * (1.0f - h);
    float ny = ay * (1.0f - h) + b.material * h;
    float nax = ax * (1.0f - keep) + rx * keep;
    float nay = ay * (1.0f - keep) + ny * keep;
    ax = nax;
    ay = nay;
  } else if (b.op == 1u) {
    float a = -dist;
    float kk = fmaxf(b.blend, 1e-6f);
    float h = clampf(0.5f - __fdiv_rn(0.5f * (ax - a), kk), 0.0f, 1.0f);
    float rx = (ax * (1.0f - h) + a * h) + kk * h * (1.0f - h);
    float hh = h * 0.85f;
    float ny = ay * (1.0f - hh) + b.material * hh;
    float nax = ax * (1.0f - keep) + rx * keep;
    float nay = ay * (1.0f - keep) + ny * keep;
    ax = nax;
    ay = nay;
  } else {
    float wv = 1.0f - smoothstepf(-fmaxf(b.blend, 1e-4f), 0.0f, dist);
    float t = wv * keep;
    ay = ay * (1.0f - t) + b.material * t;
  }
}

__global__ void __launch_bounds__(256) k_build(const BuildLevelDev L, const BrushDev* __restrict__ brushes, int nbrush) {
  __shared__ int s_ids[64];
  __shared__ int s_n;
  const int wx = blockIdx.x, wy = blockIdx.y, wz = blockIdx.z;
  const float tminx = L.ox + static_cast<float>(wx) * L.tile_size;
  const float tminy = L.oy + static_cast<float>(wy) * L.tile_size;
  const float tminz = L.oz + static_cast<float>(wz) * L.tile_size;
  if (threadIdx.x == 0) {
    float tcx = tminx + L.tile_half, tcy = tminy + L.tile_half, tcz = tminz + L.tile_half;
    int n = 0;
    for (int b = 0; b < nbrush; b++) {
      const BrushDev& B = brushes[b];
      float nx = fmaxf(fabsf(B.pos[0] - tcx) - L.tile_half, 0.0f);
      float ny = fmaxf(fabsf(B.pos[1] - tcy) - L.tile_half, 0.0f);
      float nz = fmaxf(fabsf(B.pos[2] - tcz) - L.tile_half, 0.0f);
      if (len3(nx, ny, nz) < B.bound + L.bw && n < 64) s_ids[n++] = b;
    }
    s_n = n;
  }
  __syncthreads();
  const int n = s_n;
  const int lx = threadIdx.x & 7, ly = (threadIdx.x >> 3) & 7, lz2 = threadIdx.x >> 6;
  for (int half = 0; half < 2; half++) {
    int lz = lz2 * 2 + half;
    float px = tminx + (static_cast<float>(lx) + 0.5f) * L.voxel;
    float py = tminy + (static_cast<float>(ly) + 0.5f) * L.voxel;
    float pz = tminz + (static_cast<float>(lz) + 0.5f) * L.voxel;
    float ax = L.empty, ay = 0.0f;
    for (int q = 0; q < n; q++) apply_brush(ax, ay, brushes[s_ids[q]], px, py, pz);
    int x = wx * 8 + lx, y = wy * 8 + ly, z = wz * 8 + lz;
    size_t idx = static_cast<size_t>(x) + static_cast<size_t>(L.R) * (static_cast<size_t>(y) + static_cast<size_t>(L.R) * z);
    L.dist[idx] = __float2half_rn(clampf(__fdiv_rn(ax, L.bw), -1.0f, 1.0f));
    L.mat[idx] = __float2half_rn(ay);
  }
}

// Test hook: the reference's cellIndex (fluid.ts:258-262) of every live particle, or
// 0xffffffff when the particle is outside the grid (fluid.ts:319-321).
__global__ void k_cell_index(const SceneDev* __restrict__ scenes, uint32_t* __restrict__ out) {
  const SceneDev& S = scenes[0];
  uint32_t count = work_count(S);
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float4 p = S.parts[i].a;
  int cx, cy, cz;
  cell_of(S, p.x, p.y, p.z, cx, cy, cz);
  bool in = cx >= 0 && cy >= 0 && cz >= 0 && cx < S.G && cy < S.G && cz < S.G;
  uint32_t g = static_cast<uint32_t>(S.G);
  out[i] = in ? static_cast<uint32_t>(cx) + g * (static_cast<uint32_t>(cy) + g * static_cast<uint32_t>(cz)) : kSentinel;
}

// ---------------------------------------------------------------------------------------
// Census of the algorithmic work of a frame (a measurement hook, never part of a step): the
// work the reference's own passes do, counted on the state the last step left.
//  - k_census_nbr: over the cell-ordered copies of the last substep, the neighbour candidates
//    the density pass tests (fluid.ts:346-364, with the bucket limit) and, of them, the pairs
//    within the smoothing length (self included) that it sums (:357-361).
//  - k_census_splat: the (particle, voxel) pairs of the bake whose distance passes
//    sd < bandWorld (splat.ts:246), i.e. the reference's atomicMin count, over every level
//    (blockIdx.y), with the reference's own arithmetic per voxel.
// Counts go to out[] with one 64-bit atomic per warp.
__device__ __forceinline__ void census_add(unsigned long long* out, uint32_t v) {
  const uint32_t s = __reduce_add_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, static_cast<unsigned long long>(s));
}

__global__ void k_census_nbr(const SceneDev* __restrict__ scenes, unsigned long long* __restrict__ out) {
  const SceneDev& S = scenes[0];
  const uint32_t count = work_count(S);
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t cand = 0, acc = 0;
  if (k < count) {
    const BoxInfo b = box_from_state(S.gs);
    const bool overflow = S.gs->overflow != 0u;
    const float4 me = S.spos[k];
    int cx, cy, cz;
    cell_of(S, me.x, me.y, me.z, cx, cy, cz);
    for_neighbours(S, b, overflow, cx, cy, cz, [&](uint32_t q) {
      const float4 o = S.spos[q];
      const float dx = me.x - o.x, dy = me.y - o.y, dz = me.z - o.z;
      cand++;
      if ((dx * dx + dy * dy) + dz * dz < S.h2) acc++;
    });
  }
  census_add(out, cand);
  census_add(out + 1, acc);
}

__global__ void k_census_splat(const SplatDev* __restrict__ d, unsigned long long* __restrict__ out) {
  const SplatDev& D = *d;
  const int m = static_cast<int>(blockIdx.y);
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t i = 0, hits = 0;
  if (cloud_live(D, idx, i)) {
    const float voxel = D.voxel[m], bw = D.bw[m], reach = D.reach[m], inv_voxel = D.inv_voxel[m];
    const int last = D.r[m] - 1;
    const float* pp = reinterpret_cast<const float*>(D.pos + static_cast<size_t>(i) * D.pos_stride);
    const float px = pp[0] - D.vp->origin[0], py = pp[1] - D.vp->origin[1], pz = pp[2] - D.vp->origin[2];
    const bool has_n = D.nrm != nullptr;
    float nx = 0.0f, ny = 0.0f, nz = 0.0f;
    if (has_n) {
      const float* nn = reinterpret_cast<const float*>(D.nrm + static_cast<size_t>(i) * D.nrm_stride);
      nx = nn[0];
      ny = nn[1];
      nz = nn[2];
      if (D.quat) {  // quatRotate (math/gpu.ts:21-25)
        const float qx = D.quat[0], qy = D.quat[1], qz = D.quat[2], qw = D.quat[3];
        const float tx = (qy * nz - qz * ny) * 2.0f, ty = (qz * nx - qx * nz) * 2.0f, tz = (qx * ny - qy * nx) * 2.0f;
        const float rx = (nx + tx * qw) + (qy * tz - qz * ty);
        const float ry = (ny + ty * qw) + (qz * tx - qx * tz);
        const float rz = (nz + tz * qw) + (qx * ty - qy * tx);
        nx = rx;
        ny = ry;
        nz = rz;
      }
    }
    const int lx = max(f2i(floorf((px - reach) * inv_voxel)), 0), hx = min(f2i(floorf((px + reach) * inv_voxel)), last);
    const int ly = max(f2i(floorf((py - reach) * inv_voxel)), 0), hy = min(f2i(floorf((py + reach) * inv_voxel)), last);
    const int lz = max(f2i(floorf((pz - reach) * inv_voxel)), 0), hz = min(f2i(floorf((pz + reach) * inv_voxel)), last);
    for (int z = lz; z <= hz; z++) {
      const float dz = (static_cast<float>(z) + 0.5f) * voxel - pz;
      for (int y = ly; y <= hy; y++) {
        const float dy = (static_cast<float>(y) + 0.5f) * voxel - py;
        for (int x = lx; x <= hx; x++) {
          const float dx = (static_cast<float>(x) + 0.5f) * voxel - px;
          float sd = sqrtf((dx * dx + dy * dy) + dz * dz) - D.radius;
          if (has_n) sd = fmaxf(dot3(dx, dy, dz, nx, ny, nz), sd);
          if (sd < bw) hits++;
        }
      }
    }
  }
  census_add(out, hits);
}

// ---------------------------------------------------------------------------------------
// SurfaceExtractor.extract (extract.ts:469-475): naive surface nets of the field's zero set
// on a res^3 lattice. The reference hands out particle and quad slots with atomics, so their
// order is unspecified; here a block scan gives them in lattice order (cells, then lattice
// points with their +x, +y, +z edges), which makes the output, the centre of mass included,
// deterministic and reproducible by the CPU restatement.

// Block-wide exclusive scan of one value per thread (256 threads); returns the block total.
__device__ __forceinline__ uint32_t ext_block_scan(uint32_t v, uint32_t& excl) {
  __shared__ uint32_t s_w[kExtractThreads / 32];
  const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= static_cast<uint32_t>(o)) x += y;
  }
  if (lane == 31) s_w[wid] = x;
  __syncthreads();
  uint32_t before = 0, total = 0;
  for (uint32_t k = 0; k < kExtractThreads / 32; k++) {
    const uint32_t t = s_w[k];
    if (k < wid) before += t;
    total += t;
  }
  excl = before + x - v;
  __syncthreads();
  return total;
}

// The scan origin (extract.ts:169-178) and the emitted velocity (:179-188).
__device__ __forceinline__ void ext_origin(const ExtractDev& E, float& ox, float& oy, float& oz) {
  ox = E.origin[0];
  oy = E.origin[1];
  oz = E.origin[2];
  if (E.has_motion) {
    ox = ox + E.motion[0];
    oy = oy + E.motion[1];
    oz = oz + E.motion[2];
  }
}

__device__ __forceinline__ float ext_dist(const ExtractDev& E, float px, float py, float pz) {
  float sx = 0.0f, sy = 0.0f;
  if (E.field->n > 0) field_pick(E.field, px, py, pz, sx, sy);
  return sx;
}

// reset (extract.ts:194-246): with motion and preserveMotion, the centre and mean velocity of
// the body's current particles (per-thread strided sums, then a tree) become the motion.
__global__ void __launch_bounds__(kExtractThreads) k_ext_reset(const ExtractDev* __restrict__ e) {
  const ExtractDev& E = *e;
  const uint32_t li = threadIdx.x;
  if (li == 0) {
    E.counters[0] = 0u;
    E.counters[1] = 0u;
  }
  if (!E.has_motion) return;
  __shared__ float s_sum[kExtractThreads][6];
  const unsigned char* bd = E.bodies + static_cast<size_t>(E.body) * 64;
  const uint32_t first = *reinterpret_cast<const uint32_t*>(bd + 12);
  const uint32_t count = *reinterpret_cast<const uint32_t*>(bd + 44);
  const bool keep = E.preserve != 0u;
  float s[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  if (keep) {
    for (uint32_t t = li; t < count; t += kExtractThreads) {
      const float* p = reinterpret_cast<const float*>(E.particles + static_cast<size_t>(first + t) * 96);
      s[0] = s[0] + p[0];
      s[1] = s[1] + p[1];
      s[2] = s[2] + p[2];
      s[3] = s[3] + p[8];
      s[4] = s[4] + p[9];
      s[5] = s[5] + p[10];
    }
  }
  for (int k = 0; k < 6; k++) s_sum[li][k] = s[k];
  __syncthreads();
  for (uint32_t h = kExtractThreads / 2; h > 0; h >>= 1) {
    if (li < h)
      for (int k = 0; k < 6; k++) s_sum[li][k] = s_sum[li][k] + s_sum[li + h][k];
    __syncthreads();
  }
  if (li == 0 && keep && count > 0) {
    const float inv = __fdiv_rn(1.0f, static_cast<float>(count));
    for (int k = 0; k < 3; k++) {
      E.motion[k] = s_sum[0][k] * inv;
      E.motion[4 + k] = s_sum[0][3 + k] * inv;
    }
  }
}

// (crossing point * weight, weight) of one lattice edge (extract.ts:155-163); mix(a, b, t) is
// a * (1 - t) + b * t.
__device__ __forceinline__ void ext_cross(float ax, float ay, float az, float da, float bx, float by, float bz, float db,
                                          float& sx, float& sy, float& sz, float& sw) {
  float cx = 0.0f, cy = 0.0f, cz = 0.0f, cw = 0.0f;
  if (!(da * db >= 0.0f)) {
    const float t = clampf(__fdiv_rn(da, da - db), 0.0f, 1.0f);
    const float u = 1.0f - t;
    cx = ax * u + bx * t;
    cy = ay * u + by * t;
    cz = az * u + bz * t;
    cw = 1.0f;
  }
  sx = sx + cx;
  sy = sy + cy;
  sz = sz + cz;
  sw = sw + cw;
}

// cells (extract.ts:249-327): the dual vertex of every cell whose corners straddle the
// surface, snapped onto it by one Lipschitz step; the block's count of vertices.
__global__ void __launch_bounds__(kExtractThreads) k_ext_cells(const ExtractDev* __restrict__ e) {
  const ExtractDev& E = *e;
  const uint32_t R = static_cast<uint32_t>(E.res);
  const uint32_t idx = blockIdx.x * kExtractThreads + threadIdx.x;
  uint32_t has = 0;
  if (idx < R * R * R) {
    const uint32_t gx = idx % R, gy = (idx / R) % R, gz = idx / (R * R);
    float ox, oy, oz;
    ext_origin(E, ox, oy, oz);
    const float c = E.cell;
    const float x0 = ox + static_cast<float>(gx) * c, y0 = oy + static_cast<float>(gy) * c, z0 = oz + static_cast<float>(gz) * c;
    const float x1 = x0 + c, y1 = y0 + c, z1 = z0 + c;
    const float d0 = ext_dist(E, x0, y0, z0), dx = ext_dist(E, x1, y0, z0), dy = ext_dist(E, x0, y1, z0),
                dz = ext_dist(E, x0, y0, z1), dxy = ext_dist(E, x1, y1, z0), dxz = ext_dist(E, x1, y0, z1),
                dyz = ext_dist(E, x0, y1, z1), dxyz = ext_dist(E, x1, y1, z1);
    float ax = 0.0f, ay = 0.0f, az = 0.0f, aw = 0.0f;
    // the twelve edges in the reference's order
    ext_cross(x0, y0, z0, d0, x1, y0, z0, dx, ax, ay, az, aw);
    ext_cross(x0, y1, z0, dy, x1, y1, z0, dxy, ax, ay, az, aw);
    ext_cross(x0, y0, z1, dz, x1, y0, z1, dxz, ax, ay, az, aw);
    ext_cross(x0, y1, z1, dyz, x1, y1, z1, dxyz, ax, ay, az, aw);
    ext_cross(x0, y0, z0, d0, x0, y1, z0, dy, ax, ay, az, aw);
    ext_cross(x1, y0, z0, dx, x1, y1, z0, dxy, ax, ay, az, aw);
    ext_cross(x0, y0, z1, dz, x0, y1, z1, dyz, ax, ay, az, aw);
    ext_cross(x1, y0, z1, dxz, x1, y1, z1, dxyz, ax, ay, az, aw);
    ext_cross(x0, y0, z0, d0, x0, y0, z1, dz, ax, ay, az, aw);
    ext_cross(x1, y0, z0, dx, x1, y0, z1, dxz, ax, ay, az, aw);
    ext_cross(x0, y1, z0, dy, x0, y1, z1, dyz, ax, ay, az, aw);
    ext_cross(x1, y1, z0, dxy, x1, y1, z1, dxyz, ax, ay, az, aw);
    float4 r0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), r1 = r0;
    if (!(aw < 0.5f)) {
      const float inv = __fdiv_rn(1.0f, aw);
      const float vx = ax * inv, vy = ay * inv, vz = az * inv;
      float nx = 0.0f, ny = 1.0f, nz = 0.0f, sv = 0.0f, sm = 0.0f;
      int child = -1;
      if (E.field->n > 0) {
        child = field_pick(E.field, vx, vy, vz, sv, sm);
        field_normal(E.field, child, vx, vy, vz, nx, ny, nz);
      }
      const float px = vx - nx * sv, py = vy - ny * sv, pz = vz - nz * sv;
      float mat = 0.0f;
      if (E.field->n > 0) {
        float s0, s1;
        const int ch = field_pick(E.field, px, py, pz, s0, s1);
        mat = field_material(E.field, ch, px, py, pz);
      }
      r0 = make_float4(px, py, pz, mat);
      r1 = make_float4(nx, ny, nz, 1.0f);
      has = 1;
    }
    E.rec[2 * static_cast<size_t>(idx)] = r0;
    E.rec[2 * static_cast<size_t>(idx) + 1] = r1;
  }
  uint32_t excl;
  const uint32_t total = ext_block_scan(has, excl);
  if (threadIdx.x == 0) E.blk[blockIdx.x] = total;
}

// Exclusive scan of the per-block counts of `which` (0: vertices, 1: quads) in one block,
// and the grand total into the counter.
__global__ void __launch_bounds__(1024) k_ext_scan(const ExtractDev* __restrict__ e, int which) {
  const ExtractDev& E = *e;
  uint32_t* a = which == 0 ? E.blk : E.qblk;
  const uint32_t n = static_cast<uint32_t>(E.nblocks);
  __shared__ uint32_t s_w[32];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0u;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  for (uint32_t base = 0; base < n; base += 1024) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < n ? a[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= static_cast<uint32_t>(o)) x += y;
    }
    if (lane == 31) s_w[wid] = x;
    __syncthreads();
    if (wid == 0) {
      uint32_t t = s_w[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= static_cast<uint32_t>(o)) t += y;
      }
      s_w[lane] = t;
    }
    __syncthreads();
    const uint32_t carry = s_carry;
    if (i < n) a[i] = carry + (wid > 0 ? s_w[wid - 1] : 0u) + x - v;
    __syncthreads();
    if (threadIdx.x == 0) s_carry = carry + s_w[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) E.counters[which] = s_carry;
}

// emit (extract.ts:306-326): the Particle records of the vertices in lattice order, the
// biased ids of the cells; vertices past the slice's capacity are dropped (id 0).
__global__ void __launch_bounds__(kExtractThreads) k_ext_emit(const ExtractDev* __restrict__ e) {
  const ExtractDev& E = *e;
  const uint32_t R = static_cast<uint32_t>(E.res);
  const uint32_t idx = blockIdx.x * kExtractThreads + threadIdx.x;
  const bool in = idx < R * R * R;
  float4 r0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), r1 = r0;
  if (in) {
    r0 = E.rec[2 * static_cast<size_t>(idx)];
    r1 = E.rec[2 * static_cast<size_t>(idx) + 1];
  }
  const uint32_t has = (in && r1.w > 0.5f) ? 1u : 0u;
  uint32_t excl;
  ext_block_scan(has, excl);
  if (!in) return;
  const uint32_t slot = E.blk[blockIdx.x] + excl;
  if (!has || slot >= static_cast<uint32_t>(E.capacity)) {
    E.id_grid[idx] = 0u;
    return;
  }
  const uint32_t id = static_cast<uint32_t>(E.base) + slot;
  float vx = E.vel[0], vy = E.vel[1], vz = E.vel[2];
  if (E.has_motion) {
    vx = E.motion[4];
    vy = E.motion[5];
    vz = E.motion[6];
  }
  float4* out = reinterpret_cast<float4*>(E.particles + static_cast<size_t>(id) * 96);
  out[0] = make_float4(r0.x, r0.y, r0.z, __uint_as_float(static_cast<uint32_t>(E.body)));  // pos, body
  out[1] = make_float4(r0.x, r0.y, r0.z, r0.w);                                            // prev, material
  out[2] = make_float4(vx, vy, vz, 0.0f);                                                  // vel
  out[3] = make_float4(vx, vy, vz, 0.0f);                                                  // velPrev
  out[4] = make_float4(r0.x, r0.y, r0.z, 0.0f);                                            // rest
  out[5] = make_float4(r1.x, r1.y, r1.z, 0.0f);                                            // restNormal
  E.id_grid[idx] = id + 1u;
}

__device__ __forceinline__ uint32_t ext_id(const ExtractDev& E, uint32_t x, uint32_t y, uint32_t z) {
  const uint32_t R = static_cast<uint32_t>(E.res);
  return E.id_grid[x + R * (y + R * z)];
}

// The three quads a lattice point may own (extract.ts:352-392): for edge a (0: +x, 1: +y,
// 2: +z) whose ends straddle the surface, the ids of the four cells around it in the
// reference's order; all four must hold a vertex.
__device__ __forceinline__ bool ext_quad(const ExtractDev& E, uint32_t i, uint32_t j, uint32_t k, int a, float dL, float lx,
                                         float ly, float lz, uint32_t q[4]) {
  const uint32_t hi = static_cast<uint32_t>(E.res) - 1u;
  const float c = E.cell;
  if (a == 0) {
    if (!(j >= 1 && k >= 1 && j <= hi && k <= hi)) return false;
    if (!(ext_dist(E, lx + c, ly + 0.0f, lz + 0.0f) * dL < 0.0f)) return false;
    q[0] = ext_id(E, i, j - 1, k - 1);
    q[1] = ext_id(E, i, j, k - 1);
    q[2] = ext_id(E, i, j, k);
    q[3] = ext_id(E, i, j - 1, k);
  } else if (a == 1) {
    if (!(i >= 1 && k >= 1 && i <= hi && k <= hi)) return false;
    if (!(ext_dist(E, lx + 0.0f, ly + c, lz + 0.0f) * dL < 0.0f)) return false;
    q[0] = ext_id(E, i - 1, j, k - 1);
    q[1] = ext_id(E, i - 1, j, k);
    q[2] = ext_id(E, i, j, k);
    q[3] = ext_id(E, i, j, k - 1);
  } else {
    if (!(i >= 1 && j >= 1 && i <= hi && j <= hi)) return false;
    if (!(ext_dist(E, lx + 0.0f, ly + 0.0f, lz + c) * dL < 0.0f)) return false;
    q[0] = ext_id(E, i - 1, j - 1, k);
    q[1] = ext_id(E, i, j - 1, k);
    q[2] = ext_id(E, i, j, k);
    q[3] = ext_id(E, i - 1, j, k);
  }
  return q[0] != 0u && q[1] != 0u && q[2] != 0u && q[3] != 0u;
}

// quads, pass 1: which of a lattice point's edges emit, and the block's count.
__global__ void __launch_bounds__(kExtractThreads) k_ext_qcount(const ExtractDev* __restrict__ e) {
  const ExtractDev& E = *e;
  const uint32_t R = static_cast<uint32_t>(E.res);
  const uint32_t idx = blockIdx.x * kExtractThreads + threadIdx.x;
  uint32_t m = 0;
  if (idx < R * R * R) {
    const uint32_t i = idx % R, j = (idx / R) % R, k = idx / (R * R);
    float ox, oy, oz;
    ext_origin(E, ox, oy, oz);
    const float c = E.cell;
    const float lx = ox + static_cast<float>(i) * c, ly = oy + static_cast<float>(j) * c, lz = oz + static_cast<float>(k) * c;
    const float dL = ext_dist(E, lx, ly, lz);
    uint32_t q[4];
    for (int a = 0; a < 3; a++)
      if (ext_quad(E, i, j, k, a, dL, lx, ly, lz, q)) m |= 1u << a;
    E.qmask[idx] = static_cast<unsigned char>(m);
  }
  uint32_t excl;
  const uint32_t total = ext_block_scan(static_cast<uint32_t>(__popc(m)), excl);
  if (threadIdx.x == 0) E.qblk[blockIdx.x] = total;
}

// quads, pass 2: six indices per quad (extract.ts:330-350), wound by the sign at the low end.
__global__ void __launch_bounds__(kExtractThreads) k_ext_qemit(const ExtractDev* __restrict__ e) {
  const ExtractDev& E = *e;
  const uint32_t R = static_cast<uint32_t>(E.res);
  const uint32_t idx = blockIdx.x * kExtractThreads + threadIdx.x;
  const bool in = idx < R * R * R;
  const uint32_t m = in ? static_cast<uint32_t>(E.qmask[idx]) : 0u;
  uint32_t excl;
  ext_block_scan(static_cast<uint32_t>(__popc(m)), excl);
  if (!m) return;
  const uint32_t i = idx % R, j = (idx / R) % R, k = idx / (R * R);
  float ox, oy, oz;
  ext_origin(E, ox, oy, oz);
  const float c = E.cell;
  const float lx = ox + static_cast<float>(i) * c, ly = oy + static_cast<float>(j) * c, lz = oz + static_cast<float>(k) * c;
  const float dL = ext_dist(E, lx, ly, lz);
  const bool flip = !(dL < 0.0f);
  uint32_t slot = E.qblk[blockIdx.x] + excl;
  for (int a = 0; a < 3; a++) {
    if (!(m & (1u << a))) continue;
    uint32_t q[4];
    ext_quad(E, i, j, k, a, dL, lx, ly, lz, q);
    if (slot < static_cast<uint32_t>(E.quad_cap)) {
      uint32_t* o = E.indices + static_cast<size_t>(slot) * 6;
      const uint32_t i0 = q[0] - 1u, i1 = (flip ? q[3] : q[1]) - 1u, i2 = q[2] - 1u, i3 = (flip ? q[1] : q[3]) - 1u;
      o[0] = i0;
      o[1] = i1;
      o[2] = i2;
      o[3] = i0;
      o[4] = i2;
      o[5] = i3;
    }
    slot++;
  }
}

// finish (extract.ts:395-436): the body record (first, count, rest centre of mass, rotation
// reset) and the draw arguments.
__global__ void __launch_bounds__(kExtractThreads) k_ext_finish(const ExtractDev* __restrict__ e) {
  const ExtractDev& E = *e;
  const uint32_t li = threadIdx.x;
  const uint32_t n = min(E.counters[0], static_cast<uint32_t>(E.capacity));
  __shared__ float s_g[kExtractThreads][3];
  float sx = 0.0f, sy = 0.0f, sz = 0.0f;
  for (uint32_t t = li; t < n; t += kExtractThreads) {
    const float* p = reinterpret_cast<const float*>(E.particles + static_cast<size_t>(E.base + t) * 96 + 64);  // rest
    sx = sx + p[0];
    sy = sy + p[1];
    sz = sz + p[2];
  }
  s_g[li][0] = sx;
  s_g[li][1] = sy;
  s_g[li][2] = sz;
  __syncthreads();
  for (uint32_t h = kExtractThreads / 2; h > 0; h >>= 1) {
    if (li < h)
      for (int k = 0; k < 3; k++) s_g[li][k] = s_g[li][k] + s_g[li + h][k];
    __syncthreads();
  }
  if (li != 0) return;
  const float inv = __fdiv_rn(1.0f, fmaxf(static_cast<float>(n), 1.0f));
  const float cx = s_g[0][0] * inv, cy = s_g[0][1] * inv, cz = s_g[0][2] * inv;
  unsigned char* bd = E.bodies + static_cast<size_t>(E.body) * 64;
  float* f = reinterpret_cast<float*>(bd);
  uint32_t* u = reinterpret_cast<uint32_t*>(bd);
  u[3] = static_cast<uint32_t>(E.base);  // first
  u[11] = n;                             // count
  f[8] = cx;                             // restCom
  f[9] = cy;
  f[10] = cz;
  f[0] = cx;                             // com
  f[1] = cy;
  f[2] = cz;
  f[4] = 0.0f;                           // rot
  f[5] = 0.0f;
  f[6] = 0.0f;
  f[7] = 1.0f;
  const uint32_t q = min(E.counters[1], static_cast<uint32_t>(E.quad_cap));
  E.draw_args[0] = q * 6u;
  E.draw_args[1] = 1u;
  E.draw_args[2] = 0u;
  E.draw_args[3] = 0u;
}

// ---------------------------------------------------------------------------------------
// ClaySolver (sim/pbd.ts:78-424): shape-matched particle bodies of a ParticleSet colliding
// against a field. Particle records are 96 bytes (pos 0, body 12, prev 16, material 28,
// vel 32, velPrev 48, rest 64, restNormal 80), Body records 64 (com 0, first 12, rot 16,
// restCom 32, count 44, stiffness 48, plasticity 52, material 56, flags 60).

// sin and cos of one angle, identical on the device and in the CPU restatement (WGSL leaves
// their precision to the implementation): Cody-Waite reduction by pi/2 split in three f32
// parts (the first two of 12 significant bits, so k times them is exact for |k| < 4096), then
// Taylor polynomials through x^9 (sin) and x^10 (cos) on [-pi/4, pi/4], where the truncation
// error is far below half an f32 ulp.
__host__ __device__ inline void clay_sincos(float x, float& s, float& c) {
  const float k = rintf(x * 0.636619746685028076171875f);
  const float r = ((x - k * 1.57080078125f) - k * -4.453584551811218e-06f) - k * -8.705515752716053e-10f;
  const float r2 = r * r;
  const float ps = r + r * (r2 * (-0.16666667163372039794921875f +
                                 r2 * (0.008333333767950534820556640625f +
                                       r2 * (-0.000198412701138295233249664306640625f + r2 * 2.7557318844628753140568733215332031e-06f))));
  const float pc = 1.0f + r2 * (-0.5f + r2 * (0.041666667908430099487304687500f +
                                            r2 * (-0.0013888889225199818611145019531f +
                                                  r2 * (2.4801587642286904156208038330078e-05f + r2 * -2.7557319981497130356729030609131e-07f))));
  const int q = static_cast<int>(k) & 3;
  s = q == 0 ? ps : q == 1 ? pc : q == 2 ? -ps : -pc;
  c = q == 0 ? pc : q == 1 ? -ps : q == 2 ? -pc : ps;
}

struct Q4 {
  float x, y, z, w;
};
// quatMul, quatRotate, quatConj, quatToMat3 (math/gpu.ts:5-44), in their operation order.
__device__ __forceinline__ Q4 quat_mul(Q4 a, Q4 b) {
  return {((a.w * b.x + a.x * b.w) + a.y * b.z) - a.z * b.y, ((a.w * b.y - a.x * b.z) + a.y * b.w) + a.z * b.x,
          ((a.w * b.z + a.x * b.y) - a.y * b.x) + a.z * b.w, ((a.w * b.w - a.x * b.x) - a.y * b.y) - a.z * b.z};
}
__device__ __forceinline__ void cross3(float ax, float ay, float az, float bx, float by, float bz, float& cx, float& cy,
                                       float& cz) {
  cx = ay * bz - az * by;
  cy = az * bx - ax * bz;
  cz = ax * by - ay * bx;
}
__device__ __forceinline__ void quat_rotate(Q4 q, float vx, float vy, float vz, float& ox, float& oy, float& oz) {
  float tx, ty, tz;
  cross3(q.x, q.y, q.z, vx, vy, vz, tx, ty, tz);
  tx = tx * 2.0f;
  ty = ty * 2.0f;
  tz = tz * 2.0f;
  float ux, uy, uz;
  cross3(q.x, q.y, q.z, tx, ty, tz, ux, uy, uz);
  ox = (vx + tx * q.w) + ux;
  oy = (vy + ty * q.w) + uy;
  oz = (vz + tz * q.w) + uz;
}

// extractRotation (math/gpu.ts:55-77, Müller et al. 2016): warm-started quaternion iterations
// towards the rotational part of A (columns a0, a1, a2).
__device__ __forceinline__ Q4 extract_rotation(const float a[9], Q4 q, int iters) {
  for (int it = 0; it < iters; it++) {
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    // quatToMat3 columns
    const float c0[3] = {1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + z * w), 2.0f * (x * z - y * w)};
    const float c1[3] = {2.0f * (x * y - z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + x * w)};
    const float c2[3] = {2.0f * (x * z + y * w), 2.0f * (y * z - x * w), 1.0f - 2.0f * (x * x + y * y)};
    const float d = (dot3(c0[0], c0[1], c0[2], a[0], a[1], a[2]) + dot3(c1[0], c1[1], c1[2], a[3], a[4], a[5])) +
                    dot3(c2[0], c2[1], c2[2], a[6], a[7], a[8]);
    const float denom = fabsf(d) + 1e-9f;
    float e0x, e0y, e0z, e1x, e1y, e1z, e2x, e2y, e2z;
    cross3(c0[0], c0[1], c0[2], a[0], a[1], a[2], e0x, e0y, e0z);
    cross3(c1[0], c1[1], c1[2], a[3], a[4], a[5], e1x, e1y, e1z);
    cross3(c2[0], c2[1], c2[2], a[6], a[7], a[8], e2x, e2y, e2z);
    const float inv = __fdiv_rn(1.0f, denom);
    const float ox = ((e0x + e1x) + e2x) * inv, oy = ((e0y + e1y) + e2y) * inv, oz = ((e0z + e1z) + e2z) * inv;
    const float wl = len3(ox, oy, oz);
    if (wl < 1e-9f) break;
    const float iw = __fdiv_rn(1.0f, wl);
    // quatFromAxisAngle(omega * (1 / w), w)
    float sh, ch;
    clay_sincos(wl * 0.5f, sh, ch);
    const Q4 r = {(ox * iw) * sh, (oy * iw) * sh, (oz * iw) * sh, ch};
    const Q4 m = quat_mul(r, q);
    // normalize: v / length(v)
    const float l = __fsqrt_rn(((m.x * m.x + m.y * m.y) + m.z * m.z) + m.w * m.w);
    q = {__fdiv_rn(m.x, l), __fdiv_rn(m.y, l), __fdiv_rn(m.z, l), __fdiv_rn(m.w, l)};
  }
  return q;
}

// ownerOf (pbd.ts:126-142): the particle's body when the slot lies in that body's slice,
// else max_bodies.
__device__ __forceinline__ uint32_t pbd_owner(const SolveDev& S, uint32_t i) {
  const uint32_t b = *reinterpret_cast<const uint32_t*>(S.particles + static_cast<size_t>(i) * 96 + 12);
  if (b >= static_cast<uint32_t>(S.max_bodies)) return static_cast<uint32_t>(S.max_bodies);
  const unsigned char* bd = S.bodies + static_cast<size_t>(b) * 64;
  const uint32_t first = *reinterpret_cast<const uint32_t*>(bd + 12), count = *reinterpret_cast<const uint32_t*>(bd + 44);
  if (i < first || i >= first + count) return static_cast<uint32_t>(S.max_bodies);
  return b;
}
__device__ __forceinline__ uint32_t pbd_flags(const SolveDev& S, uint32_t b) {
  return *reinterpret_cast<const uint32_t*>(S.bodies + static_cast<size_t>(b) * 64 + 60);
}

// kick (pbd.ts:144-170): the one-shot velocity change of the pushed body.
__global__ void __launch_bounds__(kSolveThreads) k_pbd_kick(const SolveDev* __restrict__ sd) {
  const SolveDev& S = *sd;
  const uint32_t i = blockIdx.x * kSolveThreads + threadIdx.x;
  if (i >= static_cast<uint32_t>(S.capacity)) return;
  const uint32_t b = pbd_owner(S, i);
  if (b != S.push_body || b >= static_cast<uint32_t>(S.max_bodies)) return;
  if (pbd_flags(S, b) & kBodyKinematic) return;
  float* p = reinterpret_cast<float*>(S.particles + static_cast<size_t>(i) * 96);
  for (int k = 0; k < 3; k++) {
    const float dv = S.kick[k];
    const float vel = p[8 + k], vp = p[12 + k], prev = p[4 + k];
    p[8 + k] = vel + dv;
    p[12 + k] = vp + dv;
    p[4 + k] = prev - dv * S.h;
  }
}

// predict (pbd.ts:172-222): BDF2 predictor, then the world collision with positional friction.
__global__ void __launch_bounds__(kSolveThreads) k_pbd_predict(const SolveDev* __restrict__ sd) {
  const SolveDev& S = *sd;
  const uint32_t i = blockIdx.x * kSolveThreads + threadIdx.x;
  if (i >= static_cast<uint32_t>(S.capacity)) return;
  const uint32_t b = pbd_owner(S, i);
  if (b >= static_cast<uint32_t>(S.max_bodies)) return;
  const uint32_t flags = pbd_flags(S, b);
  if (flags & kBodyKinematic) return;
  float* p = reinterpret_cast<float*>(S.particles + static_cast<size_t>(i) * 96);
  float acc[3];
  for (int k = 0; k < 3; k++) {
    acc[k] = (flags & kBodyWeightless) ? 0.0f : S.gravity[k];
    if (b == S.push_body) acc[k] = acc[k] + S.push[k];
  }
  const float third = 0.3333333432674407958984375f;  // f32(1 / 3)
  const float h23 = __fdiv_rn(2.0f * S.h, 3.0f);
  float q[3];
  for (int k = 0; k < 3; k++) {
    const float vpred = (p[8 + k] * 4.0f - p[12 + k]) * third + acc[k] * h23;
    q[k] = (p[k] * 4.0f - p[4 + k]) * third + vpred * h23;
  }
  float prev[3] = {p[0], p[1], p[2]};
  float sx, sy;
  const int child = field_pick(S.world, q[0], q[1], q[2], sx, sy);
  if (sx < S.radius) {
    float nx, ny, nz;
    field_normal(S.world, child, q[0], q[1], q[2], nx, ny, nz);
    const float push = S.radius - sx;
    q[0] = q[0] + nx * push;
    q[1] = q[1] + ny * push;
    q[2] = q[2] + nz * push;
    prev[0] = p[0] + nx * push;
    prev[1] = p[1] + ny * push;
    prev[2] = p[2] + nz * push;
    const float dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
    const float dn = dot3(dx, dy, dz, nx, ny, nz);
    q[0] = q[0] - (dx - nx * dn) * S.friction;
    q[1] = q[1] - (dy - ny * dn) * S.friction;
    q[2] = q[2] - (dz - nz * dn) * S.friction;
  }
  for (int k = 0; k < 3; k++) {
    p[4 + k] = prev[k];
    p[k] = q[k];
  }
}

// match (pbd.ts:224-297): per body, the current and rest centroids and the covariance
// A = sum (p - com)(r - restCom)^T by per-thread strided sums and a tree, then the rotation.
__global__ void __launch_bounds__(kSolveReduce) k_pbd_match(const SolveDev* __restrict__ sd) {
  const SolveDev& S = *sd;
  const uint32_t b = blockIdx.x, li = threadIdx.x;
  unsigned char* bd = S.bodies + static_cast<size_t>(b) * 64;
  const uint32_t first = *reinterpret_cast<const uint32_t*>(bd + 12), count = *reinterpret_cast<const uint32_t*>(bd + 44);
  // the slice clipped to the set: a record reaching past the capacity reads no further
  const uint32_t cap = static_cast<uint32_t>(S.capacity);
  const uint32_t live = first >= cap ? 0u : min(count, cap - first);
  __shared__ float g[kSolveReduce][9];
  auto reduce = [&]() {
    for (uint32_t s = kSolveReduce / 2; s > 0; s >>= 1) {
      if (li < s)
        for (int k = 0; k < 9; k++) g[li][k] = g[li][k] + g[li + s][k];
      __syncthreads();
    }
  };
  float sp[3] = {0.0f, 0.0f, 0.0f}, sr[3] = {0.0f, 0.0f, 0.0f};
  for (uint32_t t = li; t < live; t += kSolveReduce) {
    const float* p = reinterpret_cast<const float*>(S.particles + static_cast<size_t>(first + t) * 96);
    for (int k = 0; k < 3; k++) {
      sp[k] = sp[k] + p[k];
      sr[k] = sr[k] + p[16 + k];
    }
  }
  for (int k = 0; k < 3; k++) {
    g[li][k] = sp[k];
    g[li][3 + k] = sr[k];
    g[li][6 + k] = 0.0f;
  }
  __syncthreads();
  reduce();
  const float inv = __fdiv_rn(1.0f, fmaxf(static_cast<float>(count), 1.0f));
  const float com[3] = {g[0][0] * inv, g[0][1] * inv, g[0][2] * inv};
  const float rcom[3] = {g[0][3] * inv, g[0][4] * inv, g[0][5] * inv};
  __syncthreads();
  float a[9] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  for (uint32_t t = li; t < live; t += kSolveReduce) {
    const float* p = reinterpret_cast<const float*>(S.particles + static_cast<size_t>(first + t) * 96);
    const float pr[3] = {p[0] - com[0], p[1] - com[1], p[2] - com[2]};
    const float rr[3] = {p[16] - rcom[0], p[17] - rcom[1], p[18] - rcom[2]};
    for (int c = 0; c < 3; c++)
      for (int k = 0; k < 3; k++) a[3 * c + k] = a[3 * c + k] + pr[k] * rr[c];
  }
  for (int k = 0; k < 9; k++) g[li][k] = a[k];
  __syncthreads();
  reduce();
  if (li == 0 && count > 0) {
    float* f = reinterpret_cast<float*>(bd);
    const Q4 q0 = {f[4], f[5], f[6], f[7]};
    float A[9];
    for (int k = 0; k < 9; k++) A[k] = g[0][k];
    const Q4 r = extract_rotation(A, q0, S.rot_iters);
    f[0] = com[0];
    f[1] = com[1];
    f[2] = com[2];
    f[8] = rcom[0];
    f[9] = rcom[1];
    f[10] = rcom[2];
    f[4] = r.x;
    f[5] = r.y;
    f[6] = r.z;
    f[7] = r.w;
  }
}

// apply (pbd.ts:299-340): the pull towards the matched shape, a final projection out of the
// world, and plasticity letting the rest shape follow.
__global__ void __launch_bounds__(kSolveThreads) k_pbd_apply(const SolveDev* __restrict__ sd) {
  const SolveDev& S = *sd;
  const uint32_t i = blockIdx.x * kSolveThreads + threadIdx.x;
  if (i >= static_cast<uint32_t>(S.capacity)) return;
  const uint32_t b = pbd_owner(S, i);
  if (b >= static_cast<uint32_t>(S.max_bodies)) return;
  const float* bf = reinterpret_cast<const float*>(S.bodies + static_cast<size_t>(b) * 64);
  const uint32_t flags = *reinterpret_cast<const uint32_t*>(bf + 15);
  if (flags & kBodyKinematic) return;
  float* p = reinterpret_cast<float*>(S.particles + static_cast<size_t>(i) * 96);
  const Q4 rot = {bf[4], bf[5], bf[6], bf[7]};
  float tx, ty, tz;
  quat_rotate(rot, p[16] - bf[8], p[17] - bf[9], p[18] - bf[10], tx, ty, tz);
  const float target[3] = {bf[0] + tx, bf[1] + ty, bf[2] + tz};
  const float st = clampf(bf[12], 0.0f, 1.0f), om = 1.0f - st;
  float q[3];
  for (int k = 0; k < 3; k++) q[k] = p[k] * om + target[k] * st;  // mix(pos, target, st)
  float sx, sy;
  const int child = field_pick(S.world, q[0], q[1], q[2], sx, sy);
  if (sx < S.radius) {
    float nx, ny, nz;
    field_normal(S.world, child, q[0], q[1], q[2], nx, ny, nz);
    const float push = S.radius - sx;
    q[0] = q[0] + nx * push;
    q[1] = q[1] + ny * push;
    q[2] = q[2] + nz * push;
    p[4] = p[4] + nx * push;
    p[5] = p[5] + ny * push;
    p[6] = p[6] + nz * push;
  }
  const float r0[3] = {p[16], p[17], p[18]};
  p[0] = q[0];
  p[1] = q[1];
  p[2] = q[2];
  if (bf[13] > 0.0f) {
    const Q4 cj = {-rot.x, -rot.y, -rot.z, rot.w};
    float rx, ry, rz;
    quat_rotate(cj, q[0] - bf[0], q[1] - bf[1], q[2] - bf[2], rx, ry, rz);
    const float rest[3] = {rx + bf[8], ry + bf[9], rz + bf[10]};
    const float pl = clampf(bf[13], 0.0f, 1.0f), om2 = 1.0f - pl;
    for (int k = 0; k < 3; k++) p[16 + k] = r0[k] * om2 + rest[k] * pl;
  }
}

// finalize (pbd.ts:342-372): first-order velocity from the positions, damping, speed cap.
__global__ void __launch_bounds__(kSolveThreads) k_pbd_finalize(const SolveDev* __restrict__ sd) {
  const SolveDev& S = *sd;
  const uint32_t i = blockIdx.x * kSolveThreads + threadIdx.x;
  if (i >= static_cast<uint32_t>(S.capacity)) return;
  const uint32_t b = pbd_owner(S, i);
  if (b >= static_cast<uint32_t>(S.max_bodies)) return;
  if (pbd_flags(S, b) & kBodyKinematic) return;
  float* p = reinterpret_cast<float*>(S.particles + static_cast<size_t>(i) * 96);
  const float ih = __fdiv_rn(1.0f, fmaxf(S.h, 1e-6f));
  float v[3];
  for (int k = 0; k < 3; k++) v[k] = ((p[k] - p[4 + k]) * ih) * S.damping;
  const float speed = len3(v[0], v[1], v[2]);
  if (speed > S.max_speed) {
    const float sc = __fdiv_rn(S.max_speed, speed);
    for (int k = 0; k < 3; k++) v[k] = v[k] * sc;
  }
  for (int k = 0; k < 3; k++) {
    p[12 + k] = p[8 + k];
    p[8 + k] = v[k];
  }
}

// Gathers the ContactList of every scene of a batch into one array (one readback).
__global__ void k_gather_contacts(const SceneDev* __restrict__ scenes, int n, ContactsDev* __restrict__ out) {
  int s = blockIdx.x;
  if (s >= n) return;
  const uint32_t* src = reinterpret_cast<const uint32_t*>(scenes[s].contacts);
  uint32_t* dst = reinterpret_cast<uint32_t*>(out + s);
  for (int i = threadIdx.x; i < static_cast<int>(sizeof(ContactsDev) / 4); i += blockDim.x) dst[i] = src[i];
}

// Collider query (test hook): sample(p, 0) and normal(p) at n points.
__global__ void k_field_query(const FieldDev* __restrict__ f, const float* __restrict__ pts, int n, float* __restrict__ sxy,
                              float* __restrict__ nrm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float px = pts[3 * i], py = pts[3 * i + 1], pz = pts[3 * i + 2];
  float sx = 0.0f, sy = 0.0f, nx = 0.0f, ny = 1.0f, nz = 0.0f;
  if (f->n > 0) {
    int c = field_pick(f, px, py, pz, sx, sy);
    field_normal(f, c, px, py, pz, nx, ny, nz);
  }
  sxy[2 * i] = sx;
  sxy[2 * i + 1] = sy;
  nrm[3 * i] = nx;
  nrm[3 * i + 1] = ny;
  nrm[3 * i + 2] = nz;
}

// Collider query at a level: sample(p, mip) and field(p, mip) at n points.
__global__ void k_field_query_mip(const FieldDev* __restrict__ f, const float* __restrict__ pts, int n, int mip,
                                  float* __restrict__ sxy, float* __restrict__ fxy) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float sx = 0.0f, sy = 0.0f, fx = 0.0f, fy = 0.0f;
  if (f->n > 0) field_sample_mip(f, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], mip, sx, sy, fx, fy);
  sxy[2 * i] = sx;
  sxy[2 * i + 1] = sy;
  fxy[2 * i] = fx;
  fxy[2 * i + 1] = fy;
}

#endif  // CLAY_ONLY_NEIGHBOUR_PASSES

}  // namespace clay
#endif  // CLAY_DEFINE_KERNELS
