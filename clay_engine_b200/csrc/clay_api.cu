// clay_api.cu - host object model behind the C ABI of include/clay_fluid.h.
//
// Mirrors the reference's classes: SdfVolume (lib/src/field/volume.ts), volumeField /
// unionField / offsetField (lib/src/trace/field.ts), SplatField (lib/src/sim/splat.ts) and
// FluidSim (lib/src/sim/fluid.ts). Host-side derivations are done in binary64 exactly as
// the reference's JavaScript does them and rounded once to the f32 values the kernels use.
// Uniforms (FluidParams, VolumeParams, collider descriptors) live in device memory and are
// rewritten through a pinned staging ring whenever the host copy changes, which is the
// reference's `uniform.write` before a dispatch.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/clay_fluid.h"
#include "clay_device.cuh"
#include "launch.h"

using namespace clay;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

}  // namespace

namespace clay {
// The same error slot for the other host translation units (the server).
int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}
}  // namespace clay

namespace {

#define CK(x)                                                                                 \
  do {                                                                                        \
    cudaError_t e_ = (x);                                                                     \
    if (e_ != cudaSuccess) return fail(CLAY_ECUDA, "%s: %s", #x, cudaGetErrorString(e_));     \
  } while (0)

constexpr int TILE = 8;
constexpr int kMaxResolution = 4096;  // 4096^3 voxels per level: far beyond device memory, far below int64 overflow

// SplatField's default mip count, Math.max(1, Math.log2(res / TILE) | 0) (splat.ts:149):
// 1 wherever the logarithm is not a positive number (resolution 0 or below included).
int default_splat_mips(int res) {
  if (res <= 0) return 1;
  return std::max(1, static_cast<int>(std::log2(static_cast<double>(res) / TILE)));
}

// A temporary device buffer of a host query, freed on every return path (an error included).
template <class T>
struct TempDev {
  T* p = nullptr;
  TempDev() = default;
  TempDev(const TempDev&) = delete;
  TempDev& operator=(const TempDev&) = delete;
  ~TempDev() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * n); }
};

}  // namespace

int clay::report_error(int code, const char* msg) { return fail(code, "%s", msg); }

// ------------------------------------------------------------------------------------------
// Context and staging ring.
struct clay_ctx {
  int device = 0;
  std::atomic<uint64_t> bytes{0};
  // Pinned staging ring for small host->device uniform writes.
  static constexpr int kSlots = 1024;
  static constexpr size_t kSlotBytes = 1024;
  char* ring = nullptr;
  cudaEvent_t ev[kSlots];
  bool used[kSlots];
  int next = 0;
  std::mutex mu;

  int dev_alloc(void** p, size_t n) {
    cudaError_t e = cudaMalloc(p, n == 0 ? 16 : n);
    if (e != cudaSuccess) {
      *p = nullptr;
      return fail(CLAY_ENOMEM, "cudaMalloc(%zu bytes): %s", n, cudaGetErrorString(e));
    }
    bytes += n;
    return CLAY_OK;
  }
  void dev_free(void* p, size_t n) {
    if (p) {
      cudaFree(p);
      bytes -= n;
    }
  }
  // Enqueues an H2D copy of `n` bytes through a pinned slot; the host buffer may be reused
  // as soon as this returns.
  int upload(void* dst, const void* src, size_t n, cudaStream_t s) {
    if (n > kSlotBytes) {
      CK(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, s));
      return CLAY_OK;
    }
    std::lock_guard<std::mutex> lk(mu);
    int slot = next;
    next = (next + 1) % kSlots;
    if (used[slot]) CK(cudaEventSynchronize(ev[slot]));
    char* h = ring + static_cast<size_t>(slot) * kSlotBytes;
    std::memcpy(h, src, n);
    CK(cudaMemcpyAsync(dst, h, n, cudaMemcpyHostToDevice, s));
    CK(cudaEventRecord(ev[slot], s));
    used[slot] = true;
    return CLAY_OK;
  }
};

namespace {
struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
};
}  // namespace

// ------------------------------------------------------------------------------------------
struct clay_volume {
  clay_ctx* ctx = nullptr;
  int res = 0, mips = 0;
  double world = 0, band = 0, gradv = 1, origin[3] = {0, 0, 0};
  int64_t total = 0;
  int64_t off[16] = {0};
  int tile_res[16] = {0};
  int total_cells = 0;
  __half* dist = nullptr;
  __half* mat = nullptr;
  VolParamsDev h{};
  VolParamsDev* d = nullptr;
  bool dirty = true;

  void refresh_uniform() {
    double half = world / 2;
    for (int k = 0; k < 3; k++) {
      h.origin[k] = static_cast<float>(origin[k]);
      h.center[k] = static_cast<float>(origin[k] + half);
    }
    h.voxel = static_cast<float>(world / res);
    h.mips = mips;
    h.extent = static_cast<float>(world);
    h.half = static_cast<float>(half);
    h.band = static_cast<float>(band);
    // volume.ts:302: `layout.$.params.voxelSize * gradScale`, an f32 product.
    h.grad_h = h.voxel * static_cast<float>(gradv);
    h.res = res;
    h.dist = dist;
    h.mat = mat;
    dirty = true;
  }
  int flush(cudaStream_t s) {
    if (!dirty) return CLAY_OK;
    int rc = ctx->upload(d, &h, sizeof(h), s);
    if (rc == CLAY_OK) dirty = false;
    return rc;
  }
};

struct clay_field {
  clay_ctx* ctx = nullptr;
  struct Leaf {
    clay_volume* vol;
    double off[3];
    const float* dyn = nullptr;  // device offset applied outermost (an extractor's motion centre)
  };
  std::vector<Leaf> leaves;
  FieldDev h{};
  FieldDev* d = nullptr;
  bool dirty = true;

  void refresh() {
    std::memset(&h, 0, sizeof(h));
    h.n = static_cast<int>(leaves.size());
    for (size_t i = 0; i < leaves.size(); i++) {
      h.leaf[i].vp = leaves[i].vol->d;
      bool any = false;
      for (int k = 0; k < 3; k++) {
        h.leaf[i].offset[k] = static_cast<float>(leaves[i].off[k]);
        any = any || leaves[i].off[k] != 0.0;
      }
      h.leaf[i].has_offset = any ? 1 : 0;
      h.leaf[i].dyn_offset = leaves[i].dyn;
    }
    dirty = true;
  }
  int flush(cudaStream_t s) {
    for (auto& l : leaves) {
      int rc = l.vol->flush(s);
      if (rc) return rc;
    }
    if (!dirty) return CLAY_OK;
    int rc = ctx->upload(d, &h, sizeof(h), s);
    if (rc == CLAY_OK) dirty = false;
    return rc;
  }
};

struct clay_splat {
  clay_ctx* ctx = nullptr;
  clay_volume* vol = nullptr;
  clay_field* field = nullptr;
  clay_cloud_desc cloud{};
  double radius = 0, material = 0, band = 0;
  int res = 0, mips = 0;
  uint32_t* keys = nullptr;
  SplatDev h{};
  SplatDev* d = nullptr;          // cloud in index order
  SplatDev* d_ordered = nullptr;  // the fluid's cloud in cell order (fluid-owned splats)
  const uint32_t* order = nullptr;
  bool desc_dirty = true;

  int flush(cudaStream_t s) {
    int rc = vol->flush(s);
    if (rc) return rc;
    if (!desc_dirty) return CLAY_OK;
    h.order = nullptr;
    rc = ctx->upload(d, &h, sizeof(h), s);
    if (rc) return rc;
    if (d_ordered) {
      SplatDev o = h;
      o.order = order;
      rc = ctx->upload(d_ordered, &o, sizeof(o), s);
      if (rc) return rc;
    }
    desc_dirty = false;
    return CLAY_OK;
  }
};

struct clay_fluid {
  clay_ctx* ctx = nullptr;
  const clay_field* world = nullptr;
  int64_t capacity = 0;
  double spacing = 0, h = 0, radius = 0, surf_r = 0, material = 0, band = 0, world_size = 0;
  double origin[3] = {0, 0, 0};
  int bucket = 0, bake_res = 0, bake_mips = 0, substeps = 0;
  // Host state of fluid.ts:134-138.
  int64_t live = 0, cursor = 0, pending = 0;
  uint32_t seed = 1;
  clay_fluid_params frozen{};
  clay_fluid_params written{};
  bool written_valid = false;
  // Derived (fluid.ts:168-182,239-247).
  double rest = 0, poly6 = 0, spiky = 0, mass = 0;
  int G = 0;
  double gorig[3] = {0, 0, 0};
  int mode = CLAY_MODE_FAST;
  uint32_t parts_scan = 1;
  // Device memory.
  std::vector<DevBuf> bufs;
  ParticleDev* parts = nullptr;
  ParamsDev* prm = nullptr;
  ContactsDev* contacts = nullptr;
  GridState* gs = nullptr;
  SceneDev hs{};
  SceneDev* d_scene = nullptr;
  clay_splat* surface = nullptr;
  uint64_t own_bytes = 0;

  template <class T>
  int alloc(T** p, size_t count) {
    void* q = nullptr;
    int rc = ctx->dev_alloc(&q, sizeof(T) * count);
    if (rc) return rc;
    bufs.push_back({q, sizeof(T) * count});
    own_bytes += sizeof(T) * count;
    *p = static_cast<T*>(q);
    return CLAY_OK;
  }
};

// ------------------------------------------------------------------------------------------
namespace {

// SdfVolume mip rule (volume.ts:140-160).
int volume_mips(int resolution, int requested, bool has_req, int* out) {
  // Checked first: the halving loop below never ends for 0 (the reference's does not either,
  // volume.ts:148), and the cube of a larger resolution would overflow the 64-bit voxel count.
  if (resolution <= 0 || resolution > kMaxResolution)
    return fail(CLAY_EINVAL, "SdfVolume: resolution %d is outside 1..%d", resolution, kMaxResolution);
  int mips = requested;
  if (!has_req) {
    int halvings = 0;
    double n = static_cast<double>(resolution) / TILE;
    while (n == std::floor(n) && std::fmod(n, 2.0) == 0.0) {
      halvings++;
      n /= 2;
    }
    int lg = static_cast<int>(std::log2(static_cast<double>(resolution) / TILE));
    mips = std::max(1, std::min(lg, halvings + 1));
  }
  if (mips < 1 || mips > kMaxMips)
    return fail(CLAY_EINVAL, "SdfVolume: %d mip levels is outside the supported 1..%d", mips, kMaxMips);
  long long need = static_cast<long long>(TILE) << (mips - 1);
  if (resolution <= 0 || resolution % need != 0)
    return fail(CLAY_EINVAL, "SdfVolume: resolution %d must be a multiple of %lld for %d mip levels", resolution, need,
                mips);
  *out = mips;
  return CLAY_OK;
}

int make_volume(clay_ctx* ctx, int res, int mips_req, bool has_mips, double world, const double origin[3], double band,
                double gradv, clay_volume** out) {
  int mips = 0;
  int rc = volume_mips(res, mips_req, has_mips, &mips);
  if (rc) return rc;
  clay_volume* v = new clay_volume();
  v->ctx = ctx;
  v->res = res;
  v->mips = mips;
  v->world = world;
  v->band = band;
  v->gradv = gradv;
  for (int k = 0; k < 3; k++) v->origin[k] = origin[k];
  int64_t t = 0;
  int cells = 0;
  for (int m = 0; m < mips; m++) {
    int64_t r = res >> m;
    v->off[m] = t;
    t += r * r * r;
    v->tile_res[m] = (res / TILE) >> m;
    cells += v->tile_res[m] * v->tile_res[m] * v->tile_res[m];
  }
  v->total = t;
  v->total_cells = cells;
  void* p = nullptr;
  if ((rc = ctx->dev_alloc(&p, sizeof(__half) * t))) {
    delete v;
    return rc;
  }
  v->dist = static_cast<__half*>(p);
  if ((rc = ctx->dev_alloc(&p, sizeof(__half) * t))) {
    ctx->dev_free(v->dist, sizeof(__half) * t);
    delete v;
    return rc;
  }
  v->mat = static_cast<__half*>(p);
  if ((rc = ctx->dev_alloc(&p, sizeof(VolParamsDev)))) {
    ctx->dev_free(v->dist, sizeof(__half) * t);
    ctx->dev_free(v->mat, sizeof(__half) * t);
    delete v;
    return rc;
  }
  v->d = static_cast<VolParamsDev*>(p);
  // An unwritten volume reads as saturated (+1), not as a surface.
  std::vector<uint16_t> one(static_cast<size_t>(t), 0x3C00u);
  cudaMemcpy(v->dist, one.data(), sizeof(uint16_t) * t, cudaMemcpyHostToDevice);
  cudaMemset(v->mat, 0, sizeof(__half) * t);
  v->refresh_uniform();
  cudaMemcpy(v->d, &v->h, sizeof(v->h), cudaMemcpyHostToDevice);
  v->dirty = false;
  *out = v;
  return CLAY_OK;
}

void free_volume(clay_volume* v) {
  if (!v) return;
  v->ctx->dev_free(v->dist, sizeof(__half) * v->total);
  v->ctx->dev_free(v->mat, sizeof(__half) * v->total);
  v->ctx->dev_free(v->d, sizeof(VolParamsDev));
  delete v;
}

int make_field(clay_ctx* ctx, std::vector<clay_field::Leaf> leaves, clay_field** out) {
  if (leaves.empty() || leaves.size() > static_cast<size_t>(kMaxLeaves))
    return fail(CLAY_EINVAL, "a collider holds 1..%d volume leaves, got %zu", kMaxLeaves, leaves.size());
  clay_field* f = new clay_field();
  f->ctx = ctx;
  f->leaves = std::move(leaves);
  void* p = nullptr;
  int rc = ctx->dev_alloc(&p, sizeof(FieldDev));
  if (rc) {
    delete f;
    return rc;
  }
  f->d = static_cast<FieldDev*>(p);
  f->refresh();
  cudaMemcpy(f->d, &f->h, sizeof(f->h), cudaMemcpyHostToDevice);
  f->dirty = false;
  *out = f;
  return CLAY_OK;
}

void free_field(clay_field* f) {
  if (!f) return;
  f->ctx->dev_free(f->d, sizeof(FieldDev));
  delete f;
}

int make_splat(clay_ctx* ctx, const clay_cloud_desc* cloud, const clay_splat_opts* o, bool with_order,
               clay_splat** out) {
  if (!cloud || !o) return fail(CLAY_EINVAL, "SplatField: cloud and options are required");
  if (!cloud->positions && cloud->capacity > 0) return fail(CLAY_EINVAL, "SplatField: cloud has no positions");
  if (cloud->position_stride < 12 && cloud->capacity > 1)
    return fail(CLAY_EINVAL, "SplatField: position stride %u is below 12 bytes", cloud->position_stride);
  if (cloud->live_mode > CLAY_LIVE_RANGE) return fail(CLAY_EINVAL, "SplatField: unknown live mode %u", cloud->live_mode);
  if (cloud->live_mode == CLAY_LIVE_COUNT && !cloud->live_count)
    return fail(CLAY_EINVAL, "SplatField: CLAY_LIVE_COUNT needs live_count");
  if (cloud->live_mode == CLAY_LIVE_RANGE && (!cloud->live_first || !cloud->live_range_count))
    return fail(CLAY_EINVAL, "SplatField: CLAY_LIVE_RANGE needs live_first and live_range_count");
  // splat.ts:148-153
  int res = (o->set & CLAY_SPLAT_RESOLUTION) ? o->resolution : 64;
  bool has_m = (o->set & CLAY_SPLAT_MIP_LEVELS) != 0;
  int mips = has_m ? o->mip_levels : default_splat_mips(res);
  double band = (o->set & CLAY_SPLAT_BAND) ? o->band : 2.0;
  double material = (o->set & CLAY_SPLAT_MATERIAL) ? o->material : 0.0;
  double world = (o->set & CLAY_SPLAT_WORLD_SIZE) ? o->world_size : 24.0;
  double origin[3] = {-12, -4, -12};
  if (o->set & CLAY_SPLAT_ORIGIN)
    for (int k = 0; k < 3; k++) origin[k] = o->origin[k];
  if (!(o->radius >= 0)) return fail(CLAY_EINVAL, "SplatField: radius must be a non-negative number");
  clay_volume* vol = nullptr;
  int rc = make_volume(ctx, res, mips, true, world, origin, band, 1.0, &vol);
  if (rc) return rc;
  clay_splat* s = new clay_splat();
  s->ctx = ctx;
  s->vol = vol;
  s->cloud = *cloud;
  s->radius = o->radius;
  s->material = material;
  s->band = band;
  s->res = res;
  s->mips = vol->mips;
  rc = make_field(ctx, {{vol, {0, 0, 0}}}, &s->field);
  if (rc) {
    free_volume(vol);
    delete s;
    return rc;
  }
  void* p = nullptr;
  if ((rc = ctx->dev_alloc(&p, sizeof(uint32_t) * vol->total))) goto fail_out;
  s->keys = static_cast<uint32_t*>(p);
  // The key grid holds kNoHit (all bits set) between bakes (see k_resolve).
  {
    cudaMemset(s->keys, 0xff, sizeof(uint32_t) * vol->total);
    // The material channel is the constant `material` (splat.ts:273): written once here.
    uint16_t mh;
    __half hm = __float2half_rn(static_cast<float>(material));
    std::memcpy(&mh, &hm, 2);
    std::vector<uint16_t> mv(static_cast<size_t>(vol->total), mh);
    cudaMemcpy(vol->mat, mv.data(), sizeof(uint16_t) * vol->total, cudaMemcpyHostToDevice);
    // Before the first bake the volume reads as the clear value 65535 -> +1.
  }
  if ((rc = ctx->dev_alloc(&p, sizeof(SplatDev)))) goto fail_out;
  s->d = static_cast<SplatDev*>(p);
  if (with_order) {
    if ((rc = ctx->dev_alloc(&p, sizeof(SplatDev)))) goto fail_out;
    s->d_ordered = static_cast<SplatDev*>(p);
  }
  {
    SplatDev& h = s->h;
    std::memset(&h, 0, sizeof(h));
    h.pos = static_cast<const char*>(cloud->positions);
    h.nrm = static_cast<const char*>(cloud->normals);
    h.quat = cloud->rotation;
    h.live_count = cloud->live_count;
    h.live_first = cloud->live_first;
    h.live_range_count = cloud->live_range_count;
    h.keys = s->keys;
    h.dist_out = vol->dist;
    h.key_capture = nullptr;
    h.vp = vol->d;
    h.pos_stride = cloud->position_stride;
    h.nrm_stride = cloud->normal_stride;
    h.capacity = cloud->capacity;
    h.live_mode = cloud->live_mode;
    h.mips = vol->mips;
    h.radius = static_cast<float>(o->radius);
    for (int m = 0; m < vol->mips; m++) {
      // splat.ts:215-238 with voxelSizeAt(m) = (worldSize / resolution) * 2**m (volume.ts:165,336).
      double voxel = (world / res) * std::pow(2.0, m);
      double bw = band * voxel;
      h.r[m] = res >> m;
      h.off[m] = vol->off[m];
      h.voxel[m] = static_cast<float>(voxel);
      h.bw[m] = static_cast<float>(bw);
      h.reach[m] = static_cast<float>(o->radius + bw);
      h.inv_voxel[m] = static_cast<float>(1 / voxel);
    }
    h.total = vol->total;
    h.tile_ratio = kSplatTileRatio;
    h.walk_weight = kSplatWalkWeight;
    s->desc_dirty = true;
    cudaStream_t st = nullptr;
    rc = s->flush(st);
    if (rc) goto fail_out;
  }
  *out = s;
  return CLAY_OK;
fail_out:
  if (s->keys) ctx->dev_free(s->keys, sizeof(uint32_t) * vol->total);
  if (s->d) ctx->dev_free(s->d, sizeof(SplatDev));
  if (s->d_ordered) ctx->dev_free(s->d_ordered, sizeof(SplatDev));
  free_field(s->field);
  free_volume(vol);
  delete s;
  return rc;
}

void free_splat(clay_splat* s) {
  if (!s) return;
  s->ctx->dev_free(s->keys, sizeof(uint32_t) * s->vol->total);
  s->ctx->dev_free(s->d, sizeof(SplatDev));
  if (s->d_ordered) s->ctx->dev_free(s->d_ordered, sizeof(SplatDev));
  free_field(s->field);
  free_volume(s->vol);
  delete s;
}

// Blocks over the cloud's iteration space for every mip (plain bake).
int splat_bake(clay_splat* s, cudaStream_t st, bool ordered, int64_t iter_n) {
  int rc = s->flush(st);
  if (rc) return rc;
  const SplatDev* d = (ordered && s->d_ordered) ? s->d_ordered : s->d;
  int64_t n = iter_n;
  if (n > 0) {
    int blocks = static_cast<int>((n + kSplatThreads - 1) / kSplatThreads);
    CK(L_splat(d, nullptr, blocks, s->mips, s->cloud.normals ? kSplatAccVoxelsDiscs : kSplatAccVoxels, st));
  }
  int64_t quads = (s->vol->total + 3) / 4;
  int rblocks = static_cast<int>((quads + kResolveThreads - 1) / kResolveThreads);
  CK(L_resolve(d, nullptr, rblocks, st));
  return CLAY_OK;
}

}  // namespace

// ==========================================================================================
extern "C" {

const char* clay_last_error(void) { return g_err.c_str(); }
const char* clay_version(void) { return "clay-fluid-b200 0.1 (sm_100a)"; }
uint64_t clay_kernel_launch_count(void) { return clay::launch_count(); }

int clay_ctx_create(int device, clay_ctx** out) {
  if (!out) return fail(CLAY_EINVAL, "clay_ctx_create: out is NULL");
  int n = 0;
  CK(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(CLAY_EINVAL, "clay_ctx_create: device %d of %d", device, n);
  CK(cudaSetDevice(device));
  clay_ctx* c = new clay_ctx();
  c->device = device;
  cudaError_t e = cudaMallocHost(&c->ring, clay_ctx::kSlots * clay_ctx::kSlotBytes);
  if (e != cudaSuccess) {
    delete c;
    return fail(CLAY_ECUDA, "cudaMallocHost: %s", cudaGetErrorString(e));
  }
  for (int i = 0; i < clay_ctx::kSlots; i++) {
    cudaEventCreateWithFlags(&c->ev[i], cudaEventDisableTiming);
    c->used[i] = false;
  }
  *out = c;
  return CLAY_OK;
}

void clay_ctx_destroy(clay_ctx* ctx) {
  if (!ctx) return;
  cudaDeviceSynchronize();
  for (int i = 0; i < clay_ctx::kSlots; i++) cudaEventDestroy(ctx->ev[i]);
  cudaFreeHost(ctx->ring);
  delete ctx;
}

int clay_ctx_bytes_in_use(const clay_ctx* ctx, uint64_t* out) {
  if (!ctx || !out) return fail(CLAY_EINVAL, "clay_ctx_bytes_in_use: NULL argument");
  *out = ctx->bytes.load();
  return CLAY_OK;
}

// ---- SdfVolume ----------------------------------------------------------------------------
int clay_volume_create(clay_ctx* ctx, const clay_volume_opts* o, clay_volume** out) {
  if (!ctx || !out) return fail(CLAY_EINVAL, "clay_volume_create: NULL argument");
  clay_volume_opts d{};
  if (o) d = *o;
  int res = (d.set & CLAY_VOL_RESOLUTION) ? d.resolution : 128;
  double world = (d.set & CLAY_VOL_WORLD_SIZE) ? d.world_size : 16.0;
  double band = (d.set & CLAY_VOL_BAND) ? d.band : 4.0;
  double gv = (d.set & CLAY_VOL_GRADIENT_VOXELS) ? d.gradient_voxels : 1.0;
  double origin[3] = {0, 0, 0};
  if (d.set & CLAY_VOL_ORIGIN)
    for (int k = 0; k < 3; k++) origin[k] = d.origin[k];
  return make_volume(ctx, res, d.mip_levels, (d.set & CLAY_VOL_MIP_LEVELS) != 0, world, origin, band, gv, out);
}

void clay_volume_destroy(clay_volume* v) { free_volume(v); }

int clay_volume_get_info(const clay_volume* v, clay_volume_info* out) {
  if (!v || !out) return fail(CLAY_EINVAL, "clay_volume_get_info: NULL argument");
  std::memset(out, 0, sizeof(*out));
  out->resolution = v->res;
  out->mip_levels = v->mips;
  out->world_size = v->world;
  out->voxel_size = v->world / v->res;
  out->band = v->band;
  for (int k = 0; k < 3; k++) out->origin[k] = v->origin[k];
  for (int m = 0; m < v->mips; m++) {
    out->tile_res_per_mip[m] = v->tile_res[m];
    out->level_offset[m] = v->off[m];
  }
  out->total_voxels = v->total;
  out->total_cells = v->total_cells;
  return CLAY_OK;
}

int clay_volume_set_origin(clay_volume* v, double x, double y, double z) {
  if (!v) return fail(CLAY_EINVAL, "clay_volume_set_origin: NULL volume");
  v->origin[0] = x;
  v->origin[1] = y;
  v->origin[2] = z;
  v->refresh_uniform();
  return CLAY_OK;
}

double clay_volume_voxel_size_at(const clay_volume* v, int mip) {
  if (!v) return 0;
  return (v->world / v->res) * std::pow(2.0, mip);
}

int clay_volume_device_planes(clay_volume* v, void** dist, void** mat) {
  if (!v) return fail(CLAY_EINVAL, "clay_volume_device_planes: NULL volume");
  if (dist) *dist = v->dist;
  if (mat) *mat = v->mat;
  return CLAY_OK;
}

int clay_volume_upload(clay_volume* v, const uint16_t* dist, const uint16_t* mat, void* stream) {
  if (!v) return fail(CLAY_EINVAL, "clay_volume_upload: NULL volume");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dist) CK(cudaMemcpyAsync(v->dist, dist, sizeof(uint16_t) * v->total, cudaMemcpyHostToDevice, s));
  if (mat) CK(cudaMemcpyAsync(v->mat, mat, sizeof(uint16_t) * v->total, cudaMemcpyHostToDevice, s));
  return CLAY_OK;
}

int clay_volume_download(const clay_volume* v, uint16_t* dist, uint16_t* mat, void* stream) {
  if (!v) return fail(CLAY_EINVAL, "clay_volume_download: NULL volume");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dist) CK(cudaMemcpyAsync(dist, v->dist, sizeof(uint16_t) * v->total, cudaMemcpyDeviceToHost, s));
  if (mat) CK(cudaMemcpyAsync(mat, v->mat, sizeof(uint16_t) * v->total, cudaMemcpyDeviceToHost, s));
  return CLAY_OK;
}

int clay_volume_download_rgba16f(const clay_volume* v, int mip, uint16_t* rgba, void* stream) {
  if (!v || !rgba) return fail(CLAY_EINVAL, "clay_volume_download_rgba16f: NULL argument");
  if (mip < 0 || mip >= v->mips) return fail(CLAY_EINVAL, "mip %d out of range 0..%d", mip, v->mips - 1);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int64_t r = v->res >> mip;
  int64_t n = r * r * r;
  std::vector<uint16_t> d(n), m(n);
  CK(cudaMemcpyAsync(d.data(), v->dist + v->off[mip], sizeof(uint16_t) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(m.data(), v->mat + v->off[mip], sizeof(uint16_t) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int64_t i = 0; i < n; i++) {
    rgba[4 * i] = d[i];
    rgba[4 * i + 1] = m[i];
    rgba[4 * i + 2] = 0x0000u;
    rgba[4 * i + 3] = 0x3C00u;
  }
  return CLAY_OK;
}

int clay_volume_build_brushes(clay_volume* v, const clay_brush* brushes, int count, void* stream) {
  if (!v) return fail(CLAY_EINVAL, "clay_volume_build_brushes: NULL volume");
  if (count < 0 || (count > 0 && !brushes)) return fail(CLAY_EINVAL, "clay_volume_build_brushes: bad brush list");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int n = std::min(count, 256);  // builder.ts:57,148-153
  BrushDev* db = nullptr;
  void* p = nullptr;
  int rc = v->ctx->dev_alloc(&p, sizeof(BrushDev) * std::max(n, 1));
  if (rc) return rc;
  db = static_cast<BrushDev*>(p);
  if (n > 0) CK(cudaMemcpyAsync(db, brushes, sizeof(BrushDev) * n, cudaMemcpyHostToDevice, s));
  for (int m = 0; m < v->mips; m++) {
    double voxel = (v->world / v->res) * std::pow(2.0, m);
    double tile_size = voxel * TILE;
    double bw = v->band * voxel;
    BuildLevelDev L;
    L.dist = v->dist + v->off[m];
    L.mat = v->mat + v->off[m];
    L.R = v->res >> m;
    L.tiles = v->tile_res[m];
    // The builder bakes the origin the volume had at construction (builder.ts:75).
    L.ox = static_cast<float>(v->origin[0]);
    L.oy = static_cast<float>(v->origin[1]);
    L.oz = static_cast<float>(v->origin[2]);
    L.voxel = static_cast<float>(voxel);
    L.tile_size = static_cast<float>(tile_size);
    L.tile_half = static_cast<float>(tile_size / 2);
    L.bw = static_cast<float>(bw);
    L.empty = static_cast<float>(bw * 4);
    CK(L_build(L, db, n, s));
  }
  CK(cudaStreamSynchronize(s));
  v->ctx->dev_free(db, sizeof(BrushDev) * std::max(n, 1));
  return CLAY_OK;
}

// ---- TracedField --------------------------------------------------------------------------
int clay_field_from_volume(clay_volume* vol, clay_field** out) {
  if (!vol || !out) return fail(CLAY_EINVAL, "clay_field_from_volume: NULL argument");
  return make_field(vol->ctx, {{vol, {0, 0, 0}}}, out);
}

int clay_field_union(const clay_field* a, const clay_field* b, clay_field** out) {
  if (!a || !b || !out) return fail(CLAY_EINVAL, "clay_field_union: NULL argument");
  std::vector<clay_field::Leaf> l = a->leaves;
  l.insert(l.end(), b->leaves.begin(), b->leaves.end());
  return make_field(a->ctx, std::move(l), out);
}

int clay_field_offset(const clay_field* f, double dx, double dy, double dz, clay_field** out) {
  if (!f || !out) return fail(CLAY_EINVAL, "clay_field_offset: NULL argument");
  std::vector<clay_field::Leaf> l = f->leaves;
  for (auto& x : l) {
    x.off[0] += dx;
    x.off[1] += dy;
    x.off[2] += dz;
  }
  return make_field(f->ctx, std::move(l), out);
}

int clay_field_set_offset(clay_field* f, double dx, double dy, double dz) {
  if (!f) return fail(CLAY_EINVAL, "clay_field_set_offset: NULL field");
  for (auto& x : f->leaves) {
    x.off[0] = dx;
    x.off[1] = dy;
    x.off[2] = dz;
  }
  f->refresh();
  return CLAY_OK;
}

void clay_field_destroy(clay_field* f) { free_field(f); }

int clay_field_query_mip(const clay_field* f, const float* pts, int n, int mip, float* sample_xy, float* field_xy,
                         void* stream) {
  if (!f || n < 0 || (n > 0 && (!pts || !sample_xy || !field_xy)))
    return fail(CLAY_EINVAL, "clay_field_query_mip: bad argument");
  if (mip < 0) return fail(CLAY_EINVAL, "clay_field_query_mip: mip %d < 0", mip);
  if (n == 0) return CLAY_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = const_cast<clay_field*>(f)->flush(s);
  if (rc) return rc;
  TempDev<float> dp, ds, df;
  CK(dp.alloc(3 * static_cast<size_t>(n)));
  CK(ds.alloc(2 * static_cast<size_t>(n)));
  CK(df.alloc(2 * static_cast<size_t>(n)));
  CK(cudaMemcpyAsync(dp.p, pts, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s));
  CK(L_field_query_mip(f->d, dp.p, n, mip, ds.p, df.p, s));
  CK(cudaMemcpyAsync(sample_xy, ds.p, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(field_xy, df.p, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return CLAY_OK;
}

int clay_field_query_mip_device(const clay_field* f, const float* pts, int n, int mip, float* sample_xy, float* field_xy,
                                void* stream) {
  if (!f || n < 0 || (n > 0 && (!pts || !sample_xy || !field_xy)))
    return fail(CLAY_EINVAL, "clay_field_query_mip_device: bad argument");
  if (mip < 0) return fail(CLAY_EINVAL, "clay_field_query_mip_device: mip %d < 0", mip);
  if (n == 0) return CLAY_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = const_cast<clay_field*>(f)->flush(s);
  if (rc) return rc;
  CK(L_field_query_mip(f->d, pts, n, mip, sample_xy, field_xy, s));
  return CLAY_OK;
}

int clay_field_band_voxel(const clay_field* f, int mip, float* band_world, float* voxel_world) {
  if (!f || !band_world || !voxel_world || mip < 0) return fail(CLAY_EINVAL, "clay_field_band_voxel: bad argument");
  if (f->leaves.empty()) return fail(CLAY_ESTATE, "clay_field_band_voxel: empty field");
  float bw = 0.0f, vw = 0.0f;
  for (size_t i = 0; i < f->leaves.size(); i++) {
    const VolParamsDev& h = f->leaves[i].vol->h;
    const float m = std::min(static_cast<float>(mip), static_cast<float>(h.mips - 1));  // capped
    const float p2 = std::ldexp(1.0f, static_cast<int>(m));  // exp2 of an integer level
    const float b = (h.band * h.voxel) * p2;
    const float v = h.voxel * p2;
    // unionField: min of the bands, max of the voxels (trace/field.ts:294-305)
    bw = i == 0 ? b : std::min(bw, b);
    vw = i == 0 ? v : std::max(vw, v);
  }
  *band_world = bw;
  *voxel_world = vw;
  return CLAY_OK;
}

int clay_field_query(const clay_field* f, const float* pts, int n, float* sxy, float* nrm, void* stream) {
  if (!f || n < 0 || (n > 0 && (!pts || !sxy || !nrm))) return fail(CLAY_EINVAL, "clay_field_query: bad argument");
  if (n == 0) return CLAY_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = const_cast<clay_field*>(f)->flush(s);
  if (rc) return rc;
  TempDev<float> dp, ds, dn;
  CK(dp.alloc(3 * static_cast<size_t>(n)));
  CK(ds.alloc(2 * static_cast<size_t>(n)));
  CK(dn.alloc(3 * static_cast<size_t>(n)));
  CK(cudaMemcpyAsync(dp.p, pts, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s));
  CK(L_field_query(f->d, dp.p, n, ds.p, dn.p, s));
  CK(cudaMemcpyAsync(sxy, ds.p, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(nrm, dn.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return CLAY_OK;
}

// ---- SplatField ---------------------------------------------------------------------------
int clay_splat_create(clay_ctx* ctx, const clay_cloud_desc* cloud, const clay_splat_opts* opts, clay_splat** out) {
  if (!ctx || !out) return fail(CLAY_EINVAL, "clay_splat_create: NULL argument");
  return make_splat(ctx, cloud, opts, false, out);
}

void clay_splat_destroy(clay_splat* s) { free_splat(s); }

int clay_splat_set_center(clay_splat* s, double x, double y, double z) {
  if (!s) return fail(CLAY_EINVAL, "clay_splat_set_center: NULL splat");
  double half = s->vol->world / 2;  // splat.ts:284-287
  return clay_volume_set_origin(s->vol, x - half, y - half, z - half);
}

int clay_splat_bake(clay_splat* s, void* stream) {
  if (!s) return fail(CLAY_EINVAL, "clay_splat_bake: NULL splat");
  return splat_bake(s, static_cast<cudaStream_t>(stream), false, s->cloud.capacity);
}

clay_volume* clay_splat_volume(clay_splat* s) { return s ? s->vol : nullptr; }
clay_field* clay_splat_field(clay_splat* s) { return s ? s->field : nullptr; }

int clay_splat_capture_keys(clay_splat* s, uint32_t* keys_device) {
  if (!s) return fail(CLAY_EINVAL, "clay_splat_capture_keys: NULL splat");
  s->h.key_capture = keys_device;
  s->desc_dirty = true;
  return CLAY_OK;
}

// ---- FluidSim -----------------------------------------------------------------------------
static int fluid_derive(clay_fluid* f) {
  // fluid.ts:168-182
  double h = f->h;
  f->poly6 = 315 / (64 * M_PI * std::pow(h, 9));
  f->spiky = -45 / (M_PI * std::pow(h, 6));
  f->mass = std::pow(f->spacing, 3);
  double rest = 0;
  int reach = static_cast<int>(std::ceil(h / f->spacing));
  for (int z = -reach; z <= reach; z++)
    for (int y = -reach; y <= reach; y++)
      for (int x = -reach; x <= reach; x++) {
        double r2 = static_cast<double>(x * x + y * y + z * z) * f->spacing * f->spacing;
        if (r2 < h * h) rest += f->mass * f->poly6 * std::pow(h * h - r2, 3);
      }
  f->rest = rest;
  // fluid.ts:239-244
  double g = std::ceil(f->world_size / h) + 2;
  if (!(g >= 3 && g <= 1024))
    return fail(CLAY_EINVAL, "FluidSim: grid resolution %.0f (worldSize / smoothing + 2) must be in 3..1024", g);
  f->G = static_cast<int>(g);
  for (int k = 0; k < 3; k++) f->gorig[k] = f->origin[k] - h;
  return CLAY_OK;
}

static void fill_scene(clay_fluid* f) {
  SceneDev& s = f->hs;
  s.h = static_cast<float>(f->h);
  s.h2 = static_cast<float>(f->h * f->h);
  s.inv_h = static_cast<float>(1 / f->h);
  s.h6 = static_cast<float>(std::pow(f->h, 6));
  s.mass = static_cast<float>(f->mass);
  s.mass_poly6 = static_cast<float>(f->mass * f->poly6);
  s.spiky = static_cast<float>(f->spiky);
  s.rest = static_cast<float>(f->rest);
  s.rest_floor = static_cast<float>(f->rest * 0.1);
  s.radius = static_cast<float>(f->radius);
  for (int k = 0; k < 3; k++) {
    s.gorig[k] = static_cast<float>(f->gorig[k]);
    // fluid.ts:444-447: walls of the bake volume's box, summed in binary64.
    s.wlo[k] = static_cast<float>(f->origin[k] + f->radius);
    s.whi[k] = static_cast<float>(f->origin[k] + f->world_size - f->radius);
  }
  s.G = f->G;
  s.capacity = static_cast<uint32_t>(f->capacity);
  s.bucket = static_cast<uint32_t>(f->bucket);
  s.parts_scan = f->parts_scan;
  s.substeps = f->substeps;
  s.world = f->world ? f->world->d : nullptr;
}

}  // extern "C"

namespace {
// FluidSim options with the reference's defaults (fluid.ts:141-160), validated.
int fluid_options(const clay_fluid_opts& o, clay_fluid* f) {
  f->capacity = (o.set & CLAY_FLUID_CAPACITY) ? o.capacity : 8192;
  f->spacing = (o.set & CLAY_FLUID_SPACING) ? o.spacing : 0.45;
  f->h = (o.set & CLAY_FLUID_SMOOTHING) ? o.smoothing : f->spacing * 2.2;
  f->bucket = (o.set & CLAY_FLUID_BUCKET) ? o.bucket : 64;
  f->radius = (o.set & CLAY_FLUID_RADIUS) ? o.radius : f->spacing * 0.5;
  f->surf_r = (o.set & CLAY_FLUID_SURFACE_RADIUS) ? o.surface_radius : f->spacing * 1.1;
  f->material = (o.set & CLAY_FLUID_MATERIAL) ? o.material : 0.0;
  f->bake_res = (o.set & CLAY_FLUID_BAKE_RESOLUTION) ? o.bake_resolution : 64;
  f->bake_mips = (o.set & CLAY_FLUID_BAKE_MIP_LEVELS)
                     ? o.bake_mip_levels
                     : default_splat_mips(f->bake_res);
  f->band = (o.set & CLAY_FLUID_BAKE_BAND) ? o.bake_band : 2.0;
  f->world_size = (o.set & CLAY_FLUID_WORLD_SIZE) ? o.world_size : 24.0;
  double org[3] = {-12, -4, -12};
  if (o.set & CLAY_FLUID_ORIGIN)
    for (int k = 0; k < 3; k++) org[k] = o.origin[k];
  for (int k = 0; k < 3; k++) f->origin[k] = org[k];
  f->substeps = (o.set & CLAY_FLUID_SUBSTEPS) ? o.substeps : 3;
  if (f->capacity <= 0 || f->capacity > kMaxCapacity)
    return fail(CLAY_EINVAL, "FluidSim: capacity %lld must be in 1..%lld", static_cast<long long>(f->capacity),
                static_cast<long long>(kMaxCapacity));
  if (!(f->spacing > 0) || !(f->h > 0) || f->bucket <= 0 || f->substeps < 0)
    return fail(CLAY_EINVAL, "FluidSim: spacing, smoothing and bucket must be positive and substeps non-negative");
  return CLAY_OK;
}
}  // namespace

extern "C" {

int clay_fluid_estimate_bytes(const clay_fluid_opts* opts, uint64_t* out) {
  if (!out) return fail(CLAY_EINVAL, "clay_fluid_estimate_bytes: out is NULL");
  clay_fluid_opts o{};
  if (opts) o = *opts;
  clay_fluid f;
  int rc = fluid_options(o, &f);
  if (!rc) rc = fluid_derive(&f);
  if (rc) return rc;
  // the allocations of clay_fluid_create: per particle, per grid cell, fixed, then the surface
  const uint64_t C = static_cast<uint64_t>(f.capacity);
  const uint64_t cells = static_cast<uint64_t>(f.G) * f.G * f.G;
  uint64_t b = C * (sizeof(ParticleDev) + 4 * sizeof(uint32_t) + 4 * sizeof(float4) + (kMaxNbr / 4) * sizeof(uint4)) +
               (cells + 1) * sizeof(uint32_t) + (cells + 2) * sizeof(uint32_t) + sizeof(ParamsDev) + sizeof(ContactsDev) +
               sizeof(GridState) + sizeof(SceneDev);
  uint64_t t = 0;
  for (int m = 0; m < f.bake_mips; m++) {
    const uint64_t r = static_cast<uint64_t>(f.bake_res >> m);
    t += r * r * r;
  }
  // volume planes (f16 distance, f16 material) and uniform, its field, the key grid, descriptors
  b += t * (2 * sizeof(__half) + sizeof(uint32_t)) + sizeof(VolParamsDev) + sizeof(FieldDev) + 2 * sizeof(SplatDev);
  *out = b;
  return CLAY_OK;
}

int clay_fluid_create(clay_ctx* ctx, const clay_field* world, const clay_fluid_opts* opts, clay_fluid** out) {
  if (!ctx || !out) return fail(CLAY_EINVAL, "clay_fluid_create: NULL argument");
  clay_fluid_opts o{};
  if (opts) o = *opts;
  clay_fluid* f = new clay_fluid();
  f->ctx = ctx;
  f->world = world;
  {
    int rc0 = fluid_options(o, f);
    if (rc0) {
      delete f;
      return rc0;
    }
  }
  if (world && world->ctx != ctx) {
    delete f;
    return fail(CLAY_EINVAL, "FluidSim: the collider belongs to another context");
  }
  int rc = fluid_derive(f);
  if (rc) {
    delete f;
    return rc;
  }
  // frozen (fluid.ts:184-203)
  clay_fluid_params& P = f->frozen;
  std::memset(&P, 0, sizeof(P));
  double g[3] = {0, -9.81, 0};
  if (o.set & CLAY_FLUID_GRAVITY)
    for (int k = 0; k < 3; k++) g[k] = o.gravity[k];
  for (int k = 0; k < 3; k++) P.gravity[k] = static_cast<float>(g[k]);
  P.dt = static_cast<float>(1.0 / 60 / f->substeps);
  P.emit_radius = static_cast<float>(f->spacing);
  P.max_speed = static_cast<float>((o.set & CLAY_FLUID_MAX_SPEED) ? o.max_speed : 15);
  P.stiffness = static_cast<float>((o.set & CLAY_FLUID_STIFFNESS) ? o.stiffness : 220);
  P.viscosity = static_cast<float>((o.set & CLAY_FLUID_VISCOSITY) ? o.viscosity : 0.4);
  P.damping = static_cast<float>((o.set & CLAY_FLUID_DAMPING) ? o.damping : 0.995);
  P.emit_seed = 1;
  P.contact_depth = static_cast<float>(f->radius * 1.5);
  // Scan parts: enough blocks that one part covers at most ~32k cells of a full box.
  int64_t cells = static_cast<int64_t>(f->G) * f->G * f->G;
  f->parts_scan = static_cast<uint32_t>(std::min<int64_t>(kMaxParts, std::max<int64_t>(1, std::min(cells, f->capacity * 4) / 32768)));
  const int64_t C = f->capacity;
  if ((rc = f->alloc(&f->parts, C)) || (rc = f->alloc(&f->prm, 1)) || (rc = f->alloc(&f->contacts, 1)) ||
      (rc = f->alloc(&f->gs, 1)) || (rc = f->alloc(&f->hs.key, C)) || (rc = f->alloc(&f->hs.rank, C)) ||
      (rc = f->alloc(&f->hs.tmp, C)) || (rc = f->alloc(&f->hs.sorted_id, C)) || (rc = f->alloc(&f->hs.spos, C)) ||
      (rc = f->alloc(&f->hs.svel, C)) || (rc = f->alloc(&f->hs.sdp, C)) || (rc = f->alloc(&f->hs.spx, C)) ||
      (rc = f->alloc(&f->hs.nbr, C * (kMaxNbr / 4))) ||
      (rc = f->alloc(&f->hs.counts, cells + 1)) || (rc = f->alloc(&f->hs.cell_start, cells + 2)) ||
      (rc = f->alloc(&f->d_scene, 1))) {
    clay_fluid_destroy(f);
    return rc;
  }
  f->hs.parts = f->parts;
  f->hs.prm = f->prm;
  f->hs.contacts = f->contacts;
  f->hs.gs = f->gs;
  CK(cudaMemset(f->parts, 0, sizeof(ParticleDev) * C));
  CK(cudaMemset(f->contacts, 0, sizeof(ContactsDev)));
  CK(cudaMemset(f->hs.counts, 0, sizeof(uint32_t) * (cells + 1)));
  CK(cudaMemset(f->hs.cell_start, 0, sizeof(uint32_t) * (cells + 2)));
  {
    GridState gsh;
    std::memset(&gsh, 0, sizeof(gsh));
    for (int k = 0; k < 3; k++) {
      gsh.lo[k] = 0xffffffffu;
      gsh.hi_inv[k] = 0xffffffffu;
    }
    CK(cudaMemcpy(f->gs, &gsh, sizeof(gsh), cudaMemcpyHostToDevice));
    std::vector<uint32_t> ident(static_cast<size_t>(C));
    for (int64_t i = 0; i < C; i++) ident[i] = static_cast<uint32_t>(i);
    CK(cudaMemcpy(f->hs.sorted_id, ident.data(), sizeof(uint32_t) * C, cudaMemcpyHostToDevice));
  }
  fill_scene(f);
  CK(cudaMemcpy(f->d_scene, &f->hs, sizeof(SceneDev), cudaMemcpyHostToDevice));
  ParamsDev pd;
  std::memcpy(&pd, &f->frozen, sizeof(pd));
  CK(cudaMemcpy(f->prm, &pd, sizeof(pd), cudaMemcpyHostToDevice));
  // The surface (fluid.ts:215-234): live = i < params.count, position = particles[i].pos.
  clay_cloud_desc cd{};
  cd.capacity = static_cast<uint32_t>(C);
  cd.positions = f->parts;
  cd.position_stride = sizeof(ParticleDev);
  cd.live_mode = CLAY_LIVE_COUNT;
  cd.live_count = &f->prm->count;
  clay_splat_opts so{};
  so.set = CLAY_SPLAT_MATERIAL | CLAY_SPLAT_RESOLUTION | CLAY_SPLAT_MIP_LEVELS | CLAY_SPLAT_BAND | CLAY_SPLAT_ORIGIN |
           CLAY_SPLAT_WORLD_SIZE;
  so.radius = f->surf_r;
  so.material = f->material;
  so.resolution = f->bake_res;
  so.mip_levels = f->bake_mips;
  so.band = f->band;
  so.world_size = f->world_size;
  for (int k = 0; k < 3; k++) so.origin[k] = f->origin[k];
  rc = make_splat(ctx, &cd, &so, true, &f->surface);
  if (rc) {
    clay_fluid_destroy(f);
    return rc;
  }
  f->surface->order = f->hs.sorted_id;
  f->surface->desc_dirty = true;
  rc = f->surface->flush(nullptr);
  if (rc) {
    clay_fluid_destroy(f);
    return rc;
  }
  CK(cudaDeviceSynchronize());
  *out = f;
  return CLAY_OK;
}

void clay_fluid_destroy(clay_fluid* f) {
  if (!f) return;
  for (auto& b : f->bufs) f->ctx->dev_free(b.p, b.n);
  free_splat(f->surface);
  delete f;
}

int clay_fluid_set_mode(clay_fluid* f, int mode) {
  if (!f) return fail(CLAY_EINVAL, "clay_fluid_set_mode: NULL sim");
  if (mode != CLAY_MODE_FAST && mode != CLAY_MODE_REFERENCE) return fail(CLAY_EINVAL, "unknown mode %d", mode);
  f->mode = mode;
  return CLAY_OK;
}

int clay_fluid_spawn(clay_fluid* f, int64_t n, const double pos[3], const double vel[3], const double* spread) {
  if (!f || !pos || !vel) return fail(CLAY_EINVAL, "clay_fluid_spawn: NULL argument");
  // fluid.ts:511-525
  double sp = spread ? *spread : f->spacing * std::cbrt(static_cast<double>(std::max<int64_t>(n, 1))) * 0.62;
  f->pending = std::max<int64_t>(0, std::min(n, f->capacity));
  for (int k = 0; k < 3; k++) {
    f->frozen.emit_pos[k] = static_cast<float>(pos[k]);
    f->frozen.emit_vel[k] = static_cast<float>(vel[k]);
  }
  f->frozen.emit_radius = static_cast<float>(sp);
  f->frozen.emit_seed = f->seed++;
  return CLAY_OK;
}

int clay_fluid_configure(clay_fluid* f, const clay_fluid_params* p, uint32_t mask) {
  if (!f || !p) return fail(CLAY_EINVAL, "clay_fluid_configure: NULL argument");
  clay_fluid_params& q = f->frozen;
  if (mask & CLAY_P_GRAVITY) std::memcpy(q.gravity, p->gravity, sizeof(q.gravity));
  if (mask & CLAY_P_DT) q.dt = p->dt;
  if (mask & CLAY_P_EMIT_POS) std::memcpy(q.emit_pos, p->emit_pos, sizeof(q.emit_pos));
  if (mask & CLAY_P_EMIT_RADIUS) q.emit_radius = p->emit_radius;
  if (mask & CLAY_P_EMIT_VEL) std::memcpy(q.emit_vel, p->emit_vel, sizeof(q.emit_vel));
  if (mask & CLAY_P_MAX_SPEED) q.max_speed = p->max_speed;
  if (mask & CLAY_P_STIFFNESS) q.stiffness = p->stiffness;
  if (mask & CLAY_P_VISCOSITY) q.viscosity = p->viscosity;
  if (mask & CLAY_P_DAMPING) q.damping = p->damping;
  if (mask & CLAY_P_CONTACT_DEPTH) q.contact_depth = p->contact_depth;
  return CLAY_OK;
}

namespace {
// Host bookkeeping of fluid.ts:537-545: the uniform this frame writes.
clay_fluid_params fluid_frame_params(clay_fluid* f) {
  int64_t ec = f->pending;
  f->pending = 0;
  int64_t base = f->cursor;
  if (ec > 0) {
    f->cursor = (base + ec) % f->capacity;
    f->live = std::min(f->capacity, std::max(f->live, base + ec));
  }
  clay_fluid_params p = f->frozen;
  p.count = static_cast<uint32_t>(f->live);
  p.emit_base = static_cast<uint32_t>(base);
  p.emit_count = static_cast<uint32_t>(ec);
  return p;
}

// The bookkeeping, then the uniform upload if it differs from the last one written.
int fluid_begin_frame(clay_fluid* f, cudaStream_t s, uint32_t* emit_count) {
  clay_fluid_params p = fluid_frame_params(f);
  const uint32_t ec = p.emit_count;
  if (!f->written_valid || std::memcmp(&p, &f->written, sizeof(p)) != 0) {
    int rc = f->ctx->upload(f->prm, &p, sizeof(p), s);
    if (rc) return rc;
    f->written = p;
    f->written_valid = true;
  }
  *emit_count = static_cast<uint32_t>(ec);
  if (f->world) {
    int rc = const_cast<clay_field*>(f->world)->flush(s);
    if (rc) return rc;
  }
  return CLAY_OK;
}

int fluid_substep_plain(clay_fluid* f, cudaStream_t s, int sub) {
  const SceneDev* d = f->d_scene;
  const int T = kBlock;
  int pb = static_cast<int>((f->live + T - 1) / T);
  CK(L_cell_key(d, nullptr, pb, T, sub, s));
  CK(L_cell_count(d, nullptr, pb, T, sub, s));
  CK(L_scan_partial(d, nullptr, static_cast<int>(f->parts_scan), sub, s));
  CK(L_scan_final(d, nullptr, static_cast<int>(f->parts_scan), sub, s));
  CK(L_cell_scatter(d, nullptr, pb, T, sub, s));
  CK(L_cell_order(d, nullptr, pb, T, sub, s));
  if (f->mode == CLAY_MODE_REFERENCE) {
    CK(L_density_ref(d, nullptr, pb, T, sub, s));
    CK(L_forces_ref(d, nullptr, pb, T, sub, s));
  } else {
    CK(L_density_fast(d, nullptr, pb, T, sub, s));
    CK(L_forces_fast(d, nullptr, pb, T, sub, s));
  }
  return CLAY_OK;
}
}  // namespace

int clay_fluid_step(clay_fluid* f, void* stream) {
  if (!f) return fail(CLAY_EINVAL, "clay_fluid_step: NULL sim");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint32_t ec = 0;
  int rc = fluid_begin_frame(f, s, &ec);
  if (rc) return rc;
  if (ec > 0) CK(L_emit(f->d_scene, nullptr, static_cast<int>((ec + kBlock - 1) / kBlock), kBlock, s));
  // fluid.ts:550: the substep loop is skipped entirely when nothing is alive.
  for (int sub = 0; sub < f->substeps && f->live > 0; sub++) {
    rc = fluid_substep_plain(f, s, sub);
    if (rc) return rc;
  }
  bool ordered = f->substeps > 0 && f->live > 0;
  return splat_bake(f->surface, s, ordered, ordered ? f->live : f->capacity);
}

int64_t clay_fluid_particle_count(const clay_fluid* f) { return f ? f->live : -1; }

int clay_fluid_get_params(const clay_fluid* f, clay_fluid_params* out) {
  if (!f || !out) return fail(CLAY_EINVAL, "clay_fluid_get_params: NULL argument");
  *out = f->frozen;
  out->count = static_cast<uint32_t>(f->live);
  return CLAY_OK;
}

int clay_fluid_read_contacts_async(clay_fluid* f, clay_contact_list* host, void* stream) {
  if (!f || !host) return fail(CLAY_EINVAL, "clay_fluid_read_contacts_async: NULL argument");
  static_assert(sizeof(clay_contact_list) == sizeof(ContactsDev), "ContactList layout");
  CK(cudaMemcpyAsync(host, f->contacts, sizeof(ContactsDev), cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
  return CLAY_OK;
}

int clay_fluid_particles_device(clay_fluid* f, clay_fluid_particle** ptr, uint32_t* stride) {
  if (!f) return fail(CLAY_EINVAL, "clay_fluid_particles_device: NULL sim");
  static_assert(sizeof(clay_fluid_particle) == sizeof(ParticleDev), "FluidParticle layout");
  if (ptr) *ptr = reinterpret_cast<clay_fluid_particle*>(f->parts);
  if (stride) *stride = sizeof(ParticleDev);
  return CLAY_OK;
}

int clay_fluid_upload(clay_fluid* f, const clay_fluid_particle* host, int64_t count, void* stream) {
  if (!f || (count > 0 && !host)) return fail(CLAY_EINVAL, "clay_fluid_upload: NULL argument");
  if (count < 0 || count > f->capacity)
    return fail(CLAY_EINVAL, "clay_fluid_upload: count %lld outside 0..capacity %lld", static_cast<long long>(count),
                static_cast<long long>(f->capacity));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (count > 0) CK(cudaMemcpyAsync(f->parts, host, sizeof(ParticleDev) * count, cudaMemcpyHostToDevice, s));
  f->live = count;
  f->cursor = count % f->capacity;
  f->pending = 0;
  return CLAY_OK;
}

int clay_fluid_download(const clay_fluid* f, clay_fluid_particle* host, int64_t count, void* stream) {
  if (!f || (count > 0 && !host)) return fail(CLAY_EINVAL, "clay_fluid_download: NULL argument");
  if (count < 0 || count > f->capacity) return fail(CLAY_EINVAL, "clay_fluid_download: count out of range");
  if (count > 0)
    CK(cudaMemcpyAsync(host, f->parts, sizeof(ParticleDev) * count, cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
  return CLAY_OK;
}

// The sim's own uniform with its current live count, for the hooks that launch on the sim's
// own scene record: a batch steps the sim through the batch's copy of the uniform, so the
// sim's own may hold an older count.
static int fluid_sync_count(clay_fluid* f, cudaStream_t s) {
  clay_fluid_params p = f->frozen;
  p.count = static_cast<uint32_t>(f->live);
  p.emit_base = static_cast<uint32_t>(f->cursor);
  p.emit_count = 0;
  if (!f->written_valid || std::memcmp(&p, &f->written, sizeof(p)) != 0) {
    int rc = f->ctx->upload(f->prm, &p, sizeof(p), s);
    if (rc) return rc;
    f->written = p;
    f->written_valid = true;
  }
  return CLAY_OK;
}

int clay_fluid_cell_indices(clay_fluid* f, uint32_t* host, void* stream) {
  if (!f || !host) return fail(CLAY_EINVAL, "clay_fluid_cell_indices: NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (f->live == 0) return CLAY_OK;
  TempDev<uint32_t> d;
  CK(d.alloc(static_cast<size_t>(f->live)));
  int rc = fluid_sync_count(f, s);
  if (rc) return rc;
  CK(L_cell_index(f->d_scene, d.p, static_cast<int>(f->live), s));
  CK(cudaMemcpyAsync(host, d.p, sizeof(uint32_t) * f->live, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return CLAY_OK;
}

namespace {
// The bake pairs of one splat over every level, added to *d_out (device) on stream s.
int census_splat(clay_splat* sp, unsigned long long* d_out, cudaStream_t s) {
  int rc = sp->flush(s);
  if (rc) return rc;
  const uint32_t cap = sp->cloud.capacity;
  if (cap == 0) return CLAY_OK;
  CK(L_census_splat(sp->d, static_cast<int>((cap + 255) / 256), sp->mips, d_out, s));
  return CLAY_OK;
}
}  // namespace

int clay_fluid_census(clay_fluid* f, void* stream, clay_census* out) {
  if (!f || !out) return fail(CLAY_EINVAL, "clay_fluid_census: NULL argument");
  std::memset(out, 0, sizeof(*out));
  out->particles = static_cast<uint64_t>(f->live);
  if (f->live == 0) return CLAY_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = fluid_sync_count(f, s);
  if (rc) return rc;
  TempDev<unsigned long long> d;
  CK(d.alloc(3));
  CK(cudaMemsetAsync(d.p, 0, 3 * sizeof(unsigned long long), s));
  CK(L_census_nbr(f->d_scene, static_cast<int>(f->live), d.p, s));
  rc = census_splat(f->surface, d.p + 2, s);
  if (rc) return rc;
  unsigned long long h[3] = {0, 0, 0};
  CK(cudaMemcpyAsync(h, d.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  out->candidates = h[0];
  out->accepted = h[1];
  out->splat_pairs = h[2];
  return CLAY_OK;
}

int clay_splat_census(clay_splat* sp, void* stream, uint64_t* pairs_out) {
  if (!sp || !pairs_out) return fail(CLAY_EINVAL, "clay_splat_census: NULL argument");
  *pairs_out = 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  TempDev<unsigned long long> d;
  CK(d.alloc(1));
  CK(cudaMemsetAsync(d.p, 0, sizeof(unsigned long long), s));
  int rc = census_splat(sp, d.p, s);
  if (rc) return rc;
  unsigned long long h = 0;
  CK(cudaMemcpyAsync(&h, d.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *pairs_out = h;
  return CLAY_OK;
}

clay_splat* clay_fluid_surface(clay_fluid* f) { return f ? f->surface : nullptr; }
clay_field* clay_fluid_field(clay_fluid* f) { return f ? f->surface->field : nullptr; }

int clay_fluid_get_info(const clay_fluid* f, clay_fluid_info* out) {
  if (!f || !out) return fail(CLAY_EINVAL, "clay_fluid_get_info: NULL argument");
  std::memset(out, 0, sizeof(*out));
  out->capacity = f->capacity;
  out->substeps = f->substeps;
  out->bucket = f->bucket;
  out->grid_res = f->G;
  out->smoothing = f->h;
  out->rest_density = f->rest;
  for (int k = 0; k < 3; k++) out->grid_origin[k] = f->gorig[k];
  out->spacing = f->spacing;
  out->radius = f->radius;
  out->device_bytes = f->own_bytes;
  return CLAY_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Batched stepping.
struct clay_batch {
  clay_ctx* ctx = nullptr;
  std::vector<clay_fluid*> sims;
  std::vector<clay_splat*> extra;
  int mode = CLAY_MODE_FAST;
  int max_substeps = 0;
  clay_batch_tuning tune{kBlock, kSplatThreads, 1};
  // device tables
  SceneDev* d_scenes = nullptr;
  size_t n_scenes_alloc = 0;
  SplatDev* d_extra = nullptr;   // extra clouds, index order
  SplatDev* d_surf = nullptr;    // fluid surfaces, cell order
  Work *w_part = nullptr, *w_emit = nullptr, *w_scan = nullptr, *w_xsplat = nullptr, *w_xres = nullptr,
       *w_ssplat = nullptr, *w_sres = nullptr;
  int n_part = 0, n_emit = 0, n_scan = 0, n_xsplat = 0, n_xres = 0, n_ssplat = 0, n_sres = 0;
  std::vector<DevBuf> bufs;
  bool built = false;
  cudaGraphExec_t graph = nullptr;
  // Per scene-size bucket thread-block size of the particle passes: a scene whose capacity is
  // below bucket_upper[i] uses bucket_block[i]; others use tune.sph_block. One launch per
  // distinct block size per pass.
  std::vector<int64_t> bucket_upper;
  std::vector<int> bucket_block;
  // Per bucket (bucket_upper.size() + 1 entries once set, the last for the larger scenes):
  // the density variant and the splat's strategy thresholds of the scenes in it.
  std::vector<clay_bucket_tuning> bucket_tune;
  struct PartGroup {
    Work* w;
    int n;
    int T;
    int density_variant;
    bool forces_split;
  };
  std::vector<PartGroup> groups;
  // The scenes split into lanes, each stepped as its own chain of launches on its own stream
  // (forked from the frame's stream, joined at its end): the lanes' kernels run side by side,
  // so one lane's latency-bound passes overlap another's issue-bound ones and each pass's tail.
  struct Lane {
    std::vector<PartGroup> groups;
    Work *w_emit = nullptr, *w_scan = nullptr, *w_ssplat = nullptr, *w_sres = nullptr;
    int n_part = 0, n_emit = 0, n_scan = 0, n_ssplat = 0, n_sres = 0;
    cudaStream_t stream = nullptr;  // lane 0 runs on the frame's stream
    cudaEvent_t done = nullptr;
  };
  std::vector<Lane> lanes;
  int n_lanes = 1;
  int bucket_of(int64_t capacity) const {
    for (size_t i = 0; i < bucket_upper.size(); i++)
      if (capacity < bucket_upper[i]) return static_cast<int>(i);
    return static_cast<int>(bucket_upper.size());
  }
  int block_of(int64_t capacity) const {
    const size_t i = static_cast<size_t>(bucket_of(capacity));
    return i < bucket_block.size() ? bucket_block[i] : tune.sph_block;
  }
  clay_bucket_tuning tuning_of(int64_t capacity) const {
    const size_t i = static_cast<size_t>(bucket_of(capacity));
    if (i < bucket_tune.size()) return bucket_tune[i];
    clay_bucket_tuning t{};
    t.sph_block = block_of(capacity);
    t.density_variant = kDensityVariant;
    t.forces_split = 0;
    t.splat_tile_ratio = static_cast<int32_t>(kSplatTileRatio);
    t.splat_walk_weight = static_cast<int32_t>(kSplatWalkWeight);
    return t;
  }
  int64_t launches_per_step = 0;
  // The scenes' FluidParams, contiguous, written from pinned memory in one copy per frame
  // (double-buffered so the host never overwrites a copy still in flight).
  ParamsDev* d_params = nullptr;
  ParamsDev* h_params[2] = {nullptr, nullptr};
  cudaEvent_t params_ev[2] = {nullptr, nullptr};
  bool params_used[2] = {false, false};
  int params_slot = 0;
  ContactsDev* d_contacts = nullptr;
  // Subset stepping (continuous batching): per-frame work tables built on the host for the
  // scenes of that frame, double-buffered in pinned memory, one upload per frame.
  std::vector<ParamsDev> all_params;
  Work* h_sub[2] = {nullptr, nullptr};
  size_t h_sub_cap[2] = {0, 0};
  cudaEvent_t sub_ev[2] = {nullptr, nullptr};
  bool sub_used[2] = {false, false};
  int sub_slot = 0;
  Work* d_sub = nullptr;
  size_t d_sub_cap = 0;

  // A second stream for the extra clouds' bake, forked from the frame's stream and joined
  // before the first forces pass (the first reader of the bodies' volumes): the bodies bake
  // while the fluids build their cells and densities.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  ~clay_batch() {
    release();
    if (side) cudaStreamDestroy(side);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    for (auto& l : lanes) {
      if (l.stream) cudaStreamDestroy(l.stream);
      if (l.done) cudaEventDestroy(l.done);
    }
    for (int k = 0; k < 2; k++) {
      if (h_params[k]) cudaFreeHost(h_params[k]);
      if (params_ev[k]) cudaEventDestroy(params_ev[k]);
      if (h_sub[k]) cudaFreeHost(h_sub[k]);
      if (sub_ev[k]) cudaEventDestroy(sub_ev[k]);
    }
    if (d_sub) ctx->dev_free(d_sub, d_sub_cap * sizeof(Work));
  }
  void release() {
    if (graph) {
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    for (int k = 0; k < 2; k++) {
      if (h_params[k]) cudaFreeHost(h_params[k]);
      h_params[k] = nullptr;
      params_used[k] = false;
    }
    for (auto& b : bufs) ctx->dev_free(b.p, b.n);
    bufs.clear();
    built = false;
  }
  template <class T>
  int upload_table(T** d, const std::vector<T>& h) {
    void* p = nullptr;
    int rc = ctx->dev_alloc(&p, sizeof(T) * std::max<size_t>(h.size(), 1));
    if (rc) return rc;
    bufs.push_back({p, sizeof(T) * std::max<size_t>(h.size(), 1)});
    if (!h.empty()) CK(cudaMemcpy(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    *d = static_cast<T*>(p);
    return CLAY_OK;
  }
};

namespace {

void add_splat_work(std::vector<Work>& ws, std::vector<Work>& wr, uint32_t obj, const clay_splat* s, int64_t iter_n,
                    int splat_block) {
  for (int m = 0; m < s->mips; m++)
    for (int64_t f = 0; f < iter_n; f += splat_block)
      ws.push_back({obj, static_cast<uint32_t>(m), static_cast<uint32_t>(f),
                    static_cast<uint32_t>(std::min<int64_t>(splat_block, iter_n - f))});
  int64_t quads = (s->vol->total + 3) / 4;
  for (int64_t q = 0; q < quads; q += kResolveThreads) wr.push_back({obj, 0u, static_cast<uint32_t>(q), kResolveThreads});
}

// Work tables sized by capacity: blocks past a scene's live count exit at once, so the
// tables (and a captured graph) stay valid while the live counts grow.
int batch_build(clay_batch* b) {
  b->release();
  const int T = b->tune.sph_block;
  std::vector<SceneDev> scenes;
  std::vector<Work> wp, we, wsc;
  b->max_substeps = 0;
  // one group of particle-pass launches per distinct (block size, density variant)
  std::vector<std::tuple<int, int, int>> blocks;
  std::vector<std::vector<Work>> by_block;
  for (size_t i = 0; i < b->sims.size(); i++) {
    clay_fluid* f = b->sims[i];
    scenes.push_back(f->hs);
    b->max_substeps = std::max(b->max_substeps, f->substeps);
    uint32_t obj = static_cast<uint32_t>(i);
    const clay_bucket_tuning bt = b->tuning_of(f->capacity);
    const int Ts = bt.sph_block;
    const std::tuple<int, int, int> key(Ts, bt.density_variant, bt.forces_split != 0 ? 1 : 0);
    size_t gi = std::find(blocks.begin(), blocks.end(), key) - blocks.begin();
    if (gi == blocks.size()) {
      blocks.push_back(key);
      by_block.emplace_back();
    }
    for (int64_t x = 0; x < f->capacity; x += Ts) {
      Work wk{obj, 0u, static_cast<uint32_t>(x), static_cast<uint32_t>(std::min<int64_t>(Ts, f->capacity - x))};
      wp.push_back(wk);
      by_block[gi].push_back(wk);
    }
    int eb = static_cast<int>(std::min<int64_t>(8, (f->capacity + T - 1) / T));
    for (int e = 0; e < eb; e++) we.push_back({obj, 0u, static_cast<uint32_t>(e * T), static_cast<uint32_t>(eb * T)});
    for (uint32_t p = 0; p < f->parts_scan; p++) wsc.push_back({obj, p, 0u, 0u});
  }
  std::vector<SplatDev> xs, ss;
  std::vector<Work> wxs, wxr, wss, wsr;
  for (size_t i = 0; i < b->extra.size(); i++) {
    xs.push_back(b->extra[i]->h);
    xs.back().order = nullptr;
    add_splat_work(wxs, wxr, static_cast<uint32_t>(i), b->extra[i], b->extra[i]->cloud.capacity, kSplatThreads);
  }
  for (size_t i = 0; i < b->sims.size(); i++) {
    clay_splat* s = b->sims[i]->surface;
    SplatDev d = s->h;
    d.order = s->order;
    const clay_bucket_tuning bt = b->tuning_of(b->sims[i]->capacity);
    d.tile_ratio = static_cast<uint32_t>(bt.splat_tile_ratio);
    d.walk_weight = static_cast<uint32_t>(bt.splat_walk_weight);
    ss.push_back(d);
    add_splat_work(wss, wsr, static_cast<uint32_t>(i), s, b->sims[i]->capacity, kSplatThreads);
  }
  int rc;
  {
    std::vector<ParamsDev> prm(b->sims.size());
    for (size_t i = 0; i < b->sims.size(); i++) std::memcpy(&prm[i], &b->sims[i]->frozen, sizeof(ParamsDev));
    if ((rc = b->upload_table(&b->d_params, prm))) return rc;
    std::vector<ContactsDev> ct(b->sims.size());
    if ((rc = b->upload_table(&b->d_contacts, ct))) return rc;
    for (size_t i = 0; i < b->sims.size(); i++) {
      scenes[i].prm = b->d_params + i;
      ss[i].live_count = &b->d_params[i].count;
    }
    for (int k = 0; k < 2; k++) {
      CK(cudaMallocHost(&b->h_params[k], sizeof(ParamsDev) * std::max<size_t>(b->sims.size(), 1)));
      if (!b->params_ev[k]) CK(cudaEventCreateWithFlags(&b->params_ev[k], cudaEventDisableTiming));
    }
  }
  if ((rc = b->upload_table(&b->d_scenes, scenes)) || (rc = b->upload_table(&b->w_part, wp)) ||
      (rc = b->upload_table(&b->w_emit, we)) || (rc = b->upload_table(&b->w_scan, wsc)) ||
      (rc = b->upload_table(&b->d_extra, xs)) || (rc = b->upload_table(&b->d_surf, ss)) ||
      (rc = b->upload_table(&b->w_xsplat, wxs)) || (rc = b->upload_table(&b->w_xres, wxr)) ||
      (rc = b->upload_table(&b->w_ssplat, wss)) || (rc = b->upload_table(&b->w_sres, wsr)))
    return rc;
  b->n_part = static_cast<int>(wp.size());
  b->groups.clear();
  for (size_t g = 0; g < blocks.size(); g++) {
    Work* w = nullptr;
    if ((rc = b->upload_table(&w, by_block[g]))) return rc;
    b->groups.push_back({w, static_cast<int>(by_block[g].size()), std::get<0>(blocks[g]), std::get<1>(blocks[g]),
                         std::get<2>(blocks[g]) != 0});
  }
  // lanes: scenes dealt largest first to the lane with the fewest particles so far
  {
    const int nl = std::max(1, std::min(b->n_lanes, static_cast<int>(std::max<size_t>(b->sims.size(), 1))));
    std::vector<int> lane_of(b->sims.size(), 0);
    std::vector<int64_t> load(static_cast<size_t>(nl), 0);
    std::vector<size_t> by_size(b->sims.size());
    for (size_t i = 0; i < by_size.size(); i++) by_size[i] = i;
    std::stable_sort(by_size.begin(), by_size.end(),
                     [&](size_t x, size_t y) { return b->sims[x]->capacity > b->sims[y]->capacity; });
    for (size_t i : by_size) {
      const int l = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
      lane_of[i] = l;
      load[static_cast<size_t>(l)] += b->sims[i]->capacity;
    }
    const size_t old_lanes = b->lanes.size();
    for (size_t l = static_cast<size_t>(nl); l < old_lanes; l++) {
      if (b->lanes[l].stream) cudaStreamDestroy(b->lanes[l].stream);
      if (b->lanes[l].done) cudaEventDestroy(b->lanes[l].done);
    }
    b->lanes.resize(static_cast<size_t>(nl));
    for (size_t l = old_lanes; l < b->lanes.size(); l++) b->lanes[l] = clay_batch::Lane{};
    for (int l = 0; l < nl; l++) {
      clay_batch::Lane& ln = b->lanes[static_cast<size_t>(l)];
      auto mine = [&](const std::vector<Work>& all) {
        std::vector<Work> out;
        for (const Work& w : all)
          if (lane_of[w.obj] == l) out.push_back(w);
        return out;
      };
      ln.groups.clear();
      ln.n_part = 0;
      for (size_t g = 0; g < blocks.size(); g++) {
        std::vector<Work> wl = mine(by_block[g]);
        if (wl.empty()) continue;
        Work* w = nullptr;
        if ((rc = b->upload_table(&w, wl))) return rc;
        ln.groups.push_back({w, static_cast<int>(wl.size()), std::get<0>(blocks[g]), std::get<1>(blocks[g]),
                             std::get<2>(blocks[g]) != 0});
        ln.n_part += static_cast<int>(wl.size());
      }
      const std::vector<Work> le = mine(we), lsc = mine(wsc), lss = mine(wss), lsr = mine(wsr);
      if ((rc = b->upload_table(&ln.w_emit, le)) || (rc = b->upload_table(&ln.w_scan, lsc)) ||
          (rc = b->upload_table(&ln.w_ssplat, lss)) || (rc = b->upload_table(&ln.w_sres, lsr)))
        return rc;
      ln.n_emit = static_cast<int>(le.size());
      ln.n_scan = static_cast<int>(lsc.size());
      ln.n_ssplat = static_cast<int>(lss.size());
      ln.n_sres = static_cast<int>(lsr.size());
      if (l > 0 && !ln.stream) CK(cudaStreamCreateWithFlags(&ln.stream, cudaStreamNonBlocking));
      if (l > 0 && !ln.done) CK(cudaEventCreateWithFlags(&ln.done, cudaEventDisableTiming));
    }
  }
  b->n_emit = static_cast<int>(we.size());
  b->n_scan = static_cast<int>(wsc.size());
  b->n_xsplat = static_cast<int>(wxs.size());
  b->n_xres = static_cast<int>(wxr.size());
  b->n_ssplat = static_cast<int>(wss.size());
  b->n_sres = static_cast<int>(wsr.size());
  if (!b->side) CK(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking));
  if (!b->ev_fork) CK(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
  if (!b->ev_join) CK(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
  b->built = true;
  return CLAY_OK;
}

// The passes of one batched frame. Order as in a game frame: the extra clouds (clay-body
// shells, which the fluids collide with) bake first, then every fluid steps and bakes.
int batch_enqueue(clay_batch* b, cudaStream_t s) {
  const int T = b->tune.sph_block;
  const SceneDev* d = b->d_scenes;
  const bool multi = b->lanes.size() > 1;
  // the extra clouds' bake: on the side stream when there are fluids to overlap it with
  const bool fork = b->n_xsplat && b->n_part && b->max_substeps > 0;
  if (fork || multi) CK(cudaEventRecord(b->ev_fork, s));  // the stream and events exist from batch_build on
  if (fork) {
    CK(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
    CK(L_splat(b->d_extra, b->w_xsplat, b->n_xsplat, 1, kSplatAccVoxelsDiscs, b->side));
    if (b->n_xres) CK(L_resolve(b->d_extra, b->w_xres, b->n_xres, b->side));
    CK(cudaEventRecord(b->ev_join, b->side));
  } else {
    if (b->n_xsplat) CK(L_splat(b->d_extra, b->w_xsplat, b->n_xsplat, 1, kSplatAccVoxelsDiscs, s));
    if (b->n_xres) CK(L_resolve(b->d_extra, b->w_xres, b->n_xres, s));
  }
  for (size_t li = 0; li < b->lanes.size(); li++) {
    clay_batch::Lane& ln = b->lanes[li];
    cudaStream_t ls = li == 0 ? s : ln.stream;
    if (li > 0) CK(cudaStreamWaitEvent(ls, b->ev_fork, 0));
    bool joined = !fork;
    if (ln.n_part) {
      CK(L_emit(d, ln.w_emit, ln.n_emit, T, ls));
      for (int sub = 0; sub < b->max_substeps; sub++) {
        for (auto& g : ln.groups) CK(L_cell_key(d, g.w, g.n, g.T, sub, ls));
        for (auto& g : ln.groups) CK(L_cell_count(d, g.w, g.n, g.T, sub, ls));
        CK(L_scan_partial(d, ln.w_scan, ln.n_scan, sub, ls));
        CK(L_scan_final(d, ln.w_scan, ln.n_scan, sub, ls));
        for (auto& g : ln.groups) CK(L_cell_scatter(d, g.w, g.n, g.T, sub, ls));
        for (auto& g : ln.groups) CK(L_cell_order(d, g.w, g.n, g.T, sub, ls));
        for (auto& g : ln.groups) {
          if (b->mode == CLAY_MODE_REFERENCE) CK(L_density_ref(d, g.w, g.n, g.T, sub, ls, g.density_variant));
          else CK(L_density_fast(d, g.w, g.n, g.T, sub, ls, g.density_variant));
        }
        if (!joined) {  // the fluids collide with the bodies' volumes from here on
          CK(cudaStreamWaitEvent(ls, b->ev_join, 0));
          joined = true;
        }
        for (auto& g : ln.groups) {
          if (b->mode == CLAY_MODE_REFERENCE) CK(L_forces_ref(d, g.w, g.n, g.T, sub, ls, g.forces_split));
          else CK(L_forces_fast(d, g.w, g.n, g.T, sub, ls, g.forces_split));
        }
      }
    }
    if (!joined) CK(cudaStreamWaitEvent(ls, b->ev_join, 0));
    if (ln.n_ssplat) CK(L_splat(b->d_surf, ln.w_ssplat, ln.n_ssplat, 1, kSplatAccVoxels, ls));
    if (ln.n_sres) CK(L_resolve(b->d_surf, ln.w_sres, ln.n_sres, ls));
    if (li > 0) CK(cudaEventRecord(ln.done, ls));
  }
  for (size_t li = 1; li < b->lanes.size(); li++) CK(cudaStreamWaitEvent(s, b->lanes[li].done, 0));
  return CLAY_OK;
}

}  // namespace

extern "C" {

int clay_batch_create(clay_ctx* ctx, clay_fluid* const* sims, int n, clay_batch** out) {
  if (!ctx || !out || n < 0 || (n > 0 && !sims)) return fail(CLAY_EINVAL, "clay_batch_create: bad argument");
  clay_batch* b = new clay_batch();
  b->ctx = ctx;
  for (int i = 0; i < n; i++) {
    if (!sims[i] || sims[i]->ctx != ctx) {
      delete b;
      return fail(CLAY_EINVAL, "clay_batch_create: scene %d is NULL or from another context", i);
    }
    b->sims.push_back(sims[i]);
  }
  if (n > 0) {
    b->mode = sims[0]->mode;
    for (int i = 1; i < n; i++)
      if (sims[i]->mode != b->mode) {
        delete b;
        return fail(CLAY_EINVAL, "clay_batch_create: every scene of a batch must use the same arithmetic mode");
      }
  }
  *out = b;
  return CLAY_OK;
}

void clay_batch_destroy(clay_batch* b) { delete b; }

int clay_batch_add_splat(clay_batch* b, clay_splat* s) {
  if (!b || !s) return fail(CLAY_EINVAL, "clay_batch_add_splat: NULL argument");
  b->extra.push_back(s);
  b->release();
  return CLAY_OK;
}

int clay_batch_set_tuning(clay_batch* b, const clay_batch_tuning* t) {
  if (!b || !t) return fail(CLAY_EINVAL, "clay_batch_set_tuning: NULL argument");
  if (t->sph_block < 64 || t->sph_block > 256 || (t->sph_block & 31))
    return fail(CLAY_EINVAL, "sph_block %d must be a multiple of 32 in 64..256", t->sph_block);
  b->tune = *t;
  b->tune.splat_block = kSplatThreads;
  b->release();
  return CLAY_OK;
}

int clay_batch_set_bucket_blocks(clay_batch* b, const int64_t* upper, const int32_t* blocks, int n) {
  if (!b || n < 0 || (n > 0 && (!upper || !blocks))) return fail(CLAY_EINVAL, "clay_batch_set_bucket_blocks: bad argument");
  for (int i = 0; i < n; i++) {
    if (blocks[i] < 64 || blocks[i] > 256 || (blocks[i] & 31))
      return fail(CLAY_EINVAL, "bucket block %d must be a multiple of 32 in 64..256", blocks[i]);
    if (i > 0 && upper[i] <= upper[i - 1]) return fail(CLAY_EINVAL, "bucket bounds must increase");
  }
  b->bucket_upper.assign(upper, upper + n);
  b->bucket_block.assign(blocks, blocks + n);
  b->bucket_tune.clear();
  b->release();
  return CLAY_OK;
}

int clay_batch_set_lanes(clay_batch* b, int lanes) {
  if (!b || lanes < 1 || lanes > 8) return fail(CLAY_EINVAL, "clay_batch_set_lanes: lanes must be in 1..8");
  b->n_lanes = lanes;
  b->release();
  return CLAY_OK;
}

int clay_batch_set_bucket_tuning(clay_batch* b, const int64_t* upper, const clay_bucket_tuning* t, int n) {
  if (!b || n < 0 || !t || (n > 0 && !upper)) return fail(CLAY_EINVAL, "clay_batch_set_bucket_tuning: bad argument");
  for (int i = 0; i <= n; i++) {
    if (t[i].sph_block < 64 || t[i].sph_block > 256 || (t[i].sph_block & 31))
      return fail(CLAY_EINVAL, "bucket block %d must be a multiple of 32 in 64..256", t[i].sph_block);
    if (t[i].density_variant < 0 || t[i].density_variant > 2)
      return fail(CLAY_EINVAL, "bucket density variant %d is not 0, 1 or 2", t[i].density_variant);
    if (t[i].splat_tile_ratio < 1 || t[i].splat_tile_ratio > 64 || t[i].splat_walk_weight < 1 || t[i].splat_walk_weight > 64)
      return fail(CLAY_EINVAL, "bucket splat thresholds must be in 1..64");
    if (i > 0 && i < n && upper[i] <= upper[i - 1]) return fail(CLAY_EINVAL, "bucket bounds must increase");
  }
  b->bucket_upper.assign(upper, upper + n);
  b->bucket_block.clear();
  for (int i = 0; i < n; i++) b->bucket_block.push_back(t[i].sph_block);
  b->bucket_tune.assign(t, t + n + 1);
  b->release();
  return CLAY_OK;
}

int clay_batch_get_tuning(const clay_batch* b, clay_batch_tuning* t) {
  if (!b || !t) return fail(CLAY_EINVAL, "clay_batch_get_tuning: NULL argument");
  *t = b->tune;
  return CLAY_OK;
}

int clay_batch_step(clay_batch* b, void* stream) {
  if (!b) return fail(CLAY_EINVAL, "clay_batch_step: NULL batch");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc;
  if (!b->built && (rc = batch_build(b))) return rc;
  {
    // this frame's uniforms of every scene (fluid.ts:545), one pinned copy
    int k = b->params_slot;
    b->params_slot ^= 1;
    if (b->params_used[k]) CK(cudaEventSynchronize(b->params_ev[k]));
    for (size_t i = 0; i < b->sims.size(); i++) {
      clay_fluid* f = b->sims[i];
      clay_fluid_params p = fluid_frame_params(f);
      std::memcpy(&b->h_params[k][i], &p, sizeof(ParamsDev));
      if (b->all_params.size() == b->sims.size()) std::memcpy(&b->all_params[i], &p, sizeof(ParamsDev));
      if (f->world && (rc = const_cast<clay_field*>(f->world)->flush(s))) return rc;
    }
    if (!b->sims.empty()) {
      CK(cudaMemcpyAsync(b->d_params, b->h_params[k], sizeof(ParamsDev) * b->sims.size(), cudaMemcpyHostToDevice, s));
      CK(cudaEventRecord(b->params_ev[k], s));
      b->params_used[k] = true;
    }
  }
  for (clay_splat* x : b->extra)
    if ((rc = x->flush(s))) return rc;
  for (clay_fluid* f : b->sims)
    if ((rc = f->surface->flush(s))) return rc;
  if (!b->tune.use_graph) {
    uint64_t before = launch_count();
    rc = batch_enqueue(b, s);
    b->launches_per_step = static_cast<int64_t>(launch_count() - before);
    return rc;
  }
  if (!b->graph) {
    // Capture on a private stream so the caller's stream can be the legacy default.
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    uint64_t before = launch_count();
    rc = batch_enqueue(b, cs);
    b->launches_per_step = static_cast<int64_t>(launch_count() - before);
    cudaError_t e = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(CLAY_ECUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CLAY_ECUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
  }
  CK(cudaGraphLaunch(b->graph, s));
  count_launches(static_cast<uint64_t>(b->launches_per_step));
  return CLAY_OK;
}

int clay_batch_launches_per_step(const clay_batch* b, int64_t* out) {
  if (!b || !out) return fail(CLAY_EINVAL, "clay_batch_launches_per_step: NULL argument");
  *out = b->launches_per_step;
  return CLAY_OK;
}

int clay_batch_profile(clay_batch* b, void* stream, clay_phase_time* out, int cap, int* n_out) {
  if (!b || !out || !n_out) return fail(CLAY_EINVAL, "clay_batch_profile: NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc;
  if (!b->built && (rc = batch_build(b))) return rc;
  // One frame without the graph, every launch bracketed by events on `stream`.
  struct Rec {
    const char* name;
    cudaEvent_t a, z;
  };
  std::vector<Rec> recs;
  // every event is created before the frame: creating them between launches would leave the
  // device idle between an event and its kernel, and the idle time would count as the kernel's
  struct EventPool {
    std::vector<cudaEvent_t> ev;
    ~EventPool() {
      for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    }
  } pool;
  pool.ev.assign(2 * 64 * static_cast<size_t>(std::max(1, b->max_substeps) + 1), nullptr);
  size_t next_ev = 0;
  for (auto& e : pool.ev) CK(cudaEventCreate(&e));
  auto timed = [&](const char* name, auto&& launch) -> int {
    if (next_ev + 2 > pool.ev.size()) return fail(CLAY_ESTATE, "clay_batch_profile: too many launches");
    Rec r{name, pool.ev[next_ev], pool.ev[next_ev + 1]};
    next_ev += 2;
    CK(cudaEventRecord(r.a, s));
    CK(launch());
    CK(cudaEventRecord(r.z, s));
    recs.push_back(r);
    return CLAY_OK;
  };
  {
    int k = b->params_slot;
    b->params_slot ^= 1;
    if (b->params_used[k]) CK(cudaEventSynchronize(b->params_ev[k]));
    for (size_t i = 0; i < b->sims.size(); i++) {
      clay_fluid_params p = fluid_frame_params(b->sims[i]);
      std::memcpy(&b->h_params[k][i], &p, sizeof(ParamsDev));
    }
    if (!b->sims.empty()) {
      CK(cudaMemcpyAsync(b->d_params, b->h_params[k], sizeof(ParamsDev) * b->sims.size(), cudaMemcpyHostToDevice, s));
      CK(cudaEventRecord(b->params_ev[k], s));
      b->params_used[k] = true;
    }
  }
  const int T = b->tune.sph_block;
  const SceneDev* d = b->d_scenes;
  const bool ref = b->mode == CLAY_MODE_REFERENCE;
  if (b->n_xsplat && (rc = timed("body_splat", [&] { return L_splat(b->d_extra, b->w_xsplat, b->n_xsplat, 1, kSplatAccVoxelsDiscs, s); }))) return rc;
  if (b->n_xres && (rc = timed("body_resolve", [&] { return L_resolve(b->d_extra, b->w_xres, b->n_xres, s); }))) return rc;
  if (b->n_part) {
    if ((rc = timed("emit", [&] { return L_emit(d, b->w_emit, b->n_emit, T, s); }))) return rc;
    for (int sub = 0; sub < b->max_substeps; sub++) {
      for (auto& g : b->groups)
        if ((rc = timed("cell_key", [&] { return L_cell_key(d, g.w, g.n, g.T, sub, s); }))) return rc;
      for (auto& g : b->groups)
        if ((rc = timed("cell_count", [&] { return L_cell_count(d, g.w, g.n, g.T, sub, s); }))) return rc;
      if ((rc = timed("scan_partial", [&] { return L_scan_partial(d, b->w_scan, b->n_scan, sub, s); }))) return rc;
      if ((rc = timed("scan_final", [&] { return L_scan_final(d, b->w_scan, b->n_scan, sub, s); }))) return rc;
      for (auto& g : b->groups)
        if ((rc = timed("cell_scatter", [&] { return L_cell_scatter(d, g.w, g.n, g.T, sub, s); }))) return rc;
      for (auto& g : b->groups)
        if ((rc = timed("cell_order", [&] { return L_cell_order(d, g.w, g.n, g.T, sub, s); }))) return rc;
      for (auto& g : b->groups)
        if ((rc = timed("density", [&] {
               return ref ? L_density_ref(d, g.w, g.n, g.T, sub, s, g.density_variant)
                          : L_density_fast(d, g.w, g.n, g.T, sub, s, g.density_variant);
             })))
          return rc;
      for (auto& g : b->groups)
        if ((rc = timed("forces_integrate", [&] {
               return ref ? L_forces_ref(d, g.w, g.n, g.T, sub, s, g.forces_split)
                          : L_forces_fast(d, g.w, g.n, g.T, sub, s, g.forces_split);
             })))
          return rc;
    }
  }
  if (b->n_ssplat && (rc = timed("splat", [&] { return L_splat(b->d_surf, b->w_ssplat, b->n_ssplat, 1, kSplatAccVoxels, s); }))) return rc;
  if (b->n_sres && (rc = timed("resolve", [&] { return L_resolve(b->d_surf, b->w_sres, b->n_sres, s); }))) return rc;
  CK(cudaStreamSynchronize(s));
  std::vector<clay_phase_time> agg;
  for (auto& r : recs) {
    float ms = 0;
    cudaEventElapsedTime(&ms, r.a, r.z);
    bool found = false;
    for (auto& a : agg)
      if (std::strcmp(a.name, r.name) == 0) {
        a.ms += ms;
        a.launches++;
        found = true;
      }
    if (!found) {
      clay_phase_time t{};
      std::snprintf(t.name, sizeof(t.name), "%s", r.name);
      t.ms = ms;
      t.launches = 1;
      agg.push_back(t);
    }
  }
  int n = std::min(cap, static_cast<int>(agg.size()));
  for (int i = 0; i < n; i++) out[i] = agg[i];
  *n_out = n;
  return CLAY_OK;
}

int clay_batch_read_contacts_async(clay_batch* b, clay_contact_list* host, void* stream) {
  if (!b || (!host && !b->sims.empty())) return fail(CLAY_EINVAL, "clay_batch_read_contacts_async: NULL argument");
  if (!b->built) return fail(CLAY_ESTATE, "clay_batch_read_contacts_async: the batch has not stepped yet");
  if (b->sims.empty()) return CLAY_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int n = static_cast<int>(b->sims.size());
  CK(L_gather_contacts(b->d_scenes, n, b->d_contacts, s));
  CK(cudaMemcpyAsync(host, b->d_contacts, sizeof(ContactsDev) * n, cudaMemcpyDeviceToHost, s));
  return CLAY_OK;
}

int clay_batch_step_subset(clay_batch* b, const int32_t* scenes, int n, void* stream) {
  if (!b || n < 0 || (n > 0 && !scenes)) return fail(CLAY_EINVAL, "clay_batch_step_subset: bad argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc;
  if (!b->built && (rc = batch_build(b))) return rc;
  const int ns = static_cast<int>(b->sims.size());
  if (b->all_params.size() != static_cast<size_t>(ns)) {
    b->all_params.resize(ns);
    for (int i = 0; i < ns; i++) std::memcpy(&b->all_params[i], &b->sims[i]->frozen, sizeof(ParamsDev));
    for (int i = 0; i < ns; i++) b->all_params[i].count = static_cast<uint32_t>(b->sims[i]->live);
  }
  std::vector<char> seen(ns, 0);
  for (int q = 0; q < n; q++) {
    int i = scenes[q];
    if (i < 0 || i >= ns) return fail(CLAY_EINVAL, "clay_batch_step_subset: scene %d outside 0..%d", i, ns - 1);
    if (seen[i]) return fail(CLAY_EINVAL, "clay_batch_step_subset: scene %d listed twice", i);
    seen[i] = 1;
  }
  if (n == 0) return CLAY_OK;
  // The frame's uniforms (fluid.ts:537-545) for the listed scenes; the others keep theirs.
  const int T = b->tune.sph_block;
  int max_sub = 0;
  for (int q = 0; q < n; q++) {
    clay_fluid* f = b->sims[scenes[q]];
    clay_fluid_params p = fluid_frame_params(f);
    std::memcpy(&b->all_params[scenes[q]], &p, sizeof(ParamsDev));
    if (f->world && (rc = const_cast<clay_field*>(f->world)->flush(s))) return rc;
    if ((rc = f->surface->flush(s))) return rc;
    if (f->live > 0) max_sub = std::max(max_sub, f->substeps);
  }
  // Work tables sized by the live counts (known on the host): no idle blocks.
  std::vector<Work> tab;
  auto mark = [&]() { return static_cast<int>(tab.size()); };
  const int o_emit = mark();
  for (int q = 0; q < n; q++) {
    const ParamsDev& p = b->all_params[scenes[q]];
    uint32_t ec = p.emit_count;
    if (ec == 0) continue;
    int eb = static_cast<int>(std::min<int64_t>(8, (ec + T - 1) / T));
    for (int e = 0; e < eb; e++)
      tab.push_back({static_cast<uint32_t>(scenes[q]), 0u, static_cast<uint32_t>(e * T), static_cast<uint32_t>(eb * T)});
  }
  const int n_emit = mark() - o_emit;
  const int o_part = mark();
  for (int q = 0; q < n; q++) {
    clay_fluid* f = b->sims[scenes[q]];
    for (int64_t x = 0; x < f->live; x += T)
      tab.push_back({static_cast<uint32_t>(scenes[q]), 0u, static_cast<uint32_t>(x), static_cast<uint32_t>(std::min<int64_t>(T, f->live - x))});
  }
  const int n_part = mark() - o_part;
  const int o_scan = mark();
  for (int q = 0; q < n; q++) {
    clay_fluid* f = b->sims[scenes[q]];
    if (f->live == 0) continue;
    for (uint32_t p = 0; p < f->parts_scan; p++) tab.push_back({static_cast<uint32_t>(scenes[q]), p, 0u, 0u});
  }
  const int n_scan = mark() - o_scan;
  const int o_splat = mark();
  for (int q = 0; q < n; q++) {
    clay_fluid* f = b->sims[scenes[q]];
    int64_t it = (f->substeps > 0 && f->live > 0) ? f->live : 0;
    for (int m = 0; m < f->surface->mips; m++)
      for (int64_t x = 0; x < it; x += kSplatThreads)
        tab.push_back({static_cast<uint32_t>(scenes[q]), static_cast<uint32_t>(m), static_cast<uint32_t>(x),
                       static_cast<uint32_t>(std::min<int64_t>(kSplatThreads, it - x))});
  }
  const int n_splat = mark() - o_splat;
  const int o_res = mark();
  for (int q = 0; q < n; q++) {
    int64_t quads = (b->sims[scenes[q]]->surface->vol->total + 3) / 4;
    for (int64_t x = 0; x < quads; x += kResolveThreads)
      tab.push_back({static_cast<uint32_t>(scenes[q]), 0u, static_cast<uint32_t>(x), kResolveThreads});
  }
  const int n_res = mark() - o_res;
  // upload params + tables through double-buffered pinned memory
  int k = b->sub_slot;
  b->sub_slot ^= 1;
  if (b->sub_used[k]) CK(cudaEventSynchronize(b->sub_ev[k]));
  if (!b->sub_ev[k]) CK(cudaEventCreateWithFlags(&b->sub_ev[k], cudaEventDisableTiming));
  const size_t need = tab.size() + (sizeof(ParamsDev) * ns + sizeof(Work) - 1) / sizeof(Work);
  if (b->h_sub_cap[k] < need) {
    if (b->h_sub[k]) cudaFreeHost(b->h_sub[k]);
    b->h_sub_cap[k] = need * 2;
    CK(cudaMallocHost(&b->h_sub[k], b->h_sub_cap[k] * sizeof(Work)));
  }
  if (b->d_sub_cap < tab.size()) {
    // the previous frame's kernels may still read the old table: order the free behind them
    if (b->d_sub) {
      CK(cudaStreamSynchronize(s));
      b->ctx->dev_free(b->d_sub, b->d_sub_cap * sizeof(Work));
    }
    b->d_sub_cap = tab.size() * 2;
    void* p = nullptr;
    if ((rc = b->ctx->dev_alloc(&p, b->d_sub_cap * sizeof(Work)))) return rc;
    b->d_sub = static_cast<Work*>(p);
  }
  std::memcpy(b->h_sub[k], tab.data(), tab.size() * sizeof(Work));
  char* hp = reinterpret_cast<char*>(b->h_sub[k] + tab.size());
  std::memcpy(hp, b->all_params.data(), sizeof(ParamsDev) * ns);
  CK(cudaMemcpyAsync(b->d_sub, b->h_sub[k], tab.size() * sizeof(Work), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(b->d_params, hp, sizeof(ParamsDev) * ns, cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(b->sub_ev[k], s));
  b->sub_used[k] = true;
  const SceneDev* d = b->d_scenes;
  Work* W = b->d_sub;
  const bool ref = b->mode == CLAY_MODE_REFERENCE;
  if (n_emit) CK(L_emit(d, W + o_emit, n_emit, T, s));
  for (int sub = 0; sub < max_sub && n_part > 0; sub++) {
    CK(L_cell_key(d, W + o_part, n_part, T, sub, s));
    CK(L_cell_count(d, W + o_part, n_part, T, sub, s));
    CK(L_scan_partial(d, W + o_scan, n_scan, sub, s));
    CK(L_scan_final(d, W + o_scan, n_scan, sub, s));
    CK(L_cell_scatter(d, W + o_part, n_part, T, sub, s));
    CK(L_cell_order(d, W + o_part, n_part, T, sub, s));
    if (ref) {
      CK(L_density_ref(d, W + o_part, n_part, T, sub, s));
      CK(L_forces_ref(d, W + o_part, n_part, T, sub, s));
    } else {
      CK(L_density_fast(d, W + o_part, n_part, T, sub, s));
      CK(L_forces_fast(d, W + o_part, n_part, T, sub, s));
    }
  }
  if (n_splat) CK(L_splat(b->d_surf, W + o_splat, n_splat, 1, kSplatAccVoxels, s));
  if (n_res) CK(L_resolve(b->d_surf, W + o_res, n_res, s));
  return CLAY_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// SurfaceExtractor (extract.ts:84-484).
struct clay_extractor {
  clay_ctx* ctx = nullptr;
  const clay_field* field = nullptr;
  ExtractDev h{};
  ExtractDev* d = nullptr;
  std::vector<DevBuf> bufs;
  bool dirty = true;
  int blocks = 0;
  // the eight passes of one extraction, captured on the first extract and replayed after:
  // every pass reads its parameters from `d`, so one graph serves every region and motion
  cudaGraphExec_t graph = nullptr;
  int64_t launches = 0;

  template <class T>
  int alloc(T** p, size_t count) {
    void* q = nullptr;
    int rc = ctx->dev_alloc(&q, sizeof(T) * std::max<size_t>(count, 1));
    if (rc) return rc;
    bufs.push_back({q, sizeof(T) * std::max<size_t>(count, 1)});
    *p = static_cast<T*>(q);
    return CLAY_OK;
  }
  int flush(cudaStream_t s) {
    if (field) {
      int rc = const_cast<clay_field*>(field)->flush(s);
      if (rc) return rc;
      h.field = field->d;
    }
    if (!dirty) return CLAY_OK;
    int rc = ctx->upload(d, &h, sizeof(h), s);
    if (rc) return rc;
    dirty = false;
    return CLAY_OK;
  }
};

extern "C" {

int clay_extractor_create(clay_ctx* ctx, const clay_field* field, void* particles, int64_t set_capacity, void* bodies,
                          int32_t max_bodies, const clay_extractor_opts* opts, clay_extractor** out) {
  if (!ctx || !field || !particles || !bodies || !opts || !out)
    return fail(CLAY_EINVAL, "clay_extractor_create: NULL argument");
  if (field->ctx != ctx) return fail(CLAY_EINVAL, "SurfaceExtractor: the field belongs to another context");
  const int res = (opts->set & CLAY_EXTRACT_RESOLUTION) ? opts->resolution : 32;  // extract.ts:99
  if (res < 2 || res > 512) return fail(CLAY_EINVAL, "SurfaceExtractor: resolution %d outside 2..512", res);
  if (opts->capacity < 0 || opts->base < 0)
    return fail(CLAY_EINVAL, "SurfaceExtractor: base and capacity must be non-negative");
  if (static_cast<int64_t>(opts->base) + opts->capacity > set_capacity)  // extract.ts:101-103
    return fail(CLAY_EINVAL, "SurfaceExtractor: slice [%d, %lld) exceeds set capacity", opts->base,
                static_cast<long long>(opts->base) + opts->capacity);
  if (opts->body < 0 || opts->body >= max_bodies)
    return fail(CLAY_EINVAL, "SurfaceExtractor: body %d outside the set's %d bodies", opts->body, max_bodies);
  if ((reinterpret_cast<uintptr_t>(particles) & 15) || (reinterpret_cast<uintptr_t>(bodies) & 15))
    return fail(CLAY_EINVAL, "SurfaceExtractor: particle and body buffers must be 16-byte aligned");
  clay_extractor* x = new clay_extractor();
  x->ctx = ctx;
  x->field = field;
  ExtractDev& h = x->h;
  const int64_t cells = static_cast<int64_t>(res) * res * res;
  x->blocks = static_cast<int>((cells + kExtractThreads - 1) / kExtractThreads);
  h.particles = static_cast<unsigned char*>(particles);
  h.bodies = static_cast<unsigned char*>(bodies);
  h.res = res;
  h.body = opts->body;
  h.base = opts->base;
  h.capacity = opts->capacity;
  // a closed surface-nets mesh has about as many quads as vertices (extract.ts:105-107)
  h.quad_cap = static_cast<int32_t>(std::ceil(opts->capacity * 1.5));
  h.has_motion = opts->motion ? 1 : 0;
  h.motion = opts->motion;
  if (reinterpret_cast<uintptr_t>(opts->motion) & 15) {
    delete x;
    return fail(CLAY_EINVAL, "SurfaceExtractor: the motion buffer must be 16-byte aligned");
  }
  h.nblocks = x->blocks;
  h.cell = 0.1f;  // the reference's initial region (extract.ts:124-129)
  int rc;
  float4* rec = nullptr;
  if ((rc = x->alloc(&x->d, 1)) || (rc = x->alloc(&h.id_grid, cells)) || (rc = x->alloc(&rec, cells * 2)) ||
      (rc = x->alloc(&h.blk, x->blocks)) || (rc = x->alloc(&h.qblk, x->blocks)) || (rc = x->alloc(&h.qmask, cells)) ||
      (rc = x->alloc(&h.indices, static_cast<size_t>(h.quad_cap) * 6)) || (rc = x->alloc(&h.draw_args, 4)) ||
      (rc = x->alloc(&h.counters, 2))) {
    clay_extractor_destroy(x);
    return rc;
  }
  h.rec = rec;
  CK(cudaMemset(h.counters, 0, 2 * sizeof(uint32_t)));
  CK(cudaMemset(h.draw_args, 0, 4 * sizeof(uint32_t)));
  *out = x;
  return CLAY_OK;
}

void clay_extractor_destroy(clay_extractor* x) {
  if (!x) return;
  if (x->graph) cudaGraphExecDestroy(x->graph);
  for (auto& b : x->bufs) x->ctx->dev_free(b.p, b.n);
  delete x;
}

int clay_extractor_set_region(clay_extractor* x, const double origin[3], double size, const double vel[3],
                              int preserve_motion) {
  if (!x || !origin) return fail(CLAY_EINVAL, "clay_extractor_set_region: NULL argument");
  for (int k = 0; k < 3; k++) {
    x->h.origin[k] = static_cast<float>(origin[k]);
    x->h.vel[k] = vel ? static_cast<float>(vel[k]) : 0.0f;
  }
  x->h.cell = static_cast<float>(size / x->h.res);  // extract.ts:451-463: cell = size / resolution
  x->h.preserve = preserve_motion ? 1u : 0u;
  x->dirty = true;
  return CLAY_OK;
}

int clay_extractor_extract(clay_extractor* x, void* stream) {
  if (!x) return fail(CLAY_EINVAL, "clay_extractor_extract: NULL extractor");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = x->flush(s);
  if (rc) return rc;
  // A small lattice (the game's 32^3 per body) is bound by launching its eight dependent
  // passes, so they run as one CUDA graph, captured on a private stream at the first call.
  if (!x->graph) {
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = launch_count();
    cudaError_t e = L_ext_reset(x->d, cs);
    if (e == cudaSuccess) e = L_ext_cells(x->d, x->blocks, cs);
    if (e == cudaSuccess) e = L_ext_scan(x->d, 0, cs);
    if (e == cudaSuccess) e = L_ext_emit(x->d, x->blocks, cs);
    if (e == cudaSuccess) e = L_ext_qcount(x->d, x->blocks, cs);
    if (e == cudaSuccess) e = L_ext_scan(x->d, 1, cs);
    if (e == cudaSuccess) e = L_ext_qemit(x->d, x->blocks, cs);
    if (e == cudaSuccess) e = L_ext_finish(x->d, cs);
    x->launches = static_cast<int64_t>(launch_count() - before);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (e == cudaSuccess) e = ec;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&x->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      x->graph = nullptr;
      return fail(CLAY_ECUDA, "SurfaceExtractor: capturing the extraction failed: %s", cudaGetErrorString(e));
    }
  }
  CK(cudaGraphLaunch(x->graph, s));
  count_launches(static_cast<uint64_t>(x->launches));
  return CLAY_OK;
}

int clay_extractor_views(clay_extractor* x, uint32_t** indices, uint32_t** draw_args, int64_t* quad_capacity) {
  if (!x) return fail(CLAY_EINVAL, "clay_extractor_views: NULL extractor");
  if (indices) *indices = x->h.indices;
  if (draw_args) *draw_args = x->h.draw_args;
  if (quad_capacity) *quad_capacity = x->h.quad_cap;
  return CLAY_OK;
}

int clay_extractor_read_counts_async(clay_extractor* x, uint32_t* host_counts, void* stream) {
  if (!x || !host_counts) return fail(CLAY_EINVAL, "clay_extractor_read_counts_async: NULL argument");
  CK(cudaMemcpyAsync(host_counts, x->h.counters, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                     static_cast<cudaStream_t>(stream)));
  return CLAY_OK;
}

int clay_extractor_read_indices_async(clay_extractor* x, uint32_t* host_indices, uint32_t* host_draw_args, void* stream) {
  if (!x || !host_indices || !host_draw_args) return fail(CLAY_EINVAL, "clay_extractor_read_indices_async: NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  CK(cudaMemcpyAsync(host_indices, x->h.indices, sizeof(uint32_t) * 6 * static_cast<size_t>(x->h.quad_cap),
                     cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(host_draw_args, x->h.draw_args, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  return CLAY_OK;
}

int clay_field_offset_device(const clay_field* f, const float* device_offset, clay_field** out) {
  if (!f || !device_offset || !out) return fail(CLAY_EINVAL, "clay_field_offset_device: NULL argument");
  std::vector<clay_field::Leaf> l = f->leaves;
  for (auto& leaf : l) {
    if (leaf.dyn) return fail(CLAY_EINVAL, "clay_field_offset_device: the field already follows a device offset");
    leaf.dyn = device_offset;
  }
  return make_field(f->ctx, std::move(l), out);
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// ClaySolver (pbd.ts:78-424).
struct clay_solver {
  clay_ctx* ctx = nullptr;
  const clay_field* world = nullptr;
  SolveDev h{};
  SolveDev* d = nullptr;
  int substeps = 2;
  bool dirty = true;
  bool kicking = false;
  // the substeps' passes as one CUDA graph, captured for the body count they were last run
  // with (it sets the match pass's grid); every pass reads its parameters from `d`
  cudaGraphExec_t graph = nullptr;
  int32_t graph_bodies = -1;
  int64_t launches = 0;
};

extern "C" {

int clay_solver_create(clay_ctx* ctx, const clay_field* world, void* particles, int64_t capacity, void* bodies,
                       int32_t max_bodies, const clay_solver_opts* opts, clay_solver** out) {
  if (!ctx || !world || !particles || !bodies || !out) return fail(CLAY_EINVAL, "clay_solver_create: NULL argument");
  if (world->ctx != ctx) return fail(CLAY_EINVAL, "ClaySolver: the world field belongs to another context");
  if (world->leaves.empty()) return fail(CLAY_EINVAL, "ClaySolver: the world field has no volume");
  if (capacity <= 0 || capacity > (1ll << 30) || max_bodies <= 0)
    return fail(CLAY_EINVAL, "ClaySolver: capacity and max_bodies must be positive");
  if ((reinterpret_cast<uintptr_t>(particles) & 15) || (reinterpret_cast<uintptr_t>(bodies) & 15))
    return fail(CLAY_EINVAL, "ClaySolver: particle and body buffers must be 16-byte aligned");
  clay_solver_opts o{};
  if (opts) o = *opts;
  // ClaySolverOptions defaults (pbd.ts:101-118)
  const double dt = (o.set & CLAY_SOLVER_DT) ? o.dt : 1.0 / 60;
  const int substeps = (o.set & CLAY_SOLVER_SUBSTEPS) ? o.substeps : 2;
  const int iters = (o.set & CLAY_SOLVER_ROTATION_ITERATIONS) ? o.rotation_iterations : 2;
  if (!(dt > 0) || substeps < 1 || iters < 0) return fail(CLAY_EINVAL, "ClaySolver: dt > 0, substeps >= 1, iterations >= 0");
  clay_solver* sv = new clay_solver();
  sv->ctx = ctx;
  sv->world = world;
  sv->substeps = substeps;
  SolveDev& h = sv->h;
  h.particles = static_cast<unsigned char*>(particles);
  h.bodies = static_cast<unsigned char*>(bodies);
  double g[3] = {0, -9.81, 0};
  if (o.set & CLAY_SOLVER_GRAVITY)
    for (int k = 0; k < 3; k++) g[k] = o.gravity[k];
  for (int k = 0; k < 3; k++) {
    h.gravity[k] = static_cast<float>(g[k]);
    h.push[k] = 0.0f;
    h.kick[k] = 0.0f;
  }
  h.h = static_cast<float>(dt / substeps);
  h.radius = static_cast<float>((o.set & CLAY_SOLVER_RADIUS) ? o.radius : 0.1);
  h.friction = static_cast<float>((o.set & CLAY_SOLVER_FRICTION) ? o.friction : 0.35);
  h.damping = static_cast<float>((o.set & CLAY_SOLVER_DAMPING) ? o.damping : 0.995);
  h.max_speed = static_cast<float>((o.set & CLAY_SOLVER_MAX_SPEED) ? o.max_speed : 40);
  h.push_body = 0xffffffffu;
  h.capacity = static_cast<int32_t>(capacity);
  h.max_bodies = max_bodies;
  h.rot_iters = iters;
  void* p = nullptr;
  int rc = ctx->dev_alloc(&p, sizeof(SolveDev));
  if (rc) {
    delete sv;
    return rc;
  }
  sv->d = static_cast<SolveDev*>(p);
  *out = sv;
  return CLAY_OK;
}

void clay_solver_destroy(clay_solver* sv) {
  if (!sv) return;
  if (sv->graph) cudaGraphExecDestroy(sv->graph);
  sv->ctx->dev_free(sv->d, sizeof(SolveDev));
  delete sv;
}

int clay_solver_set_force(clay_solver* sv, uint32_t body, const double accel[3], const double impulse[3]) {
  if (!sv || !accel) return fail(CLAY_EINVAL, "clay_solver_set_force: NULL argument");
  bool kick = false;
  for (int k = 0; k < 3; k++) {
    sv->h.push[k] = static_cast<float>(accel[k]);
    sv->h.kick[k] = impulse ? static_cast<float>(impulse[k]) : 0.0f;
    kick = kick || (impulse && impulse[k] != 0.0);
  }
  sv->h.push_body = body;
  sv->kicking = kick;
  sv->dirty = true;
  return CLAY_OK;
}

int clay_solver_step(clay_solver* sv, int32_t body_count, void* stream) {
  if (!sv) return fail(CLAY_EINVAL, "clay_solver_step: NULL solver");
  if (body_count < 0 || body_count > sv->h.max_bodies)
    return fail(CLAY_EINVAL, "clay_solver_step: body count %d outside 0..%d", body_count, sv->h.max_bodies);
  if (body_count == 0) return CLAY_OK;  // pbd.ts:401-404
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = const_cast<clay_field*>(sv->world)->flush(s);
  if (rc) return rc;
  if (sv->h.world != sv->world->d) {  // the field rebuilt its device table
    sv->h.world = sv->world->d;
    sv->dirty = true;
  }
  if (sv->dirty) {
    if ((rc = sv->ctx->upload(sv->d, &sv->h, sizeof(SolveDev), s))) return rc;
    sv->dirty = false;
  }
  const int blocks = (sv->h.capacity + kSolveThreads - 1) / kSolveThreads;
  if (sv->kicking) {
    CK(L_pbd_kick(sv->d, blocks, s));
    sv->kicking = false;
  }
  // The substeps' 4 x substeps dependent passes run as one CUDA graph, captured on a private
  // stream the first time and again when the body count changes.
  if (!sv->graph || sv->graph_bodies != body_count) {
    if (sv->graph) cudaGraphExecDestroy(sv->graph);
    sv->graph = nullptr;
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = launch_count();
    cudaError_t e = cudaSuccess;
    for (int sub = 0; sub < sv->substeps && e == cudaSuccess; sub++) {
      e = L_pbd_predict(sv->d, blocks, cs);
      if (e == cudaSuccess) e = L_pbd_match(sv->d, body_count, cs);
      if (e == cudaSuccess) e = L_pbd_apply(sv->d, blocks, cs);
      if (e == cudaSuccess) e = L_pbd_finalize(sv->d, blocks, cs);
    }
    sv->launches = static_cast<int64_t>(launch_count() - before);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (e == cudaSuccess) e = ec;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&sv->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      sv->graph = nullptr;
      return fail(CLAY_ECUDA, "ClaySolver: capturing the substeps failed: %s", cudaGetErrorString(e));
    }
    sv->graph_bodies = body_count;
  }
  CK(cudaGraphLaunch(sv->graph, s));
  count_launches(static_cast<uint64_t>(sv->launches));
  return CLAY_OK;
}

}  // extern "C"
