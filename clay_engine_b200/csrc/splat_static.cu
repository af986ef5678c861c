// splat_static.cu - a SplatField bake that allocates no device memory.
//
// Some callers cannot allocate device memory once they are running: a game or editor that
// bakes from inside its per-frame tick, where cudaMalloc/cudaFree would synchronise the
// device and stall the frame, and plugin hosts that hand a library only buffers allocated
// up front and forbid it to grow device memory afterwards. For them this file provides
// clay_splat_bake_static: the caller passes the particle cloud (inputs) and the f16 output
// plane(s); the bake's only scratch, one 32-bit word per voxel holding the smallest distance
// lowered into it as an order-preserving integer of its f32 bits (the resolve pass turns it
// into the reference's 16-bit key), lives in a fixed file-scope device array instead of a
// per-object allocation.
//
// The array holds at most kStaticKeys keys (4 MiB) and every GPU that loads the library
// keeps it until the process exits. All calls share it: each call clears the part it uses
// before splatting, and calls whose work overlaps on the GPU (two streams at once) race on
// it, so callers must order them.
//
// Compiled with -fmad=false like every exact pass: the results are bit for bit those of
// clay_splat_bake for the same cloud and options.
#define CLAY_DEFINE_KERNELS
#define CLAY_ONLY_NEIGHBOUR_PASSES
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/clay_fluid.h"
#include "launch.h"

namespace clay {
namespace {

constexpr long long kStaticKeys = CLAY_STATIC_BAKE_MAX_VOXELS;
static_assert(kStaticKeys % 4 == 0, "the resolve pass reads keys four at a time");

// The bake's scratch key grid. In host code this name is only a stand-in for the device
// array: its device address comes from cudaGetSymbolAddress (see static_keys_address).
__device__ __align__(256) uint32_t g_static_keys[kStaticKeys];

__global__ void k_static_clear(uint32_t* __restrict__ keys, long long n) {
  long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) keys[i] = kNoHit;
}

__global__ void __launch_bounds__(32 * kSplatWarps, 4) k_static_splat(const __grid_constant__ SplatDev D, float ox, float oy,
                                                                     float oz) {
  Work w;
  w.obj = 0;
  w.sub = blockIdx.y;
  w.first = blockIdx.x * blockDim.x;
  w.n = blockDim.x;
  splat_block(D, w, ox, oy, oz, kSplatAccVoxels);
}

__global__ void k_static_resolve(const __grid_constant__ SplatDev D) {
  Work w;
  w.obj = 0;
  w.sub = 0;
  w.first = blockIdx.x * blockDim.x;
  w.n = blockDim.x;
  resolve_block(D, w);
}

__global__ void k_static_material(__half* __restrict__ out, long long n, __half v) {
  long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = v;
}

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_addr[kMaxDevices] = {};

// Set-up, once per device, with that device current: the device address of the array.
int static_keys_address(uint32_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return report_error(CLAY_ECUDA, "clay_splat_bake_static: cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxDevices) return report_error(CLAY_EINVAL, "clay_splat_bake_static: device index out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_keys);
    if (e != cudaSuccess || !p)
      return report_error(CLAY_ECUDA, "clay_splat_bake_static: cudaGetSymbolAddress of the scratch keys failed");
    // the splat's static shared memory plus its tile exceed the default 48 KB per block
    e = cudaFuncSetAttribute(k_static_splat, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSplatAccVoxels * static_cast<int>(sizeof(uint32_t)));
    if (e != cudaSuccess) return report_error(CLAY_ECUDA, "clay_splat_bake_static: cudaFuncSetAttribute failed");
    g_addr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_addr[dev];
  return CLAY_OK;
}

}  // namespace
}  // namespace clay

using namespace clay;

extern "C" int clay_splat_bake_static(const clay_cloud_desc* cloud, const clay_splat_opts* o, void* dist_out_f16,
                                      void* material_out_f16, void* stream) {
  if (!cloud || !o || !dist_out_f16) return report_error(CLAY_EINVAL, "clay_splat_bake_static: NULL argument");
  // the resolve pass stores the distance plane two halves at a time, the material pass one half
  if (reinterpret_cast<uintptr_t>(dist_out_f16) % 4 != 0)
    return report_error(CLAY_EINVAL, "clay_splat_bake_static: dist_out_f16 must be 4-byte aligned");
  if (material_out_f16 && reinterpret_cast<uintptr_t>(material_out_f16) % 2 != 0)
    return report_error(CLAY_EINVAL, "clay_splat_bake_static: material_out_f16 must be 2-byte aligned");
  if (cloud->capacity > 0 && (reinterpret_cast<uintptr_t>(cloud->positions) % 4 != 0 || cloud->position_stride % 4 != 0))
    return report_error(CLAY_EINVAL, "clay_splat_bake_static: positions must be 4-byte aligned with a stride of whole floats");
  if (!cloud->positions && cloud->capacity > 0) return report_error(CLAY_EINVAL, "clay_splat_bake_static: no positions");
  if (cloud->position_stride < 12 && cloud->capacity > 1)
    return report_error(CLAY_EINVAL, "clay_splat_bake_static: position stride below 12 bytes");
  if (cloud->live_mode > CLAY_LIVE_RANGE ||
      (cloud->live_mode == CLAY_LIVE_COUNT && !cloud->live_count) ||
      (cloud->live_mode == CLAY_LIVE_RANGE && (!cloud->live_first || !cloud->live_range_count)))
    return report_error(CLAY_EINVAL, "clay_splat_bake_static: bad live rule");
  // The options of SplatField (splat.ts:148-153) and the SdfVolume mip rule (volume.ts:156-160).
  const int res = (o->set & CLAY_SPLAT_RESOLUTION) ? o->resolution : 64;
  // Bound the resolution before anything is derived from it: no level of a bake above
  // kStaticMaxRes fits the scratch, and the cubes below stay far from 64-bit overflow.
  constexpr int kStaticMaxRes = 128;
  if (res <= 0 || res > kStaticMaxRes) {
    char msg[192];
    std::snprintf(msg, sizeof(msg),
                  "clay_splat_bake_static: resolution %d is outside 1..%d (the static scratch holds at most %lld voxels)",
                  res, kStaticMaxRes, kStaticKeys);
    return report_error(CLAY_EINVAL, msg);
  }
  if (!(o->radius >= 0)) return report_error(CLAY_EINVAL, "clay_splat_bake_static: radius must be a non-negative number");
  const int mips = (o->set & CLAY_SPLAT_MIP_LEVELS) ? o->mip_levels
                                                    : std::max(1, static_cast<int>(std::log2(static_cast<double>(res) / 8)));
  const double band = (o->set & CLAY_SPLAT_BAND) ? o->band : 2.0;
  const double material = (o->set & CLAY_SPLAT_MATERIAL) ? o->material : 0.0;
  const double world = (o->set & CLAY_SPLAT_WORLD_SIZE) ? o->world_size : 24.0;
  double origin[3] = {-12, -4, -12};
  if (o->set & CLAY_SPLAT_ORIGIN)
    for (int k = 0; k < 3; k++) origin[k] = o->origin[k];
  if (mips < 1 || mips > kMaxMips || res <= 0 || res % (8LL << (mips - 1)) != 0)
    return report_error(CLAY_EINVAL, "clay_splat_bake_static: resolution must be a multiple of 8 * 2^(mipLevels-1)");
  long long total = 0;
  for (int m = 0; m < mips; m++) {
    long long r = res >> m;
    total += r * r * r;
  }
  if (total > kStaticKeys) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "clay_splat_bake_static: a %d^3 bake with %d levels has %lld voxels; the static scratch holds at most "
                  "%lld (for example 96^3 with 3 levels)",
                  res, mips, total, kStaticKeys);
    return report_error(CLAY_EINVAL, msg);
  }
  uint32_t* keys = nullptr;
  int rc = static_keys_address(&keys);
  if (rc) return rc;

  SplatDev h;
  std::memset(&h, 0, sizeof(h));
  h.pos = static_cast<const char*>(cloud->positions);
  h.nrm = static_cast<const char*>(cloud->normals);
  h.quat = cloud->rotation;
  h.live_count = cloud->live_count;
  h.live_first = cloud->live_first;
  h.live_range_count = cloud->live_range_count;
  h.keys = keys;
  h.dist_out = static_cast<__half*>(dist_out_f16);
  h.pos_stride = cloud->position_stride;
  h.nrm_stride = cloud->normal_stride;
  h.capacity = cloud->capacity;
  h.live_mode = cloud->live_mode;
  h.mips = mips;
  h.radius = static_cast<float>(o->radius);
  long long off = 0;
  for (int m = 0; m < mips; m++) {
    double voxel = (world / res) * std::pow(2.0, m);
    double bw = band * voxel;
    h.r[m] = res >> m;
    h.off[m] = off;
    h.voxel[m] = static_cast<float>(voxel);
    h.bw[m] = static_cast<float>(bw);
    h.reach[m] = static_cast<float>(o->radius + bw);
    h.inv_voxel[m] = static_cast<float>(1 / voxel);
    off += static_cast<long long>(h.r[m]) * h.r[m] * h.r[m];
  }
  h.total = total;
  h.tile_ratio = kSplatTileRatio;
  h.walk_weight = kSplatWalkWeight;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The array keeps the last call's values: start from the clear value kNoHit.
  k_static_clear<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(keys, total);
  count_launch();
  if (cloud->capacity > 0) {
    dim3 g((cloud->capacity + kSplatThreads - 1) / kSplatThreads, mips);
    k_static_splat<<<g, kSplatThreads, kSplatAccVoxels * sizeof(uint32_t), s>>>(h, static_cast<float>(origin[0]), static_cast<float>(origin[1]),
                                               static_cast<float>(origin[2]));
    count_launch();
  }
  long long quads = (total + 3) / 4;
  k_static_resolve<<<static_cast<unsigned>((quads + kResolveThreads - 1) / kResolveThreads), kResolveThreads, 0, s>>>(h);
  count_launch();
  if (material_out_f16) {
    k_static_material<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(
        static_cast<__half*>(material_out_f16), total, __float2half_rn(static_cast<float>(material)));
    count_launch();
  }
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) return report_error(CLAY_ECUDA, cudaGetErrorString(e));
  return CLAY_OK;
}
