// kern_ref.cu - kernels whose f32 arithmetic must round exactly as written: emission, the
// cell build, the bake, the collider build and the reference-mode neighbour passes.
// Compiled with -fmad=false (no multiply-add contraction); division and square root are
// IEEE round-to-nearest (-prec-div=true -prec-sqrt=true, the nvcc defaults).
#define CLAY_DEFINE_KERNELS
#include <atomic>

#include "launch.h"

namespace clay {

static std::atomic<uint64_t> g_launches{0};
uint64_t launch_count() { return g_launches.load(); }
void count_launch() { g_launches.fetch_add(1); }
void count_launches(uint64_t n) { g_launches.fetch_add(n); }

#define CLAY_LAUNCH(kern, grid, block, st, ...)         \
  do {                                                  \
    kern<<<grid, block, 0, st>>>(__VA_ARGS__);          \
    count_launch();                                     \
    return cudaPeekAtLastError();                       \
  } while (0)

cudaError_t L_emit(const SceneDev* s, const Work* w, int blocks, int threads, cudaStream_t st) {
  CLAY_LAUNCH(k_emit, blocks, threads, st, s, w);
}
cudaError_t L_cell_key(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st) {
  CLAY_LAUNCH(k_cell_key, blocks, threads, st, s, w, sub);
}
cudaError_t L_cell_count(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st) {
  CLAY_LAUNCH(k_cell_count, blocks, threads, st, s, w, sub);
}
cudaError_t L_scan_partial(const SceneDev* s, const Work* w, int blocks, int sub, cudaStream_t st) {
  dim3 g(w ? blocks : 1, w ? 1 : blocks);
  CLAY_LAUNCH(k_scan_partial, g, kScanThreads, st, s, w, sub);
}
cudaError_t L_scan_final(const SceneDev* s, const Work* w, int blocks, int sub, cudaStream_t st) {
  dim3 g(w ? blocks : 1, w ? 1 : blocks);
  CLAY_LAUNCH(k_scan_final, g, kScanThreads, st, s, w, sub);
}
cudaError_t L_cell_scatter(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st) {
  CLAY_LAUNCH(k_cell_scatter, blocks, threads, st, s, w, sub);
}
cudaError_t L_cell_order(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st) {
  CLAY_LAUNCH(k_cell_order, blocks, threads, st, s, w, sub);
}
cudaError_t L_density_ref(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st,
                          int variant) {
  if (variant == 1) k_density<false, 1><<<blocks, threads, 0, st>>>(s, w, sub);
  else if (variant == 2) k_density<false, 2><<<blocks, threads, 0, st>>>(s, w, sub);
  else k_density<false, 0><<<blocks, threads, 0, st>>>(s, w, sub);
  count_launch();
  return cudaPeekAtLastError();
}
cudaError_t L_forces_ref(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st,
                         bool split) {
  if (split) {
    k_forces_integrate<false, true><<<blocks, threads, 0, st>>>(s, w, sub);
    count_launch();
    k_integrate<false><<<blocks, threads, 0, st>>>(s, w, sub);
  } else {
    k_forces_integrate<false, false><<<blocks, threads, 0, st>>>(s, w, sub);
  }
  count_launch();
  return cudaPeekAtLastError();
}
cudaError_t L_splat(const SplatDev* d, const Work* w, int blocks, int blocks_y, uint32_t acc_voxels, cudaStream_t st) {
  // The splat's shared memory exceeds the default per-block limit; the opt-in is a property
  // of the function on each device, so it is set once per device (from any thread).
  constexpr int kDevices = 64;
  static std::atomic<bool> attr_set[kDevices];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kDevices || !attr_set[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(k_splat, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSplatAccVoxelsDiscs * static_cast<int>(sizeof(uint32_t)));
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < kDevices) attr_set[dev].store(true, std::memory_order_release);
  }
  dim3 g(blocks, w ? 1 : blocks_y);
  k_splat<<<g, kSplatThreads, acc_voxels * sizeof(uint32_t), st>>>(d, w, acc_voxels);
  count_launch();
  return cudaPeekAtLastError();
}
cudaError_t L_resolve(const SplatDev* d, const Work* w, int blocks, cudaStream_t st) {
  CLAY_LAUNCH(k_resolve, blocks, kResolveThreads, st, d, w);
}
cudaError_t L_field_query_mip(const FieldDev* f, const float* pts, int n, int mip, float* sxy, float* fxy, cudaStream_t st) {
  CLAY_LAUNCH(k_field_query_mip, (n + 255) / 256, 256, st, f, pts, n, mip, sxy, fxy);
}
cudaError_t L_pbd_kick(const SolveDev* s, int blocks, cudaStream_t st) { CLAY_LAUNCH(k_pbd_kick, blocks, kSolveThreads, st, s); }
cudaError_t L_pbd_predict(const SolveDev* s, int blocks, cudaStream_t st) {
  CLAY_LAUNCH(k_pbd_predict, blocks, kSolveThreads, st, s);
}
cudaError_t L_pbd_match(const SolveDev* s, int bodies, cudaStream_t st) { CLAY_LAUNCH(k_pbd_match, bodies, kSolveReduce, st, s); }
cudaError_t L_pbd_apply(const SolveDev* s, int blocks, cudaStream_t st) { CLAY_LAUNCH(k_pbd_apply, blocks, kSolveThreads, st, s); }
cudaError_t L_pbd_finalize(const SolveDev* s, int blocks, cudaStream_t st) {
  CLAY_LAUNCH(k_pbd_finalize, blocks, kSolveThreads, st, s);
}
cudaError_t L_ext_reset(const ExtractDev* e, cudaStream_t st) { CLAY_LAUNCH(k_ext_reset, 1, kExtractThreads, st, e); }
cudaError_t L_ext_cells(const ExtractDev* e, int blocks, cudaStream_t st) {
  CLAY_LAUNCH(k_ext_cells, blocks, kExtractThreads, st, e);
}
cudaError_t L_ext_scan(const ExtractDev* e, int which, cudaStream_t st) { CLAY_LAUNCH(k_ext_scan, 1, 1024, st, e, which); }
cudaError_t L_ext_emit(const ExtractDev* e, int blocks, cudaStream_t st) {
  CLAY_LAUNCH(k_ext_emit, blocks, kExtractThreads, st, e);
}
cudaError_t L_ext_qcount(const ExtractDev* e, int blocks, cudaStream_t st) {
  CLAY_LAUNCH(k_ext_qcount, blocks, kExtractThreads, st, e);
}
cudaError_t L_ext_qemit(const ExtractDev* e, int blocks, cudaStream_t st) {
  CLAY_LAUNCH(k_ext_qemit, blocks, kExtractThreads, st, e);
}
cudaError_t L_ext_finish(const ExtractDev* e, cudaStream_t st) { CLAY_LAUNCH(k_ext_finish, 1, kExtractThreads, st, e); }
cudaError_t L_build(const BuildLevelDev& lv, const BrushDev* brushes, int n, cudaStream_t st) {
  dim3 g(lv.tiles, lv.tiles, lv.tiles);
  CLAY_LAUNCH(k_build, g, 256, st, lv, brushes, n);
}
cudaError_t L_cell_index(const SceneDev* s, uint32_t* out, int n, cudaStream_t st) {
  CLAY_LAUNCH(k_cell_index, (n + 255) / 256, 256, st, s, out);
}
cudaError_t L_census_nbr(const SceneDev* s, int n, unsigned long long* out, cudaStream_t st) {
  CLAY_LAUNCH(k_census_nbr, (n + 255) / 256, 256, st, s, out);
}
cudaError_t L_census_splat(const SplatDev* d, int blocks, int mips, unsigned long long* out, cudaStream_t st) {
  dim3 g(blocks, mips);
  CLAY_LAUNCH(k_census_splat, g, 256, st, d, out);
}
cudaError_t L_gather_contacts(const SceneDev* s, int n, ContactsDev* out, cudaStream_t st) {
  CLAY_LAUNCH(k_gather_contacts, n, 128, st, s, n, out);
}
cudaError_t L_field_query(const FieldDev* f, const float* pts, int n, float* sxy, float* nrm, cudaStream_t st) {
  CLAY_LAUNCH(k_field_query, (n + 127) / 128, 128, st, f, pts, n, sxy, nrm);
}

}  // namespace clay
