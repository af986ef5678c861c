// launch.h - host-side launchers of the kernels in clay_device.cuh.
//
// Every launcher takes either a work table (batched: one launch covers every scene) or
// nullptr plus a block count (one object, blocks tiling [0, n)). Each call counts one
// kernel launch in a process-wide counter.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "clay_device.cuh"

namespace clay {

// Records `msg` as the calling thread's clay_last_error() and returns `code`.
int report_error(int code, const char* msg);

uint64_t launch_count();
void count_launch();
void count_launches(uint64_t n);  // kernels replayed by a graph launch

// Threads per block of the particle passes when no tuning overrides it.
constexpr int kBlock = 256;
// The density variant used when no tuning overrides it (0: one loop, 1: two phases, 2: one
// loop over neighbour positions staged in shared memory).
constexpr int kDensityVariant = 0;

cudaError_t L_emit(const SceneDev* s, const Work* w, int blocks, int threads, cudaStream_t st);
cudaError_t L_cell_key(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st);
cudaError_t L_cell_count(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st);
cudaError_t L_scan_partial(const SceneDev* s, const Work* w, int blocks, int sub, cudaStream_t st);
cudaError_t L_scan_final(const SceneDev* s, const Work* w, int blocks, int sub, cudaStream_t st);
cudaError_t L_cell_scatter(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st);
cudaError_t L_cell_order(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st);
// Reference mode (kern_ref.cu) and fast mode (kern_fast.cu) of the neighbour passes.
// `variant` selects the density variant (all give the same visiting order).
cudaError_t L_density_ref(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st,
                          int variant = kDensityVariant);
// `split`: the forces pass without the integrate, then the integrate as a second launch.
cudaError_t L_forces_ref(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st,
                         bool split = false);
cudaError_t L_density_fast(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st,
                           int variant = kDensityVariant);
cudaError_t L_forces_fast(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st,
                          bool split = false);
// `blocks_y` = mip levels when w == nullptr.
// acc_voxels: size of the shared-memory minimum tile (dynamic shared memory, 4 B per voxel).
cudaError_t L_splat(const SplatDev* d, const Work* w, int blocks, int blocks_y, uint32_t acc_voxels, cudaStream_t st);
cudaError_t L_resolve(const SplatDev* d, const Work* w, int blocks, cudaStream_t st);
// SurfaceExtractor passes (grid passes: `blocks` blocks of kExtractThreads lattice cells).
cudaError_t L_field_query_mip(const FieldDev* f, const float* pts, int n, int mip, float* sxy, float* fxy, cudaStream_t st);
// ClaySolver passes.
cudaError_t L_pbd_kick(const SolveDev* s, int blocks, cudaStream_t st);
cudaError_t L_pbd_predict(const SolveDev* s, int blocks, cudaStream_t st);
cudaError_t L_pbd_match(const SolveDev* s, int bodies, cudaStream_t st);
cudaError_t L_pbd_apply(const SolveDev* s, int blocks, cudaStream_t st);
cudaError_t L_pbd_finalize(const SolveDev* s, int blocks, cudaStream_t st);
cudaError_t L_ext_reset(const ExtractDev* e, cudaStream_t st);
cudaError_t L_ext_cells(const ExtractDev* e, int blocks, cudaStream_t st);
cudaError_t L_ext_scan(const ExtractDev* e, int which, cudaStream_t st);
cudaError_t L_ext_emit(const ExtractDev* e, int blocks, cudaStream_t st);
cudaError_t L_ext_qcount(const ExtractDev* e, int blocks, cudaStream_t st);
cudaError_t L_ext_qemit(const ExtractDev* e, int blocks, cudaStream_t st);
cudaError_t L_ext_finish(const ExtractDev* e, cudaStream_t st);
cudaError_t L_build(const BuildLevelDev& lv, const BrushDev* brushes, int n, cudaStream_t st);
cudaError_t L_cell_index(const SceneDev* s, uint32_t* out, int n, cudaStream_t st);
// Census of a frame's algorithmic work (measurement hooks): out[0] += candidates, out[1] +=
// accepted pairs over `n` cell-ordered particles; out[0] += bake pairs over `blocks` x `mips`.
cudaError_t L_census_nbr(const SceneDev* s, int n, unsigned long long* out, cudaStream_t st);
cudaError_t L_census_splat(const SplatDev* d, int blocks, int mips, unsigned long long* out, cudaStream_t st);
cudaError_t L_gather_contacts(const SceneDev* s, int n, ContactsDev* out, cudaStream_t st);
cudaError_t L_field_query(const FieldDev* f, const float* pts, int n, float* sxy, float* nrm, cudaStream_t st);

constexpr int kScanThreads = 1024;
constexpr int kSplatThreads = 32 * kSplatWarps;
constexpr int kResolveThreads = 256;

}  // namespace clay
