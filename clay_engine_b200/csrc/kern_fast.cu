// kern_fast.cu - fast-mode neighbour passes: multiply-adds may be contracted into FMA and
// the density sum is compensated. Compiled with -fmad=true.
#define CLAY_DEFINE_KERNELS
#define CLAY_ONLY_NEIGHBOUR_PASSES
#include <atomic>

#include "launch.h"

namespace clay {

namespace {
// The neighbour passes use no shared memory (the staged density variant aside) and gather
// their neighbours through L1: ask for the largest L1 split of the SM's on-chip memory, once
// per device and kernel.
template <class K>
cudaError_t prefer_l1(K kernel, std::atomic<bool>* done) {
  constexpr int kDevices = 64;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kDevices) return e;
  if (done[dev].load(std::memory_order_acquire)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxL1);
  if (e == cudaSuccess) done[dev].store(true, std::memory_order_release);
  return e;
}
std::atomic<bool> g_l1_density[64], g_l1_forces[64];
}  // namespace

cudaError_t L_density_fast(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st,
                           int variant) {
  if (variant == 1) k_density<true, 1><<<blocks, threads, 0, st>>>(s, w, sub);
  else if (variant == 2) k_density<true, 2><<<blocks, threads, 0, st>>>(s, w, sub);
  else {
    cudaError_t e = prefer_l1(k_density<true, 0>, g_l1_density);
    if (e != cudaSuccess) return e;
    k_density<true, 0><<<blocks, threads, 0, st>>>(s, w, sub);
  }
  count_launch();
  return cudaPeekAtLastError();
}
cudaError_t L_forces_fast(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st,
                          bool split) {
  if (split) {
    k_forces_integrate<true, true><<<blocks, threads, 0, st>>>(s, w, sub);
    count_launch();
    k_integrate<true><<<blocks, threads, 0, st>>>(s, w, sub);
  } else {
    cudaError_t e = prefer_l1(k_forces_integrate<true, false>, g_l1_forces);
    if (e != cudaSuccess) return e;
    k_forces_integrate<true, false><<<blocks, threads, 0, st>>>(s, w, sub);
  }
  count_launch();
  return cudaPeekAtLastError();
}

}  // namespace clay
