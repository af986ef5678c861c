// kern_fast.cu - fast-mode neighbour passes: multiply-adds may be contracted into FMA and
// the density sum is compensated. Compiled with -fmad=true.
#define CLAY_DEFINE_KERNELS
#define CLAY_ONLY_NEIGHBOUR_PASSES
#include "launch.h"

namespace clay {

cudaError_t L_density_fast(const SceneDev* s, const Work* w, int blocks, int threads, int sub, cudaStream_t st,
                           int variant) {
  if (variant == 1) k_density<true, 1><<<blocks, threads, 0, st>>>(s, w, sub);
  else if (variant == 2) k_density<true, 2><<<blocks, threads, 0, st>>>(s, w, sub);
  else k_density<true, 0><<<blocks, threads, 0, st>>>(s, w, sub);
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
    k_forces_integrate<true, false><<<blocks, threads, 0, st>>>(s, w, sub);
  }
  count_launch();
  return cudaPeekAtLastError();
}

}  // namespace clay
