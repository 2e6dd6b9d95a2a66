// Stencil instantiations for single-precision storage.
#include "dslash_launch.cuh"

namespace iro {

cudaError_t launch_hop_single(const HopLaunch& L, cudaStream_t st) {
  return hop_dag<PREC_SINGLE, 12>(L, st);
}

}  // namespace iro
