// Stencil instantiations for half-precision storage.
#include "dslash_launch.cuh"

namespace iro {

cudaError_t launch_hop_half(const HopLaunch& L, cudaStream_t st) {
  return L.recon == 18 ? hop_dag<PREC_HALF, 18>(L, st) : hop_dag<PREC_HALF, 12>(L, st);
}

}  // namespace iro
