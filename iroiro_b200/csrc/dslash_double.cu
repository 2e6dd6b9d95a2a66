// Stencil instantiations for double-precision storage.
#include "dslash_launch.cuh"

namespace iro {

cudaError_t launch_hop_double(const HopLaunch& L, cudaStream_t st) {
  return L.recon == 12 ? hop_dag<PREC_DOUBLE, 12>(L, st) : hop_dag<PREC_DOUBLE, 18>(L, st);
}

}  // namespace iro
