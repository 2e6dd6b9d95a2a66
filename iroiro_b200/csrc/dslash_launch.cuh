// Launch dispatch of the stencil over (dagger, epilogue); included once per
// storage precision so the instantiations compile in parallel.
#pragma once

#include "dslash.cuh"
#include "internal.h"

namespace iro {

template <int SP, int GP, int RECON, bool DAG, int EPI, int VAR>
static cudaError_t hop_go(const HopLaunch& L, cudaStream_t st) {
  HopParams P;
  P.g = L.g;
  P.p0 = L.p0;
  P.nrhs = L.nrhs;
  for (int i = 0; i < 2; ++i) {
    P.in[i] = L.in[i];
    P.out[i] = L.out[i];
    P.xin[i] = L.xin[i];
    P.clov[i] = L.clov[i];
  }
  P.gauge = L.gauge;
  P.scale = L.scale;
  P.red_mask = L.red_mask;
  P.red = L.red;
  P.skip = L.skip;
  LaunchCfg c = launch_cfg(L.g.Vh, L.nrhs, L.max_blocks, L.block_cap);
  dim3 grid(c.grid, L.nparity);
  hop_kernel<SP, GP, RECON, DAG, EPI, SP, VAR><<<grid, c.block, 0, st>>>(P);
  return cudaGetLastError();
}

template <int SP, int GP, int RECON, bool DAG, int EPI>
static cudaError_t hop_var(const HopLaunch& L, cudaStream_t st) {
  switch (L.variant & 3) {
    case 0: return hop_go<SP, GP, RECON, DAG, EPI, 0>(L, st);
    case 1: return hop_go<SP, GP, RECON, DAG, EPI, 1>(L, st);
    case 2: return hop_go<SP, GP, RECON, DAG, EPI, 2>(L, st);
    default: return hop_go<SP, GP, RECON, DAG, EPI, 3>(L, st);
  }
}

template <int SP, int RECON, bool DAG>
static cudaError_t hop_epi(const HopLaunch& L, cudaStream_t st) {
  switch (L.epi) {
    case EPI_SCALE: return hop_var<SP, SP, RECON, DAG, EPI_SCALE>(L, st);
    case EPI_SCALE_CLOV: return hop_var<SP, SP, RECON, DAG, EPI_SCALE_CLOV>(L, st);
    case EPI_XPAY: return hop_var<SP, SP, RECON, DAG, EPI_XPAY>(L, st);
    case EPI_XPAY_CLOV: return hop_var<SP, SP, RECON, DAG, EPI_XPAY_CLOV>(L, st);
  }
  return cudaErrorInvalidValue;
}

template <int SP, int RECON>
static cudaError_t hop_dag(const HopLaunch& L, cudaStream_t st) {
  return L.dag ? hop_epi<SP, RECON, true>(L, st) : hop_epi<SP, RECON, false>(L, st);
}

}  // namespace iro
