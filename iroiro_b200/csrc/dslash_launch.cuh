// Launch dispatch of the stencil over (dagger, epilogue); included once per
// storage precision so the instantiations compile in parallel.
#pragma once

#include "dslash.cuh"
#include "dslash_pair.cuh"
#include "dslash_stage.cuh"
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
  P.cg = L.cg;
  P.cst = L.cst;
  for (int i = 0; i < 2; ++i) {
    P.cr[i] = L.cr[i];
  }
  P.hs0 = L.hs0;
  P.nhs = L.nhs < 0 ? L.g.Vh - L.hs0 : L.nhs;
  LaunchCfg c = launch_cfg(P.nhs, L.nrhs, L.grid_cap(),
                           L.block_cap < HopBounds<VAR>::threads ? L.block_cap
                                                                 : HopBounds<VAR>::threads);
  // programmatic dependent launch: the blocks of this grid may be scheduled
  // while the previous kernel's last blocks retire (hop_kernel waits for
  // that kernel's completion before it reads anything), hiding the launch
  // gap between the dependent stencil launches of an operator
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(c.grid, L.nparity);
  cfg.blockDim = dim3(c.block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, hop_kernel<SP, GP, RECON, DAG, EPI, SP, VAR>, P);
}

// two right-hand sides per thread (FP32/FP16, reconstruct-12, even nrhs)
template <int SP, int RECON, bool DAG, int EPI, int VAR>
static cudaError_t hop_go_pair(const HopLaunch& L, cudaStream_t st) {
  if constexpr (SP == PREC_DOUBLE || RECON != 12) {
    return cudaErrorInvalidValue;
  } else {
    if (L.nrhs % 2 != 0 || L.hs0 != 0 || (L.nhs >= 0 && L.nhs != L.g.Vh)) return cudaErrorInvalidValue;
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
    P.cg = L.cg;
    P.cst = L.cst;
    for (int i = 0; i < 2; ++i) {
      P.cr[i] = L.cr[i];
    }
    LaunchCfg c = launch_cfg(L.g.Vh, L.nrhs / 2, L.grid_cap(), L.block_cap);
    dim3 grid(c.grid, L.nparity);
    hop_pair_kernel<SP, DAG, EPI, VAR><<<grid, c.block, 0, st>>>(P);
    return cudaGetLastError();
  }
}

// two right-hand sides per thread with shared-memory staging of the neighbours
template <int SP, int RECON, bool DAG, int EPI, int VAR>
static cudaError_t hop_go_stage(const HopLaunch& L, cudaStream_t st) {
  if constexpr (SP == PREC_DOUBLE || RECON != 12) {
    return cudaErrorInvalidValue;
  } else {
    if (L.nrhs % 2 != 0 || L.hs0 != 0 || (L.nhs >= 0 && L.nhs != L.g.Vh)) return cudaErrorInvalidValue;
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
    P.cg = L.cg;
    P.cst = L.cst;
    for (int i = 0; i < 2; ++i) {
      P.cr[i] = L.cr[i];
    }
    // the staging buffers of a block must fit the 227 KiB a block can opt in
    // to (FP32: 976 B per thread, so at most 232 threads)
    int cap = L.block_cap;
    while (cap > 32 && stage_bytes<SP>() * cap > 232448) cap /= 2;
    LaunchCfg c = launch_cfg(L.g.Vh, L.nrhs / 2, L.grid_cap(), cap);
    if (stage_bytes<SP>() * c.block > 232448) return cudaErrorInvalidValue;
    const int smem = stage_bytes<SP>() * c.block;
    static int opted = 0;  // largest dynamic shared memory already allowed
    if (smem > opted) {
      cudaError_t e = cudaFuncSetAttribute(hop_stage_kernel<SP, DAG, EPI, VAR>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      opted = smem;
    }
    dim3 grid(c.grid, L.nparity);
    hop_stage_kernel<SP, DAG, EPI, VAR><<<grid, c.block, smem, st>>>(P);
    return cudaGetLastError();
  }
}

// Variants 0-3: hop_kernel (bits: see there).  FP32/FP16 with even nrhs:
// 4-7 two right-hand sides per thread with the register cap none / 128 /
// 152 / 168, 8-9 the same with the neighbours staged through shared memory.
// FP64: 4/5 the 168-register 128-thread hop_kernel (5 with the rolled loop).
// FP16 on links with three stored rows (RECON 18): only 10/11/12, the
// mixed-precision hop_kernel (VAR 8 / 9 / 10: 3 / 4 / 2 blocks per SM).
// FP16 on the 12-real links: also 13/14, the mixed-precision hop_kernel with
// row 2 rebuilt (VAR 8 / 9).
template <int SP, int GP, int RECON, bool DAG, int EPI>
static cudaError_t hop_var_more(const HopLaunch& L, cudaStream_t st);

template <int SP, int GP, int RECON, bool DAG, int EPI>
static cudaError_t hop_var(const HopLaunch& L, cudaStream_t st) {
  if constexpr (SP == PREC_HALF && RECON == 18) {
    switch (L.variant) {
      case 10: return hop_go<SP, GP, RECON, DAG, EPI, 8>(L, st);
      case 11: return hop_go<SP, GP, RECON, DAG, EPI, 9>(L, st);
      case 12: return hop_go<SP, GP, RECON, DAG, EPI, 10>(L, st);
      default: return cudaErrorInvalidValue;
    }
  } else {
    switch (L.variant) {
      case 0: return hop_go<SP, GP, RECON, DAG, EPI, 0>(L, st);
      case 1: return hop_go<SP, GP, RECON, DAG, EPI, 1>(L, st);
      case 2: return hop_go<SP, GP, RECON, DAG, EPI, 2>(L, st);
      case 3: return hop_go<SP, GP, RECON, DAG, EPI, 3>(L, st);
      default: break;
    }
    return hop_var_more<SP, GP, RECON, DAG, EPI>(L, st);
  }
}

template <int SP, int GP, int RECON, bool DAG, int EPI>
static cudaError_t hop_var_more(const HopLaunch& L, cudaStream_t st) {
  if constexpr (SP == PREC_DOUBLE) {
    switch (L.variant) {
      case 4: return hop_go<SP, GP, RECON, DAG, EPI, 4>(L, st);
      case 5: return hop_go<SP, GP, RECON, DAG, EPI, 6>(L, st);
      default: return cudaErrorInvalidValue;
    }
  } else {
    switch (L.variant) {
      case 4: return hop_go_pair<SP, RECON, DAG, EPI, 0>(L, st);
      case 5: return hop_go_pair<SP, RECON, DAG, EPI, 1>(L, st);
      case 6: return hop_go_pair<SP, RECON, DAG, EPI, 2>(L, st);
      case 7: return hop_go_pair<SP, RECON, DAG, EPI, 3>(L, st);
      case 8: return hop_go_stage<SP, RECON, DAG, EPI, 0>(L, st);
      case 9: return hop_go_stage<SP, RECON, DAG, EPI, 1>(L, st);
      default: break;
    }
    if constexpr (SP == PREC_HALF && RECON == 12) {
      switch (L.variant) {
        case 13: return hop_go<SP, GP, RECON, DAG, EPI, 8>(L, st);
        case 14: return hop_go<SP, GP, RECON, DAG, EPI, 9>(L, st);
        default: break;
      }
    }
    return cudaErrorInvalidValue;
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
