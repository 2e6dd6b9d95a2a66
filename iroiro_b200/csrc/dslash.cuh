// The Wilson(-clover) hopping stencil for sm_100a.
//
// One thread computes one output site of one right-hand side:
//   acc = sum_mu (1 - g_mu) U_mu(x) psi(x+mu) + (1 + g_mu) U_mu(x-mu)^dag psi(x-mu)
// in the direction order x+,x-,y+,y-,z+,z-,t+,t- of Dirac_Wilson::mult_offdiag
// (lib/Dirac_ops/dirac_wilson.cpp:107-113), with each neighbour first
// projected to a half spinor (two colour vectors), multiplied by the link and
// reconstructed, as the reference's improved kernel does per direction
// (lib/Dirac_ops/dirac_wilson_improved.code:5-648).  The dagger operator
// gamma5 D gamma5 (dirac_wilson.cpp:34-36) is the same stencil with the two
// projectors exchanged, since gamma5 (1 -+ g_mu) gamma5 = (1 +- g_mu).
//
// The epilogue fuses what follows the stencil in the reference's operators:
// the -kappa scale, the identity/clover diagonal term (f - kappa H f, or
// A f - kappa H f), the clover inverse of the Schur complement, and the
// FP64 norm/dot reductions a Krylov solver needs next.  Reductions are
// deterministic: a fixed tree inside each block, per-block partials in global
// scratch, and the last block to finish (ticket counter) summing the partials
// in block order and running the solver's scalar update.
#pragma once

#include "common.cuh"
#include "dslash_mix.cuh"
#include "solver_scalars.cuh"

namespace iro {

// projector (1 - S*gamma_mu) applied to psi -> half spinor h[0..2]=h0, h[3..5]=h1
// gamma matrices of GammaMatrix (lib/Dirac_ops/wilsonLikeUtils.cpp:9-40).
template <int MU, int S, typename R>
__device__ __forceinline__ void project(const Cx<R> f[12], Cx<R> h[6]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const Cx<R> f0 = f[c], f1 = f[3 + c], f2 = f[6 + c], f3 = f[9 + c];
    if (MU == 0) {  // h0 = f0 + S i f3, h1 = f1 + S i f2
      h[c] = (S > 0) ? f0 + mul_i(f3) : f0 - mul_i(f3);
      h[3 + c] = (S > 0) ? f1 + mul_i(f2) : f1 - mul_i(f2);
    } else if (MU == 1) {  // h0 = f0 + S f3, h1 = f1 - S f2
      h[c] = (S > 0) ? f0 + f3 : f0 - f3;
      h[3 + c] = (S > 0) ? f1 - f2 : f1 + f2;
    } else if (MU == 2) {  // h0 = f0 + S i f2, h1 = f1 - S i f3
      h[c] = (S > 0) ? f0 + mul_i(f2) : f0 - mul_i(f2);
      h[3 + c] = (S > 0) ? f1 - mul_i(f3) : f1 + mul_i(f3);
    } else {  // t: S=+1 keeps 2*f2, 2*f3; S=-1 keeps 2*f0, 2*f1
      h[c] = (S > 0) ? R(2) * f2 : R(2) * f0;
      h[3 + c] = (S > 0) ? R(2) * f3 : R(2) * f1;
    }
  }
}

// acc += (1 - S*gamma_mu) reconstructed from the multiplied half spinor g
template <int MU, int S, typename R>
__device__ __forceinline__ void reconstruct(Cx<R> acc[12], const Cx<R> g[6]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const Cx<R> g0 = g[c], g1 = g[3 + c];
    if (MU == 3) {
      if (S > 0) {
        acc[6 + c] = acc[6 + c] + g0;
        acc[9 + c] = acc[9 + c] + g1;
      } else {
        acc[c] = acc[c] + g0;
        acc[3 + c] = acc[3 + c] + g1;
      }
      continue;
    }
    acc[c] = acc[c] + g0;
    acc[3 + c] = acc[3 + c] + g1;
    if (MU == 0) {  // [h0, h1, -S i h1, -S i h0]
      acc[6 + c] = (S > 0) ? acc[6 + c] + mul_mi(g1) : acc[6 + c] + mul_i(g1);
      acc[9 + c] = (S > 0) ? acc[9 + c] + mul_mi(g0) : acc[9 + c] + mul_i(g0);
    } else if (MU == 1) {  // [h0, h1, -S h1, S h0]
      acc[6 + c] = (S > 0) ? acc[6 + c] - g1 : acc[6 + c] + g1;
      acc[9 + c] = (S > 0) ? acc[9 + c] + g0 : acc[9 + c] - g0;
    } else {  // MU==2: [h0, h1, -S i h0, S i h1]
      acc[6 + c] = (S > 0) ? acc[6 + c] + mul_mi(g0) : acc[6 + c] + mul_i(g0);
      acc[9 + c] = (S > 0) ? acc[9 + c] + mul_i(g1) : acc[9 + c] + mul_mi(g1);
    }
  }
}

template <typename R>
__device__ __forceinline__ void su3_mul(const Su3<R>& U, const Cx<R> h[6], Cx<R> g[6]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    g[a] = U.e[a][0] * h[0] + U.e[a][1] * h[1] + U.e[a][2] * h[2];
    g[3 + a] = U.e[a][0] * h[3] + U.e[a][1] * h[4] + U.e[a][2] * h[5];
  }
}

template <typename R>
__device__ __forceinline__ void su3_dag_mul(const Su3<R>& U, const Cx<R> h[6], Cx<R> g[6]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    g[a] = cj_mul(U.e[0][a], h[0]) + cj_mul(U.e[1][a], h[1]) + cj_mul(U.e[2][a], h[2]);
    g[3 + a] = cj_mul(U.e[0][a], h[3]) + cj_mul(U.e[1][a], h[4]) + cj_mul(U.e[2][a], h[5]);
  }
}

// Neighbour spinor projected to a half spinor.  FP16 elements are projected
// from their stored (normalised) values and the element norm is applied to
// the 6 projected complexes instead of the 12 loaded ones.
template <int MU, int S, int SP>
__device__ __forceinline__ void load_project(const SpinorPtr& in, int i,
                                             Cx<typename SpinorIO<SP>::Real> h[6]) {
  using R = typename SpinorIO<SP>::Real;
  Cx<R> f[12];
  if constexpr (SP == PREC_HALF) {
    const float n = SpinorIO<PREC_HALF>::load_raw(in, i, f);
    project<MU, S, R>(f, h);
#pragma unroll
    for (int k = 0; k < 6; ++k) h[k] = n * h[k];
  } else {
    SpinorIO<SP>::load(in, i, f);
    project<MU, S, R>(f, h);
  }
}

// Forward (x+mu) and backward (x-mu) contributions of direction MU.
template <int MU, bool DAG, int SP, int GP, int RECON>
__device__ __forceinline__ void hop_dir(const GaugePtr& gauge, const SpinorPtr& in, int p,
                                        int hs, const int nb[8], int nrhs, int r,
                                        Cx<typename SpinorIO<SP>::Real> acc[12]) {
  using R = typename SpinorIO<SP>::Real;
  Cx<R> h[6], g[6];
  // forward: (1 - g_mu) U_mu(x) psi(x+mu)   [dagger: (1 + g_mu)]
  {
    Su3<R> U;
    GaugeIO<GP, RECON>::load(gauge, p, MU, hs, U);
    constexpr int S = DAG ? -1 : 1;
    load_project<MU, S, SP>(in, nb[2 * MU] * nrhs + r, h);
    su3_mul(U, h, g);
    reconstruct<MU, S, R>(acc, g);
  }
  // backward: (1 + g_mu) U_mu(x-mu)^dag psi(x-mu)   [dagger: (1 - g_mu)]
  {
    Su3<R> U;
    GaugeIO<GP, RECON>::load(gauge, 1 - p, MU, nb[2 * MU + 1], U);
    constexpr int S = DAG ? 1 : -1;
    load_project<MU, S, SP>(in, nb[2 * MU + 1] * nrhs + r, h);
    su3_dag_mul(U, h, g);
    reconstruct<MU, S, R>(acc, g);
  }
}

struct HopParams {
  Geom g;
  int p0;  // parity of the output sites handled by blockIdx.y == 0
  int nrhs;
  SpinorPtr in[2], out[2], xin[2];  // indexed by blockIdx.y
  GaugePtr gauge;
  CloverPtr clov[2];
  double scale;
  int red_mask;
  Reduce red;
  const int* skip;  // per-rhs converged flags, or null
  // fused CG update (Solver_CG::solve_step's r update, solver_CG.cpp:120-140)
  // on the operator's output s: r -= alpha s, red[0] = |r|^2; s itself is
  // not stored.  x += alpha p is left to the p update (cg_p_kernel), which
  // reads p anyway.  Off when cg == 0.
  int cg;
  SpinorPtr cr[2];  // indexed like out[]
  const CGState* cst;
  // the output half-sites [hs0, hs0 + nhs) of this launch (all: 0, Vh)
  int hs0, nhs;
};

// VAR bit 0: at least two 256-thread blocks per SM (register cap 128);
// VAR bit 1: the four directions as a rolled loop (no hoisting of one
// direction's loads over another's, fewer live registers);
// VAR bit 2 (FP64 only): 128-thread blocks, at least three per SM (register
// cap 168: between the uncapped 254 and the spilling 128);
// VAR bit 3 (FP16 only): the mixed-precision direction code of
// dslash_mix.cuh on the links with three stored rows (RECON 18) or two
// (RECON 12, row 2 rebuilt), at least three 256-thread blocks per SM (four
// with bit 0, two with bit 1).
template <int VAR>
struct HopBounds {
  static constexpr int threads = (VAR & 4) ? 128 : 256;
  static constexpr int blocks =
      (VAR & 8) ? ((VAR & 1) ? 4 : ((VAR & 2) ? 2 : 3))
                : ((VAR & 4) ? 3 : ((VAR & 1) ? 2 : 1));
};

template <int SP, int GP, int RECON, bool DAG, int EPI, int CP, int VAR>
__global__ void __launch_bounds__(HopBounds<VAR>::threads, HopBounds<VAR>::blocks)
    hop_kernel(HopParams P) {
  using R = typename SpinorIO<SP>::Real;
  // Launched as a programmatic dependent launch (hop_go): wait until the
  // previous kernel of the stream has completed and its writes are visible
  // (its output is this launch's input; nothing global is read before), then
  // allow the next launch to be scheduled as this grid's blocks retire.  In
  // an ordinary launch both are no-ops.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int yi = blockIdx.y;
  const int p = P.p0 ^ yi;
  const int nrhs = P.nrhs;
  const int nthreads = P.nhs * nrhs;  // < 2^31, checked at context creation
  const int e0 = P.hs0 * nrhs;         // element index of the first output
  double red[3] = {0.0, 0.0, 0.0};
  // the grid stride is a multiple of nrhs, so each thread keeps one rhs
  const int r = (nrhs == 1) ? 0 : int((blockIdx.x * blockDim.x + threadIdx.x) % unsigned(nrhs));
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nthreads; t += gridDim.x * blockDim.x) {
    const int tid = e0 + t;
    const int hs = (nrhs == 1) ? tid : int(unsigned(tid) / unsigned(nrhs));
    if (P.skip && P.skip[r]) continue;
    const Coord c = coord_of(P.g, hs, p);
    int nb[8];
    neighbours(P.g, c, hs, nb);
    Cx<R> acc[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = {R(0), R(0)};
    if constexpr ((VAR & 8) != 0) {
      static_assert(SP == PREC_HALF && (RECON == 18 || RECON == 12), "mixed path: FP16 links");
      const uint32_t vh = uint32_t(P.g.Vh);
      const uint32_t lown = uint32_t(p * 4) * vh, lnb = uint32_t((1 - p) * 4) * vh;
      hop_dir_mix<0, DAG, RECON>(P.gauge, P.in[yi], lown, lnb, vh, hs, nb, nrhs, r, acc);
      hop_dir_mix<1, DAG, RECON>(P.gauge, P.in[yi], lown, lnb, vh, hs, nb, nrhs, r, acc);
      hop_dir_mix<2, DAG, RECON>(P.gauge, P.in[yi], lown, lnb, vh, hs, nb, nrhs, r, acc);
      hop_dir_mix<3, DAG, RECON>(P.gauge, P.in[yi], lown, lnb, vh, hs, nb, nrhs, r, acc);
    } else if (VAR & 2) {
#pragma unroll 1
      for (int mu = 0; mu < 4; ++mu) {
        switch (mu) {
          case 0: hop_dir<0, DAG, SP, GP, RECON>(P.gauge, P.in[yi], p, hs, nb, nrhs, r, acc); break;
          case 1: hop_dir<1, DAG, SP, GP, RECON>(P.gauge, P.in[yi], p, hs, nb, nrhs, r, acc); break;
          case 2: hop_dir<2, DAG, SP, GP, RECON>(P.gauge, P.in[yi], p, hs, nb, nrhs, r, acc); break;
          default: hop_dir<3, DAG, SP, GP, RECON>(P.gauge, P.in[yi], p, hs, nb, nrhs, r, acc); break;
        }
      }
    } else {
      hop_dir<0, DAG, SP, GP, RECON>(P.gauge, P.in[yi], p, hs, nb, nrhs, r, acc);
      hop_dir<1, DAG, SP, GP, RECON>(P.gauge, P.in[yi], p, hs, nb, nrhs, r, acc);
      hop_dir<2, DAG, SP, GP, RECON>(P.gauge, P.in[yi], p, hs, nb, nrhs, r, acc);
      hop_dir<3, DAG, SP, GP, RECON>(P.gauge, P.in[yi], p, hs, nb, nrhs, r, acc);
    }
    const R sc = R(P.scale);
    // the FP16 output of a plain hop takes the scale into the store's
    // normalisation instead of multiplying every component
    const bool fold = SP == PREC_HALF && EPI == EPI_SCALE && !P.cg;
    if (!fold) {
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[k] = sc * acc[k];
    }
    if (EPI == EPI_SCALE_CLOV) {
      CloverBlock<R> B[2];
      CloverIO<CP>::load(P.clov[yi], hs, B);
      clover_apply(B, acc);
    }
    Cx<R> xv[12];
    if (EPI == EPI_XPAY || EPI == EPI_XPAY_CLOV) {
      SpinorIO<SP>::load(P.xin[yi], tid, xv);
      Cx<R> ax[12];
#pragma unroll
      for (int k = 0; k < 12; ++k) ax[k] = xv[k];
      if (EPI == EPI_XPAY_CLOV) {
        CloverBlock<R> B[2];
        CloverIO<CP>::load(P.clov[yi], hs, B);
        clover_apply(B, ax);
      }
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[k] = ax[k] + acc[k];
    }
    if (P.cg) {
      // r -= alpha s; |r|^2 (the solver's ST_CG_BETA totals)
      const R a = R(P.cst[r].alpha);
      Cx<R> rv[12];
      SpinorIO<SP>::load(P.cr[yi], tid, rv);
      R rr = R(0);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        rv[k] = rv[k] - a * acc[k];
        rr += rv[k].re * rv[k].re + rv[k].im * rv[k].im;
      }
      SpinorIO<SP>::store(P.cr[yi], tid, rv);
      red[0] += double(rr);
      continue;
    }
    if constexpr (SP == PREC_HALF && EPI == EPI_SCALE) {
      if (fold)
        SpinorIO<SP>::store_scaled(P.out[yi], tid, acc, sc);
      else
        SpinorIO<SP>::store(P.out[yi], tid, acc);
    } else {
      SpinorIO<SP>::store(P.out[yi], tid, acc);
    }
    // per-site sums in the arithmetic precision, accumulated in FP64 across
    // sites (one conversion per sum instead of one per term)
    if (P.red_mask) {
      R o2 = R(0);
#pragma unroll
      for (int k = 0; k < 12; ++k) o2 += acc[k].re * acc[k].re + acc[k].im * acc[k].im;
      red[0] += double(fold ? o2 * sc * sc : o2);
    }
    if ((EPI == EPI_XPAY || EPI == EPI_XPAY_CLOV) && (P.red_mask & (RED_X2 | RED_XOUT))) {
      R x2 = R(0), xo = R(0);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        x2 += xv[k].re * xv[k].re + xv[k].im * xv[k].im;
        xo += xv[k].re * acc[k].re + xv[k].im * acc[k].im;
      }
      red[1] += double(x2);
      red[2] += double(xo);
    }
  }
  if (P.red_mask || P.cg)
    block_reduce_finish<3>(P.red, red, nrhs, blockIdx.y * gridDim.x + blockIdx.x,
                           gridDim.x * gridDim.y);
}

}  // namespace iro
