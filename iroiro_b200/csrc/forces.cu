// Molecular-dynamics force of the Wilson operator, the outer product of two
// spinor fields through the hopping term:
//   F_mu(x)_{ab} += w sum_s [(1 - g_mu) U_mu(x) psi(x+mu)]_{a,s} conj(chi(x)_{b,s})
// (Dirac_Wilson::mkfrc, lib/Dirac_ops/dirac_wilson.cpp:60-91, with
// mult_p[mu] the forward hop of lib/Dirac_ops/dirac_wilson_improved.code).
// md_force of the full operator (dirac_wilson.cpp:41-58) and of the e/o
// Schur operator (lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:95-117) are sums of
// such terms over both parities, with gamma5 applied to both fields in the
// "m" terms.  FP64 throughout (the force of the reference's HMC).
//
// One thread per (half-site, direction); direction-major so that a warp's
// spinor and link loads are coalesced and its branches uniform.  The force
// is accumulated in the reference's Format_G order [mu][site][3][3][re,im]
// on the device; each term is one launch that reads and writes F, so the
// summation order is fixed.
#include <cstring>

#include "dslash.cuh"
#include "internal.h"
#include "iroiro_b200.h"

namespace iro {

__device__ __forceinline__ void gamma5_swap(Cx<double> v[12]) {
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const Cx<double> t = v[k];
    v[k] = v[k + 6];
    v[k + 6] = t;
  }
}

template <int MU, int RECON>
__device__ __forceinline__ void force_term(const Geom& g, const GaugePtr& gauge, int p, int hs,
                                           const SpinorPtr& psi, const SpinorPtr& chi, bool g5,
                                           double w, double* __restrict__ F) {
  const Coord c = coord_of(g, hs, p);
  int nb[8];
  neighbours(g, c, hs, nb);
  Cx<double> f[12], h[6], gv[6], xie[12], ch[12];
  SpinorIO<PREC_DOUBLE>::load(psi, nb[2 * MU], f);
  if (g5) gamma5_swap(f);
  project<MU, 1, double>(f, h);
  Su3<double> U;
  GaugeIO<PREC_DOUBLE, RECON>::load(gauge, p, MU, hs, U);
  su3_mul(U, h, gv);
#pragma unroll
  for (int k = 0; k < 12; ++k) xie[k] = {0.0, 0.0};
  reconstruct<MU, 1, double>(xie, gv);
  SpinorIO<PREC_DOUBLE>::load(chi, hs, ch);
  if (g5) gamma5_swap(ch);
  const int64_t V = 2 * int64_t(g.Vh);
  const int64_t lex = c.x + int64_t(g.L[0]) * (c.y + int64_t(g.L[1]) * (c.z + int64_t(g.L[2]) * c.t));
  double* Fp = F + (int64_t(MU) * V + lex) * 18;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      Cx<double> s = {0.0, 0.0};
#pragma unroll
      for (int sp = 0; sp < 4; ++sp) s = s + xie[3 * sp + a] * conjx(ch[3 * sp + b]);
      Fp[2 * (3 * a + b)] += w * s.re;
      Fp[2 * (3 * a + b) + 1] += w * s.im;
    }
}

template <int RECON>
__global__ void __launch_bounds__(128) force_kernel(Geom g, GaugePtr gauge, int p, SpinorPtr psi,
                                                    SpinorPtr chi, int g5, double w, double* F) {
  const int64_t n = 4 * int64_t(g.Vh);
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int mu = int(i / g.Vh);
    const int hs = int(i - int64_t(mu) * g.Vh);
    switch (mu) {
      case 0: force_term<0, RECON>(g, gauge, p, hs, psi, chi, g5 != 0, w, F); break;
      case 1: force_term<1, RECON>(g, gauge, p, hs, psi, chi, g5 != 0, w, F); break;
      case 2: force_term<2, RECON>(g, gauge, p, hs, psi, chi, g5 != 0, w, F); break;
      default: force_term<3, RECON>(g, gauge, p, hs, psi, chi, g5 != 0, w, F); break;
    }
  }
}

cudaError_t launch_force(const Geom& g, const GaugePtr& gauge, int recon, int p, SpinorPtr psi,
                         SpinorPtr chi, int g5, double w, double* F, cudaStream_t st) {
  const int64_t n = 4 * int64_t(g.Vh);
  const int blk = 128;
  int grid = int((n + blk - 1) / blk);
  if (grid > 148 * 16) grid = 148 * 16;
  if (recon == 12)
    force_kernel<12><<<grid, blk, 0, st>>>(g, gauge, p, psi, chi, g5, w, F);
  else
    force_kernel<18><<<grid, blk, 0, st>>>(g, gauge, p, psi, chi, g5, w, F);
  return cudaGetLastError();
}

}  // namespace iro
