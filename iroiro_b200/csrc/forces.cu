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
#include <cstdint>
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

// ---- the clover term's force -----------------------------------------------------
// Dirac_Clover::md_force (lib/Dirac_ops/dirac_clover.cpp:356-367; its block
// md_force_block :369-532) adds to the Wilson force the derivative of the
// clover term T f = -kappa csw sum_k (i sigma_k (x) F_k) f, F_k = 0.25 TA(Q_k),
// Q_k(x) = L1 - L2 + L3 - L4 the four leaves at x in the plane of k
// (Staples::fieldStrength, staples.cpp:587-666), TA the traceless
// anti-hermitian part.  TA is self-adjoint for Re Tr, so
//   Re(zeta^dag T eta) = -kappa csw / 4 sum_{x,k} Re Tr(Q_k(x) Lambda_k(x)),
//   Lambda_k(x) = TA(sum_{s,t} (i sigma_k)_{st} eta_t(x) zeta_s(x)^dag),
// and a link occurring as A U B in a leaf gets U B Lambda A in its force, as
// A U^dag B gets U A^dag Lambda^dag B^dag (the convention of the Wilson force:
// Re Tr(X F_mu(x)) = d/de Re(zeta^dag D(U_mu(x) -> (1 + e X) U_mu(x)) eta)).
// FP64 throughout, on the resident Format_G links.

using M3d = Su3<double>;

__device__ __forceinline__ M3d m3_mul(const M3d& A, const M3d& B) {
  M3d C;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      Cx<double> s = A.e[a][0] * B.e[0][b];
      s = s + A.e[a][1] * B.e[1][b];
      s = s + A.e[a][2] * B.e[2][b];
      C.e[a][b] = s;
    }
  return C;
}

__device__ __forceinline__ M3d m3_dag(const M3d& A) {
  M3d C;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) C.e[a][b] = conjx(A.e[b][a]);
  return C;
}

__device__ __forceinline__ M3d m3_unit() {
  M3d C;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) C.e[a][b] = {a == b ? 1.0 : 0.0, 0.0};
  return C;
}

// link (site, mu) of a Format_G array
__device__ __forceinline__ M3d load_g(const double* __restrict__ u, int64_t V, int64_t site, int mu) {
  const double2* p = reinterpret_cast<const double2*>(u + 18 * (site + V * mu));
  M3d U;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double2 v = __ldg(p + k);
    U.e[k / 3][k % 3] = {v.x, v.y};
  }
  return U;
}

// i sigma_k, k = Bx,By,Bz,Ex,Ey,Ez (Dirac_Clover::isigma_{23,31,12,41,42,43},
// dirac_clover.cpp:221-329): row s has one entry, coef[k][s] at column perm[k][s]
__constant__ int c_sig_perm[6][4] = {{1, 0, 3, 2}, {1, 0, 3, 2}, {0, 1, 2, 3},
                                     {3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}};
__constant__ double2 c_sig_coef[6][4] = {
    {{0, 1}, {0, 1}, {0, 1}, {0, 1}},     {{1, 0}, {-1, 0}, {1, 0}, {-1, 0}},
    {{0, 1}, {0, -1}, {0, 1}, {0, -1}},   {{0, -1}, {0, -1}, {0, -1}, {0, -1}},
    {{-1, 0}, {1, 0}, {-1, 0}, {1, 0}},   {{0, -1}, {0, 1}, {0, -1}, {0, 1}}};

// Lambda_k(x) for the 6 planes, lam[(k V + lex) 9 + 3 row + col]
__global__ void __launch_bounds__(128) clover_lambda_kernel(Geom g, SpinorPtr e0, SpinorPtr e1,
                                                            SpinorPtr z0, SpinorPtr z1,
                                                            double2* __restrict__ lam) {
  const int64_t V = 2 * int64_t(g.Vh);
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < V;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int p = int(i / g.Vh);
    const int hs = int(i - int64_t(p) * g.Vh);
    const Coord c = coord_of(g, hs, p);
    const int64_t lex = c.x + int64_t(g.L[0]) * (c.y + int64_t(g.L[1]) * (c.z + int64_t(g.L[2]) * c.t));
    Cx<double> et[12], zt[12];
    SpinorIO<PREC_DOUBLE>::load(p ? e1 : e0, hs, et);
    SpinorIO<PREC_DOUBLE>::load(p ? z1 : z0, hs, zt);
    for (int k = 0; k < 6; ++k) {
      M3d M;
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          Cx<double> s = {0.0, 0.0};
#pragma unroll
          for (int sp = 0; sp < 4; ++sp) {
            const double2 cf = c_sig_coef[k][sp];
            const int t = c_sig_perm[k][sp];
            s = s + Cx<double>{cf.x, cf.y} * et[3 * t + b] * conjx(zt[3 * sp + a]);
          }
          M.e[b][a] = s;
        }
      // traceless anti-hermitian part
      M3d A;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          A.e[a][b] = {0.5 * (M.e[a][b].re - M.e[b][a].re), 0.5 * (M.e[a][b].im + M.e[b][a].im)};
        }
      const double imtr = (A.e[0][0].im + A.e[1][1].im + A.e[2][2].im) / 3.0;
#pragma unroll
      for (int a = 0; a < 3; ++a) A.e[a][a].im -= imtr;
      double2* out = lam + (int64_t(k) * V + lex) * 9;
#pragma unroll
      for (int q = 0; q < 9; ++q) out[q] = make_double2(A.e[q / 3][q % 3].re, A.e[q / 3][q % 3].im);
    }
  }
}

// One factor occurrence of a link in a leaf: the leaf of plane k with sign
// `sign`, its four factors (direction, offset from the leaf's site, dagger),
// the varied factor `i`.  Grouped by the varied factor's direction.
struct CloverTerm {
  int8_t k, sign, i, pad;
  int8_t dir[4], dag[4];
  int8_t off[4][4];
};
constexpr int kTermsPerDir = 24;
__constant__ CloverTerm c_terms[4][kTermsPerDir];

__device__ __forceinline__ int64_t wrap_site(const Geom& g, const int c[4]) {
  int w[4];
#pragma unroll
  for (int d = 0; d < 4; ++d) w[d] = c[d] < 0 ? c[d] + g.L[d] : (c[d] >= g.L[d] ? c[d] - g.L[d] : c[d]);
  return w[0] + int64_t(g.L[0]) * (w[1] + int64_t(g.L[1]) * (w[2] + int64_t(g.L[2]) * w[3]));
}

// thread per link (rho, y): F_rho(y) += w sum of its 24 occurrences, in table order
__global__ void __launch_bounds__(128) clover_force_kernel(Geom g, const double* __restrict__ u,
                                                           const double2* __restrict__ lam,
                                                           double w, double* __restrict__ F) {
  const int64_t V = 2 * int64_t(g.Vh);
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < 4 * V;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int rho = int(i / V);
    const int64_t y = i - int64_t(rho) * V;
    int cy[4];
    {
      int64_t r = y;
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        cy[d] = int(r % g.L[d]);
        r /= g.L[d];
      }
    }
    const M3d Uy = load_g(u, V, y, rho);
    M3d acc;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) acc.e[a][b] = {0.0, 0.0};
    for (int t = 0; t < kTermsPerDir; ++t) {
      const CloverTerm& T = c_terms[rho][t];
      // the leaf's site x = y - off[i]
      int cx[4];
#pragma unroll
      for (int d = 0; d < 4; ++d) cx[d] = cy[d] - T.off[T.i][d];
      M3d A = m3_unit(), B = m3_unit();
      for (int j = 0; j < 4; ++j) {
        if (j == T.i) continue;
        int cj[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) cj[d] = cx[d] + T.off[j][d];
        M3d Fj = load_g(u, V, wrap_site(g, cj), T.dir[j]);
        if (T.dag[j]) Fj = m3_dag(Fj);
        if (j < T.i) A = m3_mul(A, Fj);
        else B = m3_mul(B, Fj);
      }
      int64_t xs;
      {
        int c0[4] = {cx[0], cx[1], cx[2], cx[3]};
        xs = wrap_site(g, c0);
      }
      M3d Lam;
      const double2* lp = lam + (int64_t(T.k) * V + xs) * 9;
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        const double2 v = __ldg(lp + q);
        Lam.e[q / 3][q % 3] = {v.x, v.y};
      }
      const M3d C = T.dag[T.i] ? m3_mul(m3_mul(m3_mul(Uy, m3_dag(A)), m3_dag(Lam)), m3_dag(B))
                               : m3_mul(m3_mul(m3_mul(Uy, B), Lam), A);
      const double sg = T.sign;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) acc.e[a][b] = acc.e[a][b] + sg * C.e[a][b];
    }
    double* Fp = F + 18 * (y + V * rho);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        Fp[2 * (3 * a + b)] += w * acc.e[a][b].re;
        Fp[2 * (3 * a + b) + 1] += w * acc.e[a][b].im;
      }
  }
}

// The 96 occurrences, from the leaves of Q_{mu nu}(x) (planes in the order of
// Bx..Ez, set_csw dirac_clover.cpp:139-162):
//   L1 = U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag           (+)
//   L2 = U_mu(x) U_nu(x+mu-nu)^dag U_mu(x-nu)^dag U_nu(x-nu)      (-)
//   L3 = U_nu(x) U_mu(x-mu+nu)^dag U_nu(x-mu)^dag U_mu(x-mu)      (+)
//   L4 = U_nu(x-nu)^dag U_mu(x-mu-nu)^dag U_nu(x-mu-nu) U_mu(x-mu) (-)
static cudaError_t clover_terms_upload() {
  static bool done = false;
  if (done) return cudaSuccess;
  const int pairs[6][2] = {{1, 2}, {2, 0}, {0, 1}, {3, 0}, {3, 1}, {3, 2}};
  CloverTerm tab[4][kTermsPerDir];
  int n[4] = {0, 0, 0, 0};
  for (int k = 0; k < 6; ++k) {
    const int mu = pairs[k][0], nu = pairs[k][1];
    int e_mu[4] = {0, 0, 0, 0}, e_nu[4] = {0, 0, 0, 0};
    e_mu[mu] = 1;
    e_nu[nu] = 1;
    struct F { int dir, dag, o_mu, o_nu; };
    const F leaves[4][4] = {
        {{mu, 0, 0, 0}, {nu, 0, 1, 0}, {mu, 1, 0, 1}, {nu, 1, 0, 0}},
        {{mu, 0, 0, 0}, {nu, 1, 1, -1}, {mu, 1, 0, -1}, {nu, 0, 0, -1}},
        {{nu, 0, 0, 0}, {mu, 1, -1, 1}, {nu, 1, -1, 0}, {mu, 0, -1, 0}},
        {{nu, 1, 0, -1}, {mu, 1, -1, -1}, {nu, 0, -1, -1}, {mu, 0, -1, 0}}};
    const int signs[4] = {1, -1, 1, -1};
    for (int l = 0; l < 4; ++l)
      for (int i = 0; i < 4; ++i) {
        CloverTerm T;
        std::memset(&T, 0, sizeof(T));
        T.k = int8_t(k);
        T.sign = int8_t(signs[l]);
        T.i = int8_t(i);
        for (int j = 0; j < 4; ++j) {
          T.dir[j] = int8_t(leaves[l][j].dir);
          T.dag[j] = int8_t(leaves[l][j].dag);
          for (int d = 0; d < 4; ++d)
            T.off[j][d] = int8_t(leaves[l][j].o_mu * e_mu[d] + leaves[l][j].o_nu * e_nu[d]);
        }
        const int r = leaves[l][i].dir;
        if (n[r] >= kTermsPerDir) return cudaErrorInvalidValue;
        tab[r][n[r]++] = T;
      }
  }
  for (int r = 0; r < 4; ++r)
    if (n[r] != kTermsPerDir) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemcpyToSymbol(c_terms, tab, sizeof(tab));
  if (e == cudaSuccess) done = true;
  return e;
}

cudaError_t launch_clover_force(const Geom& g, const double* u, SpinorPtr e0, SpinorPtr e1,
                                SpinorPtr z0, SpinorPtr z1, double w, double2* lam, double* F,
                                cudaStream_t st) {
  cudaError_t e = clover_terms_upload();
  if (e != cudaSuccess) return e;
  const int64_t V = 2 * int64_t(g.Vh);
  int grid = int((V + 127) / 128);
  if (grid > 148 * 16) grid = 148 * 16;
  clover_lambda_kernel<<<grid, 128, 0, st>>>(g, e0, e1, z0, z1, lam);
  grid = int((4 * V + 127) / 128);
  if (grid > 148 * 16) grid = 148 * 16;
  clover_force_kernel<<<grid, 128, 0, st>>>(g, u, lam, w, F);
  return cudaGetLastError();
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
