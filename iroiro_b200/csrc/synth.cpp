// Seeded synthetic inputs in the reference's host layouts.
//
// Gauge links follow Format_G (include/format_G.h:34-36): 18 doubles per
// link, row-major 3x3, re/im interleaved, index 18*(site + V*mu), site
// lexicographic x + Lx*(y + Ly*(z + Lz*t)) (lib/Geometry/siteIndex.cpp:41-43).
// Spinors follow Format_F (include/format_F.h:36-42): 24 doubles per site,
// index 2*(c + 3*s) + 24*site.
//
// Each link is U = exp(i*eps*H), H = sum_a theta_a*lambda_a/2 with theta_a
// ~ N(0,1) drawn from a counter-based generator keyed by (seed, site, mu), so
// the field does not depend on thread count or traversal order.  The
// exponential is a scaling-and-squaring Taylor series (Moler & Van Loan,
// "Nineteen dubious ways to compute the exponential of a matrix", method 3);
// the result is projected back onto SU(3) by Gram-Schmidt on the first two
// rows and row3 = conj(row1 x row2), so that reconstructing the third row
// from the first two is exact up to rounding.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>

#include "iroiro_b200.h"

namespace {

using cd = std::complex<double>;

struct M3 {
  cd a[3][3];
};

inline uint64_t splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Counter-based stream: value k of stream `key`.
struct Stream {
  uint64_t key;
  uint64_t k = 0;
  explicit Stream(uint64_t key_) : key(splitmix(key_)) {}
  double uniform() {  // in (0,1)
    uint64_t r = splitmix(key ^ splitmix(k++));
    return (double((r >> 11) + 1)) * (1.0 / 9007199254740993.0);
  }
  double normal() {  // Box-Muller, one value per pair of uniforms
    double u1 = uniform(), u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925 * u2);
  }
};

inline uint64_t key_of(uint64_t seed, uint64_t a, uint64_t b, uint64_t tag) {
  return splitmix(splitmix(splitmix(seed ^ (tag << 56)) ^ a) ^ (b + 0x632BE59BD9B4E019ull));
}

M3 mul(const M3& x, const M3& y) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      cd s = 0.0;
      for (int k = 0; k < 3; ++k) s += x.a[i][k] * y.a[k][j];
      r.a[i][j] = s;
    }
  return r;
}

M3 dag(const M3& x) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = std::conj(x.a[j][i]);
  return r;
}

// i*eps*H with H = sum_a theta_a lambda_a / 2 (Gell-Mann matrices).
M3 algebra(Stream& st, double eps) {
  double th[8];
  for (int a = 0; a < 8; ++a) th[a] = st.normal();
  const double s3 = 1.0 / std::sqrt(3.0);
  cd H[3][3];
  H[0][0] = 0.5 * (th[2] + th[7] * s3);
  H[1][1] = 0.5 * (-th[2] + th[7] * s3);
  H[2][2] = 0.5 * (-2.0 * th[7] * s3);
  H[0][1] = 0.5 * cd(th[0], -th[1]);
  H[1][0] = std::conj(H[0][1]);
  H[0][2] = 0.5 * cd(th[3], -th[4]);
  H[2][0] = std::conj(H[0][2]);
  H[1][2] = 0.5 * cd(th[5], -th[6]);
  H[2][1] = std::conj(H[1][2]);
  M3 X;
  const cd ie(0.0, eps);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) X.a[i][j] = ie * H[i][j];
  return X;
}

M3 expm(const M3& X) {
  double nrm = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) nrm += std::norm(X.a[i][j]);
  nrm = std::sqrt(nrm);
  int s = 0;
  while (nrm > 0.25) {
    nrm *= 0.5;
    ++s;
  }
  const double scale = std::ldexp(1.0, -s);
  M3 A;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A.a[i][j] = X.a[i][j] * scale;
  // Horner evaluation of sum_{n<=18} A^n/n!
  M3 E;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) E.a[i][j] = (i == j) ? 1.0 : 0.0;
  for (int n = 18; n >= 1; --n) {
    M3 T = mul(A, E);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) E.a[i][j] = ((i == j) ? 1.0 : 0.0) + T.a[i][j] / double(n);
  }
  for (int k = 0; k < s; ++k) E = mul(E, E);
  return E;
}

void project_su3(M3& U) {
  double n0 = 0.0;
  for (int j = 0; j < 3; ++j) n0 += std::norm(U.a[0][j]);
  n0 = 1.0 / std::sqrt(n0);
  for (int j = 0; j < 3; ++j) U.a[0][j] *= n0;
  cd p = 0.0;
  for (int j = 0; j < 3; ++j) p += std::conj(U.a[0][j]) * U.a[1][j];
  for (int j = 0; j < 3; ++j) U.a[1][j] -= p * U.a[0][j];
  double n1 = 0.0;
  for (int j = 0; j < 3; ++j) n1 += std::norm(U.a[1][j]);
  n1 = 1.0 / std::sqrt(n1);
  for (int j = 0; j < 3; ++j) U.a[1][j] *= n1;
  U.a[2][0] = std::conj(U.a[0][1] * U.a[1][2] - U.a[0][2] * U.a[1][1]);
  U.a[2][1] = std::conj(U.a[0][2] * U.a[1][0] - U.a[0][0] * U.a[1][2]);
  U.a[2][2] = std::conj(U.a[0][0] * U.a[1][1] - U.a[0][1] * U.a[1][0]);
}

inline M3 load(const double* p) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = cd(p[2 * (3 * i + j)], p[2 * (3 * i + j) + 1]);
  return r;
}

inline void save(const M3& m, double* p) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      p[2 * (3 * i + j)] = m.a[i][j].real();
      p[2 * (3 * i + j) + 1] = m.a[i][j].imag();
    }
}

bool lattice_ok(const int L[4]) {
  if (!L) return false;
  for (int d = 0; d < 4; ++d)
    if (L[d] < 2 || (L[d] & 1)) return false;
  return true;
}

}  // namespace

extern "C" {

int iro_synth_gauge(const int L[4], double eps, uint64_t seed, int gauge_transform, double* u) {
  if (!lattice_ok(L) || !u || !(eps >= 0.0)) return IRO_BAD_ARG;
  const int64_t V = int64_t(L[0]) * L[1] * L[2] * L[3];
#pragma omp parallel for schedule(static)
  for (int64_t site = 0; site < V; ++site) {
    for (int mu = 0; mu < 4; ++mu) {
      Stream st(key_of(seed, uint64_t(site), uint64_t(mu), 1));
      M3 U = expm(algebra(st, eps));
      project_su3(U);
      save(U, u + 18 * (site + V * mu));
    }
  }
  if (!gauge_transform) return IRO_OK;
  // U_mu(x) -> G(x) U_mu(x) G(x+mu)^dagger with G(x) = exp(i*H), H from the
  // same algebra distribution with unit width.
  auto G = [&](int64_t site) {
    Stream st(key_of(seed, uint64_t(site), 0, 2));
    M3 g = expm(algebra(st, 1.0));
    project_su3(g);
    return g;
  };
#pragma omp parallel for schedule(static)
  for (int64_t site = 0; site < V; ++site) {
    int64_t c[4];
    int64_t r = site;
    for (int d = 0; d < 4; ++d) {
      c[d] = r % L[d];
      r /= L[d];
    }
    const M3 gx = G(site);
    for (int mu = 0; mu < 4; ++mu) {
      int64_t n[4] = {c[0], c[1], c[2], c[3]};
      n[mu] = (n[mu] + 1) % L[mu];
      const int64_t nb = n[0] + L[0] * (n[1] + L[1] * (n[2] + L[2] * n[3]));
      double* p = u + 18 * (site + V * mu);
      M3 U = mul(mul(gx, load(p)), dag(G(nb)));
      project_su3(U);
      save(U, p);
    }
  }
  return IRO_OK;
}

int iro_synth_gaussian(int64_t nsites, uint64_t seed, double* f) {
  if (nsites < 0 || (!f && nsites > 0)) return IRO_BAD_ARG;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < nsites; ++s) {
    Stream st(key_of(seed, uint64_t(s), 0, 3));
    for (int k = 0; k < 24; ++k) f[24 * s + k] = st.normal();
  }
  return IRO_OK;
}

int iro_synth_point_sources(int64_t nsites, int64_t site, double* f12) {
  if (nsites <= 0 || site < 0 || site >= nsites || !f12) return IRO_BAD_ARG;
  std::memset(f12, 0, sizeof(double) * size_t(12) * 24 * size_t(nsites));
  // source k = c + 3*s has 1.0 at index_r(c,s,site) (Source_local,
  // lib/Measurements/FermionicM/source_types.hpp:40-60)
  for (int k = 0; k < 12; ++k) f12[size_t(k) * 24 * nsites + 24 * site + 2 * k] = 1.0;
  return IRO_OK;
}

}  // extern "C"
