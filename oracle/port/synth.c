/* Seeded synthetic inputs for the oracle side -- TEST INFRASTRUCTURE ONLY.
 *
 * The benchmark's reference arm and the tests that run the reference's own
 * classes need the same seeded gauge fields and sources as the device path,
 * without loading the product library.  These functions restate, in plain C,
 * the generator of the product's iro_synth_gauge / iro_synth_gaussian /
 * iro_synth_point_sources, operation for operation, so that both sides see
 * bit-identical inputs (tests/test_synth.py checks this):
 *
 *   U_mu(x) = exp(i eps H), H = sum_a theta_a lambda_a / 2, theta_a ~ N(0,1)
 *   from a counter-based SplitMix64 stream keyed by (seed, site, mu); the
 *   exponential by scaling and squaring with an order-18 Taylor polynomial
 *   (Moler & Van Loan, "Nineteen dubious ways to compute the exponential of
 *   a matrix", method 3); projection to SU(3) by Gram-Schmidt on rows 0 and
 *   1, row 2 = conj(row0 x row1); an optional gauge transformation
 *   U_mu(x) -> G(x) U_mu(x) G(x+mu)^dag with G drawn the same way at eps = 1.
 *
 * Layouts are the reference's: Format_G 2*(3*a+b) + 18*(site + V*mu)
 * (include/format_G.h:34-36), Format_F 2*(c+3*s) + 24*site
 * (include/format_F.h:36-42), site = x + Lx*(y + Ly*(z + Lz*t))
 * (lib/Geometry/siteIndex.cpp:41-43).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "iro_oracle.h"

typedef double complex cplx;

typedef struct {
  cplx a[3][3];
} SM3;

static uint64_t splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

typedef struct {
  uint64_t key, k;
} Rng;

static Rng rng_of(uint64_t key) {
  Rng r = {splitmix(key), 0};
  return r;
}

static double rng_uniform(Rng* r) { /* in (0,1) */
  uint64_t v = splitmix(r->key ^ splitmix(r->k++));
  return (double)((v >> 11) + 1) * (1.0 / 9007199254740993.0);
}

static double rng_normal(Rng* r) { /* Box-Muller, one value per pair */
  double u1 = rng_uniform(r), u2 = rng_uniform(r);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925 * u2);
}

static uint64_t key_of(uint64_t seed, uint64_t a, uint64_t b, uint64_t tag) {
  return splitmix(splitmix(splitmix(seed ^ (tag << 56)) ^ a) ^ (b + 0x632BE59BD9B4E019ull));
}

static SM3 sm_mul(const SM3* x, const SM3* y) {
  SM3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      cplx s = 0.0;
      for (int k = 0; k < 3; ++k) s += x->a[i][k] * y->a[k][j];
      r.a[i][j] = s;
    }
  return r;
}

static SM3 sm_dag(const SM3* x) {
  SM3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = conj(x->a[j][i]);
  return r;
}

static cplx mk(double re, double im) {
  cplx z;
  __real__ z = re;
  __imag__ z = im;
  return z;
}

/* i*eps*H, H = sum_a theta_a lambda_a / 2 (Gell-Mann basis) */
static SM3 algebra(Rng* st, double eps) {
  double th[8];
  for (int a = 0; a < 8; ++a) th[a] = rng_normal(st);
  const double s3 = 1.0 / sqrt(3.0);
  cplx H[3][3];
  H[0][0] = mk(0.5 * (th[2] + th[7] * s3), 0.0);
  H[1][1] = mk(0.5 * (-th[2] + th[7] * s3), 0.0);
  H[2][2] = mk(0.5 * (-2.0 * th[7] * s3), 0.0);
  H[0][1] = mk(0.5 * th[0], 0.5 * -th[1]);
  H[1][0] = conj(H[0][1]);
  H[0][2] = mk(0.5 * th[3], 0.5 * -th[4]);
  H[2][0] = conj(H[0][2]);
  H[1][2] = mk(0.5 * th[5], 0.5 * -th[6]);
  H[2][1] = conj(H[1][2]);
  SM3 X;
  const cplx ie = mk(0.0, eps);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) X.a[i][j] = ie * H[i][j];
  return X;
}

static double cnorm2(cplx z) { return creal(z) * creal(z) + cimag(z) * cimag(z); }

static SM3 expm(const SM3* X) {
  double nrm = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) nrm += cnorm2(X->a[i][j]);
  nrm = sqrt(nrm);
  int s = 0;
  while (nrm > 0.25) {
    nrm *= 0.5;
    ++s;
  }
  const double scale = ldexp(1.0, -s);
  SM3 A;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A.a[i][j] = mk(creal(X->a[i][j]) * scale, cimag(X->a[i][j]) * scale);
  SM3 E;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) E.a[i][j] = (i == j) ? 1.0 : 0.0;
  for (int n = 18; n >= 1; --n) {
    SM3 T = sm_mul(&A, &E);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        E.a[i][j] = mk(((i == j) ? 1.0 : 0.0) + creal(T.a[i][j]) / (double)n,
                       cimag(T.a[i][j]) / (double)n);
  }
  for (int k = 0; k < s; ++k) E = sm_mul(&E, &E);
  return E;
}

static void project_su3(SM3* U) {
  double n0 = 0.0;
  for (int j = 0; j < 3; ++j) n0 += cnorm2(U->a[0][j]);
  n0 = 1.0 / sqrt(n0);
  for (int j = 0; j < 3; ++j) U->a[0][j] = mk(creal(U->a[0][j]) * n0, cimag(U->a[0][j]) * n0);
  cplx p = 0.0;
  for (int j = 0; j < 3; ++j) p += conj(U->a[0][j]) * U->a[1][j];
  for (int j = 0; j < 3; ++j) U->a[1][j] -= p * U->a[0][j];
  double n1 = 0.0;
  for (int j = 0; j < 3; ++j) n1 += cnorm2(U->a[1][j]);
  n1 = 1.0 / sqrt(n1);
  for (int j = 0; j < 3; ++j) U->a[1][j] = mk(creal(U->a[1][j]) * n1, cimag(U->a[1][j]) * n1);
  U->a[2][0] = conj(U->a[0][1] * U->a[1][2] - U->a[0][2] * U->a[1][1]);
  U->a[2][1] = conj(U->a[0][2] * U->a[1][0] - U->a[0][0] * U->a[1][2]);
  U->a[2][2] = conj(U->a[0][0] * U->a[1][1] - U->a[0][1] * U->a[1][0]);
}

static SM3 sm_load(const double* p) {
  SM3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = mk(p[2 * (3 * i + j)], p[2 * (3 * i + j) + 1]);
  return r;
}

static void sm_save(const SM3* m, double* p) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      p[2 * (3 * i + j)] = creal(m->a[i][j]);
      p[2 * (3 * i + j) + 1] = cimag(m->a[i][j]);
    }
}

static SM3 transform_at(uint64_t seed, int64_t site) {
  Rng st = rng_of(key_of(seed, (uint64_t)site, 0, 2));
  SM3 x = algebra(&st, 1.0);
  SM3 g = expm(&x);
  project_su3(&g);
  return g;
}

int orc_synth_gauge(const int L[4], double eps, unsigned long long seed, int gauge_transform,
                    double* u) {
  for (int d = 0; d < 4; ++d)
    if (L[d] < 2 || (L[d] & 1)) return 1;
  const int64_t V = (int64_t)L[0] * L[1] * L[2] * L[3];
#pragma omp parallel for schedule(static)
  for (int64_t site = 0; site < V; ++site) {
    for (int mu = 0; mu < 4; ++mu) {
      Rng st = rng_of(key_of(seed, (uint64_t)site, (uint64_t)mu, 1));
      SM3 x = algebra(&st, eps);
      SM3 U = expm(&x);
      project_su3(&U);
      sm_save(&U, u + 18 * (site + V * mu));
    }
  }
  if (!gauge_transform) return 0;
#pragma omp parallel for schedule(static)
  for (int64_t site = 0; site < V; ++site) {
    int64_t c[4];
    int64_t r = site;
    for (int d = 0; d < 4; ++d) {
      c[d] = r % L[d];
      r /= L[d];
    }
    const SM3 gx = transform_at(seed, site);
    for (int mu = 0; mu < 4; ++mu) {
      int64_t n[4] = {c[0], c[1], c[2], c[3]};
      n[mu] = (n[mu] + 1) % L[mu];
      const int64_t nb = n[0] + L[0] * (n[1] + L[1] * (n[2] + L[2] * n[3]));
      double* p = u + 18 * (site + V * mu);
      SM3 U0 = sm_load(p);
      SM3 gn = transform_at(seed, nb);
      SM3 gd = sm_dag(&gn);
      SM3 t = sm_mul(&gx, &U0);
      SM3 U = sm_mul(&t, &gd);
      project_su3(&U);
      sm_save(&U, p);
    }
  }
  return 0;
}

int orc_synth_gaussian(long long nsites, unsigned long long seed, double* f) {
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < nsites; ++s) {
    Rng st = rng_of(key_of(seed, (uint64_t)s, 0, 3));
    for (int k = 0; k < 24; ++k) f[24 * s + k] = rng_normal(&st);
  }
  return 0;
}
