/* CPU oracle: plain-C restatement of the reference's fermion-solve hot path.
 *
 * TEST INFRASTRUCTURE ONLY -- loaded by the tests, the smoke check and the
 * benchmark's CPU-baseline leg, to check results against; never by the product.
 *
 * Written for clarity, not speed: every operator is applied literally from
 * its definition with explicit 4x4 spin matrices, so that it checks the
 * projector algebra the GPU kernels use rather than repeating it.
 *
 * Conventions (all from the reference):
 *   Format_F  2*(c+3*s) + 24*site            include/format_F.h:36-42
 *   Format_G  2*(3*c1+c2) + 18*(site+V*mu)   include/format_G.h:34-36
 *   site      x + Lx*(y + Ly*(z + Lz*t))     lib/Geometry/siteIndex.cpp:41-43
 *   e/o half fields list the even (odd) sites in lexicographic order
 *                                            lib/Geometry/siteIndex_EvenOdd.cpp:38-47
 *   gamma matrices (Dirac-Pauli basis)       lib/Dirac_ops/wilsonLikeUtils.cpp:9-53
 *   kappa = 0.5/(4+mass)                     lib/Dirac_ops/dirac_wilson.hpp:93
 */
#include "iro_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* ---- geometry ------------------------------------------------------------ */

typedef struct {
  int L[4];
  long V, Vh;
  long* eo_site; /* [2][Vh] lexicographic site of the hs-th even/odd site */
  long* half_of; /* [V] hs of a site within its parity */
  int* parity;   /* [V] */
  long* nb;      /* [V][8] neighbour along +dir (2*dir) and -dir (2*dir+1), periodic */
} Geom;

/* The tables of the last lattice used stay cached: every operator call of a
   solve would otherwise rebuild them. */
static Geom g_cache;
static int g_cache_valid = 0;

static void geom_build(Geom* g, const int L[4]) {
  for (int d = 0; d < 4; ++d) g->L[d] = L[d];
  g->V = (long)L[0] * L[1] * L[2] * L[3];
  g->Vh = g->V / 2;
  g->eo_site = malloc(sizeof(long) * g->V);
  g->half_of = malloc(sizeof(long) * g->V);
  g->parity = malloc(sizeof(int) * g->V);
  g->nb = malloc(sizeof(long) * 8 * g->V);
  long n[2] = {0, 0};
  for (long s = 0; s < g->V; ++s) {
    long r = s;
    int sum = 0;
    for (int d = 0; d < 4; ++d) {
      sum += (int)(r % L[d]);
      r /= L[d];
    }
    int p = sum & 1;
    g->parity[s] = p;
    g->half_of[s] = n[p];
    g->eo_site[p * g->Vh + n[p]] = s;
    ++n[p];
  }
#pragma omp parallel for schedule(static)
  for (long s = 0; s < g->V; ++s) {
    long c[4];
    long r = s;
    for (int d = 0; d < 4; ++d) {
      c[d] = r % L[d];
      r /= L[d];
    }
    for (int dir = 0; dir < 4; ++dir)
      for (int k = 0; k < 2; ++k) {
        long e[4] = {c[0], c[1], c[2], c[3]};
        e[dir] = (e[dir] + (k ? -1 : 1) + L[dir]) % L[dir];
        g->nb[8 * s + 2 * dir + k] = e[0] + L[0] * (e[1] + L[1] * (e[2] + L[2] * e[3]));
      }
  }
}

static void geom_init(Geom* g, const int L[4]) {
  int same = g_cache_valid;
  for (int d = 0; d < 4 && same; ++d) same = g_cache.L[d] == L[d];
  if (!same) {
    if (g_cache_valid) {
      free(g_cache.eo_site);
      free(g_cache.half_of);
      free(g_cache.parity);
      free(g_cache.nb);
    }
    geom_build(&g_cache, L);
    g_cache_valid = 1;
  }
  *g = g_cache;
}

static void geom_free(Geom* g) { (void)g; /* the cache owns the tables */ }

/* neighbour of `site` one step along +dir (sgn=+1) or -dir (sgn=-1), periodic */
static long neighbour(const Geom* g, long site, int dir, int sgn) {
  return g->nb[8 * site + 2 * dir + (sgn < 0)];
}

/* ---- spin algebra ---------------------------------------------------------- */

/* gamma_mu as 4x4 matrices, read off GammaMatrix::gamma{X,Y,Z,T}core
   (lib/Dirac_ops/wilsonLikeUtils.cpp:9-40): (gamma f)_s = sum_t G[s][t] f_t */
static cplx GAM[4][4][4];
/* i sigma_{mu nu} spin matrices of Dirac_Clover::isigma_{23,31,12,41,42,43}
   (lib/Dirac_ops/dirac_clover.cpp:221-329), in the order Bx,By,Bz,Ex,Ey,Ez */
static cplx SIG[6][4][4];
static int spin_ready = 0;

static void spin_init(void) {
  if (spin_ready) return;
  memset(GAM, 0, sizeof(GAM));
  memset(SIG, 0, sizeof(SIG));
  /* gamma_x: w0=-i f3, w1=-i f2, w2=i f1, w3=i f0 */
  GAM[0][0][3] = -I; GAM[0][1][2] = -I; GAM[0][2][1] = I; GAM[0][3][0] = I;
  /* gamma_y: w0=-f3, w1=f2, w2=f1, w3=-f0 */
  GAM[1][0][3] = -1; GAM[1][1][2] = 1; GAM[1][2][1] = 1; GAM[1][3][0] = -1;
  /* gamma_z: w0=-i f2, w1=i f3, w2=i f0, w3=-i f1 */
  GAM[2][0][2] = -I; GAM[2][1][3] = I; GAM[2][2][0] = I; GAM[2][3][1] = -I;
  /* gamma_t = diag(1,1,-1,-1) */
  GAM[3][0][0] = 1; GAM[3][1][1] = 1; GAM[3][2][2] = -1; GAM[3][3][3] = -1;
  /* isigma_23: w0=i v1, w1=i v0, w2=i v3, w3=i v2 */
  SIG[0][0][1] = I; SIG[0][1][0] = I; SIG[0][2][3] = I; SIG[0][3][2] = I;
  /* isigma_31: w0=v1, w1=-v0, w2=v3, w3=-v2 */
  SIG[1][0][1] = 1; SIG[1][1][0] = -1; SIG[1][2][3] = 1; SIG[1][3][2] = -1;
  /* isigma_12: w0=i v0, w1=-i v1, w2=i v2, w3=-i v3 */
  SIG[2][0][0] = I; SIG[2][1][1] = -I; SIG[2][2][2] = I; SIG[2][3][3] = -I;
  /* isigma_41: w0=-i v3, w1=-i v2, w2=-i v1, w3=-i v0 */
  SIG[3][0][3] = -I; SIG[3][1][2] = -I; SIG[3][2][1] = -I; SIG[3][3][0] = -I;
  /* isigma_42: w0=-v3, w1=v2, w2=-v1, w3=v0 */
  SIG[4][0][3] = -1; SIG[4][1][2] = 1; SIG[4][2][1] = -1; SIG[4][3][0] = 1;
  /* isigma_43: w0=-i v2, w1=i v3, w2=-i v0, w3=i v1 */
  SIG[5][0][2] = -I; SIG[5][1][3] = I; SIG[5][2][0] = -I; SIG[5][3][1] = I;
  spin_ready = 1;
}

static inline cplx fget(const double* f, long site, int s, int c) {
  const double* p = f + 24 * site + 2 * (c + 3 * s);
  return p[0] + I * p[1];
}
static inline void fadd(double* f, long site, int s, int c, cplx v) {
  double* p = f + 24 * site + 2 * (c + 3 * s);
  p[0] += creal(v);
  p[1] += cimag(v);
}
static inline cplx uget(const double* u, long V, long site, int mu, int a, int b) {
  const double* p = u + 18 * (site + V * mu) + 2 * (3 * a + b);
  return p[0] + I * p[1];
}

/* GammaMatrix::gamma5core: spins 0<->2, 1<->3 (wilsonLikeUtils.cpp:42-49) */
void orc_gamma5(long nsites, const double* in, double* out) {
  for (long s = 0; s < nsites; ++s) {
    const double* f = in + 24 * s;
    double tmp[24];
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 2; ++k) {
        tmp[2 * (c + 0) + k] = f[2 * (c + 6) + k];
        tmp[2 * (c + 3) + k] = f[2 * (c + 9) + k];
        tmp[2 * (c + 6) + k] = f[2 * (c + 0) + k];
        tmp[2 * (c + 9) + k] = f[2 * (c + 3) + k];
      }
    memcpy(out + 24 * s, tmp, sizeof(tmp));
  }
}

/* ---- Wilson hopping term ------------------------------------------------- */

/* w(x) += sum_mu (1-gamma_mu) U_mu(x) f(x+mu) + (1+gamma_mu) U_mu(x-mu)^dag f(x-mu)
   for the output sites of parity `pout` (pout<0: all sites, full lattice).
   Direction order x+,x-,y+,y-,z+,z-,t+,t- as Dirac_Wilson::mult_offdiag
   (lib/Dirac_ops/dirac_wilson.cpp:107-113).  Half fields are indexed by hs. */
static void hop_accumulate(const Geom* g, const double* u, int pout, const double* in,
                           double* w) {
  spin_init();
  const long nout = pout < 0 ? g->V : g->Vh;
  /* output sites are independent: threads change nothing in the result */
#pragma omp parallel for schedule(static)
  for (long o = 0; o < nout; ++o) {
    const long x = pout < 0 ? o : g->eo_site[pout * g->Vh + o];
    for (int mu = 0; mu < 4; ++mu) {
      for (int sgn = 1; sgn >= -1; sgn -= 2) {
        const long y = neighbour(g, x, mu, sgn);
        const long yi = pout < 0 ? y : g->half_of[y];
        const long ls = sgn > 0 ? x : y; /* site of the link */
        cplx uf[4][3];
        for (int s = 0; s < 4; ++s)
          for (int a = 0; a < 3; ++a) {
            cplx acc = 0;
            for (int b = 0; b < 3; ++b) {
              cplx U = sgn > 0 ? uget(u, g->V, ls, mu, a, b) : conj(uget(u, g->V, ls, mu, b, a));
              acc += U * fget(in, yi, s, b);
            }
            uf[s][a] = acc;
          }
        /* projector 1 - sgn*gamma_mu */
        for (int s = 0; s < 4; ++s)
          for (int a = 0; a < 3; ++a) {
            cplx v = uf[s][a];
            for (int t = 0; t < 4; ++t) v -= (double)sgn * GAM[mu][s][t] * uf[t][a];
            fadd(w, o, s, a, v);
          }
      }
    }
  }
}

static double kappa_of(double mass) { return 0.5 / (4.0 + mass); }

/* Dirac_Wilson::mult / mult_dag full lattice: w = f - kappa H f, and
   gamma5 mult gamma5 (lib/Dirac_ops/dirac_wilson.cpp:28-36,115-118). */
int orc_wilson_full(const int L[4], const double* u, double mass, int dag, const double* in,
                    double* out) {
  Geom g;
  geom_init(&g, L);
  const long n = 24 * g.V;
  double* f = malloc(sizeof(double) * n);
  double* w = calloc(n, sizeof(double));
  if (dag)
    orc_gamma5(g.V, in, f);
  else
    memcpy(f, in, sizeof(double) * n);
  hop_accumulate(&g, u, -1, f, w);
  const double k = kappa_of(mass);
  for (long i = 0; i < n; ++i) w[i] = f[i] - k * w[i];
  if (dag)
    orc_gamma5(g.V, w, out);
  else
    memcpy(out, w, sizeof(double) * n);
  free(f);
  free(w);
  geom_free(&g);
  return 0;
}

/* Dirac_Wilson(mass,u,EOtag|OEtag)::mult / mult_dag: -kappa H_eo f_o (eo=0)
   or -kappa H_oe f_e (eo=1) on half fields (dirac_wilson.hpp:89-114). */
int orc_wilson_hop(const int L[4], const double* u, double mass, int eo, int dag,
                   const double* in, double* out) {
  Geom g;
  geom_init(&g, L);
  const long n = 24 * g.Vh;
  double* f = malloc(sizeof(double) * n);
  double* w = calloc(n, sizeof(double));
  if (dag)
    orc_gamma5(g.Vh, in, f);
  else
    memcpy(f, in, sizeof(double) * n);
  hop_accumulate(&g, u, eo == 0 ? 0 : 1, f, w);
  const double k = kappa_of(mass);
  for (long i = 0; i < n; ++i) w[i] *= -k;
  if (dag)
    orc_gamma5(g.Vh, w, out);
  else
    memcpy(out, w, sizeof(double) * n);
  free(f);
  free(w);
  geom_free(&g);
  return 0;
}

/* Dirac_Wilson_EvenOdd::mult = f - Deo(Doe f); mult_dag = f - Deo^dag(Doe^dag f)
   (lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:80-92). */
int orc_wilson_eo(const int L[4], const double* u, double mass, int dag, const double* in,
                  double* out) {
  long Vh = (long)L[0] * L[1] * L[2] * L[3] / 2;
  double* t = malloc(sizeof(double) * 24 * Vh);
  double* w = malloc(sizeof(double) * 24 * Vh);
  orc_wilson_hop(L, u, mass, 1, dag, in, t);
  orc_wilson_hop(L, u, mass, 0, dag, t, w);
  for (long i = 0; i < 24 * Vh; ++i) out[i] = in[i] - w[i];
  free(t);
  free(w);
  return 0;
}

/* ---- clover --------------------------------------------------------------- */

typedef struct {
  cplx a[3][3];
} M3;

static M3 m3_load(const double* u, long V, long site, int mu) {
  M3 m;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) m.a[a][b] = uget(u, V, site, mu, a, b);
  return m;
}
static M3 m3_mul(M3 x, M3 y) {
  M3 r;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      cplx s = 0;
      for (int k = 0; k < 3; ++k) s += x.a[a][k] * y.a[k][b];
      r.a[a][b] = s;
    }
  return r;
}
static M3 m3_dag(M3 x) {
  M3 r;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) r.a[a][b] = conj(x.a[b][a]);
  return r;
}
/* (M - M^dag)/2, SUNmatrix::anti_hermite (lib/Tools/sunMat.hpp:139-157) */
static M3 m3_ah(M3 x) {
  M3 r;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) r.a[a][b] = 0.5 * (x.a[a][b] - conj(x.a[b][a]));
  return r;
}

/* Staples::fieldStrength(G,mu,nu) (lib/Measurements/GaugeM/staples.cpp:587-666):
   Vup(x) = U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag        (upper, :557-567)
   Vdn(x) = c(x-nu), c(y) = U_nu(y)^dag U_mu(y) U_nu(y+mu)   (lower, :490-499)
   v = Vup^dag - Vdn^dag; F(x) = AH(U_mu(x) v(x)) + AH(v(x-mu) U_mu(x-mu));
   F = 0.25 * traceless(F)  (sunMatUtils.cpp:50-55). */
int orc_field_strength(const int L[4], const double* u, int mu, int nu, double* out) {
  Geom g;
  geom_init(&g, L);
  M3* v = malloc(sizeof(M3) * g.V);
#pragma omp parallel for schedule(static)
  for (long x = 0; x < g.V; ++x) {
    long xn = neighbour(&g, x, nu, 1), xm = neighbour(&g, x, mu, 1);
    M3 up = m3_mul(m3_mul(m3_load(u, g.V, x, nu), m3_load(u, g.V, xn, mu)),
                   m3_dag(m3_load(u, g.V, xm, nu)));
    long y = neighbour(&g, x, nu, -1), ym = neighbour(&g, y, mu, 1);
    M3 dn = m3_mul(m3_mul(m3_dag(m3_load(u, g.V, y, nu)), m3_load(u, g.V, y, mu)),
                   m3_load(u, g.V, ym, nu));
    M3 d1 = m3_dag(up), d2 = m3_dag(dn);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) v[x].a[a][b] = d1.a[a][b] - d2.a[a][b];
  }
#pragma omp parallel for schedule(static)
  for (long x = 0; x < g.V; ++x) {
    long xm = neighbour(&g, x, mu, -1);
    M3 f1 = m3_ah(m3_mul(m3_load(u, g.V, x, mu), v[x]));
    M3 f2 = m3_ah(m3_mul(v[xm], m3_load(u, g.V, xm, mu)));
    M3 f;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) f.a[a][b] = f1.a[a][b] + f2.a[a][b];
    /* traceless part: subtract i*Im(tr)/3 on the diagonal */
    double imtr = cimag(f.a[0][0] + f.a[1][1] + f.a[2][2]) / 3.0;
    for (int a = 0; a < 3; ++a) f.a[a][a] -= I * imtr;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        out[18 * x + 2 * (3 * a + b)] = 0.25 * creal(f.a[a][b]);
        out[18 * x + 2 * (3 * a + b) + 1] = 0.25 * cimag(f.a[a][b]);
      }
  }
  free(v);
  geom_free(&g);
  return 0;
}

/* Dirac_Clover::mult (lib/Dirac_ops/dirac_clover.cpp:334-349):
   w = Dw f - kappa*csw * sum_k F_k (S_k f), F = (Bx,By,Bz,Ex,Ey,Ez) =
   F(1,2),F(2,0),F(0,1),F(3,0),F(3,1),F(3,2) (set_csw, :139-162);
   mult_dag = gamma5 mult gamma5 (:351-353). */
static double* clover_fields(const int L[4], const double* u) {
  static const int PAIRS[6][2] = {{1, 2}, {2, 0}, {0, 1}, {3, 0}, {3, 1}, {3, 2}};
  const long V = (long)L[0] * L[1] * L[2] * L[3];
  double* F = malloc(sizeof(double) * 18 * V * 6);
  for (int k = 0; k < 6; ++k) orc_field_strength(L, u, PAIRS[k][0], PAIRS[k][1], F + 18 * V * k);
  return F;
}

/* the clover operator with the six field strengths F already formed */
static int clover_apply(const int L[4], const double* u, const double* F, double mass, double csw,
                        int dag, const double* in, double* out) {
  spin_init();
  Geom g;
  geom_init(&g, L);
  const long n = 24 * g.V;
  double* f = malloc(sizeof(double) * n);
  double* w = malloc(sizeof(double) * n);
  double* sw = calloc(n, sizeof(double));
  if (dag)
    orc_gamma5(g.V, in, f);
  else
    memcpy(f, in, sizeof(double) * n);
  orc_wilson_full(L, u, mass, 0, f, w);
#pragma omp parallel for schedule(static)
  for (long x = 0; x < g.V; ++x)
    for (int k = 0; k < 6; ++k)
      for (int s = 0; s < 4; ++s)
        for (int a = 0; a < 3; ++a) {
          cplx acc = 0;
          for (int t = 0; t < 4; ++t) {
            if (SIG[k][s][t] == 0) continue;
            for (int b = 0; b < 3; ++b) {
              const double* p = F + 18 * (x + g.V * k) + 2 * (3 * a + b);
              acc += (p[0] + I * p[1]) * SIG[k][s][t] * fget(f, x, t, b);
            }
          }
          fadd(sw, x, s, a, acc);
        }
  const double kc = kappa_of(mass) * csw;
  for (long i = 0; i < n; ++i) w[i] -= kc * sw[i];
  if (dag)
    orc_gamma5(g.V, w, out);
  else
    memcpy(out, w, sizeof(double) * n);
  free(f);
  free(w);
  free(sw);
  geom_free(&g);
  return 0;
}

int orc_clover_full(const int L[4], const double* u, double mass, double csw, int dag,
                    const double* in, double* out) {
  double* F = clover_fields(L, u);
  int rc = clover_apply(L, u, F, mass, csw, dag, in, out);
  free(F);
  return rc;
}

/* ---- solvers ----------------------------------------------------------------- */

typedef struct {
  const int* L;
  const double* u;
  int op;
  double mass, csw;
  long n;
  double* tmp;
  double* F; /* clover: the six field strengths, formed once per solve */
} Opr;

/* Fopr_DdagD::mult = D^dag (D f) (lib/Fopr/fopr.h:146-153) */
static void opr_apply(Opr* A, const double* in, double* out) {
  switch (A->op) {
    case ORC_WILSON_FULL:
      orc_wilson_full(A->L, A->u, A->mass, 0, in, A->tmp);
      orc_wilson_full(A->L, A->u, A->mass, 1, A->tmp, out);
      break;
    case ORC_WILSON_EO:
      orc_wilson_eo(A->L, A->u, A->mass, 0, in, A->tmp);
      orc_wilson_eo(A->L, A->u, A->mass, 1, A->tmp, out);
      break;
    default:
      clover_apply(A->L, A->u, A->F, A->mass, A->csw, 0, in, A->tmp);
      clover_apply(A->L, A->u, A->F, A->mass, A->csw, 1, A->tmp, out);
      break;
  }
}

static double dot(long n, const double* a, const double* b) {
  double s = 0;
  for (long i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

static int opr_init(Opr* A, const int L[4], const double* u, int op, double mass, double csw) {
  long V = (long)L[0] * L[1] * L[2] * L[3];
  A->L = L;
  A->u = u;
  A->op = op;
  A->mass = mass;
  A->csw = csw;
  A->n = (op == ORC_WILSON_EO) ? 12 * V : 24 * V;
  A->tmp = malloc(sizeof(double) * A->n);
  A->F = (op == ORC_CLOVER_FULL) ? clover_fields(L, u) : NULL;
  return 0;
}

/* Solver_CG::solve / solve_step (lib/Solver/solver_CG.cpp:29-160) on
   Fopr_DdagD(D): x0 = b; stop when rr/|b|^2 < prec; diff = |A x - b|/|b|. */
int orc_cg(const int L[4], const double* u, int op, double mass, double csw, const double* b,
           double* x, double prec, int maxiter, double* diff, int* iters) {
  Opr A;
  opr_init(&A, L, u, op, mass, csw);
  const long n = A.n;
  double* r = malloc(sizeof(double) * n);
  double* p = malloc(sizeof(double) * n);
  double* s = malloc(sizeof(double) * n);
  memcpy(x, b, sizeof(double) * n);
  opr_apply(&A, x, s);
  for (long i = 0; i < n; ++i) r[i] = b[i] - s[i];
  memcpy(p, r, sizeof(double) * n);
  double rr = dot(n, r, r);
  double snorm = sqrt(dot(n, b, b));
  snorm = 1.0 / (snorm * snorm);
  *iters = -1;
  for (int it = 0; it < maxiter; ++it) {
    opr_apply(&A, p, s);
    double pap = dot(n, p, s);
    double rrp = rr;
    double cr = rrp / pap;
    for (long i = 0; i < n; ++i) {
      x[i] += cr * p[i];
      r[i] -= cr * s[i];
    }
    rr = dot(n, r, r);
    cr = rr / rrp;
    for (long i = 0; i < n; ++i) p[i] = p[i] * cr + r[i];
    if (rr * snorm < prec) {
      *iters = it;
      break;
    }
  }
  opr_apply(&A, x, p);
  for (long i = 0; i < n; ++i) p[i] -= b[i];
  *diff = sqrt(dot(n, p, p)) * sqrt(snorm);
  free(r);
  free(p);
  free(s);
  free(A.tmp);
  free(A.F);
  return *iters < 0 ? 1 : 0;
}

/* MultiShiftSolver_CG::solve / solve_init / solve_step
   (lib/Solver/multiShiftSolver_CG.cpp:10-185) on Fopr_DdagD(D). */
int orc_multishift(const int L[4], const double* u, int op, double mass, double csw,
                   const double* b, int nshift, const double* sigma, double* x, double prec,
                   int maxiter, double* diff, int* nconv) {
  Opr A;
  opr_init(&A, L, u, op, mass, csw);
  const long n = A.n;
  double* p = malloc(sizeof(double) * n * nshift);
  double* r = malloc(sizeof(double) * n);
  double* s = malloc(sizeof(double) * n);
  double* zeta1 = malloc(sizeof(double) * nshift);
  double* zeta2 = malloc(sizeof(double) * nshift);
  double* csh2 = malloc(sizeof(double) * nshift);
  double* pp = malloc(sizeof(double) * nshift);
  double bnorm = sqrt(dot(n, b, b));
  double snorm = 1.0 / (bnorm * bnorm);
  for (int i = 0; i < nshift; ++i) {
    memcpy(p + i * n, b, sizeof(double) * n);
    memset(x + i * n, 0, sizeof(double) * n);
    zeta1[i] = zeta2[i] = 1.0;
    csh2[i] = sigma[i] - sigma[0];
    pp[i] = 0.0;
  }
  memcpy(r, b, sizeof(double) * n);
  double rr = dot(n, r, r);
  double alphap = 0.0, betap = 1.0;
  int nshift2 = nshift;
  *nconv = -1;
  for (int it = 0; it < maxiter; ++it) {
    double* p0 = p;
    opr_apply(&A, p0, s);
    for (long i = 0; i < n; ++i) s[i] += sigma[0] * p0[i];
    double rrp = rr;
    double pap = dot(n, s, p0);
    double beta = -rrp / pap;
    for (long i = 0; i < n; ++i) x[i] -= beta * p0[i];
    for (long i = 0; i < n; ++i) r[i] += beta * s[i];
    rr = dot(n, r, r);
    double alpha = rr / rrp;
    for (long i = 0; i < n; ++i) p0[i] = p0[i] * alpha + r[i];
    pp[0] = rr;
    double alphah = 1.0 + alphap * beta / betap;
    for (int ish = 1; ish < nshift2; ++ish) {
      double zeta = (alphah - csh2[ish] * beta) / zeta1[ish] + (1.0 - alphah) / zeta2[ish];
      zeta = 1.0 / zeta;
      double zr = zeta / zeta1[ish];
      double betas = beta * zr;
      double alphas = alpha * zr * zr;
      double* xi = x + ish * n;
      double* pi = p + ish * n;
      for (long i = 0; i < n; ++i) xi[i] -= betas * pi[i];
      for (long i = 0; i < n; ++i) pi[i] = pi[i] * alphas + zeta * r[i];
      pp[ish] = dot(n, pi, pi) * snorm;
      zeta2[ish] = zeta1[ish];
      zeta1[ish] = zeta;
    }
    for (int ish = nshift2 - 1; ish >= 0; --ish) {
      if (pp[ish] > prec) {
        nshift2 = ish + 1;
        break;
      }
    }
    alphap = alpha;
    betap = beta;
    if (rr * snorm < prec) {
      *nconv = it;
      break;
    }
  }
  double dmax = -1.0;
  for (int i = 0; i < nshift; ++i) {
    opr_apply(&A, x + i * n, s);
    for (long k = 0; k < n; ++k) s[k] += sigma[i] * x[i * n + k] - b[k];
    double d1 = dot(n, s, s) * snorm;
    if (d1 > dmax) dmax = d1;
  }
  *diff = sqrt(dmax);
  free(p);
  free(r);
  free(s);
  free(zeta1);
  free(zeta2);
  free(csh2);
  free(pp);
  free(A.tmp);
  free(A.F);
  return *nconv < 0 ? 1 : 0;
}

/* ---- callers of the solvers ------------------------------------------------ */

/* EvenOddUtils::Inverter_WilsonLike::invert for Dirac_Wilson_EvenOdd with
   Solver_CG (lib/Dirac_ops/eoUtils.cpp:43-81): be = b_e - Deo b_o; y_e by CG on
   M^dag M y_e = M^dag be; b_o -= Doe y_e; sol = (y_e, b_o) in the full
   lexicographic layout (mult_ee_inv / mult_oo_inv are the identity). */
int orc_eo_invert(const int L[4], const double* u, double mass, const double* src, double* sol,
                  double prec, int maxiter, double* diff, int* iters) {
  Geom g;
  geom_init(&g, L);
  const long nh = 24 * g.Vh;
  double* be = malloc(sizeof(double) * nh);
  double* bo = malloc(sizeof(double) * nh);
  double* t = malloc(sizeof(double) * nh);
  double* rhs = malloc(sizeof(double) * nh);
  double* ye = malloc(sizeof(double) * nh);
  for (long hs = 0; hs < g.Vh; ++hs) {
    memcpy(be + 24 * hs, src + 24 * g.eo_site[hs], sizeof(double) * 24);
    memcpy(bo + 24 * hs, src + 24 * g.eo_site[g.Vh + hs], sizeof(double) * 24);
  }
  orc_wilson_hop(L, u, mass, 0, 0, bo, t);
  for (long i = 0; i < nh; ++i) be[i] -= t[i];
  orc_wilson_eo(L, u, mass, 1, be, rhs);
  int rc = orc_cg(L, u, ORC_WILSON_EO, mass, 0.0, rhs, ye, prec, maxiter, diff, iters);
  orc_wilson_hop(L, u, mass, 1, 0, ye, t);
  for (long i = 0; i < nh; ++i) bo[i] -= t[i];
  for (long hs = 0; hs < g.Vh; ++hs) {
    memcpy(sol + 24 * g.eo_site[hs], ye + 24 * hs, sizeof(double) * 24);
    memcpy(sol + 24 * g.eo_site[g.Vh + hs], bo + 24 * hs, sizeof(double) * 24);
  }
  free(be);
  free(bo);
  free(t);
  free(rhs);
  free(ye);
  geom_free(&g);
  return rc;
}

/* RationalSolver_CG::solve (lib/Solver/rationalSolver_CG.cpp:12-39):
   sol = c0 b + sum_i r_i x_i with x_i from the multishift solve at the poles. */
int orc_rational(const int L[4], const double* u, int op, double mass, double csw,
                 const double* b, int npole, const double* poles, const double* residues,
                 double c0, double* sol, double prec, int maxiter, double* diff, int* nconv) {
  const long V = (long)L[0] * L[1] * L[2] * L[3];
  const long n = (op == ORC_WILSON_EO) ? 12 * V : 24 * V;
  double* x = malloc(sizeof(double) * n * npole);
  int rc = orc_multishift(L, u, op, mass, csw, b, npole, poles, x, prec, maxiter, diff, nconv);
  for (long i = 0; i < n; ++i) {
    double v = c0 * b[i];
    for (int k = 0; k < npole; ++k) v += residues[k] * x[k * n + i];
    sol[i] = v;
  }
  free(x);
  return rc;
}

/* ---- molecular-dynamics force --------------------------------------------- */

/* Dirac_Wilson::mkfrc (lib/Dirac_ops/dirac_wilson.cpp:60-91) on the output
   sites of parity pout (-1: every site): xie = (1 - gamma_mu) U_mu(x) eta(x+mu)
   (mult_p[mu], dirac_wilson_improved.code), F[mu](x)_{ab} += sum_s xie_{a,s}
   conj(zeta_{b,s}); half fields are indexed by hs as in hop_accumulate. */
static void mkfrc(const Geom* g, const double* u, int pout, const double* eta, const double* zeta,
                  double* F) {
  spin_init();
  const long nout = pout < 0 ? g->V : g->Vh;
  for (int mu = 0; mu < 4; ++mu)
    for (long o = 0; o < nout; ++o) {
      const long x = pout < 0 ? o : g->eo_site[pout * g->Vh + o];
      const long y = neighbour(g, x, mu, 1);
      const long yi = pout < 0 ? y : g->half_of[y];
      cplx uf[4][3], xie[4][3];
      for (int s = 0; s < 4; ++s)
        for (int a = 0; a < 3; ++a) {
          cplx acc = 0;
          for (int b = 0; b < 3; ++b) acc += uget(u, g->V, x, mu, a, b) * fget(eta, yi, s, b);
          uf[s][a] = acc;
        }
      for (int s = 0; s < 4; ++s)
        for (int a = 0; a < 3; ++a) {
          cplx v = uf[s][a];
          for (int t = 0; t < 4; ++t) v -= GAM[mu][s][t] * uf[t][a];
          xie[s][a] = v;
        }
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          cplx acc = 0;
          for (int s = 0; s < 4; ++s) acc += xie[s][a] * conj(fget(zeta, o, s, b));
          double* p = F + 18 * (x + g->V * mu) + 2 * (3 * a + b);
          p[0] += creal(acc);
          p[1] += cimag(acc);
        }
    }
}

/* Dirac_Wilson::md_force (eo=-1, full lattice; dirac_wilson.cpp:41-58) and
   Dirac_Wilson_EvenOdd::md_force (eo=1, even halves;
   dirac_wilson_EvenOdd.hpp:95-117). */
int orc_md_force(const int L[4], const double* u, double mass, int eo, const double* eta,
                 const double* zeta, double* F) {
  Geom g;
  geom_init(&g, L);
  const double k = kappa_of(mass);
  memset(F, 0, sizeof(double) * 72 * g.V);
  if (eo < 0) {
    const long n = 24 * g.V;
    double* e5 = malloc(sizeof(double) * n);
    double* z5 = malloc(sizeof(double) * n);
    orc_gamma5(g.V, eta, e5);
    orc_gamma5(g.V, zeta, z5);
    mkfrc(&g, u, -1, eta, zeta, F);
    mkfrc(&g, u, -1, z5, e5, F);
    for (long i = 0; i < 72 * g.V; ++i) F[i] *= -k;
    free(e5);
    free(z5);
  } else {
    const long n = 24 * g.Vh;
    double* A = malloc(sizeof(double) * n);  /* Doe eta */
    double* B = malloc(sizeof(double) * n);  /* Doe^dag zeta */
    double* a5 = malloc(sizeof(double) * n);
    double* b5 = malloc(sizeof(double) * n);
    double* e5 = malloc(sizeof(double) * n);
    double* z5 = malloc(sizeof(double) * n);
    orc_wilson_hop(L, u, mass, 1, 0, eta, A);
    orc_wilson_hop(L, u, mass, 1, 1, zeta, B);
    orc_gamma5(g.Vh, A, a5);
    orc_gamma5(g.Vh, B, b5);
    orc_gamma5(g.Vh, eta, e5);
    orc_gamma5(g.Vh, zeta, z5);
    mkfrc(&g, u, 0, A, zeta, F);   /* Deo.md_force_p(A, zeta) */
    mkfrc(&g, u, 1, z5, a5, F);    /* Doe.md_force_m(A, zeta) */
    mkfrc(&g, u, 1, eta, B, F);    /* Doe.md_force_p(eta, B) */
    mkfrc(&g, u, 0, b5, e5, F);    /* Deo.md_force_m(eta, B) */
    for (long i = 0; i < 72 * g.V; ++i) F[i] *= k;
    free(A);
    free(B);
    free(a5);
    free(b5);
    free(e5);
    free(z5);
  }
  geom_free(&g);
  return 0;
}
