/* CPU oracle: a plain-C restatement of the reference's fermion-solve hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only the tests, the smoke check and the CPU
 * baseline leg of the benchmark may load this library; the product never
 * calls it.  Every function works on the reference's host layouts (Format_F
 * spinors, Format_G links; see include/iroiro_b200.h) in FP64 and cites the
 * reference lines it restates.  Its parity is pinned against the reference
 * itself (compiled from its own sources by oracle/Makefile) through the
 * golden fixtures in tests/golden/.
 */
#ifndef IRO_ORACLE_H
#define IRO_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_WILSON_FULL = 0, ORC_WILSON_EO = 1, ORC_CLOVER_FULL = 2 };

void orc_gamma5(long nsites, const double* in, double* out);
int orc_wilson_full(const int L[4], const double* u, double mass, int dag, const double* in,
                    double* out);
int orc_wilson_hop(const int L[4], const double* u, double mass, int eo, int dag,
                   const double* in, double* out);
int orc_wilson_eo(const int L[4], const double* u, double mass, int dag, const double* in,
                  double* out);
int orc_field_strength(const int L[4], const double* u, int mu, int nu, double* out);
int orc_clover_full(const int L[4], const double* u, double mass, double csw, int dag,
                    const double* in, double* out);
int orc_cg(const int L[4], const double* u, int op, double mass, double csw, const double* b,
           double* x, double prec, int maxiter, double* diff, int* iters);
int orc_multishift(const int L[4], const double* u, int op, double mass, double csw,
                   const double* b, int nshift, const double* shifts, double* x, double prec,
                   int maxiter, double* diff, int* nconv);

int orc_eo_invert(const int L[4], const double* u, double mass, const double* src, double* sol,
                  double prec, int maxiter, double* diff, int* iters);
int orc_rational(const int L[4], const double* u, int op, double mass, double csw,
                 const double* b, int npole, const double* poles, const double* residues,
                 double c0, double* sol, double prec, int maxiter, double* diff, int* nconv);

int orc_md_force(const int L[4], const double* u, double mass, int eo, const double* eta,
                 const double* zeta, double* F);

/* Seeded synthetic inputs, bit-identical to the product's iro_synth_gauge and
   iro_synth_gaussian (port/synth.c), for code that must not load the product. */
int orc_synth_gauge(const int L[4], double eps, unsigned long long seed, int gauge_transform,
                    double* u);
int orc_synth_gaussian(long long nsites, unsigned long long seed, double* f);

#ifdef __cplusplus
}
#endif
#endif
