// Test-infrastructure driver around the reference's own fermion-solve classes.
//
// This file is compiled together with the reference's sources (read in place,
// never copied) into oracle/_ref/libiroiro_ref.so by oracle/Makefile.  It is
// test infrastructure: the tests, the golden-fixture script and the CPU
// baseline of bench.py call it to check results against; the product never does.
//
// Every entry point takes plain host arrays in the reference's own layouts
// (Format_F spinors, include/format_F.h:32-42; Format_G links,
// include/format_G.h:34-42), wraps them into reference `Field`s, calls the
// reference method named in its comment and copies the result back.
//
// The reference keeps the lattice geometry in process-wide singletons
// (CommonPrms::instance, lib/Main/commonPrms.cpp:22-30), so one process serves
// one lattice size: ref_init() may be called once.
//
// The reference's improved Wilson kernel puts boundary-slice buffers on the
// stack (lib/Dirac_ops/dirac_wilson_improved.code:12,23); every call therefore
// runs on a worker thread with a 512 MiB stack.
#include <pthread.h>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <iostream>
#include <sstream>
#include <streambuf>
#include <thread>
#include <vector>

#include "include/commonPrms.hpp"
#include "include/field.h"
#include "Communicator/communicator.hpp"
#include "Dirac_ops/dirac_wilson.hpp"
#include "Dirac_ops/dirac_wilson_EvenOdd.hpp"
#include "Dirac_ops/dirac_clover.hpp"
#include "Dirac_ops/eoUtils.hpp"
#include "Fopr/fopr.h"
#include "Solver/solver_CG.hpp"
#include "Solver/multiShiftSolver_CG.hpp"
#include "Measurements/GaugeM/staples.hpp"

namespace {

int g_L[4] = {0, 0, 0, 0};
bool g_init = false;

struct NullBuf : std::streambuf {
  int overflow(int c) override { return c; }
};
NullBuf g_nullbuf;

// Silences std::cout for the lifetime of the object (Dirac_Clover prints norms
// on every mult, lib/Dirac_ops/dirac_clover.cpp:125-130,345).
struct Quiet {
  std::streambuf* old;
  Quiet() : old(std::cout.rdbuf(&g_nullbuf)) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

struct Job {
  std::function<int()> fn;
  int rc;
};

void* job_entry(void* p) {
  Job* j = static_cast<Job*>(p);
  try {
    j->rc = j->fn();
  } catch (const char* msg) {
    std::cerr << "reference threw: " << msg << "\n";
    j->rc = 2;
  } catch (...) {
    j->rc = 3;
  }
  return nullptr;
}

int run_big_stack(std::function<int()> fn) {
  Job job{std::move(fn), -1};
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, size_t(512) << 20);
  pthread_t th;
  if (pthread_create(&th, &attr, job_entry, &job) != 0) return 4;
  pthread_join(th, nullptr);
  pthread_attr_destroy(&attr);
  return job.rc;
}

size_t nvol() { return size_t(g_L[0]) * g_L[1] * g_L[2] * g_L[3]; }
size_t gsize() { return 18 * 4 * nvol(); }
size_t fsize_full() { return 24 * nvol(); }
size_t fsize_half() { return 12 * nvol(); }

Field make_field(const double* p, size_t n) {
  std::valarray<double> va(p, n);
  return Field(va);
}

void store(const Field& f, double* out) {
  const std::valarray<double>& va = f.getva();
  std::memcpy(out, &va[0], sizeof(double) * va.size());
}

// Operator kinds understood by the solver entry points.
enum { OP_WILSON_FULL = 0, OP_WILSON_EO = 1, OP_CLOVER_FULL = 2 };

Dirac* make_dirac(int op, double mass, double csw, const Field* u) {
  switch (op) {
    case OP_WILSON_FULL: return new Dirac_Wilson(mass, u);
    case OP_WILSON_EO: return new Dirac_Wilson_EvenOdd<Dirac_Wilson>(mass, u);
    case OP_CLOVER_FULL: {
      Quiet q;
      // Dirac_Clover deletes the Wilson operator it is given
      // (lib/Dirac_ops/dirac_clover.hpp:71), so it is allocated with new.
      return new Dirac_Clover(new Dirac_Wilson(mass, u), csw, u);
    }
  }
  return nullptr;
}

}  // namespace

extern "C" {

// whether ref_init() has set up the lattice singletons
int ref_ready(void) { return g_init ? 1 : 0; }

// CommonPrms::instance(Lattice) with a 1x1x1x1 process grid.
int ref_init(int Lx, int Ly, int Lz, int Lt) {
  if (g_init) {
    return (Lx == g_L[0] && Ly == g_L[1] && Lz == g_L[2] && Lt == g_L[3]) ? 0 : 1;
  }
  g_L[0] = Lx; g_L[1] = Ly; g_L[2] = Lz; g_L[3] = Lt;
  Lattice latt = {false, Lx, Ly, Lz, Lt, 1, 1, 1, 1};
  CommonPrms::instance(latt);
  Communicator::instance();
  g_init = true;
  return 0;
}

// Dirac_Wilson(mass,u)::mult / mult_dag, full lattice
// (lib/Dirac_ops/dirac_wilson.cpp:28-36).
int ref_wilson_mult(const double* u, double mass, int dag, const double* in, double* out) {
  return run_big_stack([=]() {
    Field U = make_field(u, gsize());
    Field f = make_field(in, fsize_full());
    Dirac_Wilson D(mass, &U);
    store(dag ? D.mult_dag(f) : D.mult(f), out);
    return 0;
  });
}

// Dirac_Wilson(mass,u,Dop::EOtag/OEtag)::mult / mult_dag: the e/o hopping
// blocks, -kappa*D_eo (eo=0, odd->even) or -kappa*D_oe (eo=1, even->odd)
// (lib/Dirac_ops/dirac_wilson.hpp:89-114).
int ref_wilson_hop(const double* u, double mass, int eo, int dag, const double* in, double* out) {
  return run_big_stack([=]() {
    Field U = make_field(u, gsize());
    Field f = make_field(in, fsize_half());
    if (eo == 0) {
      Dirac_Wilson D(mass, &U, Dop::EOtag());
      store(dag ? D.mult_dag(f) : D.mult(f), out);
    } else {
      Dirac_Wilson D(mass, &U, Dop::OEtag());
      store(dag ? D.mult_dag(f) : D.mult(f), out);
    }
    return 0;
  });
}

// Dirac_Wilson_EvenOdd<Dirac_Wilson>::mult / mult_dag
// (lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:80-92).
int ref_wilson_eo_mult(const double* u, double mass, int dag, const double* in, double* out) {
  return run_big_stack([=]() {
    Field U = make_field(u, gsize());
    Field f = make_field(in, fsize_half());
    Dirac_Wilson_EvenOdd<Dirac_Wilson> D(mass, &U);
    store(dag ? D.mult_dag(f) : D.mult(f), out);
    return 0;
  });
}

// Dirac_Clover::mult / mult_dag, full lattice
// (lib/Dirac_ops/dirac_clover.cpp:334-353).
int ref_clover_mult(const double* u, double mass, double csw, int dag, const double* in,
                    double* out) {
  return run_big_stack([=]() {
    Quiet q;
    Field U = make_field(u, gsize());
    Field f = make_field(in, fsize_full());
    Dirac_Clover D(new Dirac_Wilson(mass, &U), csw, &U);
    store(dag ? D.mult_dag(f) : D.mult(f), out);
    return 0;
  });
}

// Staples::fieldStrength(G,mu,nu): 18*V doubles, Format_G with one direction
// (lib/Measurements/GaugeM/staples.cpp:587-666).
int ref_field_strength(const double* u, int mu, int nu, double* out) {
  return run_big_stack([=]() {
    Field U = make_field(u, gsize());
    Staples stpl;
    GaugeField1D F = stpl.fieldStrength(GaugeField(U), mu, nu);
    store(F.data, out);
    return 0;
  });
}

// Solver_CG(prec,maxiter,Fopr_DdagD(D))::solve (lib/Solver/solver_CG.cpp:29-80).
// `x` receives the solution; diff, iterations and the reference's own timing
// (ms) are returned through the pointers.  The reference aborts when the solve
// does not converge (lib/Solver/solver_CG.cpp:63-67); callers give a MaxIter
// large enough for the systems they pose.
int ref_cg_solve(const double* u, int op, double mass, double csw, const double* b, double* x,
                 double prec, int maxiter, double* diff, int* iters, double* ms) {
  return run_big_stack([=]() {
    Quiet q;
    Field U = make_field(u, gsize());
    Dirac* D = make_dirac(op, mass, csw, &U);
    Field fb = make_field(b, D->fsize());
    Fopr_DdagD A(D);
    Solver_CG slv(prec, maxiter, &A);
    Field fx(D->fsize());
    SolverOutput o = slv.solve(fx, fb);
    store(fx, x);
    *diff = o.diff;
    *iters = o.Iterations;
    *ms = o.timing;
    delete D;
    return 0;
  });
}

// MultiShiftSolver_CG(Fopr_DdagD(D),prec,maxiter)::solve for the shifts given
// (lib/Solver/multiShiftSolver_CG.cpp:95-185).  `x` holds nshift consecutive
// solutions; *diff is SolverOutput::diff, the square root of the largest
// squared relative true residual.  Returns 2 when the reference throws
// "Not converged.".
int ref_multishift_solve(const double* u, int op, double mass, double csw, const double* b,
                         int nshift, const double* shifts, double* x, double prec, int maxiter,
                         double* diff, int* nconv) {
  return run_big_stack([=]() {
    Quiet q;
    Field U = make_field(u, gsize());
    Dirac* D = make_dirac(op, mass, csw, &U);
    size_t n = D->fsize();
    Field fb = make_field(b, n);
    Fopr_DdagD A(D);
    MultiShiftSolver_CG slv(&A, prec, maxiter);
    std::vector<Field> xs(nshift, Field(n));
    std::vector<double> sig(shifts, shifts + nshift);
    double d = 0.0;
    int nc = -1;
    SolverOutput o = slv.solve(xs, fb, sig, d, nc);
    for (int i = 0; i < nshift; ++i) store(xs[i], x + i * n);
    *diff = o.diff;
    *nconv = nc;
    delete D;
    return 0;
  });
}

// EvenOddUtils::Inverter_WilsonLike(Dirac_Wilson_EvenOdd, Solver_CG on
// Fopr_DdagD)::invert (lib/Dirac_ops/eoUtils.cpp:43-81) for `nsrc`
// consecutive full-lattice sources, one after the other, as
// Qprop_EvenOdd::calc does (lib/Measurements/FermionicM/qprop_EvenOdd.cpp:10-21).
int ref_eo_invert(const double* u, double mass, const double* src, double* sol, int nsrc,
                  double prec, int maxiter) {
  return run_big_stack([=]() {
    Quiet q;
    Field U = make_field(u, gsize());
    Dirac_Wilson_EvenOdd<Dirac_Wilson> D(mass, &U);
    Fopr_DdagD A(&D);
    Solver_CG slv(prec, maxiter, &A);
    EvenOddUtils::Inverter_WilsonLike inv(&D, &slv);
    const size_t n = fsize_full();
    for (int k = 0; k < nsrc; ++k) {
      Field b = make_field(src + k * n, n);
      Field x(n);
      inv.invert(x, b);
      store(x, sol + k * n);
    }
    return 0;
  });
}

// RationalSolver_CG::solve (lib/Solver/rationalSolver_CG.cpp:12-39) with the
// reference's MultiShiftSolver_CG: the reference builds the residues, poles
// and constant with a GMP Remez algorithm (lib/Tools/RationalApprox), which
// needs GMP/MPFR and is not built here, so they are arguments and the
// reconstruction sol = c0 b + sum_i r_i x_i of rationalSolver_CG.cpp:29-36 is
// restated after the reference's multishift solve.
int ref_rational_solve(const double* u, int op, double mass, double csw, const double* b,
                       int npole, const double* poles, const double* residues, double c0,
                       double* sol, double prec, int maxiter, double* diff, int* nconv) {
  return run_big_stack([=]() {
    Quiet q;
    Field U = make_field(u, gsize());
    Dirac* D = make_dirac(op, mass, csw, &U);
    size_t n = D->fsize();
    Field fb = make_field(b, n);
    Fopr_DdagD A(D);
    MultiShiftSolver_CG slv(&A, prec, maxiter);
    std::vector<Field> xs(npole, Field(n));
    std::vector<double> sig(poles, poles + npole);
    double d = 0.0;
    int nc = -1;
    SolverOutput o = slv.solve(xs, fb, sig, d, nc);
    Field s = fb;
    s *= c0;
    for (int i = 0; i < npole; ++i) {
      Field t = xs[i];
      t *= residues[i];
      s += t;
    }
    store(s, sol);
    *diff = o.diff;
    *nconv = nc;
    delete D;
    return 0;
  });
}

// Dirac_Wilson::md_force (op OP_WILSON_FULL, lib/Dirac_ops/dirac_wilson.cpp:52-58)
// or Dirac_Wilson_EvenOdd::md_force (op OP_WILSON_EO,
// lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:108-117); `force` gets gsize() doubles.
int ref_md_force(const double* u, int op, double mass, const double* eta, const double* zeta,
                 double* force) {
  return run_big_stack([=]() {
    Quiet q;
    Field U = make_field(u, gsize());
    Dirac* D = make_dirac(op, mass, 0.0, &U);
    Field e = make_field(eta, D->fsize());
    Field z = make_field(zeta, D->fsize());
    Field F = D->md_force(e, z);
    store(F, force);
    delete D;
    return 0;
  });
}

// Throughput of Dirac_Wilson_EvenOdd<Dirac_Wilson>::mult: `nthreads`
// independent workers, each applying the operator `reps` times to its own
// copy of `in` (the reference's kernel is single-threaded per process, so
// workers stand in for one rank per core).  Wall seconds for the whole batch
// are returned in *seconds; out receives worker 0's last result.
int ref_eo_mult_throughput(const double* u, double mass, const double* in, double* out,
                           int nthreads, int reps, double* seconds) {
  Field U = make_field(u, gsize());
  Dirac_Wilson_EvenOdd<Dirac_Wilson> D(mass, &U);
  std::vector<Field> res(nthreads);
  std::vector<Job> jobs(nthreads);
  std::vector<pthread_t> th(nthreads);
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, size_t(256) << 20);
  // one untimed call initialises the lazily-built site tables
  int rc = run_big_stack([&]() {
    Field f = make_field(in, fsize_half());
    res[0] = D.mult(f);
    return 0;
  });
  if (rc) return rc;
  for (int t = 0; t < nthreads; ++t) {
    jobs[t].fn = [&, t]() {
      Field f = make_field(in, fsize_half());
      for (int r = 0; r < reps; ++r) res[t] = D.mult(f);
      return 0;
    };
    jobs[t].rc = -1;
  }
  auto t0 = std::chrono::steady_clock::now();
  for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], &attr, job_entry, &jobs[t]);
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], nullptr);
  auto t1 = std::chrono::steady_clock::now();
  pthread_attr_destroy(&attr);
  *seconds = std::chrono::duration<double>(t1 - t0).count();
  store(res[0], out);
  for (int t = 0; t < nthreads; ++t)
    if (jobs[t].rc != 0) return 5;
  return 0;
}

}  // extern "C"
