// Test-infrastructure check of the C++ adapter classes (include/iroiro_b200_adapters.hpp).
//
// Compiled with the reference's sources (read in place) and linked against
// the product library into oracle/_ref/libadapter_check.so by oracle/Makefile.
// Each entry point runs the same computation twice, once through the
// reference's own classes and once through the adapters that a maintainer
// adds to the reference (which call libiroiro_b200), and returns both, so
// that a test can compare them.  The lattice comes from ref_init()
// (ref_driver.cpp), which sets up the reference's singletons; one process
// serves one lattice.
#include <pthread.h>

#include <cstring>
#include <functional>
#include <iostream>
#include <streambuf>
#include <vector>

#include "Dirac_ops/dirac_wilson.hpp"
#include "Dirac_ops/dirac_wilson_EvenOdd.hpp"
#include "Fopr/fopr.h"
#include "Measurements/FermionicM/qprop_MultiShift.hpp"
#include "Measurements/FermionicM/source_types.hpp"
#include "Solver/multiShiftSolver_CG.hpp"
#include "Solver/solver_CG.hpp"
#include "include/commonPrms.hpp"
#include "include/field.h"
#include "include/format_F.h"
#include "iroiro_b200_adapters.hpp"

namespace {

struct NullBuf : std::streambuf {
  int overflow(int c) override { return c; }
};
NullBuf g_null;

// Silences std::cout while alive (Qprop_MultiShift prints per source).
struct Quiet {
  std::streambuf* old;
  Quiet() : old(std::cout.rdbuf(&g_null)) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

struct Task {
  std::function<int()> fn;
  int rc;
};

void* task_entry(void* p) {
  Task* t = static_cast<Task*>(p);
  try {
    t->rc = t->fn();
  } catch (const char* msg) {
    std::cerr << "threw: " << msg << "\n";
    t->rc = 2;
  } catch (...) {
    t->rc = 3;
  }
  return nullptr;
}

// The reference's improved Wilson kernel keeps boundary slices on the stack
// (lib/Dirac_ops/dirac_wilson_improved.code:12,23): run on a 512 MiB stack.
int on_big_stack(std::function<int()> fn) {
  Task t{std::move(fn), -1};
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, size_t(512) << 20);
  pthread_t th;
  if (pthread_create(&th, &attr, task_entry, &t) != 0) return 4;
  pthread_join(th, nullptr);
  pthread_attr_destroy(&attr);
  return t.rc;
}

Field wrap(const double* p, size_t n) { return Field(std::valarray<double>(p, n)); }

void put(const Field& f, double* out) { std::memcpy(out, &f.getva()[0], sizeof(double) * f.size()); }

size_t nvol() { return size_t(CommonPrms::Nvol()); }

}  // namespace

extern "C" {

// Dirac_Wilson_EvenOdd<Dirac_Wilson>::mult / mult_dag (dirac_wilson_EvenOdd.hpp:80-92)
// against Dirac_Wilson_EvenOdd_B200; even half fields (12*V doubles).
int adapter_eo_mult(const double* u, double mass, int dag, const double* in, double* out_b200,
                    double* out_ref) {
  return on_big_stack([=]() {
    Field U = wrap(u, 72 * nvol());
    Field f = wrap(in, 12 * nvol());
    Dirac_Wilson_EvenOdd<Dirac_Wilson> Dr(mass, &U);
    Dirac_Wilson_EvenOdd_B200 Db(mass, &U);
    put(dag ? Dr.mult_dag(f) : Dr.mult(f), out_ref);
    put(dag ? Db.mult_dag(f) : Db.mult(f), out_b200);
    return 0;
  });
}

// Solver_CG(prec, maxiter, Fopr_DdagD(D))::solve (solver_CG.cpp:29-80) with the
// reference's D, against Solver_CG_B200 over the adapter D; eo selects
// Dirac_Wilson_EvenOdd (12*V doubles) over the full-lattice Dirac_Wilson.
int adapter_cg(const double* u, int eo, double mass, const double* b, double prec, int maxiter,
               double* x_b200, double* x_ref, double* diff, int* iters) {
  return on_big_stack([=]() {
    Quiet q;
    Field U = wrap(u, 72 * nvol());
    const size_t n = (eo ? 12 : 24) * nvol();
    Field fb = wrap(b, n);
    Field xr(n), xb(n);
    SolverOutput o_ref, o_b200;
    if (eo) {
      Dirac_Wilson_EvenOdd<Dirac_Wilson> Dr(mass, &U);
      Fopr_DdagD A(&Dr);
      o_ref = Solver_CG(prec, maxiter, &A).solve(xr, fb);
      Dirac_Wilson_EvenOdd_B200 Db(mass, &U);
      o_b200 = Solver_CG_B200(prec, maxiter, &Db).solve(xb, fb);
    } else {
      Dirac_Wilson Dr(mass, &U);
      Fopr_DdagD A(&Dr);
      o_ref = Solver_CG(prec, maxiter, &A).solve(xr, fb);
      Dirac_Wilson_B200 Db(mass, &U);
      o_b200 = Solver_CG_B200(prec, maxiter, &Db).solve(xb, fb);
    }
    put(xr, x_ref);
    put(xb, x_b200);
    diff[0] = o_b200.diff;
    diff[1] = o_ref.diff;
    iters[0] = o_b200.Iterations;
    iters[1] = o_ref.Iterations;
    return 0;
  });
}

// Qprop_MultiShift::calc (qprop_MultiShift.cpp:10-31), the reference's caller of
// the multishift solver, unchanged, on a Source_local at `site` (x,y,z,t):
// once over Dirac_Wilson + MultiShiftSolver_CG(Fopr_DdagD), once over
// Dirac_Wilson_B200 + MultiShiftSolver_CG_B200.  Both outputs hold the
// 12 x 12 propagator fields D x_m the caller forms (24*V doubles each).
int adapter_qprop_multishift(const double* u, double mass, const int* site, int nshift,
                             const double* shifts, double prec, int maxiter, double* xq_b200,
                             double* xq_ref) {
  return on_big_stack([=]() {
    Quiet q;
    Field U = wrap(u, 72 * nvol());
    std::vector<int> sp(site, site + 4);
    Source_local<Format::Format_F> src(sp, CommonPrms::Nvol());
    std::vector<double> sh(shifts, shifts + nshift);
    prop_t xr, xb;
    {
      Dirac_Wilson Dr(mass, &U);
      Fopr_DdagD A(&Dr);
      MultiShiftSolver_CG ms(&A, prec, maxiter);
      Qprop_MultiShift(&Dr, &ms).calc(xr, src, sh);
    }
    {
      Dirac_Wilson_B200 Db(mass, &U);
      MultiShiftSolver_CG_B200 ms(&Db, prec, maxiter);
      Qprop_MultiShift(&Db, &ms).calc(xb, src, sh);
    }
    if (xr.size() != xb.size()) return 6;
    const size_t n = 24 * nvol();
    for (size_t k = 0; k < xr.size(); ++k) {
      put(xr[k], xq_ref + k * n);
      put(xb[k], xq_b200 + k * n);
    }
    return 0;
  });
}

}  // extern "C"
