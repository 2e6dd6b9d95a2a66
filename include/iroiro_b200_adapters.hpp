/* IroIro-side adapter classes over the C ABI of libiroiro_b200 (iroiro_b200.h).
 *
 * These classes implement the reference's own virtual interfaces, so that its
 * callers (Qprop, Qprop_EvenOdd, Qprop_MultiShift, Inverter_WilsonLike,
 * Action_Nf2, RationalSolver_CG) run unchanged on the GPU:
 *
 *   Dirac_Wilson_B200          : DiracWilsonLike          (dirac_wilson.hpp:36-128, full lattice)
 *   Dirac_Wilson_EvenOdd_B200  : DiracWilsonLike_EvenOdd  (dirac_wilson_EvenOdd.hpp:14-119)
 *   Dirac_Clover_B200          : DiracWilsonLike          (dirac_clover.hpp:40-112, full lattice)
 *   Solver_CG_B200             : Solver                   (solver_CG.hpp:17-60)
 *   MultiShiftSolver_CG_B200   : MultiShiftSolver         (multiShiftSolver_CG.hpp:21-74)
 *
 * It is a header for the reference's source tree (it includes the
 * reference's headers: compile with the reference's include paths, -I of
 * this directory, and link -liroiro_b200).  Host fields stay the reference's
 * Field objects in their own layouts (Format_F spinors, Format_G links);
 * every call converts at the boundary and the gauge field stays resident on
 * the device until update_internal_state() uploads it again.
 *
 * Errors: the ABI returns codes and never throws; these adapters turn a code
 * into the reference's own error handling -- Errors::ConvergenceErr where the
 * reference aborts on a solver that did not converge (solver_CG.cpp:63-67),
 * the const char* "Not converged." that MultiShiftSolver_CG throws
 * (multiShiftSolver_CG.cpp:163), Errors::BaseErr for everything else.
 */
#ifndef IROIRO_B200_ADAPTERS_HPP
#define IROIRO_B200_ADAPTERS_HPP

#include <sstream>
#include <vector>

#include "Dirac_ops/dirac_WilsonLike.hpp"
#include "Solver/multiShiftSolver.hpp"
#include "Solver/solver.hpp"
#include "include/commonPrms.hpp"
#include "include/errors.hpp"
#include "iroiro_b200.h"

namespace B200 {

/* One context per process and lattice, as the reference's CommonPrms is one
   per process (lib/Main/commonPrms.cpp:22-65); device 0 unless
   IROIRO_B200_DEVICE is defined. */
#ifndef IROIRO_B200_DEVICE
#define IROIRO_B200_DEVICE 0
#endif
inline iro_ctx* context() {
  static iro_ctx* c = nullptr;
  if (!c) {
    const int L[4] = {CommonPrms::Nx(), CommonPrms::Ny(),
                      CommonPrms::Nz(), CommonPrms::Nt()};
    if (iro_ctx_create(L, IROIRO_B200_DEVICE, &c) != IRO_OK) {
      std::ostringstream m;
      m << "iro_ctx_create failed for " << L[0] << "x" << L[1] << "x" << L[2] << "x" << L[3];
      Errors::BaseErr("B200", m);
    }
  }
  return c;
}

inline void check(int rc, const char* what) {
  if (rc != IRO_OK) {
    std::ostringstream m;
    m << what << ": " << iro_last_error(context()) << " (code " << rc << ")";
    Errors::BaseErr("B200", m);
  }
}

inline const double* in(const Field& f) { return &f.getva()[0]; }

/* What the solvers need from an operator: the ABI's operator kind and its
   parameters.  Every adapter operator below is one. */
class Operator {
 public:
  virtual ~Operator() {}
  virtual int b200_op() const = 0;
  virtual double b200_mass() const = 0;
  virtual double b200_csw() const { return 0.0; }
};

/* The adapter operator behind a Dirac*, or an error if it is not one: the
   solvers on the device apply D^dag D themselves (Fopr_DdagD, fopr.h:146-153). */
inline const Operator& operator_of(const Dirac* D) {
  const Operator* op = dynamic_cast<const Operator*>(D);
  if (!op) {
    std::ostringstream m;
    m << "the operator is not a B200 adapter (Dirac_*_B200)";
    Errors::BaseErr("B200", m);
  }
  return *op;
}

inline Field apply(int op, double mass, double csw, int dag, const Field& f) {
  Field w(f.size());
  check(iro_dirac_apply(context(), op, mass, csw, dag, IRO_PREC_DOUBLE, in(f), w.getaddr(0), 1),
        "iro_dirac_apply");
  return w;
}

}  // namespace B200

/* Drop-in for Dirac_Wilson (full lattice, dirac_wilson.hpp:36-128). */
class Dirac_Wilson_B200 : public DiracWilsonLike, public B200::Operator {
  double mass_;
  const Field* u_;

 public:
  Dirac_Wilson_B200(double mass, const Field* u) : mass_(mass), u_(u) { update_internal_state(); }
  void update_internal_state() { B200::check(iro_gauge_upload(B200::context(), B200::in(*u_)), "iro_gauge_upload"); }
  size_t fsize() const { return 24 * CommonPrms::Nvol(); }
  size_t gsize() const { return 72 * CommonPrms::Nvol(); }
  double getMass() const { return mass_; }
  const Field* getGaugeField_ptr() const { return u_; }
  const Field mult(const Field& f) const { return B200::apply(IRO_OP_WILSON_FULL, mass_, 0.0, 0, f); }
  const Field mult_dag(const Field& f) const { return B200::apply(IRO_OP_WILSON_FULL, mass_, 0.0, 1, f); }
  const Field gamma5(const Field& f) const {
    Field w(f.size());
    B200::check(iro_gamma5(B200::context(), B200::in(f), w.getaddr(0), f.size() / 24), "iro_gamma5");
    return w;
  }
  /* Dirac_Wilson::md_force (dirac_wilson.cpp:41-91): Format_G force */
  const Field md_force(const Field& eta, const Field& zeta) const {
    Field F(gsize());
    B200::check(iro_md_force(B200::context(), IRO_OP_WILSON_FULL, mass_, 0.0, B200::in(eta),
                             B200::in(zeta), F.getaddr(0)), "iro_md_force");
    return F;
  }
  int b200_op() const { return IRO_OP_WILSON_FULL; }
  double b200_mass() const { return mass_; }
};

/* Drop-in for Dirac_Wilson_EvenOdd<Dirac_Wilson> (dirac_wilson_EvenOdd.hpp:14-119):
   mult = f_e - D_eo D_oe f_e on even half fields; the hopping blocks map to
   the ABI's -kappa H_eo / -kappa H_oe (dirac_wilson.hpp:89-114). */
class Dirac_Wilson_EvenOdd_B200 : public DiracWilsonLike_EvenOdd, public B200::Operator {
  double mass_;
  const Field* u_;

 public:
  Dirac_Wilson_EvenOdd_B200(double mass, const Field* u) : mass_(mass), u_(u) {
    update_internal_state();
  }
  void update_internal_state() { B200::check(iro_gauge_upload(B200::context(), B200::in(*u_)), "iro_gauge_upload"); }
  size_t fsize() const { return 12 * CommonPrms::Nvol(); }
  size_t gsize() const { return 72 * CommonPrms::Nvol(); }
  double getMass() const { return mass_; }
  const Field* getGaugeField_ptr() const { return u_; }
  const Field mult(const Field& f) const { return B200::apply(IRO_OP_WILSON_SCHUR_EE, mass_, 0.0, 0, f); }
  const Field mult_dag(const Field& f) const { return B200::apply(IRO_OP_WILSON_SCHUR_EE, mass_, 0.0, 1, f); }
  const Field mult_eo(const Field& f) const { return B200::apply(IRO_OP_WILSON_HOP_EO, mass_, 0.0, 0, f); }
  const Field mult_oe(const Field& f) const { return B200::apply(IRO_OP_WILSON_HOP_OE, mass_, 0.0, 0, f); }
  /* Deo_.mult_dag, Doe_.mult_dag (dirac_wilson_EvenOdd.hpp:70-78) */
  const Field mult_eo_dag(const Field& f) const { return B200::apply(IRO_OP_WILSON_HOP_OE, mass_, 0.0, 1, f); }
  const Field mult_oe_dag(const Field& f) const { return B200::apply(IRO_OP_WILSON_HOP_EO, mass_, 0.0, 1, f); }
  const Field mult_ee(const Field& f) const { return f; }
  const Field mult_oo(const Field& f) const { return f; }
  const Field mult_ee_inv(const Field& f) const { return f; }
  const Field mult_oo_inv(const Field& f) const { return f; }
  const Field gamma5(const Field& f) const {
    Field w(f.size());
    B200::check(iro_gamma5(B200::context(), B200::in(f), w.getaddr(0), f.size() / 24), "iro_gamma5");
    return w;
  }
  /* Dirac_Wilson_EvenOdd::md_force (dirac_wilson_EvenOdd.hpp:95-117) */
  const Field md_force(const Field& eta, const Field& zeta) const {
    Field F(gsize());
    B200::check(iro_md_force(B200::context(), IRO_OP_WILSON_SCHUR_EE, mass_, 0.0, B200::in(eta),
                             B200::in(zeta), F.getaddr(0)), "iro_md_force");
    return F;
  }
  const DiracWilsonLike* getDeo() const { return nullptr; }
  const DiracWilsonLike* getDoe() const { return nullptr; }
  int b200_op() const { return IRO_OP_WILSON_SCHUR_EE; }
  double b200_mass() const { return mass_; }
};

/* Drop-in for Dirac_Clover (full lattice, dirac_clover.hpp:40-112).  Unlike
   the reference, it does not take ownership of a Dirac_Wilson: it is built
   from (mass, csw, u) directly. */
class Dirac_Clover_B200 : public DiracWilsonLike, public B200::Operator {
  double mass_, csw_;
  const Field* u_;

 public:
  Dirac_Clover_B200(double mass, double csw, const Field* u) : mass_(mass), csw_(csw), u_(u) {
    update_internal_state();
  }
  /* Dirac_Clover::update_internal_state recomputes F (dirac_clover.hpp:84) */
  void update_internal_state() {
    B200::check(iro_gauge_upload(B200::context(), B200::in(*u_)), "iro_gauge_upload");
    B200::check(iro_clover_setup(B200::context(), mass_, csw_), "iro_clover_setup");
  }
  size_t fsize() const { return 24 * CommonPrms::Nvol(); }
  size_t gsize() const { return 72 * CommonPrms::Nvol(); }
  double getMass() const { return mass_; }
  const Field* getGaugeField_ptr() const { return u_; }
  const Field mult(const Field& f) const { return B200::apply(IRO_OP_CLOVER_FULL, mass_, csw_, 0, f); }
  const Field mult_dag(const Field& f) const { return B200::apply(IRO_OP_CLOVER_FULL, mass_, csw_, 1, f); }
  const Field gamma5(const Field& f) const {
    Field w(f.size());
    B200::check(iro_gamma5(B200::context(), B200::in(f), w.getaddr(0), f.size() / 24), "iro_gamma5");
    return w;
  }
  /* Dirac_Clover::md_force (dirac_clover.cpp:356-532) */
  const Field md_force(const Field& eta, const Field& zeta) const {
    Field F(gsize());
    B200::check(iro_md_force(B200::context(), IRO_OP_CLOVER_FULL, mass_, csw_, B200::in(eta),
                             B200::in(zeta), F.getaddr(0)), "iro_md_force");
    return F;
  }
  int b200_op() const { return IRO_OP_CLOVER_FULL; }
  double b200_mass() const { return mass_; }
  double b200_csw() const { return csw_; }
};

/* Drop-in for Solver_CG(prec, MaxIter, new Fopr_DdagD(D)) (solver_CG.hpp:28-31):
   it takes the adapter operator D itself, since the device applies D^dag D.
   `inner` = IRO_PREC_SINGLE or IRO_PREC_HALF selects the mixed-precision
   solver, which still stops on the FP64 true residual. */
class Solver_CG_B200 : public Solver {
  double prec_;
  int maxiter_;
  const Dirac* D_;
  int inner_;
  double delta_;

 public:
  Solver_CG_B200(double prec, int MaxIter, const Dirac* D, int inner = IRO_PREC_DOUBLE,
                 double delta = 0.1)
      : prec_(prec), maxiter_(MaxIter), D_(D), inner_(inner), delta_(delta) {
    B200::operator_of(D_);
  }
  bool check_DdagD() const { return true; }
  SolverOutput solve(Field& x, const Field& b) const {
    const B200::Operator& op = B200::operator_of(D_);
    iro_cg_params p;
    p.precision = prec_;
    p.max_iter = maxiter_;
    p.inner_prec = inner_;
    p.delta = delta_;
    p.use_graph = 1;
    iro_solver_out o;
    if (x.size() != b.size()) x.resize(b.size());
    const int rc = iro_cg_solve(B200::context(), op.b200_op(), op.b200_mass(), op.b200_csw(), &p,
                                B200::in(b), x.getaddr(0), 1, &o);
    if (rc == IRO_NOT_CONVERGED) {
      std::ostringstream m;
      m << "CG solver not converged. Current residual: " << o.diff;
      Errors::ConvergenceErr(m);
    }
    B200::check(rc, "iro_cg_solve");
    SolverOutput out;
    out.diff = o.diff;
    out.Iterations = o.iterations;
    out.timing = o.timing_ms;
    out.Msg = "CG solver (B200)";
    return out;
  }
};

/* Drop-in for MultiShiftSolver_CG(new Fopr_DdagD(D), stop_cond, Niter)
   (multiShiftSolver_CG.hpp:61-65), FP64.  As the reference, it sizes x to the
   number of shifts, reports the largest relative true residual in diff and
   the converging iteration in Nconv, and throws "Not converged." otherwise. */
class MultiShiftSolver_CG_B200 : public MultiShiftSolver {
  const Dirac* D_;
  double prec_;
  int maxiter_;

 public:
  MultiShiftSolver_CG_B200(const Dirac* D, double stop_cond, int Niter)
      : D_(D), prec_(stop_cond), maxiter_(Niter) {
    B200::operator_of(D_);
  }
  SolverOutput solve(vector_Field& x, const Field& b, const vector_double& shifts, double& diff,
                     int& Nconv) const {
    const B200::Operator& op = B200::operator_of(D_);
    const size_t n = b.size(), ns = shifts.size();
    std::vector<double> xs(n * ns);
    iro_solver_out o;
    int nconv = -1;
    const int rc = iro_multishift_cg_solve(B200::context(), op.b200_op(), op.b200_mass(),
                                           op.b200_csw(), B200::in(b), int(ns), shifts.data(),
                                           xs.data(), prec_, maxiter_, &o, &nconv);
    if (rc == IRO_NOT_CONVERGED) throw "Not converged.";
    B200::check(rc, "iro_multishift_cg_solve");
    if (x.size() < ns) x.resize(ns);
    for (size_t i = 0; i < ns; ++i) {
      x[i].resize(n);
      for (size_t k = 0; k < n; ++k) x[i].set(k, xs[i * n + k]);
    }
    diff = o.diff;
    Nconv = nconv;
    SolverOutput out;
    out.diff = o.diff;
    out.Iterations = nconv;
    out.timing = o.timing_ms;
    out.Msg = "MultiShift CG solver (B200)";
    return out;
  }
};

#endif  // IROIRO_B200_ADAPTERS_HPP
