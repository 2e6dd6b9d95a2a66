/* iroiro_b200.h -- C ABI of the B200 fermion-solve library.
 *
 * Drop-in for the hot path of IroIro's Wilson-type fermion solves.  Every
 * entry point returns an int status (IRO_OK on success) and never throws or
 * aborts; the message for the last failure on a context is available from
 * iro_last_error().
 *
 * Host arrays are in the reference's own layouts:
 *   spinor  (Format_F, include/format_F.h:36-42)
 *           index_r(c,s,site) = 2*(c + 3*s) + 24*site     (24 doubles/site)
 *           full-lattice fields: site = x + Lx*(y + Ly*(z + Lz*t))
 *           e/o half fields:     site = hs, the hs-th even (odd) site in
 *                                lexicographic order, i.e. SiteIndex_EvenOdd
 *                                esec/osec (lib/Geometry/siteIndex_EvenOdd.cpp:21-62)
 *   gauge   (Format_G, include/format_G.h:34-36)
 *           index_r(c1,c2,site,mu) = 2*(3*c1 + c2) + 18*(site + V*mu)
 * They are converted once at the boundary into the device layouts; gauge and
 * clover data stay resident on the GPU until the next upload.
 *
 * Operators are given by `mass` as in the reference constructors
 * (Dirac_Wilson(double mass, const Field* u), lib/Dirac_ops/dirac_wilson.hpp:89-128);
 * kappa = 0.5/(4 + mass) exactly as dirac_wilson.hpp:93 computes it.
 */
#ifndef IROIRO_B200_H
#define IROIRO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
enum {
  IRO_OK = 0,
  IRO_NOT_CONVERGED = 1, /* Solver_CG aborts (lib/Solver/solver_CG.cpp:63-67) and
                            MultiShiftSolver_CG throws (multiShiftSolver_CG.cpp:163)
                            in this case; here the best iterate is still returned */
  IRO_BAD_ARG = 2,       /* the reference asserts on size mismatches
                            (include/common_fields.hpp:48) */
  IRO_CUDA_ERROR = 3,
  IRO_TIMEOUT = 4,       /* a device-side wait hit its time or iteration limit */
  IRO_NO_GAUGE = 5,      /* operator applied before iro_gauge_upload */
  IRO_NO_CLOVER = 6,     /* clover operator applied before iro_clover_setup */
  IRO_OUT_OF_MEMORY = 7,
  IRO_IO_ERROR = 8,      /* a file that cannot be opened, read or written; the
                            reference stops in Errors::IOErr (lib/IO/fields_io.hpp:283) */
  IRO_FORMAT_ERROR = 9,  /* a file whose header or size does not match the lattice
                            (the NERSC header checks, lib/IO/NERSC_reader.cpp:47-175) */
  IRO_UNSUPPORTED = 10   /* a format whose library is absent here (ILDG needs lime) */
};

/* ---- operators ----------------------------------------------------------- */
enum {
  /* Dirac_Wilson(mass,u)::mult, full lattice: f - kappa*H f
     (lib/Dirac_ops/dirac_wilson.cpp:28-32,115-118) */
  IRO_OP_WILSON_FULL = 0,
  /* Dirac_Wilson(mass,u,Dop::EOtag)::mult: -kappa*H_eo f_o, odd -> even
     (lib/Dirac_ops/dirac_wilson.hpp:89-100, dirac_wilson.cpp:107-113) */
  IRO_OP_WILSON_HOP_EO = 1,
  /* Dirac_Wilson(mass,u,Dop::OEtag)::mult: -kappa*H_oe f_e, even -> odd
     (lib/Dirac_ops/dirac_wilson.hpp:103-114) */
  IRO_OP_WILSON_HOP_OE = 2,
  /* Dirac_Wilson_EvenOdd<Dirac_Wilson>::mult: f_e - kappa^2 H_eo H_oe f_e
     (lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:80-84) */
  IRO_OP_WILSON_SCHUR_EE = 3,
  /* Dirac_Clover::mult, full lattice: A f - kappa*H f with
     A = 1 - kappa*csw*sum F_{mu nu} (i sigma_{mu nu})
     (lib/Dirac_ops/dirac_clover.cpp:38-136,334-349) */
  IRO_OP_CLOVER_FULL = 4,
  /* Even-odd clover Schur operator A_ee - kappa^2 H_eo A_oo^-1 H_oe.  The
     reference has no e/o clover; this is the Schur complement of
     IRO_OP_CLOVER_FULL on even sites. */
  IRO_OP_CLOVER_SCHUR_EE = 5,
  /* First half of the clover Schur operator, A_oo^-1 (-kappa H_oe f_e),
     even -> odd; it rebuilds odd sites in an even-odd solve. */
  IRO_OP_CLOVER_HOP_OE_INV = 6
};

/* ---- storage precisions -------------------------------------------------- */
enum {
  IRO_PREC_DOUBLE = 0, /* FP64 storage and arithmetic */
  IRO_PREC_SINGLE = 1, /* FP32 storage and arithmetic */
  IRO_PREC_HALF = 2    /* FP16 storage (spinors with a per-site FP32 norm),
                          FP32 arithmetic */
};

typedef struct iro_ctx iro_ctx;
typedef struct iro_field iro_field;

/* ---- context ------------------------------------------------------------- */
/* One context per lattice and device; it owns all device memory.  Replaces
   the geometry singletons CommonPrms::instance(Lattice)
   (lib/Main/commonPrms.cpp:22-65) and SiteIndex_EvenOdd
   (lib/Geometry/siteIndex_EvenOdd.cpp:21-62).  Every extent must be even
   (the reference asserts Nx%2==0, siteIndex_EvenOdd.hpp:45) and the volume
   a multiple of 64 (device arrays are blocked in groups of 32 sites). */
int iro_ctx_create(const int L[4], int device, iro_ctx** ctx);
int iro_ctx_destroy(iro_ctx* ctx);
const char* iro_last_error(const iro_ctx* ctx);
/* The CUDA stream (cudaStream_t) the context launches on.  By default the
   context creates its own; set_stream makes it use the caller's. */
void* iro_ctx_get_stream(const iro_ctx* ctx);
int iro_ctx_set_stream(iro_ctx* ctx, void* stream);
/* The stencil autotuner's choices so far, as a JSON array (one object per
   tuned launch shape: precision, reconstruction, dagger, epilogue, nrhs,
   parities -> kernel variant, block size, free_grid (1: the grid covers every
   site in one pass; 0: at most 8 blocks per SM loop over the sites), time per
   launch in ms).  The reference has no autotuner. */
int iro_autotune_report(const iro_ctx* ctx, char* buf, int len);

/* ---- gauge and clover ---------------------------------------------------- */
/* Uploads a Format_G gauge field (18*4*V doubles) and keeps it resident in
   FP64, FP32 and FP16, two-row (reconstruct-12) form when every link is in
   SU(3) to 1e-12, full 3x3 form otherwise.  This is the update_internal_state
   hook of the reference (lib/Dirac_ops/dirac.hpp:28).  Invalidates clover. */
int iro_gauge_upload(iro_ctx* ctx, const double* u);

/* Builds the clover term for (mass, csw) from the resident gauge field:
   F_{mu nu} by Staples::fieldStrength (lib/Measurements/GaugeM/staples.cpp:587-666),
   A = 1 - kappa*csw*sum F (i sigma) as two Hermitian 6x6 blocks per site in
   the gamma5 eigenbasis, and their inverses.  Dirac_Clover::set_csw
   (lib/Dirac_ops/dirac_clover.cpp:139-162). */
int iro_clover_setup(iro_ctx* ctx, double mass, double csw);

/* F_{mu nu} as computed on the device, returned in Format_G with one
   direction (18*V doubles), for checking against Staples::fieldStrength. */
int iro_field_strength(iro_ctx* ctx, int mu, int nu, double* out);

/* ---- operator application on host fields --------------------------------- */
/* out = op(in) (dagger=0) or op^dagger(in) = gamma5 op gamma5 (in)
   (dagger=1; Dirac_Wilson::mult_dag, dirac_wilson.cpp:34-36).  `in` and
   `out` hold nrhs consecutive fields of the op's size (24*V doubles for full
   lattice ops, 12*V for e/o ops).  Storage and arithmetic in `prec`.
   The Schur and full-lattice operators on one field between page-locked,
   non-overlapping `in` and `out` move the field in chunks of t-slices with
   both copy directions overlapped with each other and with the stencils
   (once the operator's stencils are tuned); the result is the same to the
   bit. */
int iro_dirac_apply(iro_ctx* ctx, int op, double mass, double csw, int dagger, int prec,
                    const double* in, double* out, int nrhs);

/* gamma5 on a host spinor of nsites sites (Dirac_Wilson::gamma5,
   dirac_wilson.cpp:120-126; GammaMatrix::gamma5core, wilsonLikeUtils.cpp:42-49). */
int iro_gamma5(iro_ctx* ctx, const double* in, double* out, int64_t nsites);

/* ---- device-resident fields ---------------------------------------------- */
/* subset: 0 = even half, 1 = odd half, 2 = full lattice (even half then odd
   half).  Fields hold nrhs right-hand sides in the device layout of `prec`. */
int iro_field_create(iro_ctx* ctx, int subset, int prec, int nrhs, iro_field** f);
int iro_field_destroy(iro_field* f);
int iro_field_upload(iro_ctx* ctx, iro_field* f, const double* host);
int iro_field_download(iro_ctx* ctx, const iro_field* f, double* host);
/* out = op(in) on device fields (no host traffic).  Subsets and precisions
   of in/out must match the operator. */
int iro_dirac_apply_field(iro_ctx* ctx, int op, double mass, double csw, int dagger,
                          const iro_field* in, iro_field* out);
/* Field::norm(), sqrt(sum x^2) over every real component, one value per
   right-hand side into out[nrhs] (include/field.h:74-78); FP64 accumulation. */
int iro_field_norm(iro_ctx* ctx, const iro_field* f, double* out);
/* Field::operator*, the real inner product sum a_i b_i, one value per
   right-hand side (lib/Fields/field.inl:58-62); FP64 accumulation. */
int iro_field_dot(iro_ctx* ctx, const iro_field* a, const iro_field* b, double* out);

/* Field norm without any device allocation.  No counterpart in the
   reference: it exists for callers that cannot call cudaMalloc, for instance
   a host code that owns all device memory through its own pool with a fixed
   budget, or that must keep its device footprint constant after set-up (the
   context API above allocates contexts, staging buffers and workspaces).
   Computes sqrt(sum d_in[i]^2) over n doubles of a device array the caller
   owns (a Format_F field has 24 doubles per site) and writes it to the
   caller's device double *d_out, on `stream` (a cudaStream_t; NULL for the
   legacy default stream), without synchronizing.  It works on the current
   device.  Limit: n <= 67108864 doubles (2796202 sites), the capacity of the
   fixed 64 KiB scratch; larger n returns IRO_BAD_ARG and launches nothing.
   The scratch is one file-scope __device__ array per GPU, held until the
   process exits and shared by every call: calls that overlap on the GPU
   (different streams or threads at the same time) race and give wrong
   results.  The first call on a device looks up the array's device address
   (cudaGetSymbolAddress), and so does the first call after the device's
   context has changed (cudaDeviceReset makes a new one); make those calls
   before any stream capture. */
int iro_norm_noalloc(const double* d_in, int64_t n, double* d_out, void* stream);

/* ---- solvers -------------------------------------------------------------- */
/* Mirrors SolverOutput (lib/Solver/solver.hpp:16-22). */
typedef struct {
  double diff;          /* final true residual |A x - b| / |b| in FP64 */
  int iterations;       /* 0-based index of the converging iteration as in
                           Solver_CG::solve (solver_CG.cpp:57-58); -1 if not */
  double timing_ms;     /* wall time of the solve on the host */
  int reliable_updates; /* FP64 residual recomputations (mixed precision) */
  int operator_applies; /* applications of the normal operator */
} iro_solver_out;

typedef struct {
  double precision; /* stop when |r|^2/|b|^2 < precision (squared, as
                       Solver_CG_Prms::GoalPrecision, solver_CG.cpp:57) */
  int max_iter;
  int inner_prec;   /* IRO_PREC_DOUBLE: the reference's FP64 CG.
                       IRO_PREC_SINGLE / IRO_PREC_HALF: reliable-update CG with
                       inner iterations in that storage, FP32 arithmetic and
                       FP64 residual recomputation, solution and reductions */
  double delta;     /* reliable update when |r| < delta * max |r| since the
                       last update (mixed precision only); <= 0 selects 0.1 */
  int use_graph;    /* capture the iteration as a CUDA graph */
} iro_cg_params;

/* Solve (D^dagger D) x = b by CG for the operator `op` (Fopr_DdagD with
   Solver_CG, lib/Fopr/fopr.h:146-153, lib/Solver/solver_CG.cpp:29-160).
   The initial guess is x0 = b as in solver_CG.cpp:40.  b and x hold nrhs
   consecutive fields; the right-hand sides are solved together, sharing
   every gauge-link load.  out receives nrhs records.  op is one of
   IRO_OP_WILSON_FULL, IRO_OP_WILSON_SCHUR_EE, IRO_OP_CLOVER_FULL,
   IRO_OP_CLOVER_SCHUR_EE. */
int iro_cg_solve(iro_ctx* ctx, int op, double mass, double csw, const iro_cg_params* prm,
                 const double* b, double* x, int nrhs, iro_solver_out* out);

/* iro_cg_solve on device-resident fields: b and x are FP64 fields of the
   operator's subset (full lattice, or the even half for the Schur operators)
   with the same nrhs; no host traffic. */
int iro_cg_solve_field(iro_ctx* ctx, int op, double mass, double csw, const iro_cg_params* prm,
                       const iro_field* b, iro_field* x, iro_solver_out* out);

/* MultiShiftSolver_CG::solve for (D^dagger D + sigma_i) x_i = b
   (lib/Solver/multiShiftSolver_CG.cpp:95-185) in FP64: x_i = 0 start,
   convergence on shift 0 only, pruning of converged shifts by
   |p_i|^2/|b|^2 <= precision.  x holds nshift consecutive fields.  *diff is
   sqrt of the largest squared relative true residual, *nconv the iteration
   index of convergence (-1 if not).  An iteration updates shift 0's vectors
   only; the residuals of up to 32 iterations are kept and folded into every
   shift's x and p in one pass.  The context keeps those residual fields (up
   to 32 of the operator's size, as many as leave 2 GiB of device memory free;
   below 8 every iteration updates all shifts) as workspaces until it is
   destroyed. */
int iro_multishift_cg_solve(iro_ctx* ctx, int op, double mass, double csw, const double* b,
                            int nshift, const double* shifts, double* x, double precision,
                            int max_iter, iro_solver_out* out, int* nconv);

/* MultiShiftSolver_CG::solve (lib/Solver/multiShiftSolver_CG.cpp:95-185) in
   mixed precision: the same result contract as iro_multishift_cg_solve (every
   shift to |b - (A + sigma_i) x_i|^2 / |b|^2 < precision in FP64), computed
   as (1) the reference's multishift iteration on FP32 vectors with its FP64
   zeta/alpha/beta recurrences and pruning, to a relative residual of 1e-6,
   then (2) one block of reliable-update CG solves, one right-hand side per
   shift, with inner_prec storage (IRO_PREC_SINGLE or IRO_PREC_HALF) and FP64
   residual recomputations, refining every x_i from there.  inner_prec =
   IRO_PREC_DOUBLE is iro_multishift_cg_solve.  Shifts ascending.  *nconv is
   the phase-1 iterations plus the refinement's (-1 if not converged). */
int iro_multishift_cg_solve_mixed(iro_ctx* ctx, int op, double mass, double csw, const double* b,
                                  int nshift, const double* shifts, double* x, double precision,
                                  int max_iter, int inner_prec, iro_solver_out* out, int* nconv);
/* The same on device-resident fields: b an FP64 field of the operator's
   subset with one right-hand side, x an FP64 field of that subset with
   nshift right-hand sides (right-hand side i = the solution of shift i);
   no host traffic.  inner_prec as above (IRO_PREC_DOUBLE: the FP64 solver). */
int iro_multishift_cg_solve_field(iro_ctx* ctx, int op, double mass, double csw,
                                  const iro_field* b, int nshift, const double* shifts,
                                  iro_field* x, double precision, int max_iter, int inner_prec,
                                  iro_solver_out* out, int* nconv);

/* RationalSolver_CG::solve (lib/Solver/rationalSolver_CG.cpp:12-39):
   sol = c0 b + sum_i residues[i] (D^dagger D + poles[i])^-1 b, the shifted
   systems solved by iro_multishift_cg_solve's algorithm (poles ascending, at
   most 16) and the sum formed on the device.  The reference obtains poles,
   residues and c0 from a GMP Remez approximation (RationalApprox); here they
   are inputs.  out / nconv as for the multishift solve. */
int iro_rational_cg_solve(iro_ctx* ctx, int op, double mass, double csw, const double* b,
                          int npole, const double* poles, const double* residues, double c0,
                          double* sol, double precision, int max_iter, iro_solver_out* out,
                          int* nconv);

/* Inverter_WilsonLike::invert (lib/Dirac_ops/eoUtils.cpp:43-81): solves the
   FULL-lattice system D sol = src through the even/odd Schur operator `op`
   (IRO_OP_WILSON_SCHUR_EE: D the full Wilson operator; IRO_OP_CLOVER_SCHUR_EE:
   the full clover operator): be = b_e - D_eo A_oo^-1 b_o, CG on
   M^dagger M y_e = M^dagger be with prm, x_o = A_oo^-1 (b_o - D_oe y_e).
   src and sol are nrhs consecutive full-lattice Format_F arrays (24*V
   doubles each).  out[r] is the CG's output for right-hand side r.
   Qprop_EvenOdd::calc (lib/Measurements/FermionicM/qprop_EvenOdd.cpp:10-21)
   is this call with the 12 spin-colour point sources as one block. */
int iro_eo_invert(iro_ctx* ctx, int op, double mass, double csw, const iro_cg_params* prm,
                  const double* src, double* sol, int nrhs, iro_solver_out* out);

/* Qprop_EvenOdd::calc (lib/Measurements/FermionicM/qprop_EvenOdd.cpp:10-28)
   on a Source_local (lib/Measurements/FermionicM/source_types.hpp:23-60):
   the spin-colour point sources r = first .. first + nrhs - 1 (r = 3 s + c,
   1 at the real part of spin s, colour c of lattice site `site`, SiteIndex
   order x + Lx (y + Ly (z + Lz t))) are built on the device and inverted as
   one block as iro_eo_invert does; sol receives the nrhs full-lattice
   Format_F solutions in that order.  first + nrhs <= 12. */
int iro_qprop_point(iro_ctx* ctx, int op, double mass, double csw, const iro_cg_params* prm,
                    int64_t site, int first, int nrhs, double* sol, iro_solver_out* out);

/* Molecular-dynamics force, FP64: the F with
   Re Tr(X F_mu(x)) = d/de Re(zeta^dag D(U_mu(x) -> (1 + e X) U_mu(x)) eta).
   op = IRO_OP_WILSON_FULL: Dirac_Wilson::md_force(eta, zeta)
        (lib/Dirac_ops/dirac_wilson.cpp:41-91), eta and zeta full-lattice
        Format_F arrays;
   op = IRO_OP_WILSON_SCHUR_EE: Dirac_Wilson_EvenOdd::md_force(eta, zeta)
        (lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:95-117), eta and zeta even
        halves (24*V/2 doubles);
   op = IRO_OP_CLOVER_FULL: Dirac_Clover::md_force(eta, zeta)
        (lib/Dirac_ops/dirac_clover.cpp:356-532): the Wilson force plus the
        derivative of the clover term, full-lattice arrays.
   csw is used by the clover operator only.  force receives the Format_G
   field (72*V doubles), overwritten. */
int iro_md_force(iro_ctx* ctx, int op, double mass, double csw, const double* eta,
                 const double* zeta, double* force);

/* ---- learned preconditioner and flexible GCR --------------------------------
   No counterpart in the reference (its solvers are CG, BiCGStab and
   multishift CG, lib/Solver/solver_Factory.cpp:10-45).  A gauge-equivariant
   network of parallel-transport convolution layers on the full lattice:
     out_o(x) = sum_{d=0..8} sum_i W_d[o][i] (T_d in_i)(x),
   T_0 = 1, T_{+mu} f(x) = U_mu(x) f(x+mu), T_{-mu} f(x) = U_mu(x-mu)^dag f(x-mu),
   channels are colour vectors (a spinor is 4 channels, one per spin), the
   channel mixing runs on the tensor cores (BF16 weights and operands, FP32
   accumulation), the transports on the CUDA cores in FP32.  The links are the
   resident gauge field (which must be SU(3)). */
typedef struct iro_ptc iro_ptc;

/* widths[0..nlayers]; widths[0] = widths[nlayers] = 4, others 4, 8 or 16. */
int iro_ptc_create(iro_ctx* ctx, int nlayers, const int* widths, iro_ptc** net);
int iro_ptc_destroy(iro_ptc* net);
/* Layer weights W_d[o][i], complex, (re, im) interleaved, [9][cout][cin]. */
int iro_ptc_set_weights(iro_ptc* net, int layer, const float* w);
/* out = N(in) for full-lattice spinors: host Format_F arrays (24*V doubles),
   or device fields (subset full, FP32 or FP64, one rhs).  The links are those
   resident in `ctx`, which must have the lattice the network was built for;
   one network serves every gauge field of that lattice. */
int iro_ptc_apply(iro_ctx* ctx, iro_ptc* net, const double* in, double* out);
int iro_ptc_apply_field(iro_ctx* ctx, iro_ptc* net, const iro_field* in, iro_field* out);
/* Training: loss = |N(in) - target|^2 / |target|^2 and, if grad is not
   NULL, dloss/dW of every layer (complex, layers concatenated in the layout of
   iro_ptc_set_weights).  Forward and backward run on the device. */
int iro_ptc_loss_grad(iro_ctx* ctx, iro_ptc* net, const iro_field* in, const iro_field* target,
                      double* loss, float* grad);

typedef struct {
  double precision; /* stop when |b - A x|^2 / |b|^2 < precision (FP64 true residual) */
  int max_iter;
  int nkrylov;      /* directions kept before a restart (1..16) */
  double delta;     /* restart when the iterated |r| fell by delta; <= 0: 0.1 */
  int krylov_half;  /* 0: the directions z_j, w_j = A z_j in FP32; 1: in FP16 (A applied
                       in mixed FP16; an SU(3) gauge field); r and the correction FP32 */
} iro_gcr_params;

typedef struct {
  double diff;         /* final FP64 true residual |b - A x| / |b| */
  int iterations;      /* GCR iterations (plus fallback CG iterations), -1 if not converged */
  double timing_ms;
  int restarts;        /* FP64 residual recomputations */
  int fallback;        /* 1 if the solve stalled and finished with mixed-precision CG */
  int precond_applies; /* network applications */
} iro_gcr_out;

/* Flexible GCR for (D^dagger D) x = b on the full lattice (op
   IRO_OP_WILSON_FULL or IRO_OP_CLOVER_FULL), right-preconditioned by `net`
   (NULL: no preconditioner).  Inner iterations in FP32, the solution and the
   restarted residual in FP64; convergence is declared on the FP64 true
   residual.  When two restart cycles in a row fail to reduce the residual by
   4x, the solve finishes with the mixed-precision reliable-update CG.  b and x
   are FP64 full-lattice device fields, x0 = 0.  Each restart cycle is
   enqueued whole, its coefficients formed on the device, and the host waits
   once per cycle; the workspaces and a small scratch are allocated by the
   context's first solve and kept. */
int iro_gcr_solve_field(iro_ctx* ctx, int op, double mass, double csw, const iro_ptc* net,
                        const iro_gcr_params* prm, const iro_field* b, iro_field* x,
                        iro_gcr_out* out);

/* Self-test of the device-side bounded waits (no counterpart in the
   reference): the tensor-core kernels wait on mbarriers for at most 1 s and
   then set an error flag that the host turns into IRO_TIMEOUT, leaving the
   context usable.  This runs the same wait on an mbarrier that nothing
   arrives at, for limit_ms (0 < limit_ms <= 1000), and returns IRO_TIMEOUT
   with the time it waited in *waited_ms. */
int iro_selftest_bounded_wait(iro_ctx* ctx, double limit_ms, double* waited_ms);

/* ---- synthetic inputs (host) ---------------------------------------------- */
/* Seeded SU(3) field U = exp(i eps H), H = sum theta_a lambda_a / 2,
   theta_a ~ N(0,1), projected onto SU(3); optionally followed by a random
   gauge transformation U_mu(x) -> G(x) U_mu(x) G(x+mu)^dagger.  Format_G. */
int iro_synth_gauge(const int L[4], double eps, uint64_t seed, int gauge_transform, double* u);
/* N(0,1) in every real component of nsites Format_F sites. */
int iro_synth_gaussian(int64_t nsites, uint64_t seed, double* f);
/* The 12 point sources (c,s) at `site`, Source_local semantics
   (lib/Measurements/FermionicM/source_types.hpp:40-60): 12 consecutive
   Format_F fields of nsites sites. */
int iro_synth_point_sources(int64_t nsites, int64_t site, double* f12);

/* ---- gauge-configuration files ------------------------------------------------
   The readers behind GaugeConf_*::init_conf (lib/Main/gaugeConf.cpp:23-228) and
   CCIO::ReadFromDisk / SaveOnDisk (lib/IO/fields_io.hpp:48-360), host-only (no
   context, no GPU): a file <-> a Format_G array u[18 * (site + V * mu)] with
   site = x + Lx (y + Ly (z + Lz t)), ready for iro_gauge_upload.  Readers
   return IRO_IO_ERROR / IRO_FORMAT_ERROR / IRO_UNSUPPORTED with a message in
   iro_io_last_error() (per thread). */
enum {
  IRO_GAUGE_BINARY = 0,       /* GaugeConf_bin: BinaryReader (lib/IO/binary_reader.cpp:21-35),
                                 [site][mu][18] big-endian doubles; BinaryWriter
                                 (binary_writer.cpp:18-24) writes host byte order */
  IRO_GAUGE_JLQCD_LEGACY = 1, /* GaugeConf_JLQCDLegacy (gaugeConf.cpp:28-33): a 4-byte
                                 Fortran record word, then [mu][site][18] host-order doubles */
  IRO_GAUGE_NERSC = 2,        /* GaugeConf_NERSC: NERSCReader (lib/IO/NERSC_reader.cpp), text
                                 header, [site][mu][12 or 18] big-endian 32/64-bit; NERSCWriter
                                 (NERSC_writer.cpp) writes 3x3 IEEE64BIG */
  IRO_GAUGE_ILDG = 3,         /* GaugeConf_ILDG: needs lime, absent -> IRO_UNSUPPORTED */
  IRO_GAUGE_ILDG_FORTRAN = 4, /* GaugeConf_ILDG_FORTRAN: likewise */
  IRO_GAUGE_CSDT = 5,         /* GaugeConf_csdt (gaugeConf.cpp:66-140): 4-byte record word,
                                 then [t][mu][z][y][x][a][b] big-endian complex doubles */
  IRO_GAUGE_TEXT = 6,         /* GaugeConf_txt (gaugeConf.cpp:142-209): text,
                                 [t][z][y][x][mu][a][b] "re im" */
  IRO_GAUGE_UNIT = 7          /* GaugeConf_unit (gaugeConf.cpp:211-228): unit links, no file */
};

typedef struct iro_gauge_info {
  double plaquette;         /* Staples::plaquette of the field read or written */
  double link_trace;        /* Staples::link_trace */
  double stored_plaquette;  /* NERSC header PLAQUETTE / LINK_TRACE / CHECKSUM */
  double stored_link_trace;
  uint32_t checksum;        /* NERSC: sum of the data's 32-bit words as in the file */
  uint32_t stored_checksum;
  int is3x2;                /* NERSC: DATATYPE 4D_SU3_GAUGE (two rows stored) */
  int bits;                 /* NERSC: 32 or 64 */
} iro_gauge_info;

/* Reads format `format` at byte `offset` (0 for the reference's own offsets)
   into u.  info (may be null) gets the plaquette and link trace of u and, for
   NERSC, the header's values and both checksums.  Like the reference, a read
   does not fail on a plaquette or checksum mismatch (ReadFromDisk's check is
   commented out, fields_io.hpp:346-352): compare info's fields to check. */
int iro_gauge_read(const char* path, int format, const int L[4], int64_t offset, double* u,
                   iro_gauge_info* info);
/* SaveOnDisk<Format_G>(u, path, append, "Binary" | "NERSC"). */
int iro_gauge_write(const char* path, int format, const int L[4], const double* u, int append);
/* Staples::plaquette and Staples::link_trace (lib/Measurements/GaugeM/staples.cpp:24-38):
   sum of Re tr over the 6 planes / (3 * 6 * V) and of Re tr U / (3 * 4 * V). */
int iro_gauge_plaquette(const int L[4], const double* u, double* plaquette, double* link_trace);
const char* iro_io_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* IROIRO_B200_H */
