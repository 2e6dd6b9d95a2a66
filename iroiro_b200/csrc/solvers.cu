// Krylov solvers on the device: the reference's FP64 CG and multishift CG,
// and the mixed-precision reliable-update CG.  The iteration scalars live on
// the device (solver_scalars.cuh); the host only launches a chunk of
// iterations (optionally as one CUDA graph) and polls the convergence flags
// between chunks.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"
#include "iroiro_b200.h"

namespace iro {
namespace host {
int apply(iro_ctx* c, int op, double mass, double csw, bool dag, const DevField& in, DevField& out,
          const Reduce* red, int red_mask, const int* skip);
int apply_cg(iro_ctx* c, int op, double mass, double csw, bool dag, const DevField& in,
             DevField& out, const Reduce& red, const int* skip, const CGFuse& fuse);
DevField* workspace(iro_ctx* c, int subset, int prec, int nrhs, int slot, int* rc);
bool workspace_exists(iro_ctx* c, int subset, int prec, int nrhs, int slot);
int import_field(iro_ctx* c, const double* host, bool full, DevField& f);
int export_field(iro_ctx* c, const DevField& f, bool full, double* host);
// host <-> device copies (large pageable ones through the context's pinned ring)
int host_to_device(iro_ctx* c, void* dev, const void* host, size_t bytes);
int device_to_host(iro_ctx* c, void* host, const void* dev, size_t bytes);
int norms(iro_ctx* c, const DevField& v, const DevField* w, std::vector<double>& nv,
          std::vector<double>* nw);
int axpby(iro_ctx* c, double a, const DevField& x, double b, const DevField& y, DevField& v);
int convert(iro_ctx* c, const DevField& in, DevField& out);
Reduce reduce(iro_ctx* c, int stage, int max_iter);
int set_error(iro_ctx* c, int code, const std::string& msg);
int cuda_error(iro_ctx* c, cudaError_t e, const char* where);
cudaStream_t stream(iro_ctx* c);
int max_blocks(iro_ctx* c);
int64_t vh(iro_ctx* c);
void* state(iro_ctx* c);
int* done(iro_ctx* c);
void* pinned(iro_ctx* c);
void* scratch(iro_ctx* c, size_t bytes, int* rc);
int device(iro_ctx* c);
bool op_is_full(int op);
int op_subset(int op);
bool op_ok(int op);
DevField* field_dev(iro_field* f);
int clover_ready(iro_ctx* c, double mass, double csw);
CloverPtr clover(iro_ctx* c, int prec, int p, bool inverse);
GaugePtr gauge_double(iro_ctx* c);
int gauge_recon(iro_ctx* c);
const double* gauge_format_g(iro_ctx* c);
bool gauge_loaded(iro_ctx* c);
const Geom& geom(iro_ctx* c);
int64_t volume(iro_ctx* c);
}  // namespace host
}  // namespace iro

using namespace iro;
using namespace iro::host;

#define CK(call)                                             \
  do {                                                       \
    cudaError_t e__ = (call);                                \
    if (e__ != cudaSuccess) return cuda_error(c, e__, #call); \
  } while (0)
#define RC(call)              \
  do {                        \
    int r__ = (call);         \
    if (r__ != IRO_OK) return r__; \
  } while (0)

namespace {

constexpr int kChunk = 8;  // iterations launched between host polls

bool solver_op_ok(int op) {
  return op == IRO_OP_WILSON_FULL || op == IRO_OP_WILSON_SCHUR_EE || op == IRO_OP_CLOVER_FULL ||
         op == IRO_OP_CLOVER_SCHUR_EE;
}

// Runs `body` (which enqueues `n` iterations) repeatedly until every
// right-hand side has left the iteration (done flag set) or max_iter is hit.
// With use_graph the chunk is captured once as a CUDA graph and replayed.
template <typename F>
int iterate(iro_ctx* c, int nrhs, int max_iter, bool use_graph, F body) {
  cudaStream_t st = stream(c);
  int* hdone = static_cast<int*>(pinned(c));
  cudaGraphExec_t exec = nullptr;
  // the legacy default stream cannot be captured: run the chunk eagerly there
  if (use_graph && st != nullptr) {
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = body(kChunk);
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_error(c, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_error(c, e, "cudaGraphInstantiate");
  }
  int launched = 0;
  int rc = IRO_OK;
  while (launched < max_iter) {
    if (exec) {
      cudaError_t e = cudaGraphLaunch(exec, st);
      if (e != cudaSuccess) {
        rc = cuda_error(c, e, "cudaGraphLaunch");
        break;
      }
    } else {
      rc = body(kChunk);
      if (rc) break;
    }
    launched += kChunk;
    cudaError_t e = cudaMemcpyAsync(hdone, done(c), sizeof(int) * nrhs, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      rc = cuda_error(c, e, "poll");
      break;
    }
    bool all = true;
    for (int r = 0; r < nrhs; ++r) all = all && hdone[r] != 0;
    if (all) break;
  }
  if (exec) cudaGraphExecDestroy(exec);
  return rc;
}

// FP64 CG on D^dag D, Solver_CG::solve (lib/Solver/solver_CG.cpp:29-80).
int cg_double(iro_ctx* c, int op, double mass, double csw, const iro_cg_params* prm,
              const DevField* B, DevField* X, int nrhs, iro_solver_out* out) {
  const int sub = op_subset(op);
  const bool full = op_is_full(op);
  int rc = IRO_OK;
  DevField* R = workspace(c, sub, PREC_DOUBLE, nrhs, 22, &rc); if (!R) return rc;
  DevField* P = workspace(c, sub, PREC_DOUBLE, nrhs, 23, &rc); if (!P) return rc;
  DevField* S = workspace(c, sub, PREC_DOUBLE, nrhs, 24, &rc); if (!S) return rc;
  DevField* Q = workspace(c, sub, PREC_DOUBLE, nrhs, 25, &rc); if (!Q) return rc;
  cudaStream_t st = stream(c);
  RC(axpby(c, 1.0, *B, 0.0, *B, *X));  // x0 = b (solver_CG.cpp:40)
  // CG state: target = GoalPrecision (scaled by |b|^2 in the init stage)
  std::vector<CGState> s0(nrhs);
  for (auto& s : s0) {
    std::memset(&s, 0, sizeof(s));
    s.target = prm->precision;
    s.conv_iter = -1;
  }
  CK(cudaMemcpyAsync(state(c), s0.data(), sizeof(CGState) * nrhs, cudaMemcpyHostToDevice, st));
  // r = b - A x, p = r, rr = (r,r)
  RC(apply(c, op, mass, csw, false, *X, *Q, nullptr, 0, nullptr));
  RC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, nullptr));
  Reduce rinit = reduce(c, ST_CG_INIT, prm->max_iter);
  CK(launch_cg_init(PREC_DOUBLE, B->sites(), nrhs, B->all(), S->all(), R->all(), P->all(), rinit,
                    max_blocks(c), st));
  const int* skip = done(c);
  Reduce ralpha = reduce(c, ST_CG_ALPHA, prm->max_iter);
  Reduce rbeta = reduce(c, ST_CG_BETA, prm->max_iter);
  auto body = [&](int n) -> int {
    for (int i = 0; i < n; ++i) {
      // (p, A p) = |D p|^2; then D^dag (D p) with r -= alpha A p and (r, r)
      // fused into its last launch; x += alpha p with the p update
      RC(apply(c, op, mass, csw, false, *P, *Q, &ralpha, RED_OUT2, skip));
      RC(apply_cg(c, op, mass, csw, true, *Q, *S, rbeta, skip,
                  CGFuse{R, static_cast<const CGState*>(state(c))}));
      CK(launch_cg_p(PREC_DOUBLE, P->sites(), nrhs, P->all(), R->all(), X->all(),
                     static_cast<const CGState*>(state(c)), done(c), st));
    }
    return IRO_OK;
  };
  RC(iterate(c, nrhs, prm->max_iter, prm->use_graph != 0, body));
  // true residual |A x - b| / |b| (solver_CG.cpp:69-71)
  RC(apply(c, op, mass, csw, false, *X, *Q, nullptr, 0, nullptr));
  RC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, nullptr));
  RC(axpby(c, 1.0, *S, -1.0, *B, *R));
  std::vector<double> rn, bn;
  RC(norms(c, *R, B, rn, &bn));
  std::vector<CGState> s1(nrhs);
  CK(cudaMemcpyAsync(s1.data(), state(c), sizeof(CGState) * nrhs, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  int status = IRO_OK;
  for (int r = 0; r < nrhs; ++r) {
    out[r].diff = std::sqrt(rn[r] / bn[r]);
    out[r].iterations = s1[r].conv_iter;
    out[r].reliable_updates = 0;
    out[r].operator_applies = s1[r].iter + 2;
    if (s1[r].conv_iter < 0) status = IRO_NOT_CONVERGED;
  }
  if (status) set_error(c, status, "CG solver not converged");
  return status;
}

}  // namespace

// sigma[r]: the shift of right-hand side r's operator (A + sigma); target[r]:
// its squared relative residual goal instead of prm->precision (both
// optional; the refinement of the mixed-precision multishift solve)
int cg_mixed(iro_ctx* c, int op, double mass, double csw, const iro_cg_params* prm,
             const DevField* B, DevField* X, int nrhs, iro_solver_out* out,
             const double* sigma = nullptr, const double* target = nullptr);

static int cg_any(iro_ctx* c, int op, double mass, double csw, const iro_cg_params* prm,
                  const DevField* B, DevField* X, int nrhs, iro_solver_out* out) {
  auto t0 = std::chrono::steady_clock::now();
  int rc = prm->inner_prec == PREC_DOUBLE ? cg_double(c, op, mass, csw, prm, B, X, nrhs, out)
                                          : cg_mixed(c, op, mass, csw, prm, B, X, nrhs, out);
  auto t1 = std::chrono::steady_clock::now();
  const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  for (int r = 0; r < nrhs; ++r) out[r].timing_ms = ms;
  return rc;
}

// CG on device fields for other solvers in this library (the fallback of the
// preconditioned GCR)
int cg_any_dev(iro_ctx* c, int op, double mass, double csw, const iro_cg_params* prm,
               const DevField* B, DevField* X, int nrhs, iro_solver_out* out) {
  return cg_any(c, op, mass, csw, prm, B, X, nrhs, out);
}

static bool cg_args_ok(const iro_cg_params* prm, int op) {
  return prm && solver_op_ok(op) && prm->inner_prec >= 0 && prm->inner_prec <= 2 &&
         prm->precision > 0.0;
}

extern "C" int iro_cg_solve(iro_ctx* c, int op, double mass, double csw,
                            const iro_cg_params* prm, const double* b, double* x, int nrhs,
                            iro_solver_out* out) {
  if (!c || !b || !x || !out || nrhs < 1 || nrhs > 16 || !cg_args_ok(prm, op))
    return set_error(c, IRO_BAD_ARG, "bad CG arguments");
  CK(cudaSetDevice(device(c)));
  const int sub = op_subset(op);
  const bool full = op_is_full(op);
  int rc = IRO_OK;
  DevField* B = workspace(c, sub, PREC_DOUBLE, nrhs, 20, &rc); if (!B) return rc;
  DevField* X = workspace(c, sub, PREC_DOUBLE, nrhs, 21, &rc); if (!X) return rc;
  RC(import_field(c, b, full, *B));
  rc = cg_any(c, op, mass, csw, prm, B, X, nrhs, out);
  if (rc != IRO_OK && rc != IRO_NOT_CONVERGED) return rc;
  int rc2 = export_field(c, *X, full, x);
  return rc2 ? rc2 : rc;
}

extern "C" int iro_cg_solve_field(iro_ctx* c, int op, double mass, double csw,
                                  const iro_cg_params* prm, const iro_field* b, iro_field* x,
                                  iro_solver_out* out) {
  const DevField* B = field_dev(const_cast<iro_field*>(b));
  DevField* X = field_dev(x);
  if (!c || !B || !X || !out || !cg_args_ok(prm, op) || B->prec != PREC_DOUBLE ||
      X->prec != PREC_DOUBLE || B->nrhs != X->nrhs || B->subset != op_subset(op) ||
      X->subset != op_subset(op) || B->data == X->data)
    return set_error(c, IRO_BAD_ARG, "bad CG field arguments");
  CK(cudaSetDevice(device(c)));
  return cg_any(c, op, mass, csw, prm, B, X, B->nrhs, out);
}

// ---- multishift CG ---------------------------------------------------------------------
// The iterations of MultiShiftSolver_CG::solve (multiShiftSolver_CG.cpp:34-93)
// with a window of W residuals.  Shift 0's x and every other shift's x and p
// are not touched per iteration: over a window that began at iteration k0,
// each is a linear combination of its value at k0 and of the residuals
// r_{k0+1}, r_{k0+2}, ... that the iteration leaves in the ring of slots:
//   p_k <- alphas_k p_k + zeta_k r_{j+1},  x_k <- x_k - betas_k p_k
// unrolled over the window's steps gives x_k = x_k + X p_k + sum_j C_j r_j
// and p_k = P p_k + sum_j D_j r_j, with X, P, C_j, D_j formed on the host in
// FP64 from the step scalars the device recorded (MSState::h*).  One pass
// (launch_msw_fold) then updates all shifts: it reads the window's residuals
// once instead of every shift's x and p once per iteration.  A shift is
// updated exactly at the steps the reference updates it (nshift2 recorded
// per step); its |p_k|^2 for the pruning test follows the recurrence of
// stage ST_MSW_P between folds and is recomputed from the stored p_k at each
// fold.  The slots: R = slot 0 holds r_0 = b; r_j goes to slot j % (W + 1).
static int ms_window(iro_ctx* c, int op, double mass, double csw, const DevField* B, int nshift,
                     int max_iter, MSState& m, const std::vector<DevField*>& slots, DevField* P0,
                     DevField* Q, DevField* S, const MSFields& f, const std::vector<DevField*>& PS,
                     double bb) {
  cudaStream_t st = stream(c);
  const int W = int(slots.size()) - 1, nslots = W + 1;
  MSState* dm = static_cast<MSState*>(state(c));
  const int* skip = done(c);
  int* hdone = static_cast<int*>(pinned(c));
  SlotList sl{};
  for (int j = 0; j < nslots; ++j) sl.s[j] = slots[j]->all();
  RC(axpby(c, 1.0, *B, 0.0, *B, *P0));  // p_0 = b, the live search direction
  m.k0 = 0;
  m.wsize = W;
  for (int k = 0; k < nshift; ++k) m.q[k] = bb;  // |p_k|^2 = |b|^2
  CK(cudaMemcpyAsync(dm, &m, sizeof(m), cudaMemcpyHostToDevice, st));
  Reduce ralpha = reduce(c, ST_MS_ALPHA, max_iter);
  Reduce rr = reduce(c, ST_MSW_R, max_iter);
  Reduce rp = reduce(c, ST_MSW_P, max_iter);
  auto body = [&](int n) -> int {
    for (int i = 0; i < n; ++i) {
      RC(apply(c, op, mass, csw, false, *P0, *Q, &ralpha, RED_OUT2 | RED_X2, skip));
      RC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, skip));
      CK(launch_msw_r(B->sites(), sl, nslots, P0->all(), S->all(), dm, rr, max_blocks(c), st));
      CK(launch_msw_p(B->sites(), sl, nslots, P0->all(), dm, rp, max_blocks(c), st));
    }
    return IRO_OK;
  };
  cudaGraphExec_t exec = nullptr;
  if (st != nullptr) {
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int brc = body(kChunk);
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (brc) return brc;
    if (e != cudaSuccess) return cuda_error(c, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_error(c, e, "cudaGraphInstantiate");
  }
  struct ExecGuard {
    cudaGraphExec_t e;
    ~ExecGuard() { if (e) cudaGraphExecDestroy(e); }
  } guard{exec};
  // x_k += X p_k + sum C r, p_k = P p_k + sum D r for the steps since k0
  auto fold = [&]() -> int {
    const int n = m.iter - m.k0;
    if (n <= 0) return IRO_OK;
    int nx = 1;
    for (int w = 0; w < n; ++w) nx = std::max(nx, m.hn2[w]);
    for (int k = 0; k < nx; ++k) {
      double X = 0.0, P = 1.0, C[MSW_MAX] = {}, D[MSW_MAX] = {};
      for (int w = 0; w < n; ++w) {
        if (k >= m.hn2[w]) continue;  // pruned before this step
        const double bs = k == 0 ? m.hbeta[w] : m.hbetas[w][k];
        const double as = k == 0 ? m.halpha[w] : m.halphas[w][k];
        const double z = k == 0 ? 1.0 : m.hzeta[w][k];
        X -= bs * P;  // x -= betas p
        for (int j = 0; j < w; ++j) C[j] -= bs * D[j];
        P *= as;  // p = alphas p + zeta r_{k0+1+w}
        for (int j = 0; j < w; ++j) D[j] *= as;
        D[w] = z;
      }
      double* cf = m.wcoef + k * kMswCoef;
      cf[0] = X;
      cf[1] = P;
      for (int j = 0; j < MSW_MAX; ++j) {
        cf[2 + j] = C[j];
        cf[2 + MSW_MAX + j] = D[j];
      }
    }
    CK(cudaMemcpyAsync(dm->wcoef, m.wcoef, sizeof(m.wcoef), cudaMemcpyHostToDevice, st));
    CK(launch_msw_fold(B->sites(), sl, nslots, (m.k0 + 1) % nslots, n, f, nx, 1, dm->wcoef, st));
    // shift 0's p is the live one; its stored copy is the next window's base
    RC(axpby(c, 1.0, *P0, 0.0, *P0, *PS[0]));
    return IRO_OK;
  };
  if (max_iter > 0) {
    for (;;) {
      if (exec) CK(cudaGraphLaunch(exec, st));
      else RC(body(kChunk));
      CK(cudaMemcpyAsync(hdone, done(c), sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (hdone[0] == RUNNING) continue;
      const int status = hdone[0];
      CK(cudaMemcpyAsync(&m, dm, sizeof(m), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      RC(fold());
      if (status != PAUSED) break;
      // the next window: |p_k|^2 from the folded p_k, the window's base, run on
      for (int k = 1; k < m.nshift2; ++k) {
        std::vector<double> pn;
        RC(norms(c, *PS[k], nullptr, pn, nullptr));
        m.q[k] = pn[0];
      }
      m.k0 = m.iter;
      const int running = RUNNING;
      CK(cudaMemcpyAsync(dm, &m, sizeof(m), cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(done(c), &running, sizeof(int), cudaMemcpyHostToDevice, st));
    }
  }
  return IRO_OK;
}

// MultiShiftSolver_CG::solve (lib/Solver/multiShiftSolver_CG.cpp:95-185) in FP64.
// The solve itself; the shifted solutions stay in the context's workspaces
// (*xs_out), and are exported to x when x is given.
// B: the FP64 source on the device.  The solutions go to the host array x
// (nshift consecutive fields) and/or the FP64 block field xblock (right-hand
// side k = shift k) when given.
static int ms_run(iro_ctx* c, int op, double mass, double csw, const DevField* B, int nshift,
                  const double* shifts, double* x, DevField* xblock, double precision,
                  int max_iter, iro_solver_out* out, int* nconv, std::vector<DevField*>* xs_out) {
  CK(cudaSetDevice(device(c)));
  auto t0 = std::chrono::steady_clock::now();
  const int sub = op_subset(op);
  const bool full = op_is_full(op);
  int rc = IRO_OK;
  DevField* R = workspace(c, sub, PREC_DOUBLE, 1, 31, &rc); if (!R) return rc;
  DevField* S = workspace(c, sub, PREC_DOUBLE, 1, 32, &rc); if (!S) return rc;
  DevField* Q = workspace(c, sub, PREC_DOUBLE, 1, 33, &rc); if (!Q) return rc;
  std::vector<DevField*> XS(nshift), PS(nshift);
  for (int k = 0; k < nshift; ++k) {
    XS[k] = workspace(c, sub, PREC_DOUBLE, 1, 40 + k, &rc); if (!XS[k]) return rc;
    PS[k] = workspace(c, sub, PREC_DOUBLE, 1, 40 + MAXSHIFT + k, &rc); if (!PS[k]) return rc;
  }
  cudaStream_t st = stream(c);
  std::vector<double> bn;
  RC(norms(c, *B, nullptr, bn, nullptr));
  // solve_init (multiShiftSolver_CG.cpp:10-32): p_i = b, x_i = 0, r = b
  for (int k = 0; k < nshift; ++k) {
    RC(axpby(c, 1.0, *B, 0.0, *B, *PS[k]));
    RC(axpby(c, 0.0, *B, 0.0, *B, *XS[k]));
  }
  RC(axpby(c, 1.0, *B, 0.0, *B, *R));
  MSState m;
  std::memset(&m, 0, sizeof(m));
  m.rr = bn[0];
  m.alphap = 0.0;
  m.betap = 1.0;
  m.snorm = 1.0 / bn[0];
  m.prec = precision;
  m.sigma0 = shifts[0];
  m.nshift = nshift;
  m.nshift2 = nshift;
  m.conv_iter = -1;
  for (int k = 0; k < nshift; ++k) {
    m.csh2[k] = shifts[k] - shifts[0];
    m.zeta1[k] = m.zeta2[k] = 1.0;
  }
  int zero = 0;
  CK(cudaMemcpyAsync(state(c), &m, sizeof(m), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(done(c), &zero, sizeof(int), cudaMemcpyHostToDevice, st));
  MSFields f;
  for (int k = 0; k < MAXSHIFT; ++k) {
    f.x[k] = XS[k < nshift ? k : 0]->all();
    f.p[k] = PS[k < nshift ? k : 0]->all();
  }
  // autotune the two operator launches outside the graph capture (scratch Q, S only)
  RC(apply(c, op, mass, csw, false, *PS[0], *Q, nullptr, 0, nullptr));
  RC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, nullptr));
  MSState* dm = static_cast<MSState*>(state(c));
  const int* skip = done(c);
  // The residual window: slot 0 is R, slots 1..W further workspaces while the
  // device keeps 2 GiB free.  With W >= 8 an iteration moves shift 0's
  // vectors only and every W iterations one pass folds the window into all
  // shifts' x and p (ms_window); otherwise every iteration updates them all.
  std::vector<DevField*> slots{R};
  for (int j = 1; j <= MSW_MAX; ++j) {
    if (!workspace_exists(c, sub, PREC_DOUBLE, 1, 200 + j)) {
      size_t fr = 0, tot = 0;
      CK(cudaMemGetInfo(&fr, &tot));
      if (fr < R->bytes_data + (size_t(2) << 30)) break;
    }
    DevField* sj = workspace(c, sub, PREC_DOUBLE, 1, 200 + j, &rc); if (!sj) return rc;
    slots.push_back(sj);
  }
  const int W = int(slots.size()) - 1;
  if (W >= 8) {
    DevField* P0 = workspace(c, sub, PREC_DOUBLE, 1, 199, &rc); if (!P0) return rc;
    RC(ms_window(c, op, mass, csw, B, nshift, max_iter, m, slots, P0, Q, S, f, PS, bn[0]));
  } else {
    Reduce ralpha = reduce(c, ST_MS_ALPHA, max_iter);
    Reduce rr = reduce(c, ST_MS_R, max_iter);
    Reduce rpp = reduce(c, ST_MS_PP, max_iter);
    auto body = [&](int n) -> int {
      for (int i = 0; i < n; ++i) {
        RC(apply(c, op, mass, csw, false, *PS[0], *Q, &ralpha, RED_OUT2 | RED_X2, skip));
        RC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, skip));
        CK(launch_ms_xr(PREC_DOUBLE, B->sites(), XS[0]->all(), R->all(), PS[0]->all(), S->all(), dm,
                        rr, max_blocks(c), st));
        CK(launch_ms_p(PREC_DOUBLE, B->sites(), nshift, f, R->all(), dm, rpp, max_blocks(c), st));
      }
      return IRO_OK;
    };
    RC(iterate(c, 1, max_iter, true, body));
  }
  CK(cudaMemcpyAsync(&m, state(c), sizeof(m), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  // true residuals of every shift (multiShiftSolver_CG.cpp:166-177)
  double dmax = -1.0;
  for (int k = 0; k < nshift; ++k) {
    RC(apply(c, op, mass, csw, false, *XS[k], *Q, nullptr, 0, nullptr));
    RC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, nullptr));
    RC(axpby(c, 1.0, *S, shifts[k], *XS[k], *S));
    RC(axpby(c, 1.0, *S, -1.0, *B, *S));
    std::vector<double> sn;
    RC(norms(c, *S, nullptr, sn, nullptr));
    const double d1 = sn[0] / bn[0];
    if (d1 > dmax) dmax = d1;
    const size_t nfield = size_t(24) * size_t(full ? 2 * vh(c) : vh(c));
    if (x) RC(export_field(c, *XS[k], full, x + size_t(k) * nfield));
  }
  if (xblock) CK(launch_ms_pack(PREC_DOUBLE, B->sites(), nshift, f, xblock->all(), st));
  if (xs_out) *xs_out = XS;
  auto t1 = std::chrono::steady_clock::now();
  out->diff = std::sqrt(dmax);
  out->iterations = m.conv_iter;
  out->timing_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  out->reliable_updates = 0;
  out->operator_applies = m.iter + nshift;
  *nconv = m.conv_iter;
  if (m.conv_iter < 0) return set_error(c, IRO_NOT_CONVERGED, "Not converged.");
  return IRO_OK;
}

static bool ms_args_ok(iro_ctx* c, int op, const double* b, int nshift, const double* shifts,
                       double precision, iro_solver_out* out, int* nconv) {
  return c && b && shifts && out && nconv && nshift >= 1 && nshift <= MAXSHIFT &&
         solver_op_ok(op) && precision > 0.0;
}

extern "C" int iro_multishift_cg_solve(iro_ctx* c, int op, double mass, double csw,
                                       const double* b, int nshift, const double* shifts,
                                       double* x, double precision, int max_iter,
                                       iro_solver_out* out, int* nconv) {
  if (!x || !ms_args_ok(c, op, b, nshift, shifts, precision, out, nconv))
    return set_error(c, IRO_BAD_ARG, "bad multishift arguments");
  CK(cudaSetDevice(device(c)));
  int rc = IRO_OK;
  DevField* B = workspace(c, op_subset(op), PREC_DOUBLE, 1, 30, &rc); if (!B) return rc;
  RC(import_field(c, b, op_is_full(op), *B));
  return ms_run(c, op, mass, csw, B, nshift, shifts, x, nullptr, precision, max_iter, out, nconv,
                nullptr);
}

// ---- mixed-precision multishift ------------------------------------------------------
// MultiShiftSolver_CG::solve with the Krylov vectors in FP32: FP64 is kept
// for the zeta/alpha/beta recurrences (MSState, the reference's update order
// as in ms_run), the reductions, the residual recomputations and the
// solutions.
//   1. The reference's multishift iteration on FP32 vectors (r, p_k and
//      per-shift FP32 accumulators of x_k) and the FP32 operator, with
//      reliable updates on shift 0 (Sleijpen & van der Vorst; for multishift
//      on GPUs, Clark et al., "Solving lattice QCD systems of equations using
//      mixed precision solvers on GPUs", CPC 181 (2010)): when |r| fell by
//      delta since the last update, or looks converged, the accumulators are
//      added to the FP64 solutions and r = b - (A + sigma_0) x_0 is
//      recomputed in FP64; shift 0 converges on that FP64 residual.
//   2. r_k = b - (A + sigma_k) x_k in FP64 for every shift: after the first
//      update the shifted residuals are no longer exactly collinear with r, so
//      the shifted systems stop near the FP32 rounding level.
//   3. A reliable-update CG on (A + sigma_k) e_k = r_k for the shifts above
//      the goal, all of them as ONE block of right-hand sides, each to
//      |r_k - (A + sigma_k) e_k|^2 < precision |b|^2; x_k += e_k.  This
//      takes a few iterations: the remaining residuals are rounding noise,
//      not unconverged low modes.
//   4. The FP64 true residual of every shift.
namespace {
// reliable-update trigger of the FP32 multishift: every two decades (the
// shifted systems' accuracy does not depend on it, the number of FP64
// recomputations does)
constexpr double kMsDelta = 0.01;

int ms_mixed(iro_ctx* c, int op, double mass, double csw, const DevField* B, int nshift,
             const double* shifts, double* x, DevField* xblock, double precision, int max_iter,
             int inner, iro_solver_out* out, int* nconv) {
  CK(cudaSetDevice(device(c)));
  auto t0 = std::chrono::steady_clock::now();
  const int sub = op_subset(op);
  const bool full = op_is_full(op);
  const int p1 = PREC_SINGLE;
  int rc = IRO_OK;
  DevField* R = workspace(c, sub, p1, 1, 31, &rc); if (!R) return rc;
  DevField* S = workspace(c, sub, p1, 1, 32, &rc); if (!S) return rc;
  DevField* Q = workspace(c, sub, p1, 1, 33, &rc); if (!Q) return rc;
  DevField* R64 = workspace(c, sub, PREC_DOUBLE, 1, 31, &rc); if (!R64) return rc;
  DevField* S64 = workspace(c, sub, PREC_DOUBLE, 1, 32, &rc); if (!S64) return rc;
  DevField* Q64 = workspace(c, sub, PREC_DOUBLE, 1, 33, &rc); if (!Q64) return rc;
  std::vector<DevField*> XS(nshift), PS(nshift), X64(nshift);
  for (int k = 0; k < nshift; ++k) {
    XS[k] = workspace(c, sub, p1, 1, 40 + k, &rc); if (!XS[k]) return rc;
    PS[k] = workspace(c, sub, p1, 1, 40 + MAXSHIFT + k, &rc); if (!PS[k]) return rc;
    X64[k] = workspace(c, sub, PREC_DOUBLE, 1, 40 + k, &rc); if (!X64[k]) return rc;
  }
  cudaStream_t st = stream(c);
  std::vector<double> bn;
  RC(norms(c, *B, nullptr, bn, nullptr));
  // ---- 1. solve_init (multiShiftSolver_CG.cpp:10-32): p_k = b, x_k = 0, r = b
  RC(convert(c, *B, *R));
  for (int k = 0; k < nshift; ++k) {
    RC(axpby(c, 1.0, *R, 0.0, *R, *PS[k]));
    RC(axpby(c, 0.0, *R, 0.0, *R, *XS[k]));
    RC(axpby(c, 0.0, *B, 0.0, *B, *X64[k]));
  }
  MSState m;
  std::memset(&m, 0, sizeof(m));
  m.rr = bn[0];
  m.maxrr = bn[0];
  m.delta2 = kMsDelta * kMsDelta;
  m.alphap = 0.0;
  m.betap = 1.0;
  m.snorm = 1.0 / bn[0];
  m.prec = precision;
  m.sigma0 = shifts[0];
  m.nshift = nshift;
  m.nshift2 = nshift;
  m.conv_iter = -1;
  for (int k = 0; k < nshift; ++k) {
    m.csh2[k] = shifts[k] - shifts[0];
    m.zeta1[k] = m.zeta2[k] = 1.0;
  }
  int zero = 0;
  CK(cudaMemcpyAsync(state(c), &m, sizeof(m), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(done(c), &zero, sizeof(int), cudaMemcpyHostToDevice, st));
  MSFields f, f64;
  for (int k = 0; k < MAXSHIFT; ++k) {
    f.x[k] = XS[k < nshift ? k : 0]->all();
    f.p[k] = PS[k < nshift ? k : 0]->all();
    f64.x[k] = X64[k < nshift ? k : 0]->all();
    f64.p[k] = f.p[k];
  }
  RC(apply(c, op, mass, csw, false, *PS[0], *Q, nullptr, 0, nullptr));  // autotuning, outside capture
  RC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, nullptr));
  const MSState* dm = static_cast<const MSState*>(state(c));
  Reduce ralpha = reduce(c, ST_MS_ALPHA, max_iter);
  Reduce rr = reduce(c, ST_MS_R, max_iter);
  Reduce rpp = reduce(c, ST_MS_PP, max_iter);
  const int* skip = done(c);
  auto body = [&](int n) -> int {
    for (int i = 0; i < n; ++i) {
      RC(apply(c, op, mass, csw, false, *PS[0], *Q, &ralpha, RED_OUT2 | RED_X2, skip));
      RC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, skip));
      CK(launch_ms_xr(p1, B->sites(), XS[0]->all(), R->all(), PS[0]->all(), S->all(), dm, rr,
                      max_blocks(c), st));
      CK(launch_ms_p(p1, B->sites(), nshift, f, R->all(), dm, rpp, max_blocks(c), st));
    }
    return IRO_OK;
  };
  cudaGraphExec_t exec = nullptr;
  if (st != nullptr) {
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int brc = body(kChunk);
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (brc) return brc;
    if (e != cudaSuccess) return cuda_error(c, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_error(c, e, "cudaGraphInstantiate");
  }
  struct ExecGuard {
    cudaGraphExec_t e;
    ~ExecGuard() { if (e) cudaGraphExecDestroy(e); }
  } guard{exec};
  int* hpin = static_cast<int*>(pinned(c));
  int merged_upto = nshift;  // shifts active since the last merge
  int updates = 0, launched = 0;
  bool converged = false;
  ShiftList s0{};
  s0.s[0] = shifts[0];
  while (launched < max_iter) {
    if (exec) CK(cudaGraphLaunch(exec, st));
    else RC(body(kChunk));
    launched += kChunk;
    CK(cudaMemcpyAsync(hpin, done(c), sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hpin[0] == RUNNING) continue;
    if (hpin[0] != PAUSED) break;  // stopped at max_iter
    // reliable update: x_k += xlo_k; r = b - (A + sigma_0) x_0 in FP64
    CK(cudaMemcpyAsync(&m, state(c), sizeof(m), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(launch_ms_merge(B->sites(), merged_upto, f64, f, st));
    merged_upto = m.nshift2;
    RC(apply(c, op, mass, csw, false, *X64[0], *Q64, nullptr, 0, nullptr));
    RC(apply(c, op, mass, csw, true, *Q64, *S64, nullptr, 0, nullptr));
    CK(launch_ms_block_residual(B->sites(), 1, B->all(), S64->all(), X64[0]->all(), s0, R64->all(), st));
    std::vector<double> rt;
    RC(norms(c, *R64, nullptr, rt, nullptr));
    RC(convert(c, *R64, *R));
    ++updates;
    m.rr = rt[0];
    m.maxrr = rt[0];
    int dflag = RUNNING;
    if (m.rr * m.snorm < precision) {
      m.conv_iter = m.iter - 1;
      dflag = CONVERGED;
      converged = true;
    } else if (m.iter >= max_iter) {
      dflag = STOPPED;
    }
    CK(cudaMemcpyAsync(state(c), &m, sizeof(m), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(done(c), &dflag, sizeof(int), cudaMemcpyHostToDevice, st));
    if (dflag != RUNNING) break;
  }
  CK(cudaMemcpyAsync(&m, state(c), sizeof(m), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (!converged) CK(launch_ms_merge(B->sites(), merged_upto, f64, f, st));
  const int iter1 = m.iter;
  // ---- 2. the shifted residuals in FP64, one block of nshift right-hand sides
  DevField* XB = workspace(c, sub, PREC_DOUBLE, nshift, 70, &rc); if (!XB) return rc;
  DevField* QB = workspace(c, sub, PREC_DOUBLE, nshift, 71, &rc); if (!QB) return rc;
  DevField* SB = workspace(c, sub, PREC_DOUBLE, nshift, 72, &rc); if (!SB) return rc;
  DevField* RB = workspace(c, sub, PREC_DOUBLE, nshift, 73, &rc); if (!RB) return rc;
  DevField* EB = workspace(c, sub, PREC_DOUBLE, nshift, 74, &rc); if (!EB) return rc;
  ShiftList sl{};
  for (int k = 0; k < nshift; ++k) sl.s[k] = shifts[k];
  CK(launch_ms_pack(PREC_DOUBLE, B->sites(), nshift, f64, XB->all(), st));
  auto residuals = [&](std::vector<double>& rn) -> int {
    RC(apply(c, op, mass, csw, false, *XB, *QB, nullptr, 0, nullptr));
    RC(apply(c, op, mass, csw, true, *QB, *SB, nullptr, 0, nullptr));
    CK(launch_ms_block_residual(B->sites(), nshift, B->all(), SB->all(), XB->all(), sl, RB->all(), st));
    return norms(c, *RB, nullptr, rn, nullptr);
  };
  std::vector<double> rn;
  RC(residuals(rn));
  // ---- 3. refinement of the shifts above the goal, one block
  bool refine = false;
  for (int k = 0; k < nshift; ++k) refine = refine || !(rn[k] < precision * bn[0]);
  int it2 = 0, upd2 = 0, applies2 = 0, rc2 = IRO_OK;
  if (refine && converged) {
    std::vector<double> goal(nshift);
    for (int k = 0; k < nshift; ++k)
      goal[k] = rn[k] > 0.0 ? 0.9 * precision * bn[0] / rn[k] : 1.0;
    iro_cg_params p2;
    p2.precision = precision;
    p2.max_iter = max_iter;
    p2.inner_prec = inner;
    // FP32 inner storage carries the refinement (3-4 decades) to one FP64
    // recomputation; FP16 needs one per decade
    p2.delta = inner == PREC_SINGLE ? 1e-4 : 0.1;
    p2.use_graph = 1;
    std::vector<iro_solver_out> o2(nshift);
    rc2 = cg_mixed(c, op, mass, csw, &p2, RB, EB, nshift, o2.data(), shifts, goal.data());
    if (rc2 != IRO_OK && rc2 != IRO_NOT_CONVERGED) return rc2;
    RC(axpby(c, 1.0, *XB, 1.0, *EB, *XB));
    // the refinement's final FP64 true residual of (A + sigma_k) e_k = r_k is
    // the shift's residual b - (A + sigma_k)(x_k + e_k), relative to |r_k|
    for (int k = 0; k < nshift; ++k) rn[k] *= o2[k].diff * o2[k].diff;
    for (int k = 0; k < nshift; ++k) {
      if (o2[k].iterations + 1 > it2) it2 = o2[k].iterations + 1;
      if (o2[k].reliable_updates > upd2) upd2 = o2[k].reliable_updates;
      applies2 += o2[k].operator_applies;
    }
  }
  // ---- 4. the true residuals
  double dmax = 0.0;
  for (int k = 0; k < nshift; ++k) {
    const double d = rn[k] / bn[0];
    if (d > dmax) dmax = d;
  }
  if (x) RC(export_field(c, *XB, full, x));
  if (xblock) RC(axpby(c, 1.0, *XB, 0.0, *XB, *xblock));
  auto t1 = std::chrono::steady_clock::now();
  const bool conv = converged && dmax < precision && rc2 == IRO_OK;
  out->diff = std::sqrt(dmax);
  out->iterations = conv ? iter1 + it2 - 1 : -1;
  out->timing_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  out->reliable_updates = updates + upd2;
  out->operator_applies = iter1 + 2 * updates + applies2 + 2 * nshift;
  *nconv = out->iterations;
  if (!conv) return set_error(c, IRO_NOT_CONVERGED, "Not converged.");
  return IRO_OK;
}
}  // namespace

extern "C" int iro_multishift_cg_solve_mixed(iro_ctx* c, int op, double mass, double csw,
                                             const double* b, int nshift, const double* shifts,
                                             double* x, double precision, int max_iter,
                                             int inner_prec, iro_solver_out* out, int* nconv) {
  if (!x || !ms_args_ok(c, op, b, nshift, shifts, precision, out, nconv) || inner_prec < 0 ||
      inner_prec > 2)
    return set_error(c, IRO_BAD_ARG, "bad multishift arguments");
  for (int k = 1; k < nshift; ++k)
    if (!(shifts[k] >= shifts[k - 1]))
      return set_error(c, IRO_BAD_ARG, "shifts must be ascending (the smallest first)");
  CK(cudaSetDevice(device(c)));
  int rc = IRO_OK;
  DevField* B = workspace(c, op_subset(op), PREC_DOUBLE, 1, 30, &rc); if (!B) return rc;
  RC(import_field(c, b, op_is_full(op), *B));
  if (inner_prec == PREC_DOUBLE)
    return ms_run(c, op, mass, csw, B, nshift, shifts, x, nullptr, precision, max_iter, out, nconv,
                  nullptr);
  if (op == IRO_OP_CLOVER_FULL || op == IRO_OP_CLOVER_SCHUR_EE) RC(clover_ready(c, mass, csw));
  return ms_mixed(c, op, mass, csw, B, nshift, shifts, x, nullptr, precision, max_iter, inner_prec,
                  out, nconv);
}

extern "C" int iro_multishift_cg_solve_field(iro_ctx* c, int op, double mass, double csw,
                                             const iro_field* b, int nshift, const double* shifts,
                                             iro_field* x, double precision, int max_iter,
                                             int inner_prec, iro_solver_out* out, int* nconv) {
  const DevField* B = field_dev(const_cast<iro_field*>(b));
  DevField* X = field_dev(x);
  if (!c || !B || !X || !shifts || !out || !nconv || nshift < 1 || nshift > MAXSHIFT ||
      !solver_op_ok(op) || !(precision > 0.0) || inner_prec < 0 || inner_prec > 2 ||
      B->prec != PREC_DOUBLE || B->nrhs != 1 || B->subset != op_subset(op) ||
      X->prec != PREC_DOUBLE || X->nrhs != nshift || X->subset != op_subset(op))
    return set_error(c, IRO_BAD_ARG, "bad multishift field arguments");
  for (int k = 1; k < nshift; ++k)
    if (!(shifts[k] >= shifts[k - 1]))
      return set_error(c, IRO_BAD_ARG, "shifts must be ascending (the smallest first)");
  CK(cudaSetDevice(device(c)));
  if (inner_prec == PREC_DOUBLE)
    return ms_run(c, op, mass, csw, B, nshift, shifts, nullptr, X, precision, max_iter, out, nconv,
                  nullptr);
  if (op == IRO_OP_CLOVER_FULL || op == IRO_OP_CLOVER_SCHUR_EE) RC(clover_ready(c, mass, csw));
  return ms_mixed(c, op, mass, csw, B, nshift, shifts, nullptr, X, precision, max_iter, inner_prec,
                  out, nconv);
}

// RationalSolver_CG::solve (lib/Solver/rationalSolver_CG.cpp:12-39): the
// multishift solve with the poles as shifts, then sol = c0 b + sum_i r_i x_i
// in one pass over the shifted solutions on the device.
extern "C" int iro_rational_cg_solve(iro_ctx* c, int op, double mass, double csw,
                                     const double* b, int npole, const double* poles,
                                     const double* residues, double c0, double* sol,
                                     double precision, int max_iter, iro_solver_out* out,
                                     int* nconv) {
  if (!sol || !residues || !ms_args_ok(c, op, b, npole, poles, precision, out, nconv))
    return set_error(c, IRO_BAD_ARG, "bad rational solver arguments");
  CK(cudaSetDevice(device(c)));
  std::vector<DevField*> xs;
  int wrc0 = IRO_OK;
  DevField* B = workspace(c, op_subset(op), PREC_DOUBLE, 1, 30, &wrc0); if (!B) return wrc0;
  RC(import_field(c, b, op_is_full(op), *B));
  const int rc = ms_run(c, op, mass, csw, B, npole, poles, nullptr, nullptr, precision, max_iter,
                        out, nconv, &xs);
  if (rc != IRO_OK && rc != IRO_NOT_CONVERGED) return rc;
  const int sub = op_subset(op);
  int wrc = IRO_OK;
  DevField* Y = workspace(c, sub, PREC_DOUBLE, 1, 34, &wrc);
  if (!Y) return wrc;
  SField list{};
  for (int k = 0; k < npole; ++k) {
    list.f[k] = xs[k]->all();
    list.a[k] = residues[k];
  }
  CK(launch_combine(B->sites(), c0, B->all(), npole, list, Y->all(), stream(c)));
  RC(export_field(c, *Y, op_is_full(op), sol));
  return rc;
}

// ---- mixed-precision reliable-update CG ----------------------------------------------
// Inner CG iterations run on FP32 or FP16 storage with FP32 arithmetic; the
// solution is accumulated in FP64 and, whenever the iterated residual has
// fallen by `delta` since the last recomputation (or looks converged), the
// residual is recomputed in FP64 as r = b - A x and the iteration continues
// from it (reliable updates: Sleijpen & van der Vorst, "Reliable updated
// residuals in hybrid Bi-CG methods", Computing 56 (1996); the FP32/FP16
// variant follows Clark et al., "Solving lattice QCD systems of equations
// using mixed precision solvers on GPUs", CPC 181 (2010)).  Convergence is
// declared only on the FP64 true residual.  The starting guess is x0 = b as
// in Solver_CG (solver_CG.cpp:40).
int cg_mixed(iro_ctx* c, int op, double mass, double csw, const iro_cg_params* prm,
             const DevField* B, DevField* X, int nrhs, iro_solver_out* out, const double* sigma,
             const double* target) {
  const int sub = op_subset(op);
  const bool full = op_is_full(op);
  const int pl = prm->inner_prec;
  int rc = IRO_OK;
  DevField* R = workspace(c, sub, PREC_DOUBLE, nrhs, 22, &rc); if (!R) return rc;
  DevField* S = workspace(c, sub, PREC_DOUBLE, nrhs, 24, &rc); if (!S) return rc;
  DevField* Q = workspace(c, sub, PREC_DOUBLE, nrhs, 25, &rc); if (!Q) return rc;
  DevField* Xl = workspace(c, sub, pl, nrhs, 26, &rc); if (!Xl) return rc;
  DevField* Rl = workspace(c, sub, pl, nrhs, 27, &rc); if (!Rl) return rc;
  DevField* Pl = workspace(c, sub, pl, nrhs, 28, &rc); if (!Pl) return rc;
  DevField* Sl = workspace(c, sub, pl, nrhs, 29, &rc); if (!Sl) return rc;
  DevField* Ql = workspace(c, sub, pl, nrhs, 19, &rc); if (!Ql) return rc;
  cudaStream_t st = stream(c);
  int* dmask = done(c) + 32;
  int* hpin = static_cast<int*>(pinned(c));
  const double delta = prm->delta > 0.0 ? prm->delta : 0.1;

  RC(axpby(c, 1.0, *B, 0.0, *B, *X));
  std::vector<CGState> hs(nrhs);
  bool shifted = false;
  for (int r = 0; r < nrhs; ++r) {
    CGState& s = hs[r];
    std::memset(&s, 0, sizeof(s));
    s.target = target ? target[r] : prm->precision;
    s.delta2 = delta * delta;
    s.conv_iter = -1;
    s.sigma = sigma ? sigma[r] : 0.0;
    shifted = shifted || s.sigma != 0.0;
  }
  const CGState* dstate = static_cast<const CGState*>(state(c));
  CK(cudaMemcpyAsync(state(c), hs.data(), sizeof(CGState) * nrhs, cudaMemcpyHostToDevice, st));
  // r = b - A x for x = b: only the inner iteration starts from this residual,
  // and the first reliable update recomputes it in FP64 from the FP64 x (which
  // is b exactly), so A x is applied in the inner precision; these launches
  // also autotune the inner operator outside the graph capture.  Then the
  // low-precision r and p, and x_lo = 0.
  RC(convert(c, *B, *Pl));
  RC(apply(c, op, mass, csw, false, *Pl, *Ql, nullptr, 0, nullptr));
  RC(apply(c, op, mass, csw, true, *Ql, *Sl, nullptr, 0, nullptr));
  RC(convert(c, *Sl, *S));
  if (shifted) CK(launch_shift_add(B->sites(), nrhs, S->all(), B->all(), dstate, st));
  Reduce rinit = reduce(c, ST_CG_INIT, prm->max_iter);
  CK(launch_cg_init(PREC_DOUBLE, B->sites(), nrhs, B->all(), S->all(), R->all(), Q->all(), rinit,
                    max_blocks(c), st));
  RC(convert(c, *R, *Rl));
  RC(convert(c, *R, *Pl));
  RC(axpby(c, 0.0, *Rl, 0.0, *Rl, *Xl));

  const int* skip = done(c);
  Reduce ralpha = reduce(c, ST_CG_ALPHA, prm->max_iter);
  Reduce rbeta = reduce(c, ST_CG_BETA, prm->max_iter);
  Reduce rnone = reduce(c, ST_NONE, 0);
  auto body = [&](int n) -> int {
    for (int i = 0; i < n; ++i) {
      if (shifted) {
        // (p, (A + sigma) p) from |M p|^2 and |p|^2; A p stored, then
        // r -= alpha (A p + sigma p) in its own pass
        RC(apply(c, op, mass, csw, false, *Pl, *Ql, &ralpha, RED_OUT2 | RED_X2, skip));
        RC(apply(c, op, mass, csw, true, *Ql, *Sl, nullptr, 0, skip));
        CK(launch_cg_shift_r(pl, Rl->sites(), nrhs, Rl->all(), Sl->all(), Pl->all(), dstate, rbeta,
                             max_blocks(c), st));
      } else {
        RC(apply(c, op, mass, csw, false, *Pl, *Ql, &ralpha, RED_OUT2, skip));
        RC(apply_cg(c, op, mass, csw, true, *Ql, *Sl, rbeta, skip, CGFuse{Rl, dstate}));
      }
      CK(launch_cg_p(pl, Pl->sites(), nrhs, Pl->all(), Rl->all(), Xl->all(), dstate, done(c), st));
    }
    return IRO_OK;
  };
  cudaGraphExec_t exec = nullptr;
  if (prm->use_graph && st != nullptr) {
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int brc = body(kChunk);
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (brc) return brc;
    if (e != cudaSuccess) return cuda_error(c, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_error(c, e, "cudaGraphInstantiate");
  }
  struct ExecGuard {
    cudaGraphExec_t e;
    ~ExecGuard() { if (e) cudaGraphExecDestroy(e); }
  } guard{exec};

  std::vector<int> updates(nrhs, 0);
  std::vector<int> hdone(nrhs), mask(nrhs);
  for (;;) {
    // inner iterations until some right-hand side pauses or all have left
    for (;;) {
      if (exec) CK(cudaGraphLaunch(exec, st));
      else RC(body(kChunk));
      CK(cudaMemcpyAsync(hpin, done(c), sizeof(int) * nrhs, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      bool any_pause = false, all_left = true;
      for (int r = 0; r < nrhs; ++r) {
        any_pause = any_pause || hpin[r] == PAUSED;
        all_left = all_left && hpin[r] != RUNNING;
      }
      if (any_pause || all_left) break;
    }
    bool any_pause = false;
    for (int r = 0; r < nrhs; ++r) {
      hdone[r] = hpin[r];
      mask[r] = hdone[r] == PAUSED ? 1 : 0;
      any_pause = any_pause || mask[r];
    }
    if (!any_pause) break;
    // reliable update of the paused right-hand sides: x += x_lo, r = b - A x
    CK(cudaMemcpyAsync(dmask, mask.data(), sizeof(int) * nrhs, cudaMemcpyHostToDevice, st));
    CK(launch_mx_merge(pl, X->sites(), nrhs, X->all(), Xl->all(), dmask, st));
    RC(apply(c, op, mass, csw, false, *X, *Q, nullptr, 0, nullptr));
    RC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, nullptr));
    if (shifted) CK(launch_shift_add(X->sites(), nrhs, S->all(), X->all(), dstate, st));
    CK(launch_mx_residual(pl, B->sites(), nrhs, B->all(), S->all(), R->all(), Rl->all(), dmask,
                          rnone, max_blocks(c), st));
    std::vector<double> rr(nrhs);
    CK(cudaMemcpyAsync(hs.data(), state(c), sizeof(CGState) * nrhs, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // the reduction's totals are in the context's output slot
    {
      Reduce tmp = rnone;
      CK(cudaMemcpyAsync(rr.data(), tmp.out, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    }
    for (int r = 0; r < nrhs; ++r) {
      if (!mask[r]) continue;
      ++updates[r];
      CGState& s = hs[r];
      s.rr = rr[r];
      s.maxrr = rr[r];
      s.beta = s.rr / s.rr_prev;
      if (s.rr < s.target) {
        s.conv_iter = s.iter - 1;
        hdone[r] = CONVERGED;
        mask[r] = 0;
      } else if (s.iter >= prm->max_iter) {
        hdone[r] = STOPPED;
        mask[r] = 0;
      } else {
        hdone[r] = RUNNING;
      }
    }
    CK(cudaMemcpyAsync(state(c), hs.data(), sizeof(CGState) * nrhs, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(dmask, mask.data(), sizeof(int) * nrhs, cudaMemcpyHostToDevice, st));
    CK(launch_mx_p(pl, Pl->sites(), nrhs, Pl->all(), Rl->all(),
                   static_cast<const CGState*>(state(c)), dmask, st));
    CK(cudaMemcpyAsync(done(c), hdone.data(), sizeof(int) * nrhs, cudaMemcpyHostToDevice, st));
    bool all_left = true;
    for (int r = 0; r < nrhs; ++r) all_left = all_left && hdone[r] != RUNNING;
    if (all_left) break;
  }
  // every right-hand side converged on an FP64 true residual just computed at
  // its last reliable update (x merged, r = b - A x): that residual is final
  bool all_conv = true;
  for (int r = 0; r < nrhs; ++r) all_conv = all_conv && hdone[r] == CONVERGED;
  if (all_conv) {
    for (int r = 0; r < nrhs; ++r) {
      // target = goal |b|^2
      const double bb = hs[r].target / (target ? target[r] : prm->precision);
      out[r].diff = std::sqrt(hs[r].rr / bb);
      out[r].iterations = hs[r].conv_iter;
      out[r].reliable_updates = updates[r];
      out[r].operator_applies = hs[r].iter + 2 * updates[r] + 1;
    }
    return IRO_OK;
  }
  // fold any remaining low-precision correction in, then the FP64 true residual
  std::vector<int> ones(nrhs, 1);
  CK(cudaMemcpyAsync(dmask, ones.data(), sizeof(int) * nrhs, cudaMemcpyHostToDevice, st));
  CK(launch_mx_merge(pl, X->sites(), nrhs, X->all(), Xl->all(), dmask, st));
  RC(apply(c, op, mass, csw, false, *X, *Q, nullptr, 0, nullptr));
  RC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, nullptr));
  if (shifted) CK(launch_shift_add(X->sites(), nrhs, S->all(), X->all(), dstate, st));
  RC(axpby(c, 1.0, *S, -1.0, *B, *R));
  std::vector<double> rn, bn;
  RC(norms(c, *R, B, rn, &bn));
  CK(cudaMemcpyAsync(hs.data(), state(c), sizeof(CGState) * nrhs, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  int status = IRO_OK;
  for (int r = 0; r < nrhs; ++r) {
    out[r].diff = std::sqrt(rn[r] / bn[r]);
    out[r].iterations = hs[r].conv_iter;
    out[r].reliable_updates = updates[r];
    out[r].operator_applies = hs[r].iter + 2 * updates[r] + 2;
    if (hs[r].conv_iter < 0) status = IRO_NOT_CONVERGED;
  }
  if (status) set_error(c, status, "mixed-precision CG not converged");
  return status;
}

// ---- even/odd inversion of the full operator -------------------------------------
namespace {
// the half `p` of a full-lattice field, as a field of its own
DevField half_view(const DevField& F, int p) {
  DevField h = F;
  const SpinorPtr s = F.half(p);
  h.subset = p;
  h.data = s.data;
  h.norm = s.norm;
  h.bytes_data = F.bytes_data / 2;
  h.bytes_norm = F.bytes_norm / 2;
  return h;
}
}  // namespace

// Inverter_WilsonLike::invert (lib/Dirac_ops/eoUtils.cpp:43-81), for nrhs
// full-lattice sources at once.  With the full operator in blocks
// D = [[A_ee, D_eo], [D_oe, A_oo]] (D_eo = -kappa H_eo; A = 1 for Wilson,
// whose mult_ee_inv / mult_oo_inv are the identity, and the clover term for
// clover):
//   be  = b_e - D_eo A_oo^-1 b_o,
//   y_e = M^-1 be by CG on M^dag M y_e = M^dag be (M the Schur operator),
//   x_o = A_oo^-1 (b_o - D_oe y_e),
// and sol = (y_e, x_o) in the full Format_F layout.  out[] holds the CG's
// outputs, as the reference prints its SolverOutput.
namespace {
// The e/o inversion of the nrhs full-lattice FP64 sources in F, in place:
// F holds the solutions on return.
int eo_invert_dev(iro_ctx* c, int op, double mass, double csw, const iro_cg_params* prm,
                  DevField* F, int nrhs, iro_solver_out* out) {
  const bool cl = op == IRO_OP_CLOVER_SCHUR_EE;
  int rc = IRO_OK;
  DevField* BE = workspace(c, 0, PREC_DOUBLE, nrhs, 51, &rc); if (!BE) return rc;
  DevField* RHS = workspace(c, 0, PREC_DOUBLE, nrhs, 52, &rc); if (!RHS) return rc;
  DevField* YE = workspace(c, 0, PREC_DOUBLE, nrhs, 53, &rc); if (!YE) return rc;
  DevField* TO = workspace(c, 1, PREC_DOUBLE, nrhs, 54, &rc); if (!TO) return rc;
  cudaStream_t st = stream(c);
  DevField fe = half_view(*F, 0), fo = half_view(*F, 1);
  // t_o = A_oo^-1 b_o;  be = b_e - D_eo t_o
  const DevField* bo = &fo;
  if (cl) {
    CK(launch_clover_mult(vh(c), nrhs, clover(c, PREC_DOUBLE, 1, true), fo.half(1), TO->half(1), st));
    bo = TO;
  }
  RC(apply(c, IRO_OP_WILSON_HOP_EO, mass, csw, false, *bo, *BE, nullptr, 0, nullptr));
  RC(axpby(c, 1.0, fe, -1.0, *BE, *BE));
  // M^dag M y_e = M^dag be
  RC(apply(c, op, mass, csw, true, *BE, *RHS, nullptr, 0, nullptr));
  const int solve_rc = cg_any(c, op, mass, csw, prm, RHS, YE, nrhs, out);
  if (solve_rc != IRO_OK && solve_rc != IRO_NOT_CONVERGED) return solve_rc;
  // x_o = A_oo^-1 (b_o - D_oe y_e), written over the odd half of F; y_e over the even half
  RC(apply(c, IRO_OP_WILSON_HOP_OE, mass, csw, false, *YE, *TO, nullptr, 0, nullptr));
  RC(axpby(c, 1.0, fo, -1.0, *TO, *TO));
  if (cl)
    CK(launch_clover_mult(vh(c), nrhs, clover(c, PREC_DOUBLE, 1, true), TO->half(1), fo.half(1), st));
  else
    RC(axpby(c, 1.0, *TO, 0.0, *TO, fo));
  RC(axpby(c, 1.0, *YE, 0.0, *YE, fe));
  return solve_rc;
}
}  // namespace

extern "C" int iro_eo_invert(iro_ctx* c, int op, double mass, double csw,
                             const iro_cg_params* prm, const double* src, double* sol, int nrhs,
                             iro_solver_out* out) {
  if (!c || !src || !sol || !out || nrhs < 1 || nrhs > 16 || !cg_args_ok(prm, op) ||
      (op != IRO_OP_WILSON_SCHUR_EE && op != IRO_OP_CLOVER_SCHUR_EE))
    return set_error(c, IRO_BAD_ARG, "bad e/o inverter arguments");
  CK(cudaSetDevice(device(c)));
  if (op == IRO_OP_CLOVER_SCHUR_EE) RC(clover_ready(c, mass, csw));
  int rc = IRO_OK;
  DevField* F = workspace(c, 2, PREC_DOUBLE, nrhs, 50, &rc); if (!F) return rc;
  RC(import_field(c, src, true, *F));
  const int solve_rc = eo_invert_dev(c, op, mass, csw, prm, F, nrhs, out);
  if (solve_rc != IRO_OK && solve_rc != IRO_NOT_CONVERGED) return solve_rc;
  RC(export_field(c, *F, true, sol));
  return solve_rc;
}

// Qprop_EvenOdd::calc (lib/Measurements/FermionicM/qprop_EvenOdd.cpp:10-28)
// on the point sources of Source_local (source_types.hpp:23-60): source
// r = 3 s + c is 1 at the real part of spin s, colour c of the lattice site
// `site` (SiteIndex::site order, x fastest).  The sources r = first ..
// first + nrhs - 1 are built on the device (the reference builds each one as
// a host field) and inverted as one block; sol receives them in that order.
extern "C" int iro_qprop_point(iro_ctx* c, int op, double mass, double csw,
                               const iro_cg_params* prm, int64_t site, int first, int nrhs,
                               double* sol, iro_solver_out* out) {
  if (!c || !sol || !out || nrhs < 1 || first < 0 || first + nrhs > 12 || !cg_args_ok(prm, op) ||
      (op != IRO_OP_WILSON_SCHUR_EE && op != IRO_OP_CLOVER_SCHUR_EE) || site < 0 ||
      site >= volume(c))
    return set_error(c, IRO_BAD_ARG, "bad point-source inverter arguments");
  CK(cudaSetDevice(device(c)));
  if (op == IRO_OP_CLOVER_SCHUR_EE) RC(clover_ready(c, mass, csw));
  int rc = IRO_OK;
  DevField* F = workspace(c, 2, PREC_DOUBLE, nrhs, 50, &rc); if (!F) return rc;
  const Geom& g = geom(c);
  const int64_t x = site % g.L[0], y = site / g.L[0] % g.L[1], z = site / (int64_t(g.L[0]) * g.L[1]) % g.L[2],
                t = site / (int64_t(g.L[0]) * g.L[1] * g.L[2]);
  CK(launch_point_sources(*F, int((x + y + z + t) & 1), site >> 1, first, stream(c)));
  const int solve_rc = eo_invert_dev(c, op, mass, csw, prm, F, nrhs, out);
  if (solve_rc != IRO_OK && solve_rc != IRO_NOT_CONVERGED) return solve_rc;
  RC(export_field(c, *F, true, sol));
  return solve_rc;
}

// ---- molecular-dynamics force ----------------------------------------------------
// Dirac_Wilson::md_force (lib/Dirac_ops/dirac_wilson.cpp:41-58):
//   F = -kappa sum_{x, mu} [mkfrc(eta, zeta) + mkfrc(g5 zeta, g5 eta)]
// Dirac_Wilson_EvenOdd::md_force (lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:95-117):
//   A = Doe eta, B = Doe^dag zeta (odd);
//   F = kappa [Deo.p(A, zeta) + Doe.m(A, zeta) + Doe.p(eta, B) + Deo.m(eta, B)]
// with X.p(e, z) = mkfrc(e, z) and X.m(e, z) = mkfrc(g5 z, g5 e) on the
// output sites of X (even for Deo, odd for Doe), in that order.
extern "C" int iro_md_force(iro_ctx* c, int op, double mass, double csw, const double* eta,
                            const double* zeta, double* force) {
  if (!c || !eta || !zeta || !force ||
      (op != IRO_OP_WILSON_FULL && op != IRO_OP_WILSON_SCHUR_EE && op != IRO_OP_CLOVER_FULL))
    return set_error(c, IRO_BAD_ARG, "bad md_force arguments");
  if (!gauge_loaded(c)) return set_error(c, IRO_NO_GAUGE, "no gauge field uploaded");
  CK(cudaSetDevice(device(c)));
  const bool full = op != IRO_OP_WILSON_SCHUR_EE;
  const double k = 0.5 / (4.0 + mass);
  int rc = IRO_OK;
  const int sub = full ? 2 : 0;
  DevField* E = workspace(c, sub, PREC_DOUBLE, 1, 60, &rc); if (!E) return rc;
  DevField* Z = workspace(c, sub, PREC_DOUBLE, 1, 61, &rc); if (!Z) return rc;
  cudaStream_t st = stream(c);
  RC(import_field(c, eta, full, *E));
  RC(import_field(c, zeta, full, *Z));
  const size_t nF = size_t(72) * size_t(volume(c));
  const bool clover_term = op == IRO_OP_CLOVER_FULL && csw != 0.0;
  const size_t nL = clover_term ? size_t(6) * 9 * size_t(volume(c)) : 0;
  // the force and (clover) Lambda_k in the context's solver scratch, which
  // stays allocated: repeated calls allocate nothing
  const size_t f_bytes = (nF * sizeof(double) + 255) / 256 * 256;
  char* scr = static_cast<char*>(scratch(c, f_bytes + nL * sizeof(double2), &rc));
  if (!scr) return rc;
  double* F = reinterpret_cast<double*>(scr);
  CK(cudaMemsetAsync(F, 0, nF * sizeof(double), st));
  const Geom& g = geom(c);
  const GaugePtr U = gauge_double(c);
  const int recon = gauge_recon(c);
  if (full) {
    for (int p = 0; p < 2; ++p) {
      CK(launch_force(g, U, recon, p, E->half(1 - p), Z->half(p), 0, -k, F, st));
      CK(launch_force(g, U, recon, p, Z->half(1 - p), E->half(p), 1, -k, F, st));
    }
    if (clover_term) {
      // the clover block of Dirac_Clover::md_force: Lambda_k for the 6 planes
      // (6 * 9 complex per site), then the leaf derivatives; its site offsets
      // reach two sites out, which one periodic wrap covers for extents >= 2
      for (int d = 0; d < 4; ++d)
        if (g.L[d] < 2) return set_error(c, IRO_BAD_ARG, "clover force needs every extent >= 2");
      double2* lam = reinterpret_cast<double2*>(scr + f_bytes);
      CK(launch_clover_force(g, gauge_format_g(c), E->half(0), E->half(1), Z->half(0), Z->half(1),
                             -k * csw / 4.0, lam, F, st));
    }
  } else {
    DevField* A = workspace(c, 1, PREC_DOUBLE, 1, 62, &rc); if (!A) return rc;
    DevField* B = workspace(c, 1, PREC_DOUBLE, 1, 63, &rc); if (!B) return rc;
    RC(apply(c, IRO_OP_WILSON_HOP_OE, mass, 0.0, false, *E, *A, nullptr, 0, nullptr));
    RC(apply(c, IRO_OP_WILSON_HOP_OE, mass, 0.0, true, *Z, *B, nullptr, 0, nullptr));
    CK(launch_force(g, U, recon, 0, A->half(1), Z->half(0), 0, k, F, st));
    CK(launch_force(g, U, recon, 1, Z->half(0), A->half(1), 1, k, F, st));
    CK(launch_force(g, U, recon, 1, E->half(0), B->half(1), 0, k, F, st));
    CK(launch_force(g, U, recon, 0, B->half(1), E->half(0), 1, k, F, st));
  }
  return device_to_host(c, force, F, nF * sizeof(double));
}
