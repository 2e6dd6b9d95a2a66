// FP64 reductions and the Krylov solvers' scalar recurrences, kept on the
// device so that an iteration needs no host round trip.
//
// A kernel that reduces hands its per-thread partial sums to
// block_reduce_finish(): a fixed-order tree inside the block, one partial per
// block in global scratch; the last block to arrive in each group of 32
// consecutive blocks sums that group's partials in block order, and the last
// group to finish sums the group partials in group order (ticket counters,
// so the result is deterministic run to run) and then applies the solver
// stage's scalar update (alpha, beta, convergence flags, multishift zeta
// recurrences).
#pragma once

#include "common.cuh"

namespace iro {

// Per right-hand side CG state (Solver_CG::solve_step, lib/Solver/solver_CG.cpp:82-160).
struct CGState {
  double rr;       // (r,r)
  double rr_prev;  // (r,r) of the previous iteration
  double pap;      // (p,Ap)
  double alpha;    // rr/pap
  double beta;     // rr/rr_prev
  double target;   // GoalPrecision * |b|^2
  double maxrr;    // (r,r) at the last reliable update (mixed precision)
  double delta2;   // reliable-update trigger delta^2; 0 for plain CG
  int iter;        // iterations completed
  int conv_iter;   // 0-based index of the converging iteration, -1 before
  int xpend;       // x += alpha p of the iteration just completed is still due
  double sigma;    // shift of the operator A + sigma (0: the plain normal operator)
};

// done[] flag values
enum { RUNNING = 0, CONVERGED = 1, STOPPED = 2, PAUSED = 3 };

// Multishift CG state (MultiShiftSolver_CG::solve_step,
// lib/Solver/multiShiftSolver_CG.cpp:34-93); shift arrays have MAXSHIFT slots.
constexpr int MAXSHIFT = 16;
// iterations per window of the FP64 multishift solver that keeps the
// residuals instead of updating every shift's x and p (ms_run)
constexpr int MSW_MAX = 32;
struct MSState {
  double rr, rrp, pap, alpha, beta, alphap, betap, snorm, prec, sigma0;
  double maxrr;   // (r,r) at the last reliable update (mixed precision)
  double delta2;  // reliable-update trigger delta^2; 0 for the FP64 solver
  int nshift, nshift2, iter, conv_iter;
  double csh2[MAXSHIFT], zeta1[MAXSHIFT], zeta2[MAXSHIFT], zeta[MAXSHIFT];
  double betas[MAXSHIFT], alphas[MAXSHIFT], pp[MAXSHIFT];
  // Residual window (stages ST_MSW_*): the window began at iteration k0 and
  // holds wsize iterations; q[k] is |p_k|^2 carried by its recurrence; the
  // step scalars of window iteration w are kept for the host's fold:
  // shift 0's beta and alpha, the shifts updated (nshift2) and every other
  // shift's betas, alphas and zeta.
  int k0, wsize;
  double q[MAXSHIFT];
  double hbeta[MSW_MAX], halpha[MSW_MAX];
  int hn2[MSW_MAX];
  double hbetas[MSW_MAX][MAXSHIFT], halphas[MSW_MAX][MAXSHIFT], hzeta[MSW_MAX][MAXSHIFT];
  // the fold's coefficients, written by the host (launch_msw_fold)
  double wcoef[MAXSHIFT * (2 + 2 * MSW_MAX)];
};

enum Stage {
  ST_NONE = 0,
  ST_CG_ALPHA = 1,  // totals[0] = (p,Ap)            -> alpha
  ST_CG_BETA = 2,   // totals[0] = (r,r)             -> beta, convergence
  ST_MS_ALPHA = 3,  // totals[0]=|Mp|^2, [1]=|p|^2   -> pap incl. sigma0, beta
  ST_MS_R = 4,      // totals[0] = (r,r)             -> alpha, zeta recurrences
  ST_MS_PP = 5,     // totals[k] = |p_k|^2 (k>=1)    -> pruning, convergence
  ST_CG_INIT = 6,   // totals[0] = (r,r), [1] = |b|^2 -> rr, target
  ST_MSW_R = 7,     // as ST_MS_R, and the step's scalars into the window history
  ST_MSW_P = 8      // |p_k|^2 by recurrence -> pruning, convergence, window full
};

// blocks per first-level group of a reduction (see block_reduce_finish)
constexpr int kReduceGroup = 32;

struct Reduce {
  double* partials;   // [blocks][nred*nrhs] scratch
  double* gpartials;  // [groups][nred*nrhs] scratch
  unsigned* counter;  // [0]: group ticket; [1 + g]: block ticket of group g; all return to zero
  double* out;        // [nred*nrhs] totals
  int stage;
  void* state;   // CGState[nrhs] or MSState
  int* done;     // per-rhs converged flags (CG)
  int max_iter;  // CG: iterations after which a right-hand side stops
};

__device__ inline void stage_update(const Reduce& R, const double* tot, int nred, int nrhs) {
  switch (R.stage) {
    case ST_CG_ALPHA: {
      CGState* s = static_cast<CGState*>(R.state);
      for (int r = 0; r < nrhs; ++r) {
        s[r].xpend = 0;  // the previous iteration's p update has run
        if (R.done[r]) continue;
        // shifted operator: (p, (A + sigma) p) = |M p|^2 + sigma |p|^2, the
        // second total being the launch's |x|^2 (x = p in its epilogue)
        s[r].pap = s[r].sigma != 0.0 ? tot[r] + s[r].sigma * tot[nrhs + r] : tot[r];
        s[r].alpha = s[r].rr / s[r].pap;
      }
    } break;
    case ST_CG_BETA: {
      CGState* s = static_cast<CGState*>(R.state);
      for (int r = 0; r < nrhs; ++r) {
        if (R.done[r]) continue;
        s[r].rr_prev = s[r].rr;
        s[r].rr = tot[r];
        s[r].xpend = 1;
        const int it = s[r].iter;
        s[r].iter = it + 1;
        if (!isfinite(s[r].rr)) {  // breakdown: stop rather than iterate to max_iter
          R.done[r] = STOPPED;
          continue;
        }
        if (s[r].delta2 > 0.0) {
          // mixed precision: pause for an FP64 residual recomputation when
          // |r| fell by delta since the last one (looking converged is
          // handled for the group below); convergence is declared on the
          // true residual only
          if (s[r].rr < s[r].delta2 * s[r].maxrr) {
            R.done[r] = PAUSED;
            continue;
          }
        } else if (s[r].rr < s[r].target) {
          s[r].beta = s[r].rr / s[r].rr_prev;
          s[r].conv_iter = it;
          R.done[r] = CONVERGED;
          continue;
        }
        s[r].beta = s[r].rr / s[r].rr_prev;
        if (s[r].iter >= R.max_iter) R.done[r] = STOPPED;
      }
      // mixed precision: when one right-hand side pauses, the others pause
      // with it, so all share one FP64 residual recomputation (which treats
      // every right-hand side in one launch anyway) instead of idling in
      // lockstep until each reaches its own trigger.  A right-hand side whose
      // iterated residual looks converged keeps iterating until every one
      // still running does: then one recomputation confirms them together,
      // instead of one per right-hand side as each crosses the target.
      bool any_pause = false, any_mixed = false, all_conv = true;
      for (int r = 0; r < nrhs; ++r) {
        any_pause = any_pause || R.done[r] == PAUSED;
        if (R.done[r] == RUNNING && s[r].delta2 > 0.0) {
          any_mixed = true;
          all_conv = all_conv && s[r].rr < s[r].target;
        }
      }
      if (any_pause || (any_mixed && all_conv))
        for (int r = 0; r < nrhs; ++r)
          if (R.done[r] == RUNNING && s[r].delta2 > 0.0) R.done[r] = PAUSED;
    } break;
    case ST_MS_ALPHA: {
      MSState* m = static_cast<MSState*>(R.state);
      if (R.done[0]) break;
      // s = A p0 + sigma0 p0 (multiShiftSolver_CG.cpp:49-50); (s,p0) =
      // |M p0|^2 + sigma0 |p0|^2
      m->pap = tot[0] + m->sigma0 * tot[1];
      m->rrp = m->rr;
      m->beta = -m->rrp / m->pap;
    } break;
    case ST_MS_R: {
      MSState* m = static_cast<MSState*>(R.state);
      if (R.done[0]) break;
      m->rr = tot[0];
      m->alpha = m->rr / m->rrp;
      m->pp[0] = m->rr;
      const double alphah = 1.0 + m->alphap * m->beta / m->betap;
      for (int k = 1; k < m->nshift2; ++k) {
        double zeta = (alphah - m->csh2[k] * m->beta) / m->zeta1[k] + (1.0 - alphah) / m->zeta2[k];
        zeta = 1.0 / zeta;
        const double zr = zeta / m->zeta1[k];
        m->betas[k] = m->beta * zr;
        m->alphas[k] = m->alpha * zr * zr;
        m->zeta[k] = zeta;
      }
    } break;
    case ST_MS_PP: {
      MSState* m = static_cast<MSState*>(R.state);
      if (R.done[0]) break;
      for (int k = 1; k < m->nshift2; ++k) {
        m->pp[k] = tot[k] * m->snorm;
        m->zeta2[k] = m->zeta1[k];
        m->zeta1[k] = m->zeta[k];
      }
      for (int k = m->nshift2 - 1; k >= 0; --k) {
        if (m->pp[k] > m->prec) {
          m->nshift2 = k + 1;
          break;
        }
      }
      m->alphap = m->alpha;
      m->betap = m->beta;
      const int it = m->iter;
      m->iter = it + 1;
      if (m->delta2 > 0.0) {
        // mixed precision: pause for a reliable update of shift 0's
        // residual when |r| fell by delta since the last one or looks
        // converged; convergence is decided on the FP64 true residual
        if (m->rr < m->delta2 * m->maxrr || m->rr * m->snorm < m->prec) R.done[0] = PAUSED;
        else if (m->iter >= R.max_iter) R.done[0] = STOPPED;
      } else if (m->rr * m->snorm < m->prec) {
        m->conv_iter = it;
        R.done[0] = 1;
      } else if (m->iter >= R.max_iter) {
        R.done[0] = 2;
      }
    } break;
    case ST_MSW_R: {
      MSState* m = static_cast<MSState*>(R.state);
      if (R.done[0]) break;
      m->rr = tot[0];
      m->alpha = m->rr / m->rrp;
      m->pp[0] = m->rr;
      const int w = m->iter - m->k0;
      m->hbeta[w] = m->beta;
      m->halpha[w] = m->alpha;
      m->hn2[w] = m->nshift2;
      const double alphah = 1.0 + m->alphap * m->beta / m->betap;
      for (int k = 1; k < m->nshift2; ++k) {
        double zeta = (alphah - m->csh2[k] * m->beta) / m->zeta1[k] + (1.0 - alphah) / m->zeta2[k];
        zeta = 1.0 / zeta;
        const double zr = zeta / m->zeta1[k];
        m->betas[k] = m->beta * zr;
        m->alphas[k] = m->alpha * zr * zr;
        m->zeta[k] = zeta;
        m->hbetas[w][k] = m->betas[k];
        m->halphas[w][k] = m->alphas[k];
        m->hzeta[w][k] = zeta;
      }
    } break;
    case ST_MSW_P: {
      MSState* m = static_cast<MSState*>(R.state);
      if (R.done[0]) break;
      // p_k' = alphas_k p_k + zeta_k r' with r' orthogonal to p_k (a CG
      // residual is orthogonal to the Krylov space of the earlier
      // iterations, which holds every p_k): |p_k'|^2 = alphas^2 |p_k|^2 +
      // zeta^2 |r'|^2, anchored to the stored p_k's norms at every fold
      for (int k = 1; k < m->nshift2; ++k) {
        m->q[k] = m->alphas[k] * m->alphas[k] * m->q[k] + m->zeta[k] * m->zeta[k] * m->rr;
        m->pp[k] = m->q[k] * m->snorm;
        m->zeta2[k] = m->zeta1[k];
        m->zeta1[k] = m->zeta[k];
      }
      for (int k = m->nshift2 - 1; k >= 0; --k) {
        if (m->pp[k] > m->prec) {
          m->nshift2 = k + 1;
          break;
        }
      }
      m->alphap = m->alpha;
      m->betap = m->beta;
      const int it = m->iter;
      m->iter = it + 1;
      if (m->rr * m->snorm < m->prec) {
        m->conv_iter = it;
        R.done[0] = CONVERGED;
      } else if (m->iter >= R.max_iter) {
        R.done[0] = STOPPED;
      } else if (m->iter - m->k0 >= m->wsize) {
        R.done[0] = PAUSED;  // the window is full: the host folds it
      }
    } break;
    case ST_CG_INIT: {
      CGState* s = static_cast<CGState*>(R.state);
      for (int r = 0; r < nrhs; ++r) {
        s[r].rr = tot[r];
        s[r].maxrr = tot[r];
        s[r].target *= tot[nrhs + r];  // GoalPrecision * |b|^2
        s[r].iter = 0;
        s[r].conv_iter = -1;
        R.done[r] = (R.max_iter <= 0) ? STOPPED : RUNNING;
      }
    } break;
    default:
      break;
  }
}

// Each thread holds RPT consecutive right-hand sides: v[j*NRED + k] is value k
// of right-hand side (RPT*t + j) mod nrhs.  Block size must be (nrhs/RPT)*2^k
// (so each thread keeps its right-hand sides across a grid-stride loop whose
// stride is a multiple of nrhs/RPT).
template <int NRED, int RPT = 1>
__device__ void block_reduce_finish(const Reduce& R, const double* v, int nrhs, int bid, int nblk) {
  __shared__ double sm[NRED][256 * RPT];
  __shared__ bool last;
  const int t = threadIdx.x;
  const int n = blockDim.x;
#pragma unroll
  for (int j = 0; j < RPT; ++j)
#pragma unroll
    for (int k = 0; k < NRED; ++k) sm[k][RPT * t + j] = v[j * NRED + k];
  __syncthreads();
  for (int s = (RPT * n / nrhs) / 2; s > 0; s >>= 1) {
    for (int u = t; u < s * nrhs; u += n) {
#pragma unroll
      for (int k = 0; k < NRED; ++k) sm[k][u] += sm[k][u + s * nrhs];
    }
    __syncthreads();
  }
  const int nv = NRED * nrhs;
  for (int u = t; u < nrhs; u += n) {
#pragma unroll
    for (int k = 0; k < NRED; ++k) R.partials[int64_t(bid) * nv + k * nrhs + u] = sm[k][u];
  }
  // level 1: the last block of each group of kReduceGroup consecutive blocks
  // sums the group's partials in block order
  const int grp = bid / kReduceGroup;
  const int first = grp * kReduceGroup;
  const int gsize = min(kReduceGroup, nblk - first);
  __threadfence();
  __syncthreads();
  if (t == 0) last = (atomicAdd(R.counter + 1 + grp, 1u) == unsigned(gsize - 1));
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int q = t; q < nv; q += n) {
    const double* src = R.partials + int64_t(first) * nv + q;
    double s = 0.0;
#pragma unroll 8
    for (int j = 0; j < gsize; ++j) s += __ldcg(src + int64_t(j) * nv);
    R.gpartials[int64_t(grp) * nv + q] = s;
  }
  if (t == 0) R.counter[1 + grp] = 0u;
  // level 2: the last group to finish sums the group partials in group order
  const int ngrp = (nblk + kReduceGroup - 1) / kReduceGroup;
  __threadfence();
  __syncthreads();
  if (t == 0) last = (atomicAdd(R.counter, 1u) == unsigned(ngrp - 1));
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ double tot[NRED * 16];
  for (int q = t; q < nv; q += n) {
    double s = 0.0;
#pragma unroll 8
    for (int g = 0; g < ngrp; ++g) s += __ldcg(R.gpartials + int64_t(g) * nv + q);
    tot[q] = s;
  }
  __syncthreads();
  if (t == 0) {
    for (int q = 0; q < nv; ++q) R.out[q] = tot[q];
    *R.counter = 0u;
    stage_update(R, tot, NRED, nrhs);
    __threadfence();
  }
}

}  // namespace iro
