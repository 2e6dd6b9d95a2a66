// Kernels of the B200 fermion-solve library other than the stencil body:
// launch dispatch of the stencil, fused linear algebra of the solvers, the
// boundary conversions between the reference's host layouts and the device
// layouts, and the clover set-up.
#include <cstring>

#include "dslash.cuh"
#include "internal.h"

namespace iro {

// ---- fields ------------------------------------------------------------------
int spinor_chunk_bytes(int prec) { return 16; }
int spinor_nchunk(int prec) {
  return prec == PREC_DOUBLE ? 12 : (prec == PREC_SINGLE ? 6 : 3);
}

SpinorPtr DevField::half(int p) const {
  // full fields store the even half, then the odd half (Vh*nrhs elements each,
  // a multiple of 32, so the two halves are whole warp blocks)
  SpinorPtr s;
  const int64_t per = Vh * nrhs;
  const int64_t off = (subset == 2 && p == 1) ? per : 0;
  s.data = static_cast<char*>(data) + off * spinor_nchunk(prec) * 16;
  s.norm = norm ? norm + off : nullptr;
  return s;
}

SpinorPtr DevField::all() const {
  SpinorPtr s;
  s.data = data;
  s.norm = norm;
  return s;
}

LaunchCfg launch_cfg(int64_t vh, int nrhs, int max_blocks, int block_cap) {
  int spb = 1;
  const int cap = block_cap < nrhs ? nrhs : (block_cap > 256 ? 256 : block_cap);
  while (nrhs * spb * 2 <= cap) spb *= 2;
  LaunchCfg c;
  c.block = nrhs * spb;
  int64_t need = (vh * nrhs + c.block - 1) / c.block;
  c.grid = int(need < max_blocks ? need : max_blocks);
  if (c.grid < 1) c.grid = 1;
  return c;
}

// ---- stencil dispatch ------------------------------------------------------------
// one translation unit per storage precision (dslash_{double,single,half}.cu)
cudaError_t launch_hop_double(const HopLaunch& L, cudaStream_t st);
cudaError_t launch_hop_single(const HopLaunch& L, cudaStream_t st);
cudaError_t launch_hop_half(const HopLaunch& L, cudaStream_t st);

cudaError_t launch_hop(const HopLaunch& L, cudaStream_t st) {
  switch (L.prec) {
    case PREC_DOUBLE: return launch_hop_double(L, st);
    case PREC_SINGLE: return launch_hop_single(L, st);
    case PREC_HALF: return launch_hop_half(L, st);
  }
  return cudaErrorInvalidValue;
}

// ---- linear algebra ------------------------------------------------------------
// Streaming kernels without per-thread scalars launch one thread per element,
// so that each thread issues all its loads at once and the whole grid keeps
// HBM busy; those that first read per-right-hand-side scalars from memory use
// a grid-stride loop over kScalarStreamGrid blocks instead.
constexpr int kScalarStreamGrid = 148 * 16;
static int stream_grid(int64_t n, int blk) {
  const int64_t g = (n + blk - 1) / blk;
  return int(g < 1 ? 1 : g);
}

template <typename RA, typename RB>
__device__ __forceinline__ void cvt12(const Cx<RA> a[12], Cx<RB> b[12]) {
#pragma unroll
  for (int k = 0; k < 12; ++k) b[k] = {RB(a[k].re), RB(a[k].im)};
}

template <int SP>
__global__ void axpby_kernel(int64_t n, double a, SpinorPtr x, double b, SpinorPtr y, SpinorPtr v) {
  using R = typename SpinorIO<SP>::Real;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    Cx<R> xv[12], yv[12];
    SpinorIO<SP>::load(x, i, xv);
    if (b != 0.0) SpinorIO<SP>::load(y, i, yv);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      xv[k] = R(a) * xv[k];
      if (b != 0.0) xv[k] = xv[k] + R(b) * yv[k];
    }
    SpinorIO<SP>::store(v, i, xv);
  }
}

// RationalSolver_CG reconstruction (lib/Solver/rationalSolver_CG.cpp:29-36)
__global__ void combine_kernel(int64_t n, double c0, SpinorPtr b, int m, SField x, SpinorPtr y) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    Cx<double> acc[12], v[12];
    SpinorIO<PREC_DOUBLE>::load(b, i, acc);
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = c0 * acc[k];
    for (int q = 0; q < m; ++q) {
      SpinorIO<PREC_DOUBLE>::load(x.f[q], i, v);
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[k] = acc[k] + x.a[q] * v[k];
    }
    SpinorIO<PREC_DOUBLE>::store(y, i, acc);
  }
}

cudaError_t launch_combine(int64_t sites, double c0, SpinorPtr b, int n, const SField& x,
                           SpinorPtr y, cudaStream_t st) {
  const int blk = 256;
  int grid = int((sites + blk - 1) / blk);
  if (grid > 148 * 16) grid = 148 * 16;
  combine_kernel<<<grid, blk, 0, st>>>(sites, c0, b, n, x, y);
  return cudaGetLastError();
}

// out = C in, C the FP64 clover block (or its inverse) of one parity
__global__ void clover_mult_kernel(int64_t vh, int nrhs, CloverPtr cl, SpinorPtr in, SpinorPtr out) {
  const int64_t n = vh * nrhs;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    Cx<double> v[12];
    SpinorIO<PREC_DOUBLE>::load(in, i, v);
    CloverBlock<double> B[2];
    CloverIO<PREC_DOUBLE>::load(cl, i / nrhs, B);
    clover_apply(B, v);
    SpinorIO<PREC_DOUBLE>::store(out, i, v);
  }
}

cudaError_t launch_clover_mult(int64_t Vh, int nrhs, CloverPtr cl, SpinorPtr in, SpinorPtr out,
                               cudaStream_t st) {
  const int64_t n = Vh * nrhs;
  const int blk = 128;
  int grid = int((n + blk - 1) / blk);
  if (grid > 148 * 16) grid = 148 * 16;
  clover_mult_kernel<<<grid, blk, 0, st>>>(Vh, nrhs, cl, in, out);
  return cudaGetLastError();
}

cudaError_t launch_axpby(int prec, int64_t Vh, int nrhs, double a, SpinorPtr x, double b,
                         SpinorPtr y, SpinorPtr v, cudaStream_t st) {
  const int64_t n = Vh * nrhs;
  const int blk = 256;
  const int grid = stream_grid(n, blk);
  switch (prec) {
    case PREC_DOUBLE: axpby_kernel<PREC_DOUBLE><<<grid, blk, 0, st>>>(n, a, x, b, y, v); break;
    case PREC_SINGLE: axpby_kernel<PREC_SINGLE><<<grid, blk, 0, st>>>(n, a, x, b, y, v); break;
    default: axpby_kernel<PREC_HALF><<<grid, blk, 0, st>>>(n, a, x, b, y, v); break;
  }
  return cudaGetLastError();
}

template <int PI, int PO>
__global__ void convert_kernel(int64_t n, SpinorPtr in, SpinorPtr out) {
  using RI = typename SpinorIO<PI>::Real;
  using RO = typename SpinorIO<PO>::Real;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    Cx<RI> a[12];
    Cx<RO> b[12];
    SpinorIO<PI>::load(in, i, a);
    cvt12(a, b);
    SpinorIO<PO>::store(out, i, b);
  }
}

cudaError_t launch_convert(int pin, SpinorPtr in, int pout, SpinorPtr out, int64_t Vh, int nrhs,
                           cudaStream_t st) {
  const int64_t n = Vh * nrhs;
  const int blk = 256;
  const int grid = stream_grid(n, blk);
#define IRO_CVT(A, B) \
  if (pin == A && pout == B) { convert_kernel<A, B><<<grid, blk, 0, st>>>(n, in, out); return cudaGetLastError(); }
  IRO_CVT(PREC_DOUBLE, PREC_DOUBLE)
  IRO_CVT(PREC_DOUBLE, PREC_SINGLE)
  IRO_CVT(PREC_DOUBLE, PREC_HALF)
  IRO_CVT(PREC_SINGLE, PREC_DOUBLE)
  IRO_CVT(PREC_SINGLE, PREC_SINGLE)
  IRO_CVT(PREC_SINGLE, PREC_HALF)
  IRO_CVT(PREC_HALF, PREC_DOUBLE)
  IRO_CVT(PREC_HALF, PREC_SINGLE)
  IRO_CVT(PREC_HALF, PREC_HALF)
#undef IRO_CVT
  return cudaErrorInvalidValue;
}

template <int SP, bool TWO>
__global__ void __launch_bounds__(256) norms_kernel(int64_t vh, int nrhs, SpinorPtr v, SpinorPtr w, Reduce red) {
  using R = typename SpinorIO<SP>::Real;
  const int64_t n = vh * nrhs;
  double acc[2] = {0.0, 0.0};
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    Cx<R> a[12];
    SpinorIO<SP>::load(v, i, a);
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[0] += double(a[k].re) * a[k].re + double(a[k].im) * a[k].im;
    if (TWO) {
      SpinorIO<SP>::load(w, i, a);
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[1] += double(a[k].re) * a[k].re + double(a[k].im) * a[k].im;
    }
  }
  block_reduce_finish<2>(red, acc, nrhs, blockIdx.x, gridDim.x);
}

cudaError_t launch_norms(int prec, int64_t Vh, int nrhs, SpinorPtr v, const SpinorPtr* w,
                         const Reduce& red, int max_blocks, cudaStream_t st) {
  LaunchCfg c = launch_cfg(Vh, nrhs, max_blocks);
  SpinorPtr ww = w ? *w : v;
#define IRO_NORMS(P)                                                                          \
  if (prec == P) {                                                                            \
    if (w) norms_kernel<P, true><<<c.grid, c.block, 0, st>>>(Vh, nrhs, v, ww, red);            \
    else norms_kernel<P, false><<<c.grid, c.block, 0, st>>>(Vh, nrhs, v, ww, red);             \
    return cudaGetLastError();                                                                \
  }
  IRO_NORMS(PREC_DOUBLE)
  IRO_NORMS(PREC_SINGLE)
  IRO_NORMS(PREC_HALF)
#undef IRO_NORMS
  return cudaErrorInvalidValue;
}

// Solver_CG::solve start (solver_CG.cpp:40-47): r = b - A x, p = r, rr = (r,r)
template <int SP>
__global__ void __launch_bounds__(256) cg_init_kernel(int64_t vh, int nrhs, SpinorPtr b, SpinorPtr s, SpinorPtr r,
                               SpinorPtr p, Reduce red) {
  using R = typename SpinorIO<SP>::Real;
  const int64_t n = vh * nrhs;
  double acc[2] = {0.0, 0.0};
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    Cx<R> bv[12], sv[12];
    SpinorIO<SP>::load(b, i, bv);
    SpinorIO<SP>::load(s, i, sv);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      acc[1] += double(bv[k].re) * bv[k].re + double(bv[k].im) * bv[k].im;
      sv[k] = bv[k] - sv[k];
      acc[0] += double(sv[k].re) * sv[k].re + double(sv[k].im) * sv[k].im;
    }
    SpinorIO<SP>::store(r, i, sv);
    SpinorIO<SP>::store(p, i, sv);
  }
  block_reduce_finish<2>(red, acc, nrhs, blockIdx.x, gridDim.x);
}

cudaError_t launch_cg_init(int prec, int64_t Vh, int nrhs, SpinorPtr b, SpinorPtr s, SpinorPtr r,
                           SpinorPtr p, const Reduce& red, int max_blocks, cudaStream_t st) {
  LaunchCfg c = launch_cfg(Vh, nrhs, max_blocks);
  switch (prec) {
    case PREC_DOUBLE: cg_init_kernel<PREC_DOUBLE><<<c.grid, c.block, 0, st>>>(Vh, nrhs, b, s, r, p, red); break;
    case PREC_SINGLE: cg_init_kernel<PREC_SINGLE><<<c.grid, c.block, 0, st>>>(Vh, nrhs, b, s, r, p, red); break;
    default: cg_init_kernel<PREC_HALF><<<c.grid, c.block, 0, st>>>(Vh, nrhs, b, s, r, p, red); break;
  }
  return cudaGetLastError();
}

// x += alpha p (solver_CG.cpp:131-136, deferred from the fused r update)
// and p = p*(rr/rrp) + r (solver_CG.cpp:150-153).  The x update runs for
// every right-hand side whose iteration just completed (CGState::xpend), also
// when it has just converged or paused; the p update only for those still
// iterating.  The block is a multiple of nrhs, so a thread keeps one
// right-hand side across the grid-stride loop, and loads its right-hand
// side's scalars once (a grid of a few blocks per SM: with one element per
// thread, the scalar loads ahead of the data would halve the bytes in
// flight).  Each element in two phases -- p and x, then r -- so that at most
// two spinors are live: 4 resident blocks per SM for FP32/FP16 storage, 2 for
// FP64.
template <int SP>
struct CgpBounds {
  static constexpr int blocks = SP == PREC_DOUBLE ? 2 : 4;
};

template <int SP>
__global__ void __launch_bounds__(256, CgpBounds<SP>::blocks) cg_p_kernel(int64_t n, int nrhs, SpinorPtr p, SpinorPtr r,
                                                   SpinorPtr x, const CGState* state,
                                                   const int* done) {
  using R = typename SpinorIO<SP>::Real;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int rhs = i0 % nrhs;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  const bool upd_x = state[rhs].xpend != 0;
  const bool upd_p = done[rhs] == RUNNING;
  if (!upd_x && !upd_p) return;
  const R a = R(state[rhs].alpha);
  const R b = R(state[rhs].beta);
  for (int64_t i = i0; i < n; i += stride) {
    Cx<R> pv[12];
    SpinorIO<SP>::load(p, i, pv);
    if (upd_x) {
      Cx<R> xv[12];
      SpinorIO<SP>::load(x, i, xv);
#pragma unroll
      for (int k = 0; k < 12; ++k) xv[k] = xv[k] + a * pv[k];
      SpinorIO<SP>::store(x, i, xv);
    }
    if (upd_p) {
      Cx<R> rv[12];
      SpinorIO<SP>::load(r, i, rv);
#pragma unroll
      for (int k = 0; k < 12; ++k) pv[k] = b * pv[k] + rv[k];
      SpinorIO<SP>::store(p, i, pv);
    }
  }
}

cudaError_t launch_cg_p(int prec, int64_t Vh, int nrhs, SpinorPtr p, SpinorPtr r, SpinorPtr x,
                        const CGState* state, const int* done, cudaStream_t st) {
  LaunchCfg c = launch_cfg(Vh, nrhs, kScalarStreamGrid);
  const int64_t n = Vh * nrhs;
  switch (prec) {
    case PREC_DOUBLE: cg_p_kernel<PREC_DOUBLE><<<c.grid, c.block, 0, st>>>(n, nrhs, p, r, x, state, done); break;
    case PREC_SINGLE: cg_p_kernel<PREC_SINGLE><<<c.grid, c.block, 0, st>>>(n, nrhs, p, r, x, state, done); break;
    default: cg_p_kernel<PREC_HALF><<<c.grid, c.block, 0, st>>>(n, nrhs, p, r, x, state, done); break;
  }
  return cudaGetLastError();
}

// ---- multishift ---------------------------------------------------------------------
// The vectors in SP: FP64 for the reference's solver, FP32 in the first phase
// of the mixed-precision solve; the scalars (MSState) are FP64 in both.
// Per-site sums are formed in the arithmetic precision and accumulated in
// FP64 (FP64 vectors: term by term, as before the FP32 phase existed).
template <int SP>
__device__ __forceinline__ void acc_norm(double& acc, const Cx<typename SpinorIO<SP>::Real> v[12]) {
  using R = typename SpinorIO<SP>::Real;
  if constexpr (SP == PREC_DOUBLE) {
#pragma unroll
    for (int k = 0; k < 12; ++k) acc += v[k].re * v[k].re + v[k].im * v[k].im;
  } else {
    R a = R(0);
#pragma unroll
    for (int k = 0; k < 12; ++k) a += v[k].re * v[k].re + v[k].im * v[k].im;
    acc += double(a);
  }
}

// multiShiftSolver_CG.cpp:49-59: x0 -= beta p0; r += beta s, s = A p0 + sigma0 p0
template <int SP>
__global__ void __launch_bounds__(256) ms_xr_kernel(int64_t vh, SpinorPtr x0, SpinorPtr r, SpinorPtr p0, SpinorPtr s,
                             const MSState* m, Reduce red) {
  using R = typename SpinorIO<SP>::Real;
  double acc = 0.0;
  if (!red.done[0]) {
    const R beta = R(m->beta), s0 = R(m->sigma0);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < vh;
         i += int64_t(gridDim.x) * blockDim.x) {
      Cx<R> xv[12], rv[12], pv[12], sv[12];
      SpinorIO<SP>::load(x0, i, xv);
      SpinorIO<SP>::load(r, i, rv);
      SpinorIO<SP>::load(p0, i, pv);
      SpinorIO<SP>::load(s, i, sv);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        sv[k] = sv[k] + s0 * pv[k];
        xv[k] = xv[k] - beta * pv[k];
        rv[k] = rv[k] + beta * sv[k];
      }
      acc_norm<SP>(acc, rv);
      SpinorIO<SP>::store(x0, i, xv);
      SpinorIO<SP>::store(r, i, rv);
    }
  }
  block_reduce_finish<1>(red, &acc, 1, blockIdx.x, gridDim.x);
}

cudaError_t launch_ms_xr(int prec, int64_t Vh, SpinorPtr x0, SpinorPtr r, SpinorPtr p0, SpinorPtr s,
                         const MSState* m, const Reduce& red, int max_blocks, cudaStream_t st) {
  LaunchCfg c = launch_cfg(Vh, 1, max_blocks);
  if (prec == PREC_DOUBLE)
    ms_xr_kernel<PREC_DOUBLE><<<c.grid, c.block, 0, st>>>(Vh, x0, r, p0, s, m, red);
  else if (prec == PREC_SINGLE)
    ms_xr_kernel<PREC_SINGLE><<<c.grid, c.block, 0, st>>>(Vh, x0, r, p0, s, m, red);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// multiShiftSolver_CG.cpp:61-83: all shifts' x and p updated in one pass
template <int SP>
__global__ void __launch_bounds__(256) ms_p_kernel(int64_t vh, MSFields f, SpinorPtr r, const MSState* m, Reduce red) {
  using R = typename SpinorIO<SP>::Real;
  double acc[MAXSHIFT];
#pragma unroll
  for (int k = 0; k < MAXSHIFT; ++k) acc[k] = 0.0;
  if (!red.done[0]) {
    const int ns2 = m->nshift2;
    const R alpha = R(m->alpha);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < vh;
         i += int64_t(gridDim.x) * blockDim.x) {
      Cx<R> rv[12], pv[12], xv[12];
      SpinorIO<SP>::load(r, i, rv);
      SpinorIO<SP>::load(f.p[0], i, pv);
#pragma unroll
      for (int k = 0; k < 12; ++k) pv[k] = alpha * pv[k] + rv[k];
      SpinorIO<SP>::store(f.p[0], i, pv);
#pragma unroll
      for (int sh = 1; sh < MAXSHIFT; ++sh) {
        if (sh >= ns2) break;
        const R bs = R(m->betas[sh]), as = R(m->alphas[sh]), z = R(m->zeta[sh]);
        SpinorIO<SP>::load(f.p[sh], i, pv);
        SpinorIO<SP>::load(f.x[sh], i, xv);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
          xv[k] = xv[k] - bs * pv[k];
          pv[k] = as * pv[k] + z * rv[k];
        }
        double a2 = 0.0;
        acc_norm<SP>(a2, pv);
        acc[sh] += a2;
        SpinorIO<SP>::store(f.x[sh], i, xv);
        SpinorIO<SP>::store(f.p[sh], i, pv);
      }
    }
  }
  block_reduce_finish<MAXSHIFT>(red, acc, 1, blockIdx.x, gridDim.x);
}

cudaError_t launch_ms_p(int prec, int64_t Vh, int nshift, const MSFields& f, SpinorPtr r,
                        const MSState* m, const Reduce& red, int max_blocks, cudaStream_t st) {
  LaunchCfg c = launch_cfg(Vh, 1, max_blocks);
  if (prec == PREC_DOUBLE)
    ms_p_kernel<PREC_DOUBLE><<<c.grid, c.block, 0, st>>>(Vh, f, r, m, red);
  else if (prec == PREC_SINGLE)
    ms_p_kernel<PREC_SINGLE><<<c.grid, c.block, 0, st>>>(Vh, f, r, m, red);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// ---- FP64 multishift with a residual window ------------------------------------
// The x and p of the shifts are not updated every iteration: the iteration
// keeps its residuals r_k in a ring of slots, and every shift's x and p after
// a window of iterations are linear combinations of its x and p before it and
// of the window's residuals, with coefficients from the step scalars (formed
// on the host, ms_run).  An iteration then moves shift 0's vectors only.

// multiShiftSolver_CG.cpp:49-57 without the x update: s += sigma0 p0,
// r += beta s, into the next slot
__global__ void __launch_bounds__(256) msw_r_kernel(int64_t vh, SlotList sl, int nslots, SpinorPtr p0,
                                                    SpinorPtr s, const MSState* m, Reduce red) {
  double acc = 0.0;
  if (!red.done[0]) {
    const double beta = m->beta, s0 = m->sigma0;
    const int it = m->iter;
    const SpinorPtr rc = sl.s[it % nslots], rn = sl.s[(it + 1) % nslots];
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < vh;
         i += int64_t(gridDim.x) * blockDim.x) {
      Cx<double> rv[12], pv[12], sv[12];
      SpinorIO<PREC_DOUBLE>::load(rc, i, rv);
      SpinorIO<PREC_DOUBLE>::load(p0, i, pv);
      SpinorIO<PREC_DOUBLE>::load(s, i, sv);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        sv[k] = sv[k] + s0 * pv[k];
        rv[k] = rv[k] + beta * sv[k];
      }
      acc_norm<PREC_DOUBLE>(acc, rv);
      SpinorIO<PREC_DOUBLE>::store(rn, i, rv);
    }
  }
  block_reduce_finish<1>(red, &acc, 1, blockIdx.x, gridDim.x);
}

cudaError_t launch_msw_r(int64_t Vh, const SlotList& sl, int nslots, SpinorPtr p0, SpinorPtr s,
                         const MSState* m, const Reduce& red, int max_blocks, cudaStream_t st) {
  LaunchCfg c = launch_cfg(Vh, 1, max_blocks);
  msw_r_kernel<<<c.grid, c.block, 0, st>>>(Vh, sl, nslots, p0, s, m, red);
  return cudaGetLastError();
}

// multiShiftSolver_CG.cpp:59-63: p0 = alpha p0 + r; the reduction only
// carries the stage (pruning, convergence, window full) to the last block
__global__ void __launch_bounds__(256) msw_p_kernel(int64_t vh, SlotList sl, int nslots, SpinorPtr p0,
                                                    const MSState* m, Reduce red) {
  double acc = 0.0;
  if (!red.done[0]) {
    const double alpha = m->alpha;
    const SpinorPtr rn = sl.s[(m->iter + 1) % nslots];
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < vh;
         i += int64_t(gridDim.x) * blockDim.x) {
      Cx<double> rv[12], pv[12];
      SpinorIO<PREC_DOUBLE>::load(rn, i, rv);
      SpinorIO<PREC_DOUBLE>::load(p0, i, pv);
#pragma unroll
      for (int k = 0; k < 12; ++k) pv[k] = alpha * pv[k] + rv[k];
      SpinorIO<PREC_DOUBLE>::store(p0, i, pv);
    }
  }
  block_reduce_finish<1>(red, &acc, 1, blockIdx.x, gridDim.x);
}

cudaError_t launch_msw_p(int64_t Vh, const SlotList& sl, int nslots, SpinorPtr p0, const MSState* m,
                         const Reduce& red, int max_blocks, cudaStream_t st) {
  LaunchCfg c = launch_cfg(Vh, 1, max_blocks);
  msw_p_kernel<<<c.grid, c.block, 0, st>>>(Vh, sl, nslots, p0, m, red);
  return cudaGetLastError();
}

// One thread per (element, chunk, group of four shifts): lanes are 32
// consecutive elements (a warp block's chunk q is 512 contiguous bytes),
// threadIdx.y the chunk q of 12, and consecutive blocks the shift groups of
// one tile of 32 elements, so that a tile's residual chunks come from DRAM
// once and from L2 for the other groups.  A thread keeps its shifts' x and p
// chunks in registers (few registers: several blocks per SM to cover the
// load latency); the coefficients are staged in shared memory.
constexpr int kFoldGroup = 4;
__global__ void __launch_bounds__(32 * 12) msw_fold_kernel(int64_t vh, SlotList sl, int nslots, int s1, int n,
                                                           MSFields f, int nx, int plo, int ngroups,
                                                           const double* __restrict__ coef) {
  __shared__ double cs[kFoldGroup * kMswCoef];
  const int64_t tile = blockIdx.x / ngroups;
  const int k0 = (blockIdx.x % ngroups) * kFoldGroup;
  const int nk = min(kFoldGroup, nx - k0);
  for (int t = threadIdx.y * 32 + threadIdx.x; t < nk * kMswCoef; t += 32 * 12)
    cs[t] = coef[k0 * kMswCoef + t];
  __syncthreads();
  const int64_t i = tile * 32 + threadIdx.x;
  if (i >= vh) return;
  const int q = threadIdx.y;
  double2 xa[kFoldGroup], pa[kFoldGroup];
#pragma unroll
  for (int k = 0; k < kFoldGroup; ++k) xa[k] = pa[k] = make_double2(0.0, 0.0);
#pragma unroll 8
  for (int j = 0; j < n; ++j) {
    const double2 rv =
        __ldg(chunk0<12>(static_cast<const double2*>(sl.s[(s1 + j) % nslots].data), i) + 32 * q);
#pragma unroll
    for (int k = 0; k < kFoldGroup; ++k) {
      if (k < nk) {
        const double C = cs[k * kMswCoef + 2 + j], D = cs[k * kMswCoef + 2 + MSW_MAX + j];
        xa[k] = make_double2(fma(C, rv.x, xa[k].x), fma(C, rv.y, xa[k].y));
        pa[k] = make_double2(fma(D, rv.x, pa[k].x), fma(D, rv.y, pa[k].y));
      }
    }
  }
  double2 pv[kFoldGroup], xv[kFoldGroup];
#pragma unroll
  for (int k = 0; k < kFoldGroup; ++k) {
    if (k < nk) {
      pv[k] = *(chunk0<12>(static_cast<const double2*>(f.p[k0 + k].data), i) + 32 * q);
      xv[k] = *(chunk0<12>(static_cast<const double2*>(f.x[k0 + k].data), i) + 32 * q);
    }
  }
#pragma unroll
  for (int k = 0; k < kFoldGroup; ++k) {
    if (k < nk) {
      const double X = cs[k * kMswCoef], P = cs[k * kMswCoef + 1];
      *(chunk0<12>(static_cast<double2*>(f.x[k0 + k].data), i) + 32 * q) =
          make_double2(xv[k].x + fma(X, pv[k].x, xa[k].x), xv[k].y + fma(X, pv[k].y, xa[k].y));
      if (k0 + k >= plo)
        *(chunk0<12>(static_cast<double2*>(f.p[k0 + k].data), i) + 32 * q) =
            make_double2(fma(P, pv[k].x, pa[k].x), fma(P, pv[k].y, pa[k].y));
    }
  }
}

cudaError_t launch_msw_fold(int64_t Vh, const SlotList& sl, int nslots, int s1, int n,
                            const MSFields& f, int nx, int plo, const double* coef, cudaStream_t st) {
  if (nx < 1 || nx > MAXSHIFT || n < 1 || n > MSW_MAX) return cudaErrorInvalidValue;
  const int ngroups = (nx + kFoldGroup - 1) / kFoldGroup;
  const int64_t grid = (Vh + 31) / 32 * ngroups;
  if (grid > 0x7fffffff) return cudaErrorInvalidValue;
  msw_fold_kernel<<<unsigned(grid), dim3(32, 12), 0, st>>>(Vh, sl, nslots, s1, n, f, nx, plo, ngroups,
                                                           coef);
  return cudaGetLastError();
}

// reliable update of the mixed-precision multishift: x64_k += xlo_k, xlo_k = 0
// for the shifts k < n (FP32 accumulators into the FP64 solutions)
__global__ void ms_merge_kernel(int64_t vh, int n, MSFields x64, MSFields xlo) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < vh;
       i += int64_t(gridDim.x) * blockDim.x) {
    for (int k = 0; k < n; ++k) {
      Cx<double> a[12];
      Cx<float> b[12], z[12];
      SpinorIO<PREC_DOUBLE>::load(x64.x[k], i, a);
      SpinorIO<PREC_SINGLE>::load(xlo.x[k], i, b);
#pragma unroll
      for (int j = 0; j < 12; ++j) {
        a[j] = a[j] + Cx<double>{double(b[j].re), double(b[j].im)};
        z[j] = {0.f, 0.f};
      }
      SpinorIO<PREC_DOUBLE>::store(x64.x[k], i, a);
      SpinorIO<PREC_SINGLE>::store(xlo.x[k], i, z);
    }
  }
}

cudaError_t launch_ms_merge(int64_t Vh, int n, const MSFields& x64, const MSFields& xlo,
                            cudaStream_t st) {
  const int blk = 256;
  ms_merge_kernel<<<stream_grid(Vh, blk), blk, 0, st>>>(Vh, n, x64, xlo);
  return cudaGetLastError();
}

// ---- shifted CG (the refinement of the mixed-precision multishift solve) ----------
// r -= alpha (s + sigma p) per right-hand side (s = A p from the operator, the
// shift sigma from the right-hand side's CGState); reduce |r|^2 (stage
// ST_CG_BETA).  Right-hand sides that have left the iteration are skipped.
template <int SP>
__global__ void __launch_bounds__(256) cg_shift_r_kernel(int64_t n, int nrhs, SpinorPtr r, SpinorPtr s,
                                                       SpinorPtr p, const CGState* state, Reduce red) {
  using R = typename SpinorIO<SP>::Real;
  double acc = 0.0;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int rhs = i0 % nrhs;  // the block is a multiple of nrhs: one rhs per thread
  if (!red.done[rhs]) {
    const R a = R(state[rhs].alpha), sg = R(state[rhs].sigma);
    for (int64_t i = i0; i < n; i += int64_t(gridDim.x) * blockDim.x) {
      Cx<R> rv[12], sv[12], pv[12];
      SpinorIO<SP>::load(r, i, rv);
      SpinorIO<SP>::load(s, i, sv);
      SpinorIO<SP>::load(p, i, pv);
#pragma unroll
      for (int k = 0; k < 12; ++k) rv[k] = rv[k] - a * (sv[k] + sg * pv[k]);
      acc_norm<SP>(acc, rv);
      SpinorIO<SP>::store(r, i, rv);
    }
  }
  block_reduce_finish<1>(red, &acc, nrhs, blockIdx.x, gridDim.x);
}

cudaError_t launch_cg_shift_r(int prec, int64_t Vh, int nrhs, SpinorPtr r, SpinorPtr s, SpinorPtr p,
                              const CGState* state, const Reduce& red, int max_blocks,
                              cudaStream_t st) {
  LaunchCfg c = launch_cfg(Vh, nrhs, max_blocks);
  const int64_t n = Vh * nrhs;
  switch (prec) {
    case PREC_DOUBLE: cg_shift_r_kernel<PREC_DOUBLE><<<c.grid, c.block, 0, st>>>(n, nrhs, r, s, p, state, red); break;
    case PREC_SINGLE: cg_shift_r_kernel<PREC_SINGLE><<<c.grid, c.block, 0, st>>>(n, nrhs, r, s, p, state, red); break;
    default: cg_shift_r_kernel<PREC_HALF><<<c.grid, c.block, 0, st>>>(n, nrhs, r, s, p, state, red); break;
  }
  return cudaGetLastError();
}

// s += sigma_rhs x over FP64 elements (the shift of the shifted operator in
// the FP64 residual recomputations)
__global__ void shift_add_kernel(int64_t n, int nrhs, SpinorPtr s, SpinorPtr x, const CGState* state) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const double sg = state[i % nrhs].sigma;
    if (sg == 0.0) continue;
    Cx<double> sv[12], xv[12];
    SpinorIO<PREC_DOUBLE>::load(s, i, sv);
    SpinorIO<PREC_DOUBLE>::load(x, i, xv);
#pragma unroll
    for (int k = 0; k < 12; ++k) sv[k] = sv[k] + sg * xv[k];
    SpinorIO<PREC_DOUBLE>::store(s, i, sv);
  }
}

cudaError_t launch_shift_add(int64_t sites, int nrhs, SpinorPtr s, SpinorPtr x, const CGState* state,
                             cudaStream_t st) {
  const int64_t n = sites * nrhs;
  const int blk = 256;
  shift_add_kernel<<<stream_grid(n, blk), blk, 0, st>>>(n, nrhs, s, x, state);
  return cudaGetLastError();
}

// FP64 block field (right-hand side k = shift k) from the shifts' single fields
// in precision SPI: out[hs * ns + k] = x_k[hs]
template <int SPI>
__global__ void ms_pack_kernel(int64_t sites, int ns, MSFields f, SpinorPtr out) {
  using RI = typename SpinorIO<SPI>::Real;
  const int64_t n = sites * ns;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int k = int(i % ns);
    Cx<RI> a[12];
    Cx<double> b[12];
    SpinorIO<SPI>::load(f.x[k], i / ns, a);
    cvt12(a, b);
    SpinorIO<PREC_DOUBLE>::store(out, i, b);
  }
}

cudaError_t launch_ms_pack(int prec, int64_t sites, int ns, const MSFields& f, SpinorPtr out,
                           cudaStream_t st) {
  const int64_t n = sites * ns;
  const int blk = 256;
  if (prec == PREC_SINGLE)
    ms_pack_kernel<PREC_SINGLE><<<stream_grid(n, blk), blk, 0, st>>>(sites, ns, f, out);
  else if (prec == PREC_DOUBLE)
    ms_pack_kernel<PREC_DOUBLE><<<stream_grid(n, blk), blk, 0, st>>>(sites, ns, f, out);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// r_k = b - s_k - sigma_k x_k over an FP64 block of ns right-hand sides (one
// per shift), b a single FP64 field: the residuals of the shifted systems
__global__ void ms_block_residual_kernel(int64_t sites, int ns, SpinorPtr b, SpinorPtr s, SpinorPtr x,
                                         ShiftList sg, SpinorPtr r) {
  const int64_t n = sites * ns;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const double sk = sg.s[i % ns];
    Cx<double> bv[12], sv[12], xv[12];
    SpinorIO<PREC_DOUBLE>::load(b, i / ns, bv);
    SpinorIO<PREC_DOUBLE>::load(s, i, sv);
    SpinorIO<PREC_DOUBLE>::load(x, i, xv);
#pragma unroll
    for (int k = 0; k < 12; ++k) bv[k] = bv[k] - sv[k] - sk * xv[k];
    SpinorIO<PREC_DOUBLE>::store(r, i, bv);
  }
}

cudaError_t launch_ms_block_residual(int64_t sites, int ns, SpinorPtr b, SpinorPtr s, SpinorPtr x,
                                     const ShiftList& sg, SpinorPtr r, cudaStream_t st) {
  const int64_t n = sites * ns;
  const int blk = 256;
  ms_block_residual_kernel<<<stream_grid(n, blk), blk, 0, st>>>(sites, ns, b, s, x, sg, r);
  return cudaGetLastError();
}

// ---- boundary conversion ------------------------------------------------------------
__device__ __forceinline__ int64_t host_site(const Geom& g, int layout, int p, int hs) {
  if (layout == 1) return hs;
  const Coord c = coord_of(g, hs, p);
  return int64_t(c.x) + int64_t(g.L[0]) * c.row;
}

template <int SP>
__global__ void import_kernel(Geom g, const double* stage, int layout, int p, int64_t host_sites,
                              int nrhs, SpinorPtr out, int64_t i0, int64_t n) {
  using R = typename SpinorIO<SP>::Real;
  for (int64_t i = i0 + int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < i0 + n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int hs = int(i / nrhs);
    const int r = int(i - int64_t(hs) * nrhs);
    const double* src = stage + (int64_t(r) * host_sites + host_site(g, layout, p, hs)) * 24;
    Cx<R> v[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) v[k] = {R(src[2 * k]), R(src[2 * k + 1])};
    SpinorIO<SP>::store(out, i, v);
  }
}

template <int SP>
__global__ void export_kernel(Geom g, double* stage, int layout, int p, int64_t host_sites,
                              int nrhs, SpinorPtr in, int64_t i0, int64_t n) {
  using R = typename SpinorIO<SP>::Real;
  for (int64_t i = i0 + int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < i0 + n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int hs = int(i / nrhs);
    const int r = int(i - int64_t(hs) * nrhs);
    double* dst = stage + (int64_t(r) * host_sites + host_site(g, layout, p, hs)) * 24;
    Cx<R> v[12];
    SpinorIO<SP>::load(in, i, v);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      dst[2 * k] = double(v[k].re);
      dst[2 * k + 1] = double(v[k].im);
    }
  }
}

static int grid_for(int64_t n, int blk) {
  int64_t g = (n + blk - 1) / blk;
  return int(g > 148 * 32 ? 148 * 32 : (g < 1 ? 1 : g));
}

__global__ void point_source_kernel(SpinorPtr s, int64_t hs, int nrhs, int first) {
  const int j = threadIdx.x;
  if (j < nrhs) chunk0<12>(static_cast<double2*>(s.data), hs * nrhs + j)[32 * (first + j)] = make_double2(1.0, 0.0);
}

cudaError_t launch_point_sources(const DevField& F, int p, int64_t hs, int first, cudaStream_t st) {
  if (F.prec != PREC_DOUBLE || F.subset != 2 || hs < 0 || hs >= F.Vh || first < 0 || first + F.nrhs > 12)
    return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(F.data, 0, F.bytes_data, st);
  if (e != cudaSuccess) return e;
  point_source_kernel<<<1, 32, 0, st>>>(F.half(p), hs, F.nrhs, first);
  return cudaGetLastError();
}

cudaError_t launch_import_spinor(const Geom& g, const double* stage, int layout, int p,
                                 int64_t host_sites, int nrhs, int prec, SpinorPtr out,
                                 cudaStream_t st, int64_t hs0, int64_t nhs) {
  if (nhs < 0) nhs = g.Vh - hs0;
  const int64_t i0 = hs0 * nrhs, n = nhs * nrhs;
  const int grid = grid_for(n, 256);
  switch (prec) {
    case PREC_DOUBLE: import_kernel<PREC_DOUBLE><<<grid, 256, 0, st>>>(g, stage, layout, p, host_sites, nrhs, out, i0, n); break;
    case PREC_SINGLE: import_kernel<PREC_SINGLE><<<grid, 256, 0, st>>>(g, stage, layout, p, host_sites, nrhs, out, i0, n); break;
    default: import_kernel<PREC_HALF><<<grid, 256, 0, st>>>(g, stage, layout, p, host_sites, nrhs, out, i0, n); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_export_spinor(const Geom& g, double* stage, int layout, int p,
                                 int64_t host_sites, int nrhs, int prec, SpinorPtr in,
                                 cudaStream_t st, int64_t hs0, int64_t nhs) {
  if (nhs < 0) nhs = g.Vh - hs0;
  const int64_t i0 = hs0 * nrhs, n = nhs * nrhs;
  const int grid = grid_for(n, 256);
  switch (prec) {
    case PREC_DOUBLE: export_kernel<PREC_DOUBLE><<<grid, 256, 0, st>>>(g, stage, layout, p, host_sites, nrhs, in, i0, n); break;
    case PREC_SINGLE: export_kernel<PREC_SINGLE><<<grid, 256, 0, st>>>(g, stage, layout, p, host_sites, nrhs, in, i0, n); break;
    default: export_kernel<PREC_HALF><<<grid, 256, 0, st>>>(g, stage, layout, p, host_sites, nrhs, in, i0, n); break;
  }
  return cudaGetLastError();
}

// GammaMatrix::gamma5core (lib/Dirac_ops/wilsonLikeUtils.cpp:42-49): spins 0<->2, 1<->3
__global__ void gamma5_aos_kernel(double* f, int64_t nsites) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nsites * 6;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t site = i / 6;
    const int k = int(i - site * 6);  // complex k of spins 0,1 (k = c + 3*s)
    double2* p = reinterpret_cast<double2*>(f + site * 24);
    double2 a = p[k], b = p[k + 6];
    p[k] = b;
    p[k + 6] = a;
  }
}

cudaError_t launch_gamma5_aos(double* stage, int64_t nsites, cudaStream_t st) {
  gamma5_aos_kernel<<<grid_for(nsites * 6, 256), 256, 0, st>>>(stage, nsites);
  return cudaGetLastError();
}

// ---- gauge import -------------------------------------------------------------------
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* a, double v) {
  atomicMax(a, static_cast<unsigned long long>(__double_as_longlong(v)));
}

__global__ void import_gauge_kernel(Geom g, const double* raw, GaugeArrays ga,
                                    unsigned long long* maxdev) {
  const int64_t Vh = g.Vh;
  const int64_t V = 2 * Vh;
  const int64_t n = 2 * 4 * Vh;
  double dev = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t hs = i % Vh;
    const int mu = int((i / Vh) % 4);
    const int p = int(i / (4 * Vh));
    const Coord c = coord_of(g, int(hs), p);
    const int64_t site = int64_t(c.x) + int64_t(g.L[0]) * c.row;
    const double* u = raw + 18 * (site + V * mu);
    Su3<double> U;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) U.e[a][b] = {u[2 * (3 * a + b)], u[2 * (3 * a + b) + 1]};
    const int64_t base = int64_t(p * 4 + mu);
#pragma unroll
    for (int k = 0; k < 6; ++k) ga.d12[link0<6>(Vh, p, mu, hs) + 32 * k] = make_double2(U.e[k / 3][k % 3].re, U.e[k / 3][k % 3].im);
#pragma unroll
    for (int k = 0; k < 9; ++k) ga.d18[link0<9>(Vh, p, mu, hs) + 32 * k] = make_double2(U.e[k / 3][k % 3].re, U.e[k / 3][k % 3].im);
    ga.s12[link0<3>(Vh, p, mu, hs)] = make_float4(U.e[0][0].re, U.e[0][0].im, U.e[0][1].re, U.e[0][1].im);
    ga.s12[link0<3>(Vh, p, mu, hs) + 32] = make_float4(U.e[0][2].re, U.e[0][2].im, U.e[1][0].re, U.e[1][0].im);
    ga.s12[link0<3>(Vh, p, mu, hs) + 64] = make_float4(U.e[1][1].re, U.e[1][1].im, U.e[1][2].re, U.e[1][2].im);
    uint4 ha;
    ha.x = pack_h2(float(U.e[0][0].re), float(U.e[0][0].im));
    ha.y = pack_h2(float(U.e[0][1].re), float(U.e[0][1].im));
    ha.z = pack_h2(float(U.e[0][2].re), float(U.e[0][2].im));
    ha.w = pack_h2(float(U.e[1][0].re), float(U.e[1][0].im));
    uint2 hb;
    hb.x = pack_h2(float(U.e[1][1].re), float(U.e[1][1].im));
    hb.y = pack_h2(float(U.e[1][2].re), float(U.e[1][2].im));
    ga.h12a[base * Vh + hs] = ha;
    ga.h12b[base * Vh + hs] = hb;
    uint32_t hw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
      hw[k] = pack_h2(float(U.e[k / 3][k % 3].re), float(U.e[k / 3][k % 3].im));
    ga.h18a[2 * (base * Vh + hs)] = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    ga.h18a[2 * (base * Vh + hs) + 1] = make_uint4(hw[4], hw[5], hw[6], hw[7]);
    ga.h18b[base * Vh + hs] = pack_h2(float(U.e[2][2].re), float(U.e[2][2].im));
    // SU(3) check: rows 0,1 orthonormal and row 2 = conj(row0 x row1)
    Su3<double> W = U;
    reconstruct_row2(W);
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      dev = fmax(dev, fabs(W.e[2][b].re - U.e[2][b].re));
      dev = fmax(dev, fabs(W.e[2][b].im - U.e[2][b].im));
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int a2 = 0; a2 < 2; ++a2) {
        Cx<double> s = {0.0, 0.0};
#pragma unroll
        for (int b = 0; b < 3; ++b) s = s + cj_mul(U.e[a][b], U.e[a2][b]);
        dev = fmax(dev, fabs(s.re - (a == a2 ? 1.0 : 0.0)));
        dev = fmax(dev, fabs(s.im));
      }
  }
  dev = warp_max(dev);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(maxdev, dev);
}

cudaError_t launch_import_gauge(const Geom& g, const double* raw, GaugeArrays ga,
                                unsigned long long* maxdev_bits, cudaStream_t st) {
  import_gauge_kernel<<<grid_for(int64_t(8) * g.Vh, 256), 256, 0, st>>>(g, raw, ga, maxdev_bits);
  return cudaGetLastError();
}

// ---- clover set-up (FP64) -------------------------------------------------------------
// Spin matrices i*sigma_{mu nu} of Dirac_Clover::isigma_{23,31,12,41,42,43}
// (lib/Dirac_ops/dirac_clover.cpp:221-329) reduced to the two chirality
// blocks: s_pm[k][a][b] = S_k[a][b] +- S_k[a][b+2] for a,b in {0,1}.
__constant__ double2 c_spm[2][6][2][2];

struct M3d {
  Cx<double> e[3][3];
};

__device__ __forceinline__ M3d m3_load(const double* raw, int64_t V, int64_t site, int mu) {
  M3d m;
  const double* u = raw + 18 * (site + V * mu);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) m.e[a][b] = {u[2 * (3 * a + b)], u[2 * (3 * a + b) + 1]};
  return m;
}
__device__ __forceinline__ M3d m3_mul(const M3d& x, const M3d& y) {
  M3d r;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) r.e[a][b] = x.e[a][0] * y.e[0][b] + x.e[a][1] * y.e[1][b] + x.e[a][2] * y.e[2][b];
  return r;
}
__device__ __forceinline__ M3d m3_dag(const M3d& x) {
  M3d r;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) r.e[a][b] = conjx(x.e[b][a]);
  return r;
}
__device__ __forceinline__ M3d m3_ah(const M3d& x) {
  M3d r;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) r.e[a][b] = 0.5 * (x.e[a][b] - conjx(x.e[b][a]));
  return r;
}

__device__ __forceinline__ int64_t lex_shift(const Geom& g, int64_t site, int dir, int sgn) {
  int c[4];
  int64_t r = site;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    c[d] = int(r % g.L[d]);
    r /= g.L[d];
  }
  c[dir] = (c[dir] + sgn + g.L[dir]) % g.L[dir];
  return c[0] + int64_t(g.L[0]) * (c[1] + int64_t(g.L[1]) * (c[2] + int64_t(g.L[2]) * c[3]));
}

// v(x) = Vup(x)^dag - Vdn(x)^dag (staples.cpp:596-597, 641-643)
__device__ M3d leaves(const Geom& g, const double* raw, int64_t V, int64_t x, int mu, int nu) {
  const int64_t xn = lex_shift(g, x, nu, 1), xm = lex_shift(g, x, mu, 1);
  M3d up = m3_mul(m3_mul(m3_load(raw, V, x, nu), m3_load(raw, V, xn, mu)), m3_dag(m3_load(raw, V, xm, nu)));
  const int64_t y = lex_shift(g, x, nu, -1), ym = lex_shift(g, y, mu, 1);
  M3d dn = m3_mul(m3_mul(m3_dag(m3_load(raw, V, y, nu)), m3_load(raw, V, y, mu)), m3_load(raw, V, ym, nu));
  M3d a = m3_dag(up), b = m3_dag(dn), v;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) v.e[i][j] = a.e[i][j] - b.e[i][j];
  return v;
}

// Staples::fieldStrength (lib/Measurements/GaugeM/staples.cpp:587-666)
__device__ M3d field_strength_at(const Geom& g, const double* raw, int64_t V, int64_t x, int mu, int nu) {
  const int64_t xm = lex_shift(g, x, mu, -1);
  M3d f1 = m3_ah(m3_mul(m3_load(raw, V, x, mu), leaves(g, raw, V, x, mu, nu)));
  M3d f2 = m3_ah(m3_mul(leaves(g, raw, V, xm, mu, nu), m3_load(raw, V, xm, mu)));
  M3d f;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) f.e[i][j] = f1.e[i][j] + f2.e[i][j];
  // traceless anti-Hermitian part (anti_hermite_traceless, sunMatUtils.cpp:50-55), x 0.25
  const double imtr = (f.e[0][0].im + f.e[1][1].im + f.e[2][2].im) / 3.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) f.e[i][i].im -= imtr;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) f.e[i][j] = 0.25 * f.e[i][j];
  return f;
}

__global__ void field_strength_kernel(Geom g, const double* raw, int mu, int nu, double* out) {
  const int64_t V = 2 * int64_t(g.Vh);
  for (int64_t x = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < V;
       x += int64_t(gridDim.x) * blockDim.x) {
    M3d f = field_strength_at(g, raw, V, x, mu, nu);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        out[18 * x + 2 * (3 * i + j)] = f.e[i][j].re;
        out[18 * x + 2 * (3 * i + j) + 1] = f.e[i][j].im;
      }
  }
}

cudaError_t launch_field_strength(const Geom& g, const double* raw, int mu, int nu, double* out,
                                  cudaStream_t st) {
  field_strength_kernel<<<grid_for(2 * int64_t(g.Vh), 128), 128, 0, st>>>(g, raw, mu, nu, out);
  return cudaGetLastError();
}

// complex 6x6 inverse by Gauss-Jordan elimination with partial pivoting
__device__ bool inv6(Cx<double> a[6][6], Cx<double> inv[6][6]) {
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) inv[i][j] = {i == j ? 1.0 : 0.0, 0.0};
  for (int c = 0; c < 6; ++c) {
    int piv = c;
    double best = a[c][c].re * a[c][c].re + a[c][c].im * a[c][c].im;
    for (int r = c + 1; r < 6; ++r) {
      const double m = a[r][c].re * a[r][c].re + a[r][c].im * a[r][c].im;
      if (m > best) {
        best = m;
        piv = r;
      }
    }
    if (!(best > 0.0)) return false;
    if (piv != c)
      for (int j = 0; j < 6; ++j) {
        Cx<double> t = a[c][j]; a[c][j] = a[piv][j]; a[piv][j] = t;
        t = inv[c][j]; inv[c][j] = inv[piv][j]; inv[piv][j] = t;
      }
    const double den = a[c][c].re * a[c][c].re + a[c][c].im * a[c][c].im;
    const Cx<double> rp = {a[c][c].re / den, -a[c][c].im / den};
    for (int j = 0; j < 6; ++j) {
      a[c][j] = a[c][j] * rp;
      inv[c][j] = inv[c][j] * rp;
    }
    for (int r = 0; r < 6; ++r) {
      if (r == c) continue;
      const Cx<double> f = a[r][c];
      for (int j = 0; j < 6; ++j) {
        a[r][j] = a[r][j] - f * a[c][j];
        inv[r][j] = inv[r][j] - f * inv[c][j];
      }
    }
  }
  return true;
}

__device__ void store_block(const CloverArrays& ca, bool inverse, int p, int64_t Vh, int64_t hs,
                            int blk, Cx<double> m[6][6]) {
  // Hermitian parts: real diagonal and upper triangle (averaged with the lower)
  double v[36];
  for (int i = 0; i < 6; ++i) v[i] = m[i][i].re;
  for (int i = 0; i < 6; ++i)
    for (int j = i + 1; j < 6; ++j) {
      const int k = tri(i, j);
      v[6 + 2 * k] = 0.5 * (m[i][j].re + m[j][i].re);
      v[7 + 2 * k] = 0.5 * (m[i][j].im - m[j][i].im);
    }
  void* const* arr = inverse ? ca.Ainv[0] : ca.A[0];
  double2* d = static_cast<double2*>(arr[p]);
  for (int k = 0; k < 18; ++k) d[blk0<36>(hs) + 32 * (blk * 18 + k)] = make_double2(v[2 * k], v[2 * k + 1]);
  float* fptr = reinterpret_cast<float*>(static_cast<float4*>((inverse ? ca.Ainv[1] : ca.A[1])[p]));
  // FP32: 18 float4 chunks over both blocks, values v_all[36*blk + j]
  for (int q = 0; q < 9; ++q) {
    float4 f4 = make_float4(float(v[4 * q]), float(v[4 * q + 1]), float(v[4 * q + 2]), float(v[4 * q + 3]));
    reinterpret_cast<float4*>(fptr)[blk0<18>(hs) + 32 * (blk * 9 + q)] = f4;
  }
  uint4* h = static_cast<uint4*>((inverse ? ca.Ainv[2] : ca.A[2])[p]);
  // FP16: 9 chunks of 8 halves over both blocks: block 0 owns values 0..35,
  // block 1 36..71; chunk 4 straddles the two blocks (values 32..39).
  // Written per half-word pair so the two blocks can be stored independently.
  unsigned short* hs16 = reinterpret_cast<unsigned short*>(h);
  for (int j = 0; j < 36; ++j) {
    const int gidx = 36 * blk + j;
    const int q = gidx / 8, w = gidx % 8;
    __half hv = __float2half_rn(float(v[j]));
    hs16[(blk0<9>(hs) + 32 * q) * 8 + w] = *reinterpret_cast<unsigned short*>(&hv);
  }
}

__global__ void clover_build_kernel(Geom g, const double* raw, double kc, CloverArrays ca, int* singular) {
  const int64_t Vh = g.Vh;
  const int64_t V = 2 * Vh;
  const int PAIRS[6][2] = {{1, 2}, {2, 0}, {0, 1}, {3, 0}, {3, 1}, {3, 2}};
  for (int64_t x = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < V;
       x += int64_t(gridDim.x) * blockDim.x) {
    int c4[4];
    int64_t rr = x;
    for (int d = 0; d < 4; ++d) {
      c4[d] = int(rr % g.L[d]);
      rr /= g.L[d];
    }
    const int p = (c4[0] + c4[1] + c4[2] + c4[3]) & 1;
    const int64_t hs = x >> 1;
    Cx<double> B[2][6][6];
    for (int s = 0; s < 2; ++s)
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) B[s][i][j] = {i == j ? 1.0 : 0.0, 0.0};
    for (int k = 0; k < 6; ++k) {
      const M3d F = field_strength_at(g, raw, V, x, PAIRS[k][0], PAIRS[k][1]);
      for (int s = 0; s < 2; ++s)
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) {
            const double2 sv = c_spm[s][k][a][b];
            if (sv.x == 0.0 && sv.y == 0.0) continue;
            const Cx<double> sc = {-kc * sv.x, -kc * sv.y};
            for (int i = 0; i < 3; ++i)
              for (int j = 0; j < 3; ++j) B[s][a * 3 + i][b * 3 + j] = B[s][a * 3 + i][b * 3 + j] + sc * F.e[i][j];
          }
    }
    for (int s = 0; s < 2; ++s) {
      Cx<double> inv[6][6], work[6][6];
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) work[i][j] = B[s][i][j];
      if (!inv6(work, inv)) atomicExch(singular, 1);
      store_block(ca, false, p, Vh, hs, s, B[s]);
      store_block(ca, true, p, Vh, hs, s, inv);
    }
  }
}

cudaError_t launch_clover_build(const Geom& g, const double* raw, double kappa_csw,
                                CloverArrays ca, int* singular, cudaStream_t st) {
  clover_build_kernel<<<grid_for(2 * int64_t(g.Vh), 64), 64, 0, st>>>(g, raw, kappa_csw, ca, singular);
  return cudaGetLastError();
}

void clover_init_tables() {
  // S_k[s_out][s_in] as (re, im), from Dirac_Clover::isigma_* (dirac_clover.cpp:221-329)
  double S[6][4][4][2];
  std::memset(S, 0, sizeof(S));
  auto set = [&](int k, int a, int b, double re, double im) {
    S[k][a][b][0] = re;
    S[k][a][b][1] = im;
  };
  // isigma_23: w0 = i v1, w1 = i v0, w2 = i v3, w3 = i v2
  set(0, 0, 1, 0, 1); set(0, 1, 0, 0, 1); set(0, 2, 3, 0, 1); set(0, 3, 2, 0, 1);
  // isigma_31: w0 = v1, w1 = -v0, w2 = v3, w3 = -v2
  set(1, 0, 1, 1, 0); set(1, 1, 0, -1, 0); set(1, 2, 3, 1, 0); set(1, 3, 2, -1, 0);
  // isigma_12: w0 = i v0, w1 = -i v1, w2 = i v2, w3 = -i v3
  set(2, 0, 0, 0, 1); set(2, 1, 1, 0, -1); set(2, 2, 2, 0, 1); set(2, 3, 3, 0, -1);
  // isigma_41: w0 = -i v3, w1 = -i v2, w2 = -i v1, w3 = -i v0
  set(3, 0, 3, 0, -1); set(3, 1, 2, 0, -1); set(3, 2, 1, 0, -1); set(3, 3, 0, 0, -1);
  // isigma_42: w0 = -v3, w1 = v2, w2 = -v1, w3 = v0
  set(4, 0, 3, -1, 0); set(4, 1, 2, 1, 0); set(4, 2, 1, -1, 0); set(4, 3, 0, 1, 0);
  // isigma_43: w0 = -i v2, w1 = i v3, w2 = -i v0, w3 = i v1
  set(5, 0, 2, 0, -1); set(5, 1, 3, 0, 1); set(5, 2, 0, 0, -1); set(5, 3, 1, 0, 1);
  double2 spm[2][6][2][2];
  for (int s = 0; s < 2; ++s)
    for (int k = 0; k < 6; ++k)
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
          const double sg = s == 0 ? 1.0 : -1.0;
          spm[s][k][a][b].x = S[k][a][b][0] + sg * S[k][a][b + 2][0];
          spm[s][k][a][b].y = S[k][a][b][1] + sg * S[k][a][b + 2][1];
        }
  cudaMemcpyToSymbol(c_spm, spm, sizeof(spm));
}

}  // namespace iro

namespace iro {

// ---- mixed-precision reliable updates -------------------------------------------------
// The blocks are multiples of nrhs (launch_cfg), so a thread keeps one
// right-hand side across its grid-stride loop.
// x64 += xlo; xlo = 0   for right-hand sides with mask[r] != 0
template <int PL>
__global__ void mx_merge_kernel(int64_t n, int nrhs, SpinorPtr x64, SpinorPtr xlo, const int* mask) {
  using RL = typename SpinorIO<PL>::Real;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (!mask[i0 % nrhs]) return;
  for (int64_t i = i0; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    Cx<double> a[12];
    Cx<RL> l[12];
    SpinorIO<PREC_DOUBLE>::load(x64, i, a);
    SpinorIO<PL>::load(xlo, i, l);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      a[k] = a[k] + Cx<double>{double(l[k].re), double(l[k].im)};
      l[k] = {RL(0), RL(0)};
    }
    SpinorIO<PREC_DOUBLE>::store(x64, i, a);
    SpinorIO<PL>::store(xlo, i, l);
  }
}

// r64 = b - s64; rlo = r64; reduce |r64|^2   for mask[r] != 0
template <int PL>
__global__ void __launch_bounds__(256) mx_residual_kernel(int64_t n, int nrhs, SpinorPtr b, SpinorPtr s64, SpinorPtr r64,
                                   SpinorPtr rlo, const int* mask, Reduce red) {
  using RL = typename SpinorIO<PL>::Real;
  double acc = 0.0;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const bool on = mask[i0 % nrhs] != 0;
  for (int64_t i = i0; on && i < n; i += int64_t(gridDim.x) * blockDim.x) {
    Cx<double> bv[12], sv[12];
    Cx<RL> l[12];
    SpinorIO<PREC_DOUBLE>::load(b, i, bv);
    SpinorIO<PREC_DOUBLE>::load(s64, i, sv);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      sv[k] = bv[k] - sv[k];
      acc += sv[k].re * sv[k].re + sv[k].im * sv[k].im;
      l[k] = {RL(sv[k].re), RL(sv[k].im)};
    }
    SpinorIO<PREC_DOUBLE>::store(r64, i, sv);
    SpinorIO<PL>::store(rlo, i, l);
  }
  block_reduce_finish<1>(red, &acc, nrhs, blockIdx.x, gridDim.x);
}

// p = beta p + r   for mask[r] != 0
template <int PL>
__global__ void mx_p_kernel(int64_t n, int nrhs, SpinorPtr p, SpinorPtr r, const CGState* state,
                            const int* mask) {
  using RL = typename SpinorIO<PL>::Real;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int rhs = i0 % nrhs;
  if (!mask[rhs]) return;
  const RL beta = RL(state[rhs].beta);
  for (int64_t i = i0; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    Cx<RL> pv[12], rv[12];
    SpinorIO<PL>::load(p, i, pv);
    SpinorIO<PL>::load(r, i, rv);
#pragma unroll
    for (int k = 0; k < 12; ++k) pv[k] = beta * pv[k] + rv[k];
    SpinorIO<PL>::store(p, i, pv);
  }
}

cudaError_t launch_mx_merge(int plo, int64_t sites, int nrhs, SpinorPtr x64, SpinorPtr xlo,
                            const int* mask, cudaStream_t st) {
  const int64_t n = sites * nrhs;
  LaunchCfg c = launch_cfg(sites, nrhs, kScalarStreamGrid);
  if (plo == PREC_SINGLE) mx_merge_kernel<PREC_SINGLE><<<c.grid, c.block, 0, st>>>(n, nrhs, x64, xlo, mask);
  else if (plo == PREC_HALF) mx_merge_kernel<PREC_HALF><<<c.grid, c.block, 0, st>>>(n, nrhs, x64, xlo, mask);
  else mx_merge_kernel<PREC_DOUBLE><<<c.grid, c.block, 0, st>>>(n, nrhs, x64, xlo, mask);
  return cudaGetLastError();
}

cudaError_t launch_mx_residual(int plo, int64_t sites, int nrhs, SpinorPtr b, SpinorPtr s64,
                               SpinorPtr r64, SpinorPtr rlo, const int* mask, const Reduce& red,
                               int max_blocks, cudaStream_t st) {
  LaunchCfg c = launch_cfg(sites, nrhs, max_blocks);
  const int64_t n = sites * nrhs;
  if (plo == PREC_SINGLE) mx_residual_kernel<PREC_SINGLE><<<c.grid, c.block, 0, st>>>(n, nrhs, b, s64, r64, rlo, mask, red);
  else if (plo == PREC_HALF) mx_residual_kernel<PREC_HALF><<<c.grid, c.block, 0, st>>>(n, nrhs, b, s64, r64, rlo, mask, red);
  else mx_residual_kernel<PREC_DOUBLE><<<c.grid, c.block, 0, st>>>(n, nrhs, b, s64, r64, rlo, mask, red);
  return cudaGetLastError();
}

cudaError_t launch_mx_p(int plo, int64_t sites, int nrhs, SpinorPtr p, SpinorPtr r,
                        const CGState* state, const int* mask, cudaStream_t st) {
  const int64_t n = sites * nrhs;
  LaunchCfg c = launch_cfg(sites, nrhs, kScalarStreamGrid);
  if (plo == PREC_SINGLE) mx_p_kernel<PREC_SINGLE><<<c.grid, c.block, 0, st>>>(n, nrhs, p, r, state, mask);
  else if (plo == PREC_HALF) mx_p_kernel<PREC_HALF><<<c.grid, c.block, 0, st>>>(n, nrhs, p, r, state, mask);
  else mx_p_kernel<PREC_DOUBLE><<<c.grid, c.block, 0, st>>>(n, nrhs, p, r, state, mask);
  return cudaGetLastError();
}

// ---- Field::operator* (lib/Fields/field.inl:58-62): sum_i a_i b_i per rhs ------------
template <int SP>
__global__ void __launch_bounds__(256) dot_kernel(int64_t n, int nrhs, SpinorPtr a, SpinorPtr b, Reduce red) {
  using R = typename SpinorIO<SP>::Real;
  double acc = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    Cx<R> av[12], bv[12];
    SpinorIO<SP>::load(a, i, av);
    SpinorIO<SP>::load(b, i, bv);
#pragma unroll
    for (int k = 0; k < 12; ++k) acc += double(av[k].re) * bv[k].re + double(av[k].im) * bv[k].im;
  }
  block_reduce_finish<1>(red, &acc, nrhs, blockIdx.x, gridDim.x);
}

cudaError_t launch_dot(int prec, int64_t sites, int nrhs, SpinorPtr a, SpinorPtr b,
                       const Reduce& red, int max_blocks, cudaStream_t st) {
  LaunchCfg c = launch_cfg(sites, nrhs, max_blocks);
  const int64_t n = sites * nrhs;
  if (prec == PREC_SINGLE) dot_kernel<PREC_SINGLE><<<c.grid, c.block, 0, st>>>(n, nrhs, a, b, red);
  else if (prec == PREC_HALF) dot_kernel<PREC_HALF><<<c.grid, c.block, 0, st>>>(n, nrhs, a, b, red);
  else dot_kernel<PREC_DOUBLE><<<c.grid, c.block, 0, st>>>(n, nrhs, a, b, red);
  return cudaGetLastError();
}

}  // namespace iro
