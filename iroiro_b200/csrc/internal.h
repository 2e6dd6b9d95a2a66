// Host-side interface between the C ABI layer and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "solver_scalars.cuh"

namespace iro {

// A device spinor field of one parity (or both, for full-lattice fields: the
// even half followed by the odd half), nrhs right-hand sides.
struct DevField {
  int subset;  // 0 even, 1 odd, 2 full
  int prec;
  int nrhs;
  int64_t Vh;
  void* data;   // chunks
  float* norm;  // FP16 norms
  size_t bytes_data, bytes_norm;
  // pointer to the half of parity p (p must be contained in the subset)
  SpinorPtr half(int p) const;
  // the whole field as one vector of sites() sites
  SpinorPtr all() const;
  int64_t sites() const { return (subset == 2 ? 2 : 1) * Vh; }
};

int spinor_chunk_bytes(int prec);  // bytes of one chunk element
int spinor_nchunk(int prec);

struct LaunchCfg {
  int block;  // nrhs * 2^k, at most 256
  int grid;
};
LaunchCfg launch_cfg(int64_t vh, int nrhs, int max_blocks, int block_cap = 256);

// ---- stencil ---------------------------------------------------------------
struct HopLaunch {
  Geom g;
  int p0;     // output parity of grid row 0
  int nparity;  // 1 or 2 (both parities in one launch)
  int nrhs;
  SpinorPtr in[2], out[2], xin[2];
  GaugePtr gauge;
  int recon;
  CloverPtr clov[2];
  int prec;
  bool dag;
  int epi;
  double scale;
  int red_mask;
  Reduce red;
  const int* skip;
  int max_blocks;
  int variant;    // kernel variant (see hop_kernel), chosen by the autotuner
  int block_cap;  // largest block size (128 or 256), chosen by the autotuner
  // fused CG update on the output (see HopParams::cg)
  int cg = 0;
  SpinorPtr cr[2];
  const CGState* cst = nullptr;
  // output half-sites [hs0, hs0 + nhs) only (nhs < 0: all); one-RHS-per-thread
  // variants only (the overlapped host-array path)
  int hs0 = 0;
  int nhs = -1;
  // grid over every site instead of max_blocks (ignored when the launch
  // reduces: the reduction scratch holds max_blocks partials per parity)
  int grid_free = 0;
  int grid_cap() const { return (grid_free && !red_mask && !cg) ? 0x7fffffff : max_blocks; }
};
cudaError_t launch_hop(const HopLaunch& L, cudaStream_t st);

// the residual updated by the CG step fused into the last launch of D^dag D
struct CGFuse {
  const DevField* r;
  const CGState* st;
};

// ---- linear algebra on fields ------------------------------------------------
// v = a*x + b*y for nrhs fields of one parity (scalars uniform)
cudaError_t launch_axpby(int prec, int64_t Vh, int nrhs, double a, SpinorPtr x, double b,
                         SpinorPtr y, SpinorPtr v, cudaStream_t st);
// precision conversion of one parity
cudaError_t launch_convert(int pin, SpinorPtr in, int pout, SpinorPtr out, int64_t Vh, int nrhs,
                           cudaStream_t st);
// sum |v|^2 (k=0) and, if w given, |w|^2 (k=1) per rhs with a stage update
cudaError_t launch_norms(int prec, int64_t Vh, int nrhs, SpinorPtr v, const SpinorPtr* w,
                         const Reduce& red, int max_blocks, cudaStream_t st);
// sum_i a_i b_i (real parts) per rhs
cudaError_t launch_dot(int prec, int64_t sites, int nrhs, SpinorPtr a, SpinorPtr b,
                       const Reduce& red, int max_blocks, cudaStream_t st);
// CG: r = b - s, p = r; reduce |r|^2, |b|^2 (stage ST_CG_INIT)
cudaError_t launch_cg_init(int prec, int64_t Vh, int nrhs, SpinorPtr b, SpinorPtr s, SpinorPtr r,
                           SpinorPtr p, const Reduce& red, int max_blocks, cudaStream_t st);
// CG: p = beta p + r
cudaError_t launch_cg_p(int prec, int64_t Vh, int nrhs, SpinorPtr p, SpinorPtr r, SpinorPtr x,
                        const CGState* state, const int* done, cudaStream_t st);

// Multishift, vectors in FP64 or FP32 (prec), FP64 scalars:
// x0 -= beta p0; r += beta (s + sigma0 p0); reduce |r|^2
cudaError_t launch_ms_xr(int prec, int64_t Vh, SpinorPtr x0, SpinorPtr r, SpinorPtr p0, SpinorPtr s,
                         const MSState* m, const Reduce& red, int max_blocks, cudaStream_t st);
// p0 = alpha p0 + r; x_k -= betas_k p_k; p_k = alphas_k p_k + zeta_k r; reduce |p_k|^2
struct MSFields {
  SpinorPtr x[MAXSHIFT], p[MAXSHIFT];
};
cudaError_t launch_ms_p(int prec, int64_t Vh, int nshift, const MSFields& f, SpinorPtr r,
                        const MSState* m, const Reduce& red, int max_blocks, cudaStream_t st);
// FP64 multishift with a residual window: the ring of residual slots and the
// fold's fields
struct SlotList {
  SpinorPtr s[MSW_MAX + 1];
};
// r_{k+1} = r_k + beta (s + sigma0 p0) from slot k % nslots into slot
// (k + 1) % nslots, |r_{k+1}|^2 (stage ST_MSW_R)
cudaError_t launch_msw_r(int64_t Vh, const SlotList& sl, int nslots, SpinorPtr p0, SpinorPtr s,
                         const MSState* m, const Reduce& red, int max_blocks, cudaStream_t st);
// p0 = alpha p0 + r_{k+1} (stage ST_MSW_P)
cudaError_t launch_msw_p(int64_t Vh, const SlotList& sl, int nslots, SpinorPtr p0, const MSState* m,
                         const Reduce& red, int max_blocks, cudaStream_t st);
// Fold of a window of n iterations that began at k0, for shifts k < nx:
//   x_k += X_k p_k + sum_{j<n} C_kj r_{k0+1+j};
//   p_k  = P_k p_k + sum_{j<n} D_kj r_{k0+1+j}   (p formed for plo <= k < nx)
// coef[k * kMswCoef + {0, 1, 2 + j, 2 + MSW_MAX + j}] = X_k, P_k, C_kj, D_kj;
// r_{k0+1+j} is in slot (s1 + j) % nslots
constexpr int kMswCoef = 2 + 2 * MSW_MAX;
cudaError_t launch_msw_fold(int64_t Vh, const SlotList& sl, int nslots, int s1, int n,
                            const MSFields& f, int nx, int plo, const double* coef, cudaStream_t st);
// x64_k += xlo_k (FP32), xlo_k = 0 for k < n
cudaError_t launch_ms_merge(int64_t Vh, int n, const MSFields& x64, const MSFields& xlo,
                            cudaStream_t st);
// shifted CG: r -= alpha (s + sigma p) per rhs (CGState::alpha, ::sigma);
// reduce |r|^2 (stage ST_CG_BETA)
cudaError_t launch_cg_shift_r(int prec, int64_t Vh, int nrhs, SpinorPtr r, SpinorPtr s, SpinorPtr p,
                              const CGState* state, const Reduce& red, int max_blocks,
                              cudaStream_t st);
// s += sigma_rhs x (FP64)
cudaError_t launch_shift_add(int64_t sites, int nrhs, SpinorPtr s, SpinorPtr x, const CGState* state,
                             cudaStream_t st);
// FP64 block of ns right-hand sides from the single fields f.x[k] (prec)
cudaError_t launch_ms_pack(int prec, int64_t sites, int ns, const MSFields& f, SpinorPtr out,
                           cudaStream_t st);
struct ShiftList {
  double s[MAXSHIFT];
};
// r_k = b - s_k - sigma_k x_k (FP64 block, b a single field)
cudaError_t launch_ms_block_residual(int64_t sites, int ns, SpinorPtr b, SpinorPtr s, SpinorPtr x,
                                     const ShiftList& sg, SpinorPtr r, cudaStream_t st);

// ---- mixed precision (reliable updates), masked by mask[rhs] != 0 ----------------
cudaError_t launch_mx_merge(int plo, int64_t sites, int nrhs, SpinorPtr x64, SpinorPtr xlo,
                            const int* mask, cudaStream_t st);
cudaError_t launch_mx_residual(int plo, int64_t sites, int nrhs, SpinorPtr b, SpinorPtr s64,
                               SpinorPtr r64, SpinorPtr rlo, const int* mask, const Reduce& red,
                               int max_blocks, cudaStream_t st);
cudaError_t launch_mx_p(int plo, int64_t sites, int nrhs, SpinorPtr p, SpinorPtr r,
                        const CGState* state, const int* mask, cudaStream_t st);

// ---- boundary conversion ---------------------------------------------------------
// host Format_F doubles (already on the device in `stage`) <-> device field.
// layout 0: full lexicographic lattice; 1: half field of parity p (hs order).
// nrhs consecutive host fields of `host_sites` sites each.
// [hs0, hs0 + nhs): the half-sites converted (nhs < 0: to the end)
cudaError_t launch_import_spinor(const Geom& g, const double* stage, int layout, int p,
                                 int64_t host_sites, int nrhs, int prec, SpinorPtr out,
                                 cudaStream_t st, int64_t hs0 = 0, int64_t nhs = -1);
cudaError_t launch_export_spinor(const Geom& g, double* stage, int layout, int p,
                                 int64_t host_sites, int nrhs, int prec, SpinorPtr in,
                                 cudaStream_t st, int64_t hs0 = 0, int64_t nhs = -1);
// F (a full-lattice FP64 field of F.nrhs right-hand sides) = the spin-colour
// point sources r = first .. first + F.nrhs - 1 at half-site hs of parity p:
// right-hand side j is 1 at the real part of spin-colour component first + j
cudaError_t launch_point_sources(const DevField& F, int p, int64_t hs, int first, cudaStream_t st);
// gamma5 on a Format_F staging buffer in place
cudaError_t launch_gamma5_aos(double* stage, int64_t nsites, cudaStream_t st);

// Format_G doubles on the device -> link arrays.  Also returns (in *maxdev)
// the largest deviation of row 2 from conj(row0 x row1) and of the first two
// rows from orthonormality.
struct GaugeArrays {
  double2* d12;  // [2][4][6][Vh]
  double2* d18;  // [2][4][9][Vh]
  float4* s12;   // [2][4][3][Vh]
  uint4* h12a;   // [2][4][Vh]
  uint2* h12b;   // [2][4][Vh]
  uint4* h18a;   // [2][4][Vh][2]: FP16 U00..U21 (all three rows stored)
  uint32_t* h18b;  // [2][4][Vh]: FP16 U22
};
cudaError_t launch_import_gauge(const Geom& g, const double* raw, GaugeArrays ga,
                                unsigned long long* maxdev_bits, cudaStream_t st);

// ---- clover ------------------------------------------------------------------------
struct CloverArrays {
  void* A[3][2];     // [prec][parity]
  void* Ainv[3][2];
};
cudaError_t launch_clover_build(const Geom& g, const double* raw, double kappa_csw,
                                CloverArrays ca, int* singular, cudaStream_t st);
cudaError_t launch_field_strength(const Geom& g, const double* raw, int mu, int nu, double* out,
                                  cudaStream_t st);
void clover_init_tables();

// ---- rational-function reconstruction and clover fields (kernels.cu) --------------
constexpr int kMaxCombine = 16;
struct SField {
  SpinorPtr f[kMaxCombine];
  double a[kMaxCombine];
};
// y = c0 b + sum_{k<n} a_k x_k over `sites` FP64 elements
cudaError_t launch_combine(int64_t sites, double c0, SpinorPtr b, int n, const SField& x,
                           SpinorPtr y, cudaStream_t st);
// out = C in for an FP64 half field of nrhs right-hand sides (C: a clover block or its inverse)
cudaError_t launch_clover_mult(int64_t Vh, int nrhs, CloverPtr cl, SpinorPtr in, SpinorPtr out,
                               cudaStream_t st);

// ---- molecular-dynamics force (forces.cu) ------------------------------------------
// F[mu][lex site][18] += w (1 - g_mu) U_mu(x) psi(x+mu) (x) chi(x)^dag over the
// sites x of parity p (gamma5 on both fields when g5)
// the clover block of Dirac_Clover::md_force, added to F (Format_G) with weight
// w = -kappa csw / 4; lam: scratch of 6 * 9 * V double2
cudaError_t launch_clover_force(const Geom& g, const double* u_format_g, SpinorPtr e0, SpinorPtr e1,
                                SpinorPtr z0, SpinorPtr z1, double w, double2* lam, double* F,
                                cudaStream_t st);
cudaError_t launch_force(const Geom& g, const GaugePtr& gauge, int recon, int p, SpinorPtr psi,
                         SpinorPtr chi, int g5, double w, double* F, cudaStream_t st);

// ---- learned preconditioner (learned.cu) -------------------------------------------
struct PtcGeo;
constexpr int kMaxVec = 16;
constexpr int kMaxList = kMaxVec + 2;  // a cycle's directions and two more fields
struct CFieldList {
  SpinorPtr f[kMaxList];
};
// The state of one GCR restart cycle on the device: its coefficients are
// formed there (gcr_coef_kernel), so that the host enqueues a whole cycle and
// reads back once.  Iteration k of the cycle is skipped (every kernel of it
// returns at once) when skip[k] is set, which the coefficient kernel does for
// the iterations after the one that met the restart test.
struct GcrState {
  double nw[kMaxVec];                   // |w'_q|^2
  double tre[kMaxVec * kMaxVec];        // T[i][j] at i * kMaxVec + j: z'_j = sum_i T[i][j] z_i
  double tim[kMaxVec * kMaxVec];
  double are[kMaxVec], aim[kMaxVec];    // alpha_j
  double bre[kMaxVec], bim[kMaxVec];    // the current iteration's Gram-Schmidt coefficients
  double rr_it, rr_start, target, d2;   // iterated |r|^2, its value at the cycle start, the
                                        // solve's target and delta^2
  int limit;                            // iterations the cycle may take
  int jdone;                            // iterations done
  int skip[kMaxVec];                    // iteration k is not needed
  int plain[kMaxVec];                   // iteration k needs no second pass
  float cre[kMaxList], cim[kMaxList];   // the current coefficients in FP32 (update / correction)
  float ure, uim;                       // the current alpha in FP32
};
// The Krylov fields w, z (and t) are FP32 or FP16 (pw/px = PREC_SINGLE or
// PREC_HALF); the residual r and the correction are FP32.
// <w_q, t> (q < m; w_{m-1} is r): block partials into part, their
// sums (a fixed order) into out[2m]; nothing when skip is set
cudaError_t launch_cdot(int64_t n, int m, const CFieldList& w, SpinorPtr t, double* part, int blocks,
                        double* out, const int* skip, int pw, cudaStream_t st);
// y += sum_{q < m} c_q x_q with the coefficients s->cre/cim (q < *count when
// count is given; sign -1: y -= ...); nothing when skip is set
cudaError_t launch_caxpy_dev(int64_t n, int m, const CFieldList& x, int px, const GcrState* s,
                             const int* count, float sign, SpinorPtr y, const int* skip,
                             cudaStream_t st);
// one Gram-Schmidt step of GCR in one pass: wj += sum_{q<m} c_q w_q, then, if
// s->plain[j], r -= alpha wj with the updated wj (coefficients from s) and,
// given feat, the network's input features of the new r
cudaError_t launch_gcr_update(int64_t n, int m, const CFieldList& w, int pw, const GcrState* s, int j,
                              SpinorPtr wj, SpinorPtr r, float2* feat, cudaStream_t st);
// the cycle's state at its start
cudaError_t launch_gcr_init(GcrState* s, double rr, double target, double d2, int limit,
                            cudaStream_t st);
// iteration j's coefficients from g = (<w_q, w_j> (q < j), |w_j|^2, <r, w_j>)
// (second = 0), or, when the first pass found w_j nearly in the span of the
// w_q, from g = (|w'_j|^2, <r, w'_j>) of the orthogonalised w'_j (second = 1)
cudaError_t launch_gcr_coef(GcrState* s, const double* g, int j, int m, int second,
                            cudaStream_t st);
// the correction coefficients gamma = T alpha of the finished cycle into
// s->cre/cim
cudaError_t launch_gcr_gamma(GcrState* s, cudaStream_t st);

}  // namespace iro
