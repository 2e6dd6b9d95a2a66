// C ABI of the B200 fermion-solve library: contexts, resident gauge and
// clover data, boundary conversion of host fields, operator composition and
// the Krylov solvers.  See include/iroiro_b200.h for the contract of each
// entry point and the reference interface it replaces.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "internal.h"
#include "iroiro_b200.h"

using namespace iro;

struct iro_field {
  iro_ctx* ctx;
  int dev;  // device of the buffers (iro_field_destroy does not touch the context)
  DevField f;
};

// an autotuner choice: stencil variant, block size cap, and whether the grid
// covers every site (one pass) or is capped at max_blocks (grid-stride loop)
struct Tune {
  int variant, block, free_grid;
};

struct iro_ctx {
  int L[4];
  Geom g;
  int64_t V, Vh;
  int device;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  int sms = 148;
  int max_blocks = 148 * 8;

  // gauge
  bool has_gauge = false;
  int recon = 12;
  double* raw = nullptr;  // Format_G, FP64, on the device
  GaugeArrays ga{};
  unsigned long long* d_maxdev = nullptr;

  // clover
  bool has_clover = false;
  double cl_kc = 0.0;  // kappa*csw the clover was built for
  void* clA[3][2] = {};
  void* clAinv[3][2] = {};
  int* d_singular = nullptr;

  // boundary staging
  double* stage = nullptr;
  size_t stage_bytes = 0;
  // pinned host ring for large copies to and from pageable host memory
  char* ring[2] = {nullptr, nullptr};
  cudaEvent_t ring_ev[2] = {nullptr, nullptr};
  // copy streams (host-to-device, device-to-host) and chunk events of the
  // overlapped Schur operator between pinned host arrays
  cudaStream_t xs[2] = {nullptr, nullptr};
  std::vector<cudaEvent_t> xev;

  // reduction scratch and solver state
  double* partials = nullptr;
  unsigned* counter = nullptr;
  double* redout = nullptr;
  void* state = nullptr;  // CGState[16] or MSState
  int* done = nullptr;    // [16]
  void* h_pinned = nullptr;  // host mirror of state + done

  std::map<std::tuple<int, int, int, int>, DevField> ws;
  // small device scratch of the solvers that keep per-call state (GCR),
  // allocated once and grown on demand: no allocation inside a solve
  void* scratch = nullptr;
  size_t scratch_bytes = 0;

  // stencil autotuner: (prec, recon, dag, epilogue, nrhs, nparity) -> (variant, block cap)
  std::map<std::tuple<int, int, int, int, int, int>, Tune> tuned;
  std::map<std::tuple<int, int, int, int, int, int>, float> tuned_ms;
};

namespace {

constexpr int kMaxRhs = 16;
constexpr size_t kPartialsPerBlock = 64;

int fail(iro_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_fail(iro_ctx* c, cudaError_t e, const char* where) {
  return fail(c, e == cudaErrorMemoryAllocation ? IRO_OUT_OF_MEMORY : IRO_CUDA_ERROR,
              std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                        \
  do {                                                  \
    cudaError_t e__ = (call);                           \
    if (e__ != cudaSuccess) return cuda_fail(c, e__, #call); \
  } while (0)

#define RCK(call)             \
  do {                        \
    const int r__ = (call);   \
    if (r__) return r__;      \
  } while (0)

double kappa_of(double mass) { return 0.5 / (4.0 + mass); }

int alloc_field(iro_ctx* c, int subset, int prec, int nrhs, DevField& f) {
  f.subset = subset;
  f.prec = prec;
  f.nrhs = nrhs;
  f.Vh = c->Vh;
  const int np = subset == 2 ? 2 : 1;
  f.bytes_data = size_t(np) * c->Vh * nrhs * spinor_nchunk(prec) * 16;
  f.bytes_norm = prec == PREC_HALF ? size_t(np) * c->Vh * nrhs * sizeof(float) : 0;
  f.data = nullptr;
  f.norm = nullptr;
  cudaError_t e = cudaMalloc(&f.data, f.bytes_data);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc(field)");
  if (f.bytes_norm) {
    e = cudaMalloc(reinterpret_cast<void**>(&f.norm), f.bytes_norm);
    if (e != cudaSuccess) {
      cudaFree(f.data);
      return cuda_fail(c, e, "cudaMalloc(norm)");
    }
  }
  return IRO_OK;
}

void free_field(DevField& f) {
  if (f.data) cudaFree(f.data);
  if (f.norm) cudaFree(f.norm);
  f.data = nullptr;
  f.norm = nullptr;
}

// workspace field (cached per subset, precision, nrhs and slot)
DevField* ws(iro_ctx* c, int subset, int prec, int nrhs, int slot, int* rc) {
  auto key = std::make_tuple(subset, prec, nrhs, slot);
  auto it = c->ws.find(key);
  if (it != c->ws.end()) return &it->second;
  DevField f;
  *rc = alloc_field(c, subset, prec, nrhs, f);
  if (*rc != IRO_OK) return nullptr;
  return &(c->ws[key] = f);
}

// ---- host copies -----------------------------------------------------------------
// The driver copies pageable host memory through its own staging on one host
// thread (~21 GB/s for 4.8 GB device to host, measured on a B200 host).
// Large copies to or from pageable memory go through two pinned chunks
// instead: the DMA of one chunk overlaps the copy of the other, which
// kCopyThreads host threads split (~46 GB/s measured).  Pinned (registered)
// host memory, and copies below two chunks, take the direct DMA.
constexpr size_t kRingChunk = size_t(128) << 20;
constexpr int kCopyThreads = 8;

bool host_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// the stripes no thread took (thread creation can fail) are copied by the caller
void parallel_copy(void* dst, const void* src, size_t bytes) {
  const int nt = int(std::min<unsigned>(kCopyThreads, std::max(1u, std::thread::hardware_concurrency())));
  const size_t stripe = ((bytes / nt) + 63) & ~size_t(63);
  auto part = [=](int k) {
    const size_t a = std::min(bytes, k * stripe), b = std::min(bytes, a + stripe);
    if (b > a) std::memcpy(static_cast<char*>(dst) + a, static_cast<const char*>(src) + a, b - a);
  };
  std::vector<std::thread> th;
  int k = 1;
  try {
    for (; k < nt; ++k) th.emplace_back(part, k);
  } catch (...) {
  }
  part(0);
  for (int j = k; j < nt; ++j) part(j);
  for (auto& t : th) t.join();
}

int ensure_ring(iro_ctx* c) {
  for (int i = 0; i < 2; ++i) {
    if (!c->ring[i]) CK(cudaHostAlloc(reinterpret_cast<void**>(&c->ring[i]), kRingChunk, cudaHostAllocDefault));
    if (!c->ring_ev[i]) CK(cudaEventCreateWithFlags(&c->ring_ev[i], cudaEventDisableTiming));
  }
  return IRO_OK;
}

// device -> host, returns with the copy complete
int copy_d2h(iro_ctx* c, void* host, const void* dev, size_t bytes) {
  if (bytes < 2 * kRingChunk || host_pinned(host)) {
    CK(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return IRO_OK;
  }
  RCK(ensure_ring(c));
  const size_t nch = (bytes + kRingChunk - 1) / kRingChunk;
  // chunk i goes to slot i % 2; the host copy of chunk i - 1 (slot (i - 1) % 2)
  // runs while the DMA of chunk i is in flight
  for (size_t i = 0; i <= nch; ++i) {
    if (i < nch) {
      const size_t off = i * kRingChunk, len = std::min(kRingChunk, bytes - off);
      CK(cudaMemcpyAsync(c->ring[i % 2], static_cast<const char*>(dev) + off, len, cudaMemcpyDeviceToHost,
                         c->stream));
      CK(cudaEventRecord(c->ring_ev[i % 2], c->stream));
    }
    if (i >= 1) {
      const size_t j = i - 1, off = j * kRingChunk, len = std::min(kRingChunk, bytes - off);
      CK(cudaEventSynchronize(c->ring_ev[j % 2]));
      parallel_copy(static_cast<char*>(host) + off, c->ring[j % 2], len);
    }
  }
  return IRO_OK;
}

// host -> device, enqueued on the context's stream (the host buffer may be
// reused once this returns)
int copy_h2d(iro_ctx* c, void* dev, const void* host, size_t bytes) {
  if (bytes < 2 * kRingChunk || host_pinned(host)) {
    CK(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, c->stream));
    return IRO_OK;
  }
  RCK(ensure_ring(c));
  const size_t nch = (bytes + kRingChunk - 1) / kRingChunk;
  for (size_t i = 0; i < nch; ++i) {
    const size_t off = i * kRingChunk, len = std::min(kRingChunk, bytes - off);
    // slot i % 2 is free once the DMA of chunk i - 2 has completed
    if (i >= 2) CK(cudaEventSynchronize(c->ring_ev[i % 2]));
    parallel_copy(c->ring[i % 2], static_cast<const char*>(host) + off, len);
    CK(cudaMemcpyAsync(static_cast<char*>(dev) + off, c->ring[i % 2], len, cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(c->ring_ev[i % 2], c->stream));
  }
  // the pinned chunks are reused by the next call: wait for the last DMAs
  for (size_t i = nch >= 2 ? nch - 2 : 0; i < nch; ++i) CK(cudaEventSynchronize(c->ring_ev[i % 2]));
  return IRO_OK;
}

int ensure_stage(iro_ctx* c, size_t bytes) {
  if (c->stage_bytes >= bytes) return IRO_OK;
  if (c->stage) cudaFree(c->stage);
  c->stage = nullptr;
  c->stage_bytes = 0;
  CK(cudaMalloc(&c->stage, bytes));
  c->stage_bytes = bytes;
  return IRO_OK;
}

Reduce make_reduce(iro_ctx* c, int stage, int max_iter) {
  Reduce r;
  r.partials = c->partials;
  r.gpartials = c->partials + kPartialsPerBlock * size_t(c->max_blocks) * 2;
  r.counter = c->counter;
  r.out = c->redout;
  r.stage = stage;
  r.state = c->state;
  r.done = c->done;
  r.max_iter = max_iter;
  return r;
}

GaugePtr gauge_ptr(iro_ctx* c, int prec) {
  GaugePtr g;
  g.Vh = c->Vh;
  g.b = nullptr;
  if (prec == PREC_DOUBLE)
    g.a = c->recon == 12 ? static_cast<const void*>(c->ga.d12) : static_cast<const void*>(c->ga.d18);
  else if (prec == PREC_SINGLE)
    g.a = c->ga.s12;
  else {
    g.a = c->ga.h12a;
    g.b = c->ga.h12b;
  }
  return g;
}

bool is_clover(int op) {
  return op == IRO_OP_CLOVER_FULL || op == IRO_OP_CLOVER_SCHUR_EE || op == IRO_OP_CLOVER_HOP_OE_INV;
}
bool is_full(int op) { return op == IRO_OP_WILSON_FULL || op == IRO_OP_CLOVER_FULL; }
bool op_valid(int op) { return op >= IRO_OP_WILSON_FULL && op <= IRO_OP_CLOVER_HOP_OE_INV; }

int input_subset(int op) {
  switch (op) {
    case IRO_OP_WILSON_HOP_EO: return 1;
    case IRO_OP_WILSON_HOP_OE:
    case IRO_OP_CLOVER_HOP_OE_INV: return 0;
    case IRO_OP_WILSON_SCHUR_EE:
    case IRO_OP_CLOVER_SCHUR_EE: return 0;
    default: return 2;
  }
}
int output_subset(int op) {
  switch (op) {
    case IRO_OP_WILSON_HOP_EO: return 0;
    case IRO_OP_WILSON_HOP_OE:
    case IRO_OP_CLOVER_HOP_OE_INV: return 1;
    case IRO_OP_WILSON_SCHUR_EE:
    case IRO_OP_CLOVER_SCHUR_EE: return 0;
    default: return 2;
  }
}

int clover_build(iro_ctx* c, double kc);

int ensure_clover(iro_ctx* c, double mass, double csw) {
  const double kc = kappa_of(mass) * csw;
  if (c->has_clover && c->cl_kc == kc) return IRO_OK;
  return clover_build(c, kc);
}

CloverPtr clover_ptr(iro_ctx* c, int prec, int p, bool inverse) {
  CloverPtr cp;
  cp.data = inverse ? c->clAinv[prec][p] : c->clA[prec][p];
  cp.Vh = c->Vh;
  return cp;
}

HopLaunch base_launch(iro_ctx* c, int prec, bool dag, int nrhs) {
  HopLaunch L{};
  L.g = c->g;
  L.nparity = 1;
  L.nrhs = nrhs;
  L.gauge = gauge_ptr(c, prec);
  L.recon = prec == PREC_DOUBLE ? c->recon : 12;
  L.prec = prec;
  L.dag = dag;
  L.max_blocks = c->max_blocks;
  L.skip = nullptr;
  L.red_mask = 0;
  L.variant = 0;
  L.block_cap = 256;
  return L;
}

// Launches the stencil with the variant and block size the autotuner picked
// for this (precision, reconstruction, dagger, epilogue, nrhs, parities).
// An untuned shape is timed once in every candidate configuration on the
// caller's own fields (without reductions, so solver state is untouched; the
// launch is idempotent) before the real launch; during stream capture the
// default configuration is used.  IRO_HOP_VARIANT="<variant>,<block>[,<free
// grid 0/1>]" fixes the choice.  The grid is either capped at max_blocks
// blocks, whose threads loop over the sites, or covers every site in one
// pass (launches with a reduction keep the cap: the reduction's scratch
// holds max_blocks partials per parity).
// Candidates (see hop_var): all precisions 0..3; FP64 4, 5 and, on an SU(3)
// field, 6..11 = 0..5 on the stored 18-real links (no third-row
// reconstruction: fewer FP64 operations, more link bytes); FP32/FP16 with an
// even nrhs 4..9 (two right-hand sides per thread); FP16 10..12 (the
// mixed-precision kernel on the FP16 links with three stored rows at 3, 4 or
// 2 blocks per SM, any nrhs) and 13..14 (the same kernel on the 12-real FP16
// links, row 2 rebuilt per link, at 3 or 4 blocks per SM).
constexpr int kHopVariants = 15;

static bool variant_ok(const HopLaunch& L, int v) {
  if (v < 0 || v >= kHopVariants) return false;
  if (v < 4) return true;
  if (L.prec == PREC_DOUBLE) return v < 12 && (v < 6 || L.recon == 12);
  if (v < 10) return L.recon == 12 && L.nrhs % 2 == 0;
  return L.prec == PREC_HALF && L.recon == 12;
}

static cudaError_t launch_variant(iro_ctx* c, HopLaunch L, cudaStream_t st) {
  if (L.prec == PREC_DOUBLE && L.variant >= 6) {
    L.variant -= 6;
    L.recon = 18;
    L.gauge.a = c->ga.d18;
  } else if (L.prec == PREC_HALF && L.variant >= 10 && L.variant <= 12) {
    L.recon = 18;
    L.gauge.a = c->ga.h18a;
    L.gauge.b = c->ga.h18b;
  }
  return launch_hop(L, st);
}

std::tuple<int, int, int, int, int, int> tune_key(const HopLaunch& L) {
  return std::make_tuple(L.prec, L.recon, int(L.dag), L.epi, L.nrhs, L.nparity);
}

int launch_tuned(iro_ctx* c, HopLaunch L) {
  const auto key = tune_key(L);
  cudaStream_t st = c->stream;
  static const char* forced = std::getenv("IRO_HOP_VARIANT");
  auto it = c->tuned.find(key);
  if (forced) {
    // the forced variant, modulo the candidates of the shape: FP64 6 (12 on
    // an SU(3) field); otherwise 13, a variant the shape lacks falling back
    // to its number modulo 4
    int v = 0, b = 256, g = 0;
    std::sscanf(forced, "%d,%d,%d", &v, &b, &g);
    if (L.prec == PREC_DOUBLE) v %= (L.recon == 12 ? 12 : 6);
    else if (!variant_ok(L, v % kHopVariants)) v %= 4;
    else v %= kHopVariants;
    c->tuned[key] = Tune{v, b, g != 0};
    it = c->tuned.find(key);
  }
  if (it == c->tuned.end()) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) {
      L.variant = 0;
      L.block_cap = 256;
      CK(launch_hop(L, st));
      return IRO_OK;
    }
    HopLaunch T = L;
    T.red_mask = 0;
    T.cg = 0;  // tuning launches must not touch the solver's fields
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best = 1e30f;
    Tune pick{0, 256, 0};
    for (int v = 0; v < kHopVariants; ++v)
      for (int b : {256, 128})
        for (int g : {0, 1}) {
          if (!variant_ok(L, v)) continue;
          T.variant = v;
          T.block_cap = b;
          T.grid_free = g;
          CK(launch_variant(c, T, st));  // warm-up
          CK(cudaEventRecord(e0, st));
          for (int i = 0; i < 3; ++i) CK(launch_variant(c, T, st));
          CK(cudaEventRecord(e1, st));
          CK(cudaEventSynchronize(e1));
          float ms = 0.f;
          CK(cudaEventElapsedTime(&ms, e0, e1));
          if (ms < best) {
            best = ms;
            pick = {v, b, g};
          }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->tuned[key] = pick;
    c->tuned_ms[key] = best / 3;
    it = c->tuned.find(key);
  }
  L.variant = it->second.variant;
  L.block_cap = it->second.block;
  L.grid_free = it->second.free_grid;
  CK(launch_variant(c, L, st));
  return IRO_OK;
}

// The two stencils of the even/odd Schur operator on fields of L1's
// precision, dagger and nrhs (L1 comes from base_launch):
//   L1: t_o   = [A_oo^-1] (-kappa H_oe f_e)
//   L2: out_e = [A_ee] f_e + kappa H_eo t_o  =  f - Deo(Doe f)
// (Dirac_Wilson_EvenOdd::mult, lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:79-83)
void schur_launches(iro_ctx* c, bool cl, double k, const DevField& in, DevField& t,
                    DevField& out, HopLaunch& L1, HopLaunch& L2) {
  L2 = L1;
  L1.p0 = 1;
  L1.in[0] = in.half(0);
  L1.out[0] = t.half(1);
  L1.epi = cl ? EPI_SCALE_CLOV : EPI_SCALE;
  if (cl) L1.clov[0] = clover_ptr(c, L1.prec, 1, true);
  L1.scale = -k;
  L2.p0 = 0;
  L2.in[0] = t.half(1);
  L2.out[0] = out.half(0);
  L2.xin[0] = in.half(0);
  L2.epi = cl ? EPI_XPAY_CLOV : EPI_XPAY;
  if (cl) L2.clov[0] = clover_ptr(c, L1.prec, 0, false);
  L2.scale = k;
}

// The full-lattice operator as one launch over both parities (L from
// base_launch): out_p = [A_pp] in_p - kappa H_{p,1-p} in_{1-p}
// (Dirac_Wilson::mult, lib/Dirac_ops/dirac_wilson.cpp:28-32)
void full_launch(iro_ctx* c, bool cl, double k, const DevField& in, DevField& out, HopLaunch& L) {
  L.p0 = 0;
  L.nparity = 2;
  for (int y = 0; y < 2; ++y) {
    L.in[y] = in.half(1 - y);
    L.out[y] = out.half(y);
    L.xin[y] = in.half(y);
    if (cl) L.clov[y] = clover_ptr(c, L.prec, y, false);
  }
  L.epi = cl ? EPI_XPAY_CLOV : EPI_XPAY;
  L.scale = -k;
}

// out = op(in) on device fields.  `red`/`red_mask`, when given, attach a
// reduction to the last kernel of the operator (|out|^2, |xin|^2, (xin,out)),
// and `skip` lets converged right-hand sides be left untouched.
int apply_dev(iro_ctx* c, int op, double mass, double csw, bool dag, const DevField& in,
              DevField& out, const Reduce* red, int red_mask, const int* skip,
              const CGFuse* fuse = nullptr) {
  if (fuse && (!red || op == IRO_OP_WILSON_HOP_EO || op == IRO_OP_WILSON_HOP_OE ||
               op == IRO_OP_CLOVER_HOP_OE_INV))
    return fail(c, IRO_BAD_ARG, "fused CG update needs a full or Schur operator and a reduction");
  if (!c->has_gauge) return fail(c, IRO_NO_GAUGE, "no gauge field uploaded");
  if (!op_valid(op)) return fail(c, IRO_BAD_ARG, "unknown operator");
  if (in.prec != out.prec || in.nrhs != out.nrhs)
    return fail(c, IRO_BAD_ARG, "operator fields differ in precision or nrhs");
  if ((in.subset != input_subset(op) && !(in.subset == 2 && input_subset(op) != 2)) ||
      (out.subset != output_subset(op) && !(out.subset == 2 && output_subset(op) != 2)))
    return fail(c, IRO_BAD_ARG, "field subset does not match the operator");
  if (in.data == out.data) return fail(c, IRO_BAD_ARG, "in and out must differ");
  const int prec = in.prec;
  const int nrhs = in.nrhs;
  if (prec != PREC_DOUBLE && c->recon != 12)
    return fail(c, IRO_BAD_ARG, "single/half precision need an SU(3) gauge field");
  if (is_clover(op)) {
    int rc = ensure_clover(c, mass, csw);
    if (rc) return rc;
  }
  const double k = kappa_of(mass);
  HopLaunch L = base_launch(c, prec, dag, nrhs);
  L.skip = skip;
  cudaStream_t st = c->stream;
  switch (op) {
    case IRO_OP_WILSON_HOP_EO:
    case IRO_OP_WILSON_HOP_OE: {
      const int pout = op == IRO_OP_WILSON_HOP_EO ? 0 : 1;
      L.p0 = pout;
      L.in[0] = in.half(1 - pout);
      L.out[0] = out.half(pout);
      L.epi = EPI_SCALE;
      L.scale = -k;
      if (red) { L.red = *red; L.red_mask = red_mask; }
      { int rt = launch_tuned(c, L); if (rt) return rt; }
    } break;
    case IRO_OP_CLOVER_HOP_OE_INV: {
      L.p0 = 1;
      L.in[0] = in.half(0);
      L.out[0] = out.half(1);
      L.epi = EPI_SCALE_CLOV;
      L.clov[0] = clover_ptr(c, prec, 1, true);
      L.scale = -k;
      if (red) { L.red = *red; L.red_mask = red_mask; }
      { int rt = launch_tuned(c, L); if (rt) return rt; }
    } break;
    case IRO_OP_WILSON_SCHUR_EE:
    case IRO_OP_CLOVER_SCHUR_EE: {
      int rc = IRO_OK;
      DevField* t = ws(c, 1, prec, nrhs, 0, &rc);
      if (!t) return rc;
      HopLaunch L2;
      schur_launches(c, op == IRO_OP_CLOVER_SCHUR_EE, k, in, *t, out, L, L2);
      L2.skip = skip;
      { int rt = launch_tuned(c, L); if (rt) return rt; }
      if (red) { L2.red = *red; L2.red_mask = red_mask; }
      if (fuse) {
        L2.cg = 1;
        L2.cst = fuse->st;
        L2.cr[0] = fuse->r->half(0);
      }
      { int rt = launch_tuned(c, L2); if (rt) return rt; }
    } break;
    case IRO_OP_WILSON_FULL:
    case IRO_OP_CLOVER_FULL: {
      full_launch(c, op == IRO_OP_CLOVER_FULL, k, in, out, L);
      if (red) { L.red = *red; L.red_mask = red_mask; }
      if (fuse) {
        L.cg = 1;
        L.cst = fuse->st;
        for (int y = 0; y < 2; ++y) L.cr[y] = fuse->r->half(y);
      }
      { int rt = launch_tuned(c, L); if (rt) return rt; }
    } break;
  }
  return IRO_OK;
}

int clover_build(iro_ctx* c, double kc) {
  if (!c->has_gauge) return fail(c, IRO_NO_GAUGE, "no gauge field uploaded");
  if (!c->clA[0][0]) {
    const size_t bytes[3] = {size_t(36) * 16, size_t(18) * 16, size_t(9) * 16};
    for (int pr = 0; pr < 3; ++pr)
      for (int p = 0; p < 2; ++p) {
        CK(cudaMalloc(&c->clA[pr][p], bytes[pr] * c->Vh));
        CK(cudaMalloc(&c->clAinv[pr][p], bytes[pr] * c->Vh));
      }
  }
  CloverArrays ca;
  for (int pr = 0; pr < 3; ++pr)
    for (int p = 0; p < 2; ++p) {
      ca.A[pr][p] = c->clA[pr][p];
      ca.Ainv[pr][p] = c->clAinv[pr][p];
    }
  CK(cudaMemsetAsync(c->d_singular, 0, sizeof(int), c->stream));
  CK(launch_clover_build(c->g, c->raw, kc, ca, c->d_singular, c->stream));
  int singular = 0;
  CK(cudaMemcpyAsync(&singular, c->d_singular, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (singular) return fail(c, IRO_BAD_ARG, "clover block not invertible");
  c->has_clover = true;
  c->cl_kc = kc;
  return IRO_OK;
}

// host Format_F (nrhs fields) -> device field
int import_host(iro_ctx* c, const double* host, int host_layout_full, DevField& f) {
  const int64_t host_sites = host_layout_full ? c->V : c->Vh;
  const size_t bytes = size_t(host_sites) * 24 * sizeof(double) * f.nrhs;
  int rc = ensure_stage(c, bytes);
  if (rc) return rc;
  RCK(copy_h2d(c, c->stage, host, bytes));
  if (f.subset == 2) {
    for (int p = 0; p < 2; ++p)
      CK(launch_import_spinor(c->g, c->stage, 0, p, host_sites, f.nrhs, f.prec, f.half(p), c->stream));
  } else {
    CK(launch_import_spinor(c->g, c->stage, host_layout_full ? 0 : 1, f.subset, host_sites, f.nrhs,
                            f.prec, f.half(f.subset), c->stream));
  }
  return IRO_OK;
}

int export_host(iro_ctx* c, const DevField& f, int host_layout_full, double* host) {
  const int64_t host_sites = host_layout_full ? c->V : c->Vh;
  const size_t bytes = size_t(host_sites) * 24 * sizeof(double) * f.nrhs;
  int rc = ensure_stage(c, bytes);
  if (rc) return rc;
  if (f.subset == 2) {
    for (int p = 0; p < 2; ++p)
      CK(launch_export_spinor(c->g, c->stage, 0, p, host_sites, f.nrhs, f.prec, f.half(p), c->stream));
  } else {
    CK(launch_export_spinor(c->g, c->stage, host_layout_full ? 0 : 1, f.subset, host_sites, f.nrhs,
                            f.prec, f.half(f.subset), c->stream));
  }
  return copy_d2h(c, host, c->stage, bytes);
}

// sum |v|^2 per rhs (and |w|^2) into host arrays
int norms_host(iro_ctx* c, const DevField& v, const DevField* w, std::vector<double>& nv,
               std::vector<double>* nw) {
  Reduce r = make_reduce(c, ST_NONE, 0);
  nv.assign(v.nrhs, 0.0);
  if (nw) nw->assign(v.nrhs, 0.0);
  std::vector<double> tmp(2 * v.nrhs);
  SpinorPtr wp;
  if (w) wp = w->all();
  CK(launch_norms(v.prec, v.sites(), v.nrhs, v.all(), w ? &wp : nullptr, r, c->max_blocks, c->stream));
  CK(cudaMemcpyAsync(tmp.data(), c->redout, sizeof(double) * 2 * v.nrhs, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < v.nrhs; ++k) {
    nv[k] = tmp[k];
    if (nw) (*nw)[k] = tmp[v.nrhs + k];
  }
  return IRO_OK;
}

// v = a x + b y over the whole field
int axpby_dev(iro_ctx* c, double a, const DevField& x, double b, const DevField& y, DevField& v) {
  CK(launch_axpby(v.prec, v.sites(), v.nrhs, a, x.all(), b, y.all(), v.all(), c->stream));
  return IRO_OK;
}

int convert_dev(iro_ctx* c, const DevField& in, DevField& out) {
  CK(launch_convert(in.prec, in.all(), out.prec, out.all(), out.sites(), out.nrhs, c->stream));
  return IRO_OK;
}

}  // namespace

// =====================================================================================
extern "C" {

int iro_ctx_create(const int L[4], int device, iro_ctx** out) {
  if (!out || !L) return IRO_BAD_ARG;
  *out = nullptr;
  for (int d = 0; d < 4; ++d)
    if (L[d] < 2 || (L[d] & 1)) return IRO_BAD_ARG;
  const int64_t V = int64_t(L[0]) * L[1] * L[2] * L[3];
  // 32-bit element indices for up to 16 right-hand sides, and warp-blocked
  // arrays whose half-lattice element counts are multiples of 32
  if (V / 2 * kMaxRhs >= int64_t(1) << 31 || V % 64 != 0) return IRO_BAD_ARG;
  std::unique_ptr<iro_ctx> c(new iro_ctx());
  for (int d = 0; d < 4; ++d) c->L[d] = L[d];
  c->V = V;
  c->Vh = V / 2;
  c->g.L[0] = L[0]; c->g.L[1] = L[1]; c->g.L[2] = L[2]; c->g.L[3] = L[3];
  c->g.Lxh = L[0] / 2;
  c->g.Vh = int(c->Vh);
  c->g.sy = c->g.Lxh;
  c->g.sz = c->g.Lxh * L[1];
  c->g.st = c->g.Lxh * L[1] * L[2];
  c->g.dxh = make_fastdiv(uint32_t(c->g.Lxh));
  c->g.dy = make_fastdiv(uint32_t(L[1]));
  c->g.dz = make_fastdiv(uint32_t(L[2]));
  c->device = device;
  iro_ctx* cp = c.get();
  {
    iro_ctx* c = cp;
    CK(cudaSetDevice(device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    c->sms = prop.multiProcessorCount;
    c->max_blocks = c->sms * 8;
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
    // block partials of up to 2 * max_blocks blocks, then their group partials
    const size_t groups = size_t(2 * c->max_blocks + kReduceGroup - 1) / kReduceGroup;
    CK(cudaMalloc(&c->partials, sizeof(double) * kPartialsPerBlock * (2 * c->max_blocks + groups)));
    CK(cudaMalloc(&c->counter, sizeof(unsigned) * (1 + groups)));
    CK(cudaMemset(c->counter, 0, sizeof(unsigned) * (1 + groups)));
    CK(cudaMalloc(&c->redout, sizeof(double) * kPartialsPerBlock));
    CK(cudaMalloc(&c->state, sizeof(MSState) > sizeof(CGState) * kMaxRhs ? sizeof(MSState) : sizeof(CGState) * kMaxRhs));
    CK(cudaMalloc(&c->done, sizeof(int) * 64));
    CK(cudaMemset(c->done, 0, sizeof(int) * 64));
    CK(cudaMallocHost(&c->h_pinned, 4096 + sizeof(MSState)));
    CK(cudaMalloc(&c->d_maxdev, sizeof(unsigned long long)));
    CK(cudaMalloc(&c->d_singular, sizeof(int)));
    clover_init_tables();
    CK(cudaGetLastError());
  }
  *out = c.release();
  return IRO_OK;
}

int iro_ctx_destroy(iro_ctx* c) {
  if (!c) return IRO_BAD_ARG;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& kv : c->ws) free_field(kv.second);
  void* ptrs[] = {c->raw, c->ga.d12, c->ga.d18, c->ga.s12, c->ga.h12a, c->ga.h12b, c->ga.h18a,
                  c->ga.h18b, c->d_maxdev,
                  c->d_singular, c->stage, c->partials, c->counter, c->redout, c->state, c->done};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int pr = 0; pr < 3; ++pr)
    for (int p = 0; p < 2; ++p) {
      if (c->clA[pr][p]) cudaFree(c->clA[pr][p]);
      if (c->clAinv[pr][p]) cudaFree(c->clAinv[pr][p]);
    }
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  if (c->scratch) cudaFree(c->scratch);
  for (int i = 0; i < 2; ++i) {
    if (c->ring[i]) cudaFreeHost(c->ring[i]);
    if (c->ring_ev[i]) cudaEventDestroy(c->ring_ev[i]);
    if (c->xs[i]) cudaStreamDestroy(c->xs[i]);
  }
  for (cudaEvent_t e : c->xev)
    if (e) cudaEventDestroy(e);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return IRO_OK;
}

const char* iro_last_error(const iro_ctx* c) { return c ? c->err.c_str() : "null context"; }

int iro_autotune_report(const iro_ctx* c, char* buf, int len) {
  if (!c || !buf || len < 3) return IRO_BAD_ARG;
  std::string s = "[";
  for (const auto& kv : c->tuned) {
    const auto& k = kv.first;
    char item[256];
    auto ms = c->tuned_ms.find(k);
    std::snprintf(item, sizeof(item),
                  "%s{\"prec\":%d,\"recon\":%d,\"dag\":%d,\"epilogue\":%d,\"nrhs\":%d,"
                  "\"parities\":%d,\"variant\":%d,\"block\":%d,\"free_grid\":%d,\"ms\":%.5f}",
                  s.size() > 1 ? "," : "", std::get<0>(k), std::get<1>(k), std::get<2>(k),
                  std::get<3>(k), std::get<4>(k), std::get<5>(k), kv.second.variant, kv.second.block,
                  kv.second.free_grid, ms == c->tuned_ms.end() ? -1.0 : double(ms->second));
    s += item;
  }
  s += "]";
  if (int(s.size()) + 1 > len) return IRO_BAD_ARG;
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return IRO_OK;
}

void* iro_ctx_get_stream(const iro_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

int iro_ctx_set_stream(iro_ctx* c, void* stream) {
  if (!c) return IRO_BAD_ARG;
  CK(cudaStreamSynchronize(c->stream));
  if (c->own_stream) cudaStreamDestroy(c->stream);
  c->stream = static_cast<cudaStream_t>(stream);
  c->own_stream = false;
  return IRO_OK;
}

int iro_gauge_upload(iro_ctx* c, const double* u) {
  if (!c || !u) return fail(c, IRO_BAD_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  const size_t raw_bytes = size_t(18) * 4 * c->V * sizeof(double);
  if (!c->raw) {
    CK(cudaMalloc(&c->raw, raw_bytes));
    CK(cudaMalloc(&c->ga.d12, size_t(2) * 4 * 6 * c->Vh * sizeof(double2)));
    CK(cudaMalloc(&c->ga.d18, size_t(2) * 4 * 9 * c->Vh * sizeof(double2)));
    CK(cudaMalloc(&c->ga.s12, size_t(2) * 4 * 3 * c->Vh * sizeof(float4)));
    CK(cudaMalloc(&c->ga.h12a, size_t(2) * 4 * c->Vh * sizeof(uint4)));
    CK(cudaMalloc(&c->ga.h12b, size_t(2) * 4 * c->Vh * sizeof(uint2)));
    CK(cudaMalloc(&c->ga.h18a, size_t(2) * 4 * 2 * c->Vh * sizeof(uint4)));
    CK(cudaMalloc(&c->ga.h18b, size_t(2) * 4 * c->Vh * sizeof(uint32_t)));
  }
  RCK(copy_h2d(c, c->raw, u, raw_bytes));
  CK(cudaMemsetAsync(c->d_maxdev, 0, sizeof(unsigned long long), c->stream));
  CK(launch_import_gauge(c->g, c->raw, c->ga, c->d_maxdev, c->stream));
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, c->d_maxdev, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double dev;
  std::memcpy(&dev, &bits, sizeof(dev));
  c->recon = (dev <= 1e-12) ? 12 : 18;
  c->has_gauge = true;
  c->has_clover = false;
  return IRO_OK;
}

int iro_clover_setup(iro_ctx* c, double mass, double csw) {
  if (!c) return IRO_BAD_ARG;
  CK(cudaSetDevice(c->device));
  return clover_build(c, kappa_of(mass) * csw);
}

int iro_field_strength(iro_ctx* c, int mu, int nu, double* out) {
  if (!c || !out || mu < 0 || mu > 3 || nu < 0 || nu > 3 || mu == nu)
    return fail(c, IRO_BAD_ARG, "bad field-strength arguments");
  if (!c->has_gauge) return fail(c, IRO_NO_GAUGE, "no gauge field uploaded");
  CK(cudaSetDevice(c->device));
  const size_t bytes = size_t(18) * c->V * sizeof(double);
  int rc = ensure_stage(c, bytes);
  if (rc) return rc;
  CK(launch_field_strength(c->g, c->raw, mu, nu, c->stage, c->stream));
  return copy_d2h(c, out, c->stage, bytes);
}

// The even/odd Schur operator between pinned host arrays with the copies
// overlapped.  The even half field moves in chunks of whole t-slices, host to
// device on one copy stream and device to host on another, so that both
// directions of the host link are busy at once, and the stencils of a chunk
// run as soon as the chunks they read have arrived: chunk j of the odd
// intermediate reads input chunks j-1..j+1 (a t hop crosses one slice), and
// chunk j of the output reads intermediate chunks j-1..j+1.  The input goes
// in the order n-1, 0, 1, ..., n-2; output chunk j leaves once its
// neighbourhood is complete, the five around chunk n-2 last.  The stage
// buffer holds both directions: output chunk j overwrites input chunk j
// after the import of j has read it (both on the compute stream).  Every
// site is computed by the kernels of apply_dev, so the result is the same to
// the bit.  Returns with *handled false (and nothing done) when the
// stencils are not tuned yet: the caller takes the plain path, which tunes.
constexpr int kPipeMaxChunks = 64;
constexpr size_t kPipeMinChunkBytes = size_t(8) << 20;

// The chunks' first t-slices b[0..n-1] (b[n] = Lt); returns n.  Chunks of
// `per` slices (at least kPipeMinChunkBytes); when that is more than one
// slice, chunks 0..3 and n-4..n-1 (the first input chunks to arrive and the
// output chunks that wait for the last one) are single slices, which
// shortens the pipeline's fill and drain.
int pipe_plan(const iro_ctx* c, int* b) {
  const int Lt = c->L[3];
  const size_t slice = size_t(c->g.st) * 24 * sizeof(double);
  int per = int((kPipeMinChunkBytes + slice - 1) / slice);
  if (const char* e = std::getenv("IRO_PIPE_SLICES")) per = std::max(1, std::atoi(e));
  int n = 0;
  if (per > 1 && Lt - 8 >= 2 * per) {
    const int mid = Lt - 8, m = std::min(mid / per, kPipeMaxChunks - 8);
    for (int k = 0; k < 4; ++k) b[n++] = k;
    for (int i = 0; i < m; ++i) b[n++] = 4 + i * mid / m;
    for (int k = 0; k < 4; ++k) b[n++] = Lt - 4 + k;
  } else {
    const int m = std::min(std::max(Lt / per, 1), kPipeMaxChunks);
    for (int i = 0; i < m; ++i) b[n++] = i * Lt / m;
  }
  b[n] = Lt;
  return n;
}

int pipe_chunks(const iro_ctx* c) {
  int b[kPipeMaxChunks + 1];
  return pipe_plan(c, b);
}

int schur_host_pipelined(iro_ctx* c, int op, double mass, double csw, bool dag, int prec,
                         const double* in, double* out, bool* handled) {
  *handled = false;
  int b[kPipeMaxChunks + 1];
  const int n = pipe_plan(c, b);
  const bool cl = op == IRO_OP_CLOVER_SCHUR_EE;
  if (cl) RCK(ensure_clover(c, mass, csw));
  int rc = IRO_OK;
  DevField* fi = ws(c, 0, prec, 1, 10, &rc);
  if (!fi) return rc;
  DevField* fo = ws(c, 0, prec, 1, 11, &rc);
  if (!fo) return rc;
  DevField* t = ws(c, 1, prec, 1, 0, &rc);
  if (!t) return rc;
  HopLaunch L1 = base_launch(c, prec, dag, 1), L2;
  schur_launches(c, cl, kappa_of(mass), *fi, *t, *fo, L1, L2);
  if (!c->tuned.count(tune_key(L1)) || !c->tuned.count(tune_key(L2))) return IRO_OK;
  RCK(ensure_stage(c, size_t(c->Vh) * 24 * sizeof(double)));
  for (int i = 0; i < 2; ++i)
    if (!c->xs[i]) CK(cudaStreamCreateWithFlags(&c->xs[i], cudaStreamNonBlocking));
  while (c->xev.size() < size_t(2 * kPipeMaxChunks + 1)) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c->xev.push_back(e);
  }
  *handled = true;
  cudaStream_t cs = c->stream, h2d = c->xs[0], d2h = c->xs[1];
  cudaEvent_t* arrived = c->xev.data();
  cudaEvent_t* exported = arrived + kPipeMaxChunks;
  cudaEvent_t start = arrived[2 * kPipeMaxChunks];
  // chunk j: half-sites [lo(j), lo(j + 1)), whole t-slices (host index = half-site)
  auto lo = [&](int j) { return int64_t(b[j]) * c->g.st; };
  auto run = [&]() -> int {
    CK(cudaEventRecord(start, cs));  // earlier work of the stream may still use the stage
    CK(cudaStreamWaitEvent(h2d, start, 0));
    for (int q = 0; q < n; ++q) {
      const int j = (q + n - 1) % n;
      CK(cudaMemcpyAsync(c->stage + lo(j) * 24, in + lo(j) * 24,
                         size_t(lo(j + 1) - lo(j)) * 24 * sizeof(double), cudaMemcpyHostToDevice, h2d));
      CK(cudaEventRecord(arrived[j], h2d));
    }
    auto import = [&](int j) -> int {
      CK(cudaStreamWaitEvent(cs, arrived[j], 0));
      CK(launch_import_spinor(c->g, c->stage, 1, 0, c->Vh, 1, prec, fi->half(0), cs, lo(j),
                              lo(j + 1) - lo(j)));
      return IRO_OK;
    };
    auto hop1 = [&](int j) -> int {
      L1.hs0 = int(lo(j));
      L1.nhs = int(lo(j + 1) - lo(j));
      return launch_tuned(c, L1);
    };
    auto hop2 = [&](int j) -> int {
      L2.hs0 = int(lo(j));
      L2.nhs = int(lo(j + 1) - lo(j));
      RCK(launch_tuned(c, L2));
      CK(launch_export_spinor(c->g, c->stage, 1, 0, c->Vh, 1, prec, fo->half(0), cs, lo(j),
                              lo(j + 1) - lo(j)));
      CK(cudaEventRecord(exported[j], cs));
      CK(cudaStreamWaitEvent(d2h, exported[j], 0));
      CK(cudaMemcpyAsync(out + lo(j) * 24, c->stage + lo(j) * 24,
                         size_t(lo(j + 1) - lo(j)) * 24 * sizeof(double), cudaMemcpyDeviceToHost, d2h));
      return IRO_OK;
    };
    RCK(import(n - 1));
    RCK(import(0));
    RCK(import(1));
    RCK(hop1(0));
    for (int k = 2; k <= n - 2; ++k) {
      RCK(import(k));
      RCK(hop1(k - 1));
      if (k >= 3) RCK(hop2(k - 2));
    }
    RCK(hop1(n - 2));
    RCK(hop1(n - 1));
    for (int j : {n - 3, n - 2, n - 1, 0}) RCK(hop2(j));
    return IRO_OK;
  };
  rc = run();
  // the copies read and write the caller's arrays: wait for them on every path
  const cudaError_t e1 = cudaStreamSynchronize(h2d);
  const cudaError_t e2 = cudaStreamSynchronize(d2h);
  const cudaError_t e3 = cudaStreamSynchronize(cs);
  if (rc) return rc;
  CK(e1);
  CK(e2);
  CK(e3);
  return IRO_OK;
}

// The full-lattice operators between pinned host arrays, overlapped like the
// Schur operator above (same chunks of t-slices, streams and events): the
// host array is lexicographic, so a chunk of t-slices is one contiguous host
// range and one half-site range in each parity.  Output chunk j reads input
// chunks j-1..j+1, so it is computed and sent back as soon as input chunk j+1
// has arrived.  The same single launch over both parities as apply_dev, on
// the chunk's half-sites: the result is the same to the bit.
int full_host_pipelined(iro_ctx* c, int op, double mass, double csw, bool dag, int prec,
                        const double* in, double* out, bool* handled) {
  *handled = false;
  int b[kPipeMaxChunks + 1];
  const int n = pipe_plan(c, b);
  const bool cl = op == IRO_OP_CLOVER_FULL;
  if (cl) RCK(ensure_clover(c, mass, csw));
  int rc = IRO_OK;
  DevField* fi = ws(c, 2, prec, 1, 10, &rc);
  if (!fi) return rc;
  DevField* fo = ws(c, 2, prec, 1, 11, &rc);
  if (!fo) return rc;
  HopLaunch L = base_launch(c, prec, dag, 1);
  full_launch(c, cl, kappa_of(mass), *fi, *fo, L);
  if (!c->tuned.count(tune_key(L))) return IRO_OK;
  RCK(ensure_stage(c, size_t(c->V) * 24 * sizeof(double)));
  for (int i = 0; i < 2; ++i)
    if (!c->xs[i]) CK(cudaStreamCreateWithFlags(&c->xs[i], cudaStreamNonBlocking));
  while (c->xev.size() < size_t(2 * kPipeMaxChunks + 1)) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c->xev.push_back(e);
  }
  *handled = true;
  cudaStream_t cs = c->stream, h2d = c->xs[0], d2h = c->xs[1];
  cudaEvent_t* arrived = c->xev.data();
  cudaEvent_t* exported = arrived + kPipeMaxChunks;
  cudaEvent_t start = arrived[2 * kPipeMaxChunks];
  // chunk j: half-sites [lo(j), lo(j + 1)) of each parity; host sites
  // [2 lo(j), 2 lo(j + 1)) (a t-slice holds 2 st lexicographic sites)
  auto lo = [&](int j) { return int64_t(b[j]) * c->g.st; };
  auto bytes = [&](int j) { return size_t(lo(j + 1) - lo(j)) * 2 * 24 * sizeof(double); };
  auto run = [&]() -> int {
    CK(cudaEventRecord(start, cs));
    CK(cudaStreamWaitEvent(h2d, start, 0));
    for (int q = 0; q < n; ++q) {
      const int j = (q + n - 1) % n;
      CK(cudaMemcpyAsync(c->stage + 2 * lo(j) * 24, in + 2 * lo(j) * 24, bytes(j),
                         cudaMemcpyHostToDevice, h2d));
      CK(cudaEventRecord(arrived[j], h2d));
    }
    auto import = [&](int j) -> int {
      CK(cudaStreamWaitEvent(cs, arrived[j], 0));
      for (int p = 0; p < 2; ++p)
        CK(launch_import_spinor(c->g, c->stage, 0, p, c->V, 1, prec, fi->half(p), cs, lo(j),
                                lo(j + 1) - lo(j)));
      return IRO_OK;
    };
    auto apply_chunk = [&](int j) -> int {
      L.hs0 = int(lo(j));
      L.nhs = int(lo(j + 1) - lo(j));
      RCK(launch_tuned(c, L));
      for (int p = 0; p < 2; ++p)
        CK(launch_export_spinor(c->g, c->stage, 0, p, c->V, 1, prec, fo->half(p), cs, lo(j),
                                lo(j + 1) - lo(j)));
      CK(cudaEventRecord(exported[j], cs));
      CK(cudaStreamWaitEvent(d2h, exported[j], 0));
      CK(cudaMemcpyAsync(out + 2 * lo(j) * 24, c->stage + 2 * lo(j) * 24, bytes(j),
                         cudaMemcpyDeviceToHost, d2h));
      return IRO_OK;
    };
    RCK(import(n - 1));
    RCK(import(0));
    RCK(import(1));
    RCK(apply_chunk(0));
    for (int k = 2; k <= n - 2; ++k) {
      RCK(import(k));
      RCK(apply_chunk(k - 1));
    }
    RCK(apply_chunk(n - 2));
    RCK(apply_chunk(n - 1));
    return IRO_OK;
  };
  rc = run();
  const cudaError_t e1 = cudaStreamSynchronize(h2d);
  const cudaError_t e2 = cudaStreamSynchronize(d2h);
  const cudaError_t e3 = cudaStreamSynchronize(cs);
  if (rc) return rc;
  CK(e1);
  CK(e2);
  CK(e3);
  return IRO_OK;
}

int iro_dirac_apply(iro_ctx* c, int op, double mass, double csw, int dagger, int prec,
                    const double* in, double* out, int nrhs) {
  if (!c || !in || !out || nrhs < 1 || nrhs > kMaxRhs || prec < 0 || prec > 2 || !op_valid(op))
    return fail(c, IRO_BAD_ARG, "bad operator arguments");
  CK(cudaSetDevice(c->device));
  int rc = IRO_OK;
  const bool schur = op == IRO_OP_WILSON_SCHUR_EE || op == IRO_OP_CLOVER_SCHUR_EE;
  const bool full = op == IRO_OP_WILSON_FULL || op == IRO_OP_CLOVER_FULL;
  const int64_t len = (full ? c->V : c->Vh) * 24;
  if (nrhs == 1 && (schur || full) && c->has_gauge && (prec == PREC_DOUBLE || c->recon == 12) &&
      pipe_chunks(c) >= 6 && (out + len <= in || in + len <= out) && host_pinned(in) &&
      host_pinned(out)) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(c->stream, &cs));
    if (cs == cudaStreamCaptureStatusNone) {
      bool handled = false;
      rc = schur ? schur_host_pipelined(c, op, mass, csw, dagger != 0, prec, in, out, &handled)
                 : full_host_pipelined(c, op, mass, csw, dagger != 0, prec, in, out, &handled);
      if (rc || handled) return rc;
    }
  }
  const int si = input_subset(op), so = output_subset(op);
  DevField* fi = ws(c, si, prec, nrhs, 10, &rc);
  if (!fi) return rc;
  DevField* fo = ws(c, so, prec, nrhs, 11, &rc);
  if (!fo) return rc;
  rc = import_host(c, in, is_full(op), *fi);
  if (rc) return rc;
  rc = apply_dev(c, op, mass, csw, dagger != 0, *fi, *fo, nullptr, 0, nullptr);
  if (rc) return rc;
  return export_host(c, *fo, is_full(op), out);
}

int iro_gamma5(iro_ctx* c, const double* in, double* out, int64_t nsites) {
  if (!c || !in || !out || nsites < 0) return fail(c, IRO_BAD_ARG, "bad gamma5 arguments");
  CK(cudaSetDevice(c->device));
  const size_t bytes = size_t(nsites) * 24 * sizeof(double);
  int rc = ensure_stage(c, bytes);
  if (rc) return rc;
  RCK(copy_h2d(c, c->stage, in, bytes));
  CK(launch_gamma5_aos(c->stage, nsites, c->stream));
  return copy_d2h(c, out, c->stage, bytes);
}

int iro_field_create(iro_ctx* c, int subset, int prec, int nrhs, iro_field** f) {
  if (!c || !f || subset < 0 || subset > 2 || prec < 0 || prec > 2 || nrhs < 1 || nrhs > kMaxRhs)
    return fail(c, IRO_BAD_ARG, "bad field arguments");
  CK(cudaSetDevice(c->device));
  std::unique_ptr<iro_field> h(new iro_field());
  h->ctx = c;
  h->dev = c->device;
  int rc = alloc_field(c, subset, prec, nrhs, h->f);
  if (rc) return rc;
  CK(cudaMemset(h->f.data, 0, h->f.bytes_data));
  if (h->f.norm) CK(cudaMemset(h->f.norm, 0, h->f.bytes_norm));
  *f = h.release();
  return IRO_OK;
}

int iro_field_destroy(iro_field* f) {
  if (!f) return IRO_BAD_ARG;
  cudaSetDevice(f->dev);  // the context may already be destroyed
  free_field(f->f);
  delete f;
  return IRO_OK;
}

int iro_field_upload(iro_ctx* c, iro_field* f, const double* host) {
  if (!c || !f || !host) return fail(c, IRO_BAD_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  return import_host(c, host, f->f.subset == 2, f->f);
}

int iro_field_download(iro_ctx* c, const iro_field* f, double* host) {
  if (!c || !f || !host) return fail(c, IRO_BAD_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  return export_host(c, f->f, f->f.subset == 2, host);
}

int iro_dirac_apply_field(iro_ctx* c, int op, double mass, double csw, int dagger,
                          const iro_field* in, iro_field* out) {
  if (!c || !in || !out) return fail(c, IRO_BAD_ARG, "null argument");
  return apply_dev(c, op, mass, csw, dagger != 0, in->f, out->f, nullptr, 0, nullptr);
}

int iro_field_norm(iro_ctx* c, const iro_field* f, double* out) {
  if (!c || !f || !out) return fail(c, IRO_BAD_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  std::vector<double> n2;
  int rc = norms_host(c, f->f, nullptr, n2, nullptr);
  if (rc) return rc;
  for (int r = 0; r < f->f.nrhs; ++r) out[r] = std::sqrt(n2[r]);
  return IRO_OK;
}

int iro_field_dot(iro_ctx* c, const iro_field* a, const iro_field* b, double* out) {
  if (!c || !a || !b || !out) return fail(c, IRO_BAD_ARG, "null argument");
  if (a->f.subset != b->f.subset || a->f.prec != b->f.prec || a->f.nrhs != b->f.nrhs)
    return fail(c, IRO_BAD_ARG, "dot: fields differ in subset, precision or nrhs");
  CK(cudaSetDevice(c->device));
  Reduce r = make_reduce(c, ST_NONE, 0);
  CK(launch_dot(a->f.prec, a->f.sites(), a->f.nrhs, a->f.all(), b->f.all(), r, c->max_blocks,
                c->stream));
  CK(cudaMemcpyAsync(out, c->redout, sizeof(double) * a->f.nrhs, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return IRO_OK;
}

// ---- CG ------------------------------------------------------------------------------
int iro_cg_solve(iro_ctx* c, int op, double mass, double csw, const iro_cg_params* prm,
                 const double* b, double* x, int nrhs, iro_solver_out* out);

int iro_multishift_cg_solve(iro_ctx* c, int op, double mass, double csw, const double* b,
                            int nshift, const double* shifts, double* x, double precision,
                            int max_iter, iro_solver_out* out, int* nconv);

}  // extern "C"

// The solvers live in solvers.cu; these helpers are shared with it.
namespace iro {
namespace host {
int apply(iro_ctx* c, int op, double mass, double csw, bool dag, const DevField& in, DevField& out,
          const Reduce* red, int red_mask, const int* skip) {
  return apply_dev(c, op, mass, csw, dag, in, out, red, red_mask, skip);
}
int apply_cg(iro_ctx* c, int op, double mass, double csw, bool dag, const DevField& in,
             DevField& out, const Reduce& red, const int* skip, const CGFuse& fuse) {
  return apply_dev(c, op, mass, csw, dag, in, out, &red, 0, skip, &fuse);
}
DevField* workspace(iro_ctx* c, int subset, int prec, int nrhs, int slot, int* rc) {
  return ws(c, subset, prec, nrhs, slot, rc);
}
bool workspace_exists(iro_ctx* c, int subset, int prec, int nrhs, int slot) {
  return c->ws.count(std::make_tuple(subset, prec, nrhs, slot)) != 0;
}
int import_field(iro_ctx* c, const double* host, bool full, DevField& f) {
  return import_host(c, host, full ? 1 : 0, f);
}
int host_to_device(iro_ctx* c, void* dev, const void* host, size_t bytes) { return copy_h2d(c, dev, host, bytes); }
int device_to_host(iro_ctx* c, void* host, const void* dev, size_t bytes) { return copy_d2h(c, host, dev, bytes); }
int export_field(iro_ctx* c, const DevField& f, bool full, double* host) {
  return export_host(c, f, full ? 1 : 0, host);
}
int norms(iro_ctx* c, const DevField& v, const DevField* w, std::vector<double>& nv,
          std::vector<double>* nw) {
  return norms_host(c, v, w, nv, nw);
}
int axpby(iro_ctx* c, double a, const DevField& x, double b, const DevField& y, DevField& v) {
  return axpby_dev(c, a, x, b, y, v);
}
int convert(iro_ctx* c, const DevField& in, DevField& out) { return convert_dev(c, in, out); }
Reduce reduce(iro_ctx* c, int stage, int max_iter) { return make_reduce(c, stage, max_iter); }
int set_error(iro_ctx* c, int code, const std::string& msg) { return fail(c, code, msg); }
int cuda_error(iro_ctx* c, cudaError_t e, const char* where) { return cuda_fail(c, e, where); }
cudaStream_t stream(iro_ctx* c) { return c->stream; }
int max_blocks(iro_ctx* c) { return c->max_blocks; }
int64_t vh(iro_ctx* c) { return c->Vh; }
void* state(iro_ctx* c) { return c->state; }
int* done(iro_ctx* c) { return c->done; }
void* pinned(iro_ctx* c) { return c->h_pinned; }
void* scratch(iro_ctx* c, size_t bytes, int* rc) {
  if (c->scratch_bytes < bytes) {
    if (c->scratch) {
      // the previous scratch may still be read by enqueued work
      cudaError_t e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) { *rc = cuda_fail(c, e, "cudaStreamSynchronize"); return nullptr; }
      cudaFree(c->scratch);
      c->scratch = nullptr;
      c->scratch_bytes = 0;
    }
    cudaError_t e = cudaMalloc(&c->scratch, bytes);
    if (e != cudaSuccess) {
      c->scratch = nullptr;
      *rc = cuda_fail(c, e, "cudaMalloc (solver scratch)");
      return nullptr;
    }
    c->scratch_bytes = bytes;
  }
  return c->scratch;
}
int device(iro_ctx* c) { return c->device; }
DevField* field_dev(iro_field* f) { return f ? &f->f : nullptr; }
const Geom& geom(iro_ctx* c) { return c->g; }
GaugePtr gauge_single(iro_ctx* c) { return gauge_ptr(c, PREC_SINGLE); }
bool gauge_su3(iro_ctx* c) { return c->has_gauge && c->recon == 12; }
int64_t volume(iro_ctx* c) { return c->V; }
bool op_is_full(int op) { return is_full(op); }
int op_subset(int op) { return input_subset(op); }
bool op_ok(int op) { return op_valid(op); }
int clover_ready(iro_ctx* c, double mass, double csw) { return ensure_clover(c, mass, csw); }
GaugePtr gauge_double(iro_ctx* c) { return gauge_ptr(c, PREC_DOUBLE); }
int gauge_recon(iro_ctx* c) { return c->recon; }
const double* gauge_format_g(iro_ctx* c) { return c->raw; }
bool gauge_loaded(iro_ctx* c) { return c->has_gauge; }
CloverPtr clover(iro_ctx* c, int prec, int p, bool inverse) { return clover_ptr(c, prec, p, inverse); }
}  // namespace host
}  // namespace iro
