// Gauge-equivariant learned preconditioner: parallel-transport convolution
// (PTC) layers and their gradients.
//
// A layer maps C_in colour-vector channels to C_out channels on every site of
// the full lattice:
//     out_o(x) = sum_{d=0..8} sum_i W_d[o][i] (T_d in_i)(x)
// with T_0 the identity and, for d = 1 + 2*mu + s,
//     T_{+mu} f(x) = U_mu(x) f(x+mu),   T_{-mu} f(x) = U_mu(x-mu)^dag f(x-mu),
// so the layer commutes with gauge transformations (the weights act on the
// channel index only, the links on colour).  A Wilson spinor is 4 channels
// (its spins).  The reference has no learned part; this follows the
// parallel-transport convolutions of Lehner & Wettig, "Gauge-equivariant
// neural networks as preconditioners in lattice QCD", PRD 108 (2023).
//
// Forward kernel, one CTA per tile of 42 sites = 126 rows (site, colour):
//  1. the CUDA cores transport every input channel along the 9 displacements
//     and write the real GEMM operand A[row][k], k = (2d + re/im)*C_in + i,
//     in BF16 into shared memory in the canonical K-major no-swizzle UMMA
//     layout (8x16-byte core matrices);
//  2. one thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32, M=128)
//     against the packed real weight matrix B[n][k] (n = 2*o + re/im), the
//     accumulator lives in tensor memory;
//  3. the four warps read their 32 accumulator lanes back (tcgen05.ld) and
//     store the output channels in FP32.
// Every wait on the MMA's mbarrier is bounded: on time-out the kernel sets
// an error flag, skips the read-back, frees its tensor memory and returns.
//
// Backward: dA = dY B (tcgen05, same machinery), then the adjoint transport
// (a gather) gives d in; dB = A^T dY per tile on the CUDA cores with a
// deterministic reduction over tiles.
#include <cuda_bf16.h>

#include <cstring>
#include <vector>

#include "dslash_pair.cuh"
#include "internal.h"
#include "iroiro_b200.h"

namespace iro {

// ---- tcgen05 / mbarrier primitives ------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// A wait on an mbarrier gives up after kWaitNs nanoseconds of global time
// (or kWaitLimit polls, whichever comes first): the kernel then sets its
// error flag and leaves, and the host reports IRO_TIMEOUT.
constexpr int kWaitLimit = 1 << 24;
constexpr uint64_t kWaitNs = 1000000000ull;

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Polls the barrier until `phase` completes; false after limit_ns of global
// time or kWaitLimit polls
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase,
                                                  uint64_t limit_ns = kWaitNs) {
  const uint64_t t0 = global_ns();
  for (int it = 0; it < kWaitLimit; ++it) {
    if (mbar_try_wait(bar, phase)) return true;
    if ((it & 63) == 63 && global_ns() - t0 > limit_ns) return false;
  }
  return false;
}
// D(tmem) (+)= A(smem) * B(smem)^T, BF16 inputs, FP32 accumulation
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n.reg .pred p;\n"
      "setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}
// 16 consecutive FP32 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// Shared-memory matrix descriptor, K-major, no swizzle: 8-row x 16-byte core
// matrices, LBO = byte step between the two K-halves of an MMA's K=16, SBO =
// byte step between 8-row groups; version 1 (sm100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}
// Instruction descriptor: FP32 accumulate, BF16 A and B, both K-major, M=128, N.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(128 >> 4) << 24);
}
// byte offset of element (r, k) of a K-major R x K BF16 operand in the canonical layout
__host__ __device__ __forceinline__ uint32_t canon(int r, int k, int K) {
  return uint32_t((r >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

constexpr int kTileSites = 42;  // 126 of the 128 MMA rows
constexpr int kThreads = 128;

template <int CIN, int COUT>
struct Ptc {
  static constexpr int KF = 18 * CIN;
  static constexpr int KP = (KF + 15) / 16 * 16;
  static constexpr int NF = 2 * COUT;
  static constexpr int NP = NF < 16 ? 16 : (NF + 15) / 16 * 16;
  static constexpr int TCOLS = NP <= 32 ? 32 : 64;
  static constexpr int A_BYTES = 128 * KP * 2;
  static constexpr int B_BYTES = NP * KP * 2;
  // forward kernel: A holds the 96 rows of 32 sites; the MMA's rows 96..127
  // read the bytes that follow (the weights, padded to at least 32 rows),
  // which only feed accumulator rows that are never read back
  static constexpr int A96_BYTES = 96 * KP * 2;
  static constexpr int BF_BYTES = NP >= 32 ? B_BYTES : 32 * KP * 2;
};

// Feature element (site s, channel o, colour a) of a V-site field.  Channels
// are stored in pairs, structure-of-arrays over sites in 16-byte units: pair
// q = o/2 and colour a occupy the float4 row (3q + a)*V + s holding
// (re o=2q, re o=2q+1, im o=2q, im o=2q+1).  A warp reading one row for 32
// consecutive (or uniformly shifted) sites is coalesced, and a row is
// directly the packed FP32x2 operand pair of the two channels.
__host__ __device__ __forceinline__ size_t fidx(int s, int o, int a, int V) {
  return (size_t((o >> 1) * 3 + a) * V + s) * 4 + (o & 1);
}
__device__ __forceinline__ float2 feat_get(const float2* f, int s, int o, int a, int V) {
  const float* p = reinterpret_cast<const float*>(f) + fidx(s, o, a, V);
  return make_float2(p[0], p[2]);
}
__device__ __forceinline__ void feat_set(float2* f, int s, int o, int a, int V, float2 v) {
  float* p = reinterpret_cast<float*>(f) + fidx(s, o, a, V);
  p[0] = v.x;
  p[2] = v.y;
}

struct PtcGeo {
  Geom g;
  GaugePtr gauge;  // FP32 two-row links
  int V;
  int* err;
  const int* skip;  // forward only: when set and nonzero the launch does nothing
};

// Builds the BF16 A tile: rows (site, colour) of the tile, columns
// (2d + part)*CIN + i; padding rows/columns are zero.
template <int CIN, int KP>
__device__ void build_a_tile(const PtcGeo& G, const float2* __restrict__ in, int site0,
                             unsigned char* A) {
  // zero the tile (padding rows and columns must not hold stale values)
  for (int b = threadIdx.x * 16; b < 128 * KP * 2; b += kThreads * 16)
    *reinterpret_cast<uint4*>(A + b) = make_uint4(0, 0, 0, 0);
  __syncthreads();
  const int Vh = G.g.Vh;
  for (int j = threadIdx.x; j < kTileSites * 9; j += kThreads) {
    const int sl = j / 9, d = j - sl * 9;
    const int s = site0 + sl;
    if (s >= G.V) continue;
    const int p = s >= Vh ? 1 : 0;
    const int hs = s - p * Vh;
    int src = s;
    Su3<float> U;
    bool fwd = true;
    if (d > 0) {
      const Coord c = coord_of(G.g, hs, p);
      int nb[8];
      neighbours(G.g, c, hs, nb);
      const int mu = (d - 1) >> 1;
      fwd = ((d - 1) & 1) == 0;
      const int n = nb[d - 1];
      src = (1 - p) * Vh + n;
      if (fwd)
        GaugeIO<PREC_SINGLE, 12>::load(G.gauge, p, mu, hs, U);
      else
        GaugeIO<PREC_SINGLE, 12>::load(G.gauge, 1 - p, mu, n, U);
    }
#pragma unroll 4
    for (int i = 0; i < CIN; ++i) {
      Cx<float> v[3], w[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float2 t = feat_get(in, src, i, a, G.V);
        v[a] = {t.x, t.y};
      }
      if (d == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) w[a] = v[a];
      } else if (fwd) {
#pragma unroll
        for (int a = 0; a < 3; ++a) w[a] = U.e[a][0] * v[0] + U.e[a][1] * v[1] + U.e[a][2] * v[2];
      } else {
#pragma unroll
        for (int a = 0; a < 3; ++a)
          w[a] = cj_mul(U.e[0][a], v[0]) + cj_mul(U.e[1][a], v[1]) + cj_mul(U.e[2][a], v[2]);
      }
      const int kre = (2 * d) * CIN + i, kim = (2 * d + 1) * CIN + i;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int r = sl * 3 + a;
        *reinterpret_cast<__nv_bfloat16*>(A + canon(r, kre, KP)) = __float2bfloat16_rn(w[a].re);
        *reinterpret_cast<__nv_bfloat16*>(A + canon(r, kim, KP)) = __float2bfloat16_rn(w[a].im);
      }
    }
  }
}

// Loads an N x K row-major BF16 matrix into the canonical K-major layout.
template <int N, int K>
__device__ void load_b(const __nv_bfloat16* __restrict__ B, unsigned char* Bs) {
  for (int idx = threadIdx.x; idx < N * K; idx += kThreads) {
    const int n = idx / K, k = idx - n * K;
    *reinterpret_cast<__nv_bfloat16*>(Bs + canon(n, k, K)) = B[idx];
  }
}

// Issues the K/16 MMAs of D = A B^T into TMEM, commits to the mbarrier and
// waits (bounded).  Only warp 0 polls the barrier (the other warps wait at
// the block barrier without taking issue slots); the block barrier then
// orders everyone's tcgen05 accesses after the completed MMAs.  Returns false
// on time-out, in every thread.
template <int K>
__device__ bool mma_and_wait(const unsigned char* A, const unsigned char* B, uint32_t tmem,
                             uint32_t idesc, uint64_t* bar, uint32_t phase, int* err) {
  __shared__ int mma_ok;
  fence_async_smem();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32) {
    if (threadIdx.x == 0) {
      const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
      constexpr uint32_t sbo = (K / 8) * 128;
#pragma unroll 1
      for (int kb = 0; kb < K / 16; ++kb)
        umma_bf16(tmem, smem_desc(a0 + kb * 256, 128, sbo), smem_desc(b0 + kb * 256, 128, sbo),
                  idesc, kb > 0 ? 1u : 0u);
      umma_commit(bar);
    }
    __syncwarp();
    const bool ok = mbar_wait_bounded(bar, phase);
    if (threadIdx.x == 0) {
      mma_ok = ok ? 1 : 0;
      if (!ok && err) atomicExch(err, 1);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  return mma_ok != 0;
}

// ---- forward ----------------------------------------------------------------------
// Writes the A-tile entries of one (site, displacement) job: the CIN
// transported channel vectors of the tile's site sl, as BF16 in columns
// (2d + re/im)*CIN + i of rows 3*sl + colour.  Channels are handled in pairs
// in the packed FP32x2 arithmetic (su3_row); each colour row receives CIN/8
// 16-byte stores (8-byte stores for CIN = 4).
template <int CIN, int KP>
__device__ __forceinline__ void a_tile_job(const PtcGeo& G, const float2* __restrict__ in, int s,
                                           int sl, int d, unsigned char* A) {
  constexpr int NW = CIN / 2;  // BF16x2 words per colour and part
  uint32_t wre[3][NW], wim[3][NW];
  if (s < G.V) {
    const int Vh = G.g.Vh;
    const int p = s >= Vh ? 1 : 0;
    const int hs = s - p * Vh;
    int src = s;
    Su3<float> U;
    bool fwd = true;
    int mu = 0, n = hs;
    if (d > 0) {
      const Coord c = coord_of(G.g, hs, p);
      int nb[8];
      neighbours(G.g, c, hs, nb);
      mu = (d - 1) >> 1;
      fwd = ((d - 1) & 1) == 0;
      n = nb[d - 1];
      src = (1 - p) * Vh + n;
    }
    // channels 2q, 2q+1 of the source site, one float4 row per colour (see fidx)
    const float4* f4 = reinterpret_cast<const float4*>(in) + src;
    const size_t V = size_t(G.V);
    // all of the job's feature rows requested at once (into L1), so that the
    // loads below, which the register budget spreads over the channel
    // pairs, find them there instead of each pair waiting on memory
#pragma unroll
    for (int q = 0; q < 3 * NW; ++q) asm volatile("prefetch.global.L1 [%0];" ::"l"(f4 + q * V));
    if (d > 0) {
      if (fwd)
        GaugeIO<PREC_SINGLE, 12>::load(G.gauge, p, mu, hs, U);
      else
        GaugeIO<PREC_SINGLE, 12>::load(G.gauge, 1 - p, mu, n, U);
    }
#pragma unroll
    for (int q = 0; q < NW; ++q) {
      const float4 a = __ldg(f4 + (3 * q) * V), b = __ldg(f4 + (3 * q + 1) * V),
                   e = __ldg(f4 + (3 * q + 2) * V);
      const Cp h0 = {make_float2(a.x, a.y), make_float2(a.z, a.w)};
      const Cp h1 = {make_float2(b.x, b.y), make_float2(b.z, b.w)};
      const Cp h2 = {make_float2(e.x, e.y), make_float2(e.z, e.w)};
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        Cp w;
        if (d == 0)
          w = r == 0 ? h0 : (r == 1 ? h1 : h2);
        else if (fwd)
          w = su3_row<false>(U, r, h0, h1, h2);
        else
          w = su3_row<true>(U, r, h0, h1, h2);
        const __nv_bfloat162 br = __floats2bfloat162_rn(w.re.x, w.re.y);
        const __nv_bfloat162 bi = __floats2bfloat162_rn(w.im.x, w.im.y);
        wre[r][q] = *reinterpret_cast<const uint32_t*>(&br);
        wim[r][q] = *reinterpret_cast<const uint32_t*>(&bi);
      }
    }
  } else {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < NW; ++q) wre[r][q] = wim[r][q] = 0u;
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const int row = 3 * sl + r;
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      const uint32_t* w = part ? wim[r] : wre[r];
      const int k0 = (2 * d + part) * CIN;
      if constexpr (CIN == 4) {
        *reinterpret_cast<uint2*>(A + canon(row, k0, KP)) = make_uint2(w[0], w[1]);
      } else {
#pragma unroll
        for (int q = 0; q < NW; q += 4)
          *reinterpret_cast<uint4*>(A + canon(row, k0 + 2 * q, KP)) =
              make_uint4(w[q], w[q + 1], w[q + 2], w[q + 3]);
      }
    }
  }
}

// Persistent forward kernel: each CTA allocates its tensor memory, loads the
// weights and zeroes its A tile once, then loops over tiles of 32 sites
// (96 of the 128 MMA rows).  The 9 warps build the A tile, warp d handling
// displacement d for the 32 sites (lane = site): branches on the displacement
// are warp-uniform, a warp's gathers are the neighbours of 32 consecutive
// sites, and its 16-byte stores into the canonical layout hit 8 different
// bank groups per 128 bytes.  One thread issues the MMAs; warps 0-2 read the
// accumulator back.  The mbarrier phase alternates per tile; every wait is
// bounded and a time-out stops the CTA with the error flag set.
constexpr int kFwdSites = 32;

// First site of forward tile `tile`: even and odd tiles alternate (tile 2k is
// even-parity half-sites [32k, 32k + 32), tile 2k + 1 the same odd ones), so
// that a feature or link read as a neighbour by one parity's tiles is read
// again as the centre of the other parity's tiles shortly after, from L2.
// Tiling the even sites before the odd ones read each of them from DRAM twice
// (8->8 layer at 24^3x48: 512 MB of DRAM reads per launch, 261 MB now, the
// input features and links once).
// (The volume is a multiple of 64, so each parity is a whole number of tiles.)
__device__ __forceinline__ int fwd_tile_site0(const PtcGeo& G, int tile) {
  return (tile & 1) * G.g.Vh + (tile >> 1) * kFwdSites;
}
constexpr int kFwdThreads = 288;

template <int CIN, int COUT>
__global__ void __launch_bounds__(kFwdThreads) ptc_fwd_kernel(PtcGeo G, const float2* __restrict__ in,
                                                              float2* __restrict__ out,
                                                              const __nv_bfloat16* __restrict__ bop,
                                                              int ntiles) {
  if (G.skip && *G.skip) return;  // the same value in every thread, before any allocation
  using S = Ptc<CIN, COUT>;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* A = smem;
  unsigned char* B = smem + S::A96_BYTES;
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) tmem_alloc(&tslot, S::TCOLS);
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  // zero the weights' padding rows (read only as A rows 96..127), then the
  // weights: NP x KP row-major BF16, copied in 16-byte pieces into the canonical layout
  for (int b = S::B_BYTES + threadIdx.x * 16; b < S::BF_BYTES; b += kFwdThreads * 16)
    *reinterpret_cast<uint4*>(B + b) = make_uint4(0, 0, 0, 0);
  for (int idx = threadIdx.x; idx < S::NP * (S::KP / 8); idx += kFwdThreads) {
    const int n = idx / (S::KP / 8), k0 = (idx - n * (S::KP / 8)) * 8;
    *reinterpret_cast<uint4*>(B + canon(n, k0, S::KP)) =
        __ldg(reinterpret_cast<const uint4*>(bop + size_t(n) * S::KP + k0));
  }
  // columns KF..KP are never written by a job
  for (int b = threadIdx.x * 16; b < S::A96_BYTES; b += kFwdThreads * 16)
    *reinterpret_cast<uint4*>(A + b) = make_uint4(0, 0, 0, 0);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tslot;
  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int site0 = fwd_tile_site0(G, tile);
    a_tile_job<CIN, S::KP>(G, in, site0 + lane, lane, warp, A);
    const bool ok = mma_and_wait<S::KP>(A, B, tmem, idesc_bf16(S::NP), &bar, phase, G.err);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) break;  // all threads leave together on a time-out
    if (warp < 3) {
      const int r = warp * 32 + lane;
      float v[S::NP];
#pragma unroll
      for (int c = 0; c < S::NP; c += 16) tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + c, v + c);
      const int sl = r / 3, a = r - sl * 3;
      const int s = site0 + sl;
      if (s < G.V) {
        // channel pair (2q, 2q+1) of colour a: one 16-byte store
        float4* o4 = reinterpret_cast<float4*>(out) + size_t(a) * G.V + s;
#pragma unroll
        for (int q = 0; q < COUT / 2; ++q)
          o4[size_t(3 * q) * G.V] = make_float4(v[4 * q], v[4 * q + 2], v[4 * q + 1], v[4 * q + 3]);
      }
    }
    // the accumulator is read and the MMA has consumed A before the next tile
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, S::TCOLS);
}

// Double-buffered forward kernel (two A tiles, two accumulators): the A tile
// of tile t+1 is built while the MMAs of tile t run; then the MMAs of tile t+1
// are issued and tile t is read back while they run.  A CTA's tile
// otherwise spends about a third of its time waiting for its MMAs (measured
// with clock64 at 32^3x64: 3.5k of 9.5k cycles for an 8->8 layer).  The
// shared memory holds [A1 | A0 | weights]: the MMA's rows 96..127 of A1 read
// the first rows of A0, those of A0 the weights (padded to >= 32 rows); those
// rows feed accumulator rows that are never read back.
template <int CIN, int COUT>
// (register budget: 4 CTAs per SM for 4 input channels, 3 for 8 -- what the
// shared memory allows -- instead of the 2 that 84 registers left for 8;
// 2.7 % less time per (4,8,8,4) application at 32^3x64)
__global__ void __launch_bounds__(kFwdThreads, (CIN <= 4 ? 4 : (CIN <= 8 ? 3 : 1))) ptc_fwd2_kernel(PtcGeo G, const float2* __restrict__ in,
                                                               float2* __restrict__ out,
                                                               const __nv_bfloat16* __restrict__ bop,
                                                               int ntiles) {
  if (G.skip && *G.skip) return;  // the same value in every thread, before any allocation
  using S = Ptc<CIN, COUT>;
  extern __shared__ __align__(1024) unsigned char smem[];
  // A tile of buffer b: A0 = smem + A96, A1 = smem
  auto abuf = [&](int b) { return smem + (b ? 0 : S::A96_BYTES); };
  unsigned char* B = smem + 2 * S::A96_BYTES;
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tslot;
  __shared__ int mma_ok;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) tmem_alloc(&tslot, 2 * S::TCOLS);
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
  }
  for (int b = S::B_BYTES + threadIdx.x * 16; b < S::BF_BYTES; b += kFwdThreads * 16)
    *reinterpret_cast<uint4*>(B + b) = make_uint4(0, 0, 0, 0);
  for (int idx = threadIdx.x; idx < S::NP * (S::KP / 8); idx += kFwdThreads) {
    const int n = idx / (S::KP / 8), k0 = (idx - n * (S::KP / 8)) * 8;
    *reinterpret_cast<uint4*>(B + canon(n, k0, S::KP)) =
        __ldg(reinterpret_cast<const uint4*>(bop + size_t(n) * S::KP + k0));
  }
  // columns KF..KP of both tiles are never written by a job
  for (int b = threadIdx.x * 16; b < 2 * S::A96_BYTES; b += kFwdThreads * 16)
    *reinterpret_cast<uint4*>(smem + b) = make_uint4(0, 0, 0, 0);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem0 = tslot;
  const uint32_t idesc = idesc_bf16(S::NP);
  uint32_t ph = 0u;  // bit b: the mbarrier phase to wait for on buffer b
  int prev = -1;     // the tile whose MMAs are in flight
  for (int tile = blockIdx.x, it = 0;; tile += gridDim.x, ++it) {
    const bool have = tile < ntiles;
    const int sb = it & 1;
    if (have) a_tile_job<CIN, S::KP>(G, in, fwd_tile_site0(G, tile) + lane, lane, warp, abuf(sb));
    fence_async_smem();
    __syncthreads();
    tc_fence_after();
    if (prev >= 0) {
      // the previous tile: wait for its MMAs (bounded), read its accumulator back
      const int pb = sb ^ 1;
      if (warp == 0) {
        const bool ok = mbar_wait_bounded(&bar[pb], (ph >> pb) & 1u);
        if (lane == 0) {
          mma_ok = ok ? 1 : 0;
          if (!ok) atomicExch(G.err, 1);
        }
      }
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      ph ^= 1u << pb;
      if (!mma_ok) break;  // the same flag in every thread: the CTA leaves together
    }
    // This tile's MMAs go out before the previous tile is read back, so that
    // the read-back overlaps them (the two use different accumulators; A of
    // this tile and its accumulator were last used two tiles ago, which the
    // barriers above have ordered).
    if (have && threadIdx.x == 0) {
      const uint32_t a0 = smem_u32(abuf(sb)), b0 = smem_u32(B);
      constexpr uint32_t sbo = (S::KP / 8) * 128;
#pragma unroll 1
      for (int kb = 0; kb < S::KP / 16; ++kb)
        umma_bf16(tmem0 + uint32_t(sb * S::TCOLS), smem_desc(a0 + kb * 256, 128, sbo),
                  smem_desc(b0 + kb * 256, 128, sbo), idesc, kb > 0 ? 1u : 0u);
      umma_commit(&bar[sb]);
    }
    if (prev >= 0 && warp < 3) {
      const int pb = sb ^ 1;
      const int r = warp * 32 + lane;
      float v[S::NP];
#pragma unroll
      for (int c = 0; c < S::NP; c += 16)
        tmem_ld16(tmem0 + uint32_t(pb * S::TCOLS) + (uint32_t(warp * 32) << 16) + c, v + c);
      const int sl = r / 3, a = r - sl * 3;
      const int s = fwd_tile_site0(G, prev) + sl;
      if (s < G.V) {
        float4* o4 = reinterpret_cast<float4*>(out) + size_t(a) * G.V + s;
#pragma unroll
        for (int q = 0; q < COUT / 2; ++q)
          o4[size_t(3 * q) * G.V] = make_float4(v[4 * q], v[4 * q + 2], v[4 * q + 1], v[4 * q + 3]);
      }
    }
    // the read-back's tensor-memory loads are ordered before the next
    // iteration's barrier, after which that accumulator is written again
    tc_fence_before();
    if (!have) break;
    prev = tile;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem0, 2 * S::TCOLS);
}

// ---- backward: dA = dY B, stored as FP32 rows (site, colour) x KP ------------------
template <int CIN, int COUT>
__global__ void __launch_bounds__(kThreads) ptc_da_kernel(PtcGeo G, const float2* __restrict__ dy,
                                                          float* __restrict__ da,
                                                          const __nv_bfloat16* __restrict__ bopT) {
  using S = Ptc<CIN, COUT>;
  // operand A' = dY tile: 128 rows x NP (K' = NP); operand B' = B^T: KP rows x NP
  constexpr int NCH = S::KP <= 256 ? S::KP : S::KP / 2;  // output columns per MMA pass
  static_assert(NCH % 16 == 0 && NCH <= 256, "bad pass width");
  constexpr int NPASS = S::KP / NCH;
  constexpr int TC = NCH <= 32 ? 32 : (NCH <= 64 ? 64 : (NCH <= 128 ? 128 : 256));
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* A = smem;                 // 128 x NP
  unsigned char* B = smem + 128 * S::NP * 2;  // KP x NP
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) tmem_alloc(&tslot, TC);
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  load_b<S::KP, S::NP>(bopT, B);
  const int site0 = blockIdx.x * kTileSites;
  for (int idx = threadIdx.x; idx < 128 * S::NP; idx += kThreads) {
    const int r = idx / S::NP, n = idx - r * S::NP;
    const int sl = r / 3, a = r - sl * 3, s = site0 + sl;
    float val = 0.f;
    if (sl < kTileSites && s < G.V && n < S::NF) {
      const float2 t = feat_get(dy, s, n >> 1, a, G.V);
      val = (n & 1) ? t.y : t.x;
    }
    *reinterpret_cast<__nv_bfloat16*>(A + canon(r, n, S::NP)) = __float2bfloat16_rn(val);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tslot;
  const int r = warp * 32 + lane;
  const int sl = r / 3, a = r - sl * 3, s = site0 + sl;
  for (int pass = 0; pass < NPASS; ++pass) {
    const bool ok = mma_and_wait<S::NP>(A, B + pass * NCH * S::NP * 2 / 1, tmem, idesc_bf16(NCH), &bar,
                                        uint32_t(pass & 1), G.err);
    if (!ok) break;
    float v[16];
    for (int c = 0; c < NCH; c += 16) {
      tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + c, v);
      if (sl < kTileSites && s < G.V) {
#pragma unroll
        for (int k = 0; k < 16; ++k) da[(size_t(s) * 3 + a) * S::KP + pass * NCH + c + k] = v[k];
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, TC);
}

// d in(y)_i = dA_0(y) + sum_mu U_mu(y-mu)^dag dA_{+mu}(y-mu) + U_mu(y) dA_{-mu}(y+mu)
template <int CIN, int KP>
__global__ void ptc_gather_kernel(PtcGeo G, const float* __restrict__ da, float2* __restrict__ din) {
  const int Vh = G.g.Vh;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < G.V; s += gridDim.x * blockDim.x) {
    const int p = s >= Vh ? 1 : 0;
    const int hs = s - p * Vh;
    const Coord c = coord_of(G.g, hs, p);
    int nb[8];
    neighbours(G.g, c, hs, nb);
    for (int i = 0; i < CIN; ++i) {
      Cx<float> acc[3];
      auto grad = [&](int site, int d, Cx<float> g[3]) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
          g[a] = {da[(size_t(site) * 3 + a) * KP + (2 * d) * CIN + i],
                  da[(size_t(site) * 3 + a) * KP + (2 * d + 1) * CIN + i]};
      };
      grad(s, 0, acc);
#pragma unroll 1
      for (int mu = 0; mu < 4; ++mu) {
        Cx<float> g[3];
        Su3<float> U;
        // from x = y - mu (d = +mu): U_mu(x)^dag g
        const int xm = nb[2 * mu + 1];
        grad((1 - p) * Vh + xm, 1 + 2 * mu, g);
        GaugeIO<PREC_SINGLE, 12>::load(G.gauge, 1 - p, mu, xm, U);
#pragma unroll
        for (int a = 0; a < 3; ++a)
          acc[a] = acc[a] + cj_mul(U.e[0][a], g[0]) + cj_mul(U.e[1][a], g[1]) + cj_mul(U.e[2][a], g[2]);
        // from x = y + mu (d = -mu): U_mu(y) g
        const int xp = nb[2 * mu];
        grad((1 - p) * Vh + xp, 2 + 2 * mu, g);
        GaugeIO<PREC_SINGLE, 12>::load(G.gauge, p, mu, hs, U);
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[a] = acc[a] + U.e[a][0] * g[0] + U.e[a][1] * g[1] + U.e[a][2] * g[2];
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) feat_set(din, s, i, a, G.V, make_float2(acc[a].re, acc[a].im));
    }
  }
}

// dB[n][k] = sum_rows dY[row][n] A[row][k], one partial per tile (CUDA cores)
template <int CIN, int COUT>
__global__ void __launch_bounds__(kThreads) ptc_db_kernel(PtcGeo G, const float2* __restrict__ in,
                                                          const float2* __restrict__ dy,
                                                          float* __restrict__ partial) {
  using S = Ptc<CIN, COUT>;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* A = smem;
  float* Y = reinterpret_cast<float*>(smem + S::A_BYTES);  // 128 x NF
  const int site0 = blockIdx.x * kTileSites;
  build_a_tile<CIN, S::KP>(G, in, site0, A);
  for (int idx = threadIdx.x; idx < 128 * S::NF; idx += kThreads) {
    const int r = idx / S::NF, n = idx - r * S::NF;
    const int sl = r / 3, a = r - sl * 3, s = site0 + sl;
    float val = 0.f;
    if (sl < kTileSites && s < G.V) {
      const float2 t = feat_get(dy, s, n >> 1, a, G.V);
      val = (n & 1) ? t.y : t.x;
    }
    Y[idx] = val;
  }
  __syncthreads();
  float* out = partial + size_t(blockIdx.x) * S::NF * S::KF;
  for (int q = threadIdx.x; q < S::NF * S::KF; q += kThreads) {
    const int n = q / S::KF, k = q - n * S::KF;
    float acc = 0.f;
    for (int r = 0; r < 126; ++r)
      acc += Y[r * S::NF + n] * __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(A + canon(r, k, S::KP)));
    out[q] = acc;
  }
}

// deterministic sum over tiles
__global__ void sum_partials_kernel(const float* __restrict__ partial, int ntiles, int n, float* out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int t = 0; t < ntiles; ++t) acc += partial[size_t(t) * n + q];
    out[q] = float(acc);
  }
}

// spinor field (FP32, full lattice) <-> 4-channel features [site][spin][colour]
__global__ void spinor_to_feat_kernel(int Vh, SpinorPtr e, SpinorPtr o, float2* feat, const int* skip) {
  if (skip && *skip) return;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < 2 * Vh; s += gridDim.x * blockDim.x) {
    const int p = s >= Vh ? 1 : 0;
    Cx<float> v[12];
    SpinorIO<PREC_SINGLE>::load(p ? o : e, s - p * Vh, v);
#pragma unroll
    for (int k = 0; k < 12; ++k) feat_set(feat, s, k / 3, k % 3, 2 * Vh, make_float2(v[k].re, v[k].im));
  }
}
template <int PO>
__global__ void feat_to_spinor_kernel(int Vh, const float2* feat, SpinorPtr e, SpinorPtr o, const int* skip) {
  if (skip && *skip) return;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < 2 * Vh; s += gridDim.x * blockDim.x) {
    const int p = s >= Vh ? 1 : 0;
    Cx<float> v[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      const float2 t = feat_get(feat, s, k / 3, k % 3, 2 * Vh);
      v[k] = {t.x, t.y};
    }
    SpinorIO<PO>::store(p ? o : e, s - p * Vh, v);
  }
}

// ---- host launchers ------------------------------------------------------------------
static int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n < 1) n = 1;
  }
  return n;
}

// CTAs of `threads` threads of kernel f that fit on one SM by registers (65536
// per SM, allocated per warp in units of 256): the persistent forward kernels
// launch no more than this many per SM, so that no CTA waits for another to
// finish before it starts its share of the tiles
static int fit_by_registers(const void* f, int threads) {
  cudaFuncAttributes a;
  if (cudaFuncGetAttributes(&a, f) != cudaSuccess || a.numRegs <= 0) return 1 << 20;
  const int per_warp = (a.numRegs * 32 + 255) / 256 * 256;
  const int n = 65536 / (per_warp * ((threads + 31) / 32));
  return n > 0 ? n : 1;
}

template <int CIN, int COUT>
static cudaError_t fwd_t(const PtcGeo& G, const float2* in, float2* out, const __nv_bfloat16* bop,
                         cudaStream_t st) {
  using S = Ptc<CIN, COUT>;
  const int ntiles2 = (G.V + kFwdSites - 1) / kFwdSites;
  // double-buffered where two A tiles leave room for at least two CTAs per SM
  // in ~200 KB of shared memory (CIN <= 8); one tile otherwise
  const int smem2 = 2 * S::A96_BYTES + S::BF_BYTES;
  if ((200 * 1024) / (smem2 + 1024) >= 2) {
    static bool attr2 = false;
    if (!attr2) {
      cudaError_t e = cudaFuncSetAttribute(ptc_fwd2_kernel<CIN, COUT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem2);
      if (e != cudaSuccess) return e;
      attr2 = true;
    }
    int per_sm = (200 * 1024) / (smem2 + 1024);
    if (per_sm > 2048 / kFwdThreads) per_sm = 2048 / kFwdThreads;
    const int regs = fit_by_registers(reinterpret_cast<const void*>(ptc_fwd2_kernel<CIN, COUT>), kFwdThreads);
    if (per_sm > regs) per_sm = regs;
    int grid = sm_count() * per_sm;
    if (grid > ntiles2) grid = ntiles2;
    ptc_fwd2_kernel<CIN, COUT><<<grid, kFwdThreads, smem2, st>>>(G, in, out, bop, ntiles2);
    return cudaGetLastError();
  }
  const int smem = S::A96_BYTES + S::BF_BYTES;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(ptc_fwd_kernel<CIN, COUT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int ntiles = (G.V + kFwdSites - 1) / kFwdSites;
  // persistent: as many CTAs as fit on the device (threads, and shared memory
  // up to ~150 KB per SM so that the rest of the SM's 256 KB stays L1 cache
  // for the neighbour gathers), at most one per tile
  int per_sm = (150 * 1024) / (smem + 1024);
  if (per_sm > 2048 / kFwdThreads) per_sm = 2048 / kFwdThreads;
  const int regs = fit_by_registers(reinterpret_cast<const void*>(ptc_fwd_kernel<CIN, COUT>), kFwdThreads);
  if (per_sm > regs) per_sm = regs;
  if (per_sm < 1) per_sm = 1;
  int grid = sm_count() * per_sm;
  if (grid > ntiles) grid = ntiles;
  ptc_fwd_kernel<CIN, COUT><<<grid, kFwdThreads, smem, st>>>(G, in, out, bop, ntiles);
  return cudaGetLastError();
}

template <int CIN, int COUT>
static cudaError_t bwd_t(const PtcGeo& G, const float2* in, const float2* dy, float* da, float2* din,
                         const __nv_bfloat16* bopT, float* partial, float* db, cudaStream_t st) {
  using S = Ptc<CIN, COUT>;
  const int grid = (G.V + kTileSites - 1) / kTileSites;
  if (din) {
    // the pass accumulator takes up to 256 TMEM columns: ask for enough shared
    // memory that at most two CTAs share an SM (2 x 256 = its 512 columns),
    // so tensor-memory allocation never has to wait
    constexpr int NCH = S::KP <= 256 ? S::KP : S::KP / 2;
    constexpr int TC = NCH <= 32 ? 32 : (NCH <= 64 ? 64 : (NCH <= 128 ? 128 : 256));
    const int need = 128 * S::NP * 2 + S::KP * S::NP * 2;
    const int cap = TC >= 256 ? 100 * 1024 : (TC >= 128 ? 52 * 1024 : 0);
    const int smem = need > cap ? need : cap;
    static bool attr = false;
    if (!attr) {
      cudaError_t e = cudaFuncSetAttribute(ptc_da_kernel<CIN, COUT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      attr = true;
    }
    ptc_da_kernel<CIN, COUT><<<grid, kThreads, smem, st>>>(G, dy, da, bopT);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    ptc_gather_kernel<CIN, S::KP><<<(G.V + 255) / 256, 256, 0, st>>>(G, da, din);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (db) {
    const int smem = S::A_BYTES + 128 * S::NF * 4;
    static bool attr = false;
    if (!attr) {
      cudaError_t e = cudaFuncSetAttribute(ptc_db_kernel<CIN, COUT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      attr = true;
    }
    ptc_db_kernel<CIN, COUT><<<grid, kThreads, smem, st>>>(G, in, dy, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    sum_partials_kernel<<<(S::NF * S::KF + 255) / 256, 256, 0, st>>>(partial, grid, S::NF * S::KF, db);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int ptc_shape_ok(int cin, int cout) {
  return (cin == 4 || cin == 8 || cin == 16) && (cout == 4 || cout == 8 || cout == 16);
}

#define IRO_PTC_DISPATCH(CALL)                              \
  switch (cin * 100 + cout) {                               \
    case 404: return CALL(4, 4);                            \
    case 408: return CALL(4, 8);                            \
    case 416: return CALL(4, 16);                           \
    case 804: return CALL(8, 4);                            \
    case 808: return CALL(8, 8);                            \
    case 816: return CALL(8, 16);                           \
    case 1604: return CALL(16, 4);                          \
    case 1608: return CALL(16, 8);                          \
    case 1616: return CALL(16, 16);                         \
  }                                                         \
  return cudaErrorInvalidValue;

cudaError_t launch_ptc_fwd(int cin, int cout, const PtcGeo& G, const float2* in, float2* out,
                           const void* bop, cudaStream_t st) {
#define IRO_F(A, B) fwd_t<A, B>(G, in, out, static_cast<const __nv_bfloat16*>(bop), st)
  IRO_PTC_DISPATCH(IRO_F)
#undef IRO_F
}

cudaError_t launch_ptc_bwd(int cin, int cout, const PtcGeo& G, const float2* in, const float2* dy,
                           float* da, float2* din, const void* bopT, float* partial, float* db,
                           cudaStream_t st) {
#define IRO_B(A, B) bwd_t<A, B>(G, in, dy, da, din, static_cast<const __nv_bfloat16*>(bopT), partial, db, st)
  IRO_PTC_DISPATCH(IRO_B)
#undef IRO_B
}

void ptc_dims(int cin, int cout, int* kf, int* kp, int* nf, int* np) {
  *kf = 18 * cin;
  *kp = (*kf + 15) / 16 * 16;
  *nf = 2 * cout;
  *np = *nf < 16 ? 16 : (*nf + 15) / 16 * 16;
}

cudaError_t launch_spinor_to_feat(int Vh, SpinorPtr e, SpinorPtr o, float2* feat, cudaStream_t st,
                                  const int* skip = nullptr) {
  spinor_to_feat_kernel<<<(2 * Vh + 255) / 256, 256, 0, st>>>(Vh, e, o, feat, skip);
  return cudaGetLastError();
}
// to an FP32 (or, prec = PREC_HALF, FP16) spinor field
cudaError_t launch_feat_to_spinor(int Vh, const float2* feat, SpinorPtr e, SpinorPtr o, cudaStream_t st,
                                  const int* skip = nullptr, int prec = PREC_SINGLE) {
  if (prec == PREC_HALF)
    feat_to_spinor_kernel<PREC_HALF><<<(2 * Vh + 255) / 256, 256, 0, st>>>(Vh, feat, e, o, skip);
  else
    feat_to_spinor_kernel<PREC_SINGLE><<<(2 * Vh + 255) / 256, 256, 0, st>>>(Vh, feat, e, o, skip);
  return cudaGetLastError();
}

// ---- loss of a training pair: |y - t|^2 and |t|^2, and dy = 2 (y - t) / |t|^2 ------------
constexpr int kRedBlocks = 296;

__global__ void loss_partials_kernel(int n, const float2* y, const float2* t, double* part) {
  __shared__ double sa[256], sb[256];
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float2 yy = y[i], tt = t[i];
    const double dr = double(yy.x) - tt.x, di = double(yy.y) - tt.y;
    a += dr * dr + di * di;
    b += double(tt.x) * tt.x + double(tt.y) * tt.y;
  }
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      sa[threadIdx.x] += sa[threadIdx.x + h];
      sb[threadIdx.x] += sb[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sa[0];
    part[2 * blockIdx.x + 1] = sb[0];
  }
}

__global__ void loss_grad_kernel(int n, const float2* y, const float2* t, float scale, float2* dy) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float2 yy = y[i], tt = t[i];
    dy[i] = make_float2(scale * (yy.x - tt.x), scale * (yy.y - tt.y));
  }
}

cudaError_t launch_loss_partials(int n, const float2* y, const float2* t, double* part, cudaStream_t st) {
  loss_partials_kernel<<<kRedBlocks, 256, 0, st>>>(n, y, t, part);
  return cudaGetLastError();
}
cudaError_t launch_loss_grad(int n, const float2* y, const float2* t, float scale, float2* dy,
                             cudaStream_t st) {
  loss_grad_kernel<<<kRedBlocks, 256, 0, st>>>(n, y, t, scale, dy);
  return cudaGetLastError();
}
int loss_blocks() { return kRedBlocks; }

// ---- complex linear algebra for GCR on FP32 fields ---------------------------------------
// <w_q, t> = sum conj(w_q) t for q < m, per-block partials [block][2m]; the
// last listed field is FP32 (GCR's residual), the others and t of type PW
// M fields (a compile-time count: the loads of every field of a site can be
// issued together and only 2M accumulators are live), 128-thread blocks
constexpr int kCdotThreads = 128;
template <int PW, int M>
__global__ void __launch_bounds__(kCdotThreads) cdot_kernel(int64_t n, CFieldList w, SpinorPtr t,
                                                            double* part, const int* skip) {
  if (skip && *skip) return;  // the same value in every thread
  __shared__ double sm[2 * M][kCdotThreads / 32];
  double acc[2 * M];
#pragma unroll
  for (int q = 0; q < 2 * M; ++q) acc[q] = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    Cx<float> tv[12];
    SpinorIO<PW>::load(t, i, tv);
#pragma unroll
    for (int q = 0; q < M; ++q) {
      Cx<float> wv[12];
      if (q == M - 1)
        SpinorIO<PREC_SINGLE>::load(w.f[q], i, wv);
      else
        SpinorIO<PW>::load(w.f[q], i, wv);
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        re += double(wv[k].re) * tv[k].re + double(wv[k].im) * tv[k].im;
        im += double(wv[k].re) * tv[k].im - double(wv[k].im) * tv[k].re;
      }
      acc[2 * q] += re;
      acc[2 * q + 1] += im;
    }
  }
#pragma unroll
  for (int q = 0; q < 2 * M; ++q) {
    double v = acc[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 2 * M) {
    double v = 0.0;
#pragma unroll
    for (int wv = 0; wv < kCdotThreads / 32; ++wv) v += sm[threadIdx.x][wv];
    part[size_t(blockIdx.x) * 2 * M + threadIdx.x] = v;
  }
}

// the block partials of cdot_kernel summed in a fixed order: one warp per
// real component (block q), lane l summing blocks l, l + 32, ..., then a
// shuffle tree over the lanes
__global__ void cdot_finish_kernel(int blocks, int m2, const double* part, double* out, const int* skip) {
  if (skip && *skip) return;
  const int q = blockIdx.x, l = threadIdx.x;
  if (q >= m2) return;
  double v = 0.0;
  for (int b = l; b < blocks; b += 32) v += part[size_t(b) * m2 + q];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (l == 0) out[q] = v;
}

// y += sign sum_q c_q x_q  (complex coefficients from the cycle state; the
// first *count of the m fields when count is given); x of type PX, y FP32
template <int PX>
__global__ void caxpy_dev_kernel(int64_t n, int m, CFieldList x, const GcrState* s, const int* count,
                                 float sign, SpinorPtr y, const int* skip) {
  if (skip && *skip) return;
  __shared__ float cre[kMaxList], cim[kMaxList];
  __shared__ int mm;
  if (threadIdx.x < kMaxList) {
    cre[threadIdx.x] = sign * s->cre[threadIdx.x];
    cim[threadIdx.x] = sign * s->cim[threadIdx.x];
  }
  if (threadIdx.x == 0) mm = count ? min(*count, m) : m;
  __syncthreads();
  const int k = mm;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    Cx<float> yv[12], xv[12];
    SpinorIO<PREC_SINGLE>::load(y, i, yv);
    for (int q = 0; q < k; ++q) {
      SpinorIO<PX>::load(x.f[q], i, xv);
      const Cx<float> cq = {cre[q], cim[q]};
#pragma unroll
      for (int c = 0; c < 12; ++c) yv[c] = yv[c] + cq * xv[c];
    }
    SpinorIO<PREC_SINGLE>::store(y, i, yv);
  }
}

// iteration j (the w of type PW, r FP32): wj += sum_{q<m} c_q w_q; then, unless the coefficient kernel
// found w_j nearly in the span of the w_q (s->plain[j] = 0: a second pass
// forms |w'_j|^2 and <r, w'_j> first), r -= alpha wj with the updated wj,
// and, given feat, the network's input features of the new r
template <int PW>
__global__ void gcr_update_kernel(int64_t n, int m, CFieldList w, const GcrState* s, int j,
                                  SpinorPtr wj, SpinorPtr r, float2* feat) {
  if (s->skip[j]) return;
  __shared__ float cre[kMaxList], cim[kMaxList];
  if (threadIdx.x < kMaxList) {
    cre[threadIdx.x] = s->cre[threadIdx.x];
    cim[threadIdx.x] = s->cim[threadIdx.x];
  }
  __syncthreads();
  const bool plain = s->plain[j] != 0;
  const Cx<float> a = {s->ure, s->uim};
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    Cx<float> yv[12], xv[12];
    SpinorIO<PW>::load(wj, i, yv);
    for (int q = 0; q < m; ++q) {
      SpinorIO<PW>::load(w.f[q], i, xv);
      const Cx<float> cq = {cre[q], cim[q]};
#pragma unroll
      for (int k = 0; k < 12; ++k) yv[k] = yv[k] + cq * xv[k];
    }
    SpinorIO<PW>::store(wj, i, yv);
    if (plain) {
      SpinorIO<PREC_SINGLE>::load(r, i, xv);
#pragma unroll
      for (int k = 0; k < 12; ++k) xv[k] = xv[k] - a * yv[k];
      SpinorIO<PREC_SINGLE>::store(r, i, xv);
      if (feat) {
        // the network's input features of the new r (as spinor_to_feat: site
        // i of the full field, spin pair q and colour c in float4 row 3q + c)
        float4* f4 = reinterpret_cast<float4*>(feat);
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const Cx<float> lo = xv[6 * q + c], hi = xv[6 * q + 3 + c];
            f4[size_t(3 * q + c) * size_t(n) + size_t(i)] = make_float4(lo.re, hi.re, lo.im, hi.im);
          }
      }
    }
  }
}

__global__ void gcr_init_kernel(GcrState* s, double rr, double target, double d2, int limit) {
  const int t = threadIdx.x;
  if (t < kMaxVec) {
    s->skip[t] = 0;
    s->plain[t] = 1;
  }
  for (int i = t; i < kMaxVec * kMaxVec; i += blockDim.x) s->tre[i] = s->tim[i] = 0.0;
  if (t == 0) {
    s->rr_it = s->rr_start = rr;
    s->target = target;
    s->d2 = d2;
    s->limit = limit;
    s->jdone = 0;
  }
}

// alpha_j, column j of T, the iterated |r|^2 and the restart test, from
// |w'_j|^2 and <r, w'_j> (r is orthogonal to every earlier w'_q, so
// <r, w'_j> = <r, w_j>); the beta_q of the iteration are in s->bre/bim
__device__ void gcr_finish_iteration(GcrState* s, int j, int m, double nwj, double rre, double rim) {
  constexpr int K = kMaxVec;
  s->nw[j] = nwj;
  const double ar = rre / nwj, ai = -rim / nwj;  // alpha = conj(<r, w'_j>) / |w'_j|^2
  s->are[j] = ar;
  s->aim[j] = ai;
  s->ure = float(ar);
  s->uim = float(ai);
  // z'_j = z_j + sum_q beta_q z'_q
  s->tre[j * K + j] = 1.0;
  for (int q = 0; q < j; ++q) {
    const double br = s->bre[q], bi = s->bim[q];
    for (int i = 0; i <= q; ++i) {
      const double tr = s->tre[i * K + q], ti = s->tim[i * K + q];
      s->tre[i * K + j] += br * tr - bi * ti;
      s->tim[i * K + j] += br * ti + bi * tr;
    }
  }
  // r minus its projection on w'_j; only the restart test reads it, the FP64
  // residual decides
  s->rr_it = s->rr_it - (rre * rre + rim * rim) / nwj;
  s->jdone = j + 1;
  if (s->rr_it < s->target || s->rr_it < s->d2 * s->rr_start || s->jdone >= s->limit)
    for (int k = j + 1; k < m; ++k) s->skip[k] = 1;
}

// One thread.  First pass (second = 0): g = <w_q, w_j> (q < j), |w_j|^2,
// <r, w_j> as (re, im) pairs.  The w_q are orthogonal, hence for w'_j = w_j +
// sum_q beta_q w_q with beta_q = -<w_q, w_j>/|w_q|^2, |w'_j|^2 = |w_j|^2 -
// sum_q |<w_q, w_j>|^2/|w_q|^2; when that falls below 1e-4 |w_j|^2 the
// orthogonalised vector is formed first and a second pass (second = 1, g =
// |w'_j|^2, <r, w'_j>) finishes the iteration.
__global__ void gcr_coef_kernel(GcrState* s, const double* g, int j, int m, int second) {
  if (s->skip[j]) return;
  if (!second) {
    double nwj = g[2 * j];
    for (int q = 0; q < j; ++q) {
      const double gr = g[2 * q], gi = g[2 * q + 1], nq = s->nw[q];
      const double br = -gr / nq, bi = -gi / nq;
      s->bre[q] = br;
      s->bim[q] = bi;
      s->cre[q] = float(br);
      s->cim[q] = float(bi);
      nwj -= (gr * gr + gi * gi) / nq;
    }
    if (nwj > 1e-4 * g[2 * j]) {
      gcr_finish_iteration(s, j, m, nwj, g[2 * j + 2], g[2 * j + 3]);
    } else {
      s->plain[j] = 0;
      s->ure = s->uim = 0.f;
    }
  } else {
    if (s->plain[j]) return;
    gcr_finish_iteration(s, j, m, g[0], g[2], g[3]);
    s->cre[0] = s->ure;  // r -= alpha w'_j (caxpy with sign -1)
    s->cim[0] = s->uim;
  }
}

// gamma_i = sum_{j >= i} T[i][j] alpha_j over the cycle's iterations, into
// s->cre/cim (zero beyond them)
__global__ void gcr_gamma_kernel(GcrState* s) {
  const int jd = s->jdone;
  for (int i = threadIdx.x; i < kMaxList; i += blockDim.x) {
    double gr = 0.0, gi = 0.0;
    for (int j = i; j < jd; ++j) {
      const double tr = s->tre[i * kMaxVec + j], ti = s->tim[i * kMaxVec + j];
      gr += tr * s->are[j] - ti * s->aim[j];
      gi += tr * s->aim[j] + ti * s->are[j];
    }
    s->cre[i] = float(gr);
    s->cim[i] = float(gi);
  }
}

// Self-test of the bounded wait (iro_selftest_bounded_wait): one thread waits
// on an mbarrier that nothing arrives at, gives up after limit_ns, and
// records the time it waited and the error flag, as the tensor-core kernels
// do on a wait that runs out.
__global__ void bounded_wait_probe_kernel(uint64_t limit_ns, int* err, unsigned long long* waited_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint64_t t0 = global_ns();
    const bool ok = mbar_wait_bounded(&bar, 0u, limit_ns);
    *waited_ns = global_ns() - t0;
    if (!ok) atomicExch(err, 1);
  }
}

cudaError_t launch_bounded_wait_probe(uint64_t limit_ns, int* err, unsigned long long* waited_ns,
                                      cudaStream_t st) {
  bounded_wait_probe_kernel<<<1, 32, 0, st>>>(limit_ns, err, waited_ns);
  return cudaGetLastError();
}

template <int PW, int M>
static void cdot_go(int64_t n, const CFieldList& w, SpinorPtr t, double* part, int blocks,
                    const int* skip, cudaStream_t st) {
  cdot_kernel<PW, M><<<blocks, kCdotThreads, 0, st>>>(n, w, t, part, skip);
}
template <int PW>
static cudaError_t cdot_count(int64_t n, int m, const CFieldList& w, SpinorPtr t, double* part,
                              int blocks, const int* skip, cudaStream_t st) {
  static_assert(kMaxList == 18, "one case per field count");
  switch (m) {
#define IRO_CD(M) \
  case M: cdot_go<PW, M>(n, w, t, part, blocks, skip, st); break;
    IRO_CD(1) IRO_CD(2) IRO_CD(3) IRO_CD(4) IRO_CD(5) IRO_CD(6) IRO_CD(7) IRO_CD(8) IRO_CD(9)
    IRO_CD(10) IRO_CD(11) IRO_CD(12) IRO_CD(13) IRO_CD(14) IRO_CD(15) IRO_CD(16) IRO_CD(17)
    IRO_CD(18)
#undef IRO_CD
    default: return cudaErrorInvalidValue;
  }
  return cudaSuccess;
}
cudaError_t launch_cdot(int64_t n, int m, const CFieldList& w, SpinorPtr t, double* part, int blocks,
                        double* out, const int* skip, int pw, cudaStream_t st) {
  const cudaError_t e = pw == PREC_HALF ? cdot_count<PREC_HALF>(n, m, w, t, part, blocks, skip, st)
                                        : cdot_count<PREC_SINGLE>(n, m, w, t, part, blocks, skip, st);
  if (e != cudaSuccess) return e;
  cdot_finish_kernel<<<2 * m, 32, 0, st>>>(blocks, 2 * m, part, out, skip);
  return cudaGetLastError();
}
static int blas_grid(int64_t n) {
  int grid = int((n + 255) / 256);
  return grid > 148 * 16 ? 148 * 16 : grid;
}
cudaError_t launch_caxpy_dev(int64_t n, int m, const CFieldList& x, int px, const GcrState* s,
                             const int* count, float sign, SpinorPtr y, const int* skip,
                             cudaStream_t st) {
  if (px == PREC_HALF)
    caxpy_dev_kernel<PREC_HALF><<<blas_grid(n), 256, 0, st>>>(n, m, x, s, count, sign, y, skip);
  else
    caxpy_dev_kernel<PREC_SINGLE><<<blas_grid(n), 256, 0, st>>>(n, m, x, s, count, sign, y, skip);
  return cudaGetLastError();
}
cudaError_t launch_gcr_update(int64_t n, int m, const CFieldList& w, int pw, const GcrState* s, int j,
                              SpinorPtr wj, SpinorPtr r, float2* feat, cudaStream_t st) {
  if (pw == PREC_HALF)
    gcr_update_kernel<PREC_HALF><<<blas_grid(n), 256, 0, st>>>(n, m, w, s, j, wj, r, feat);
  else
    gcr_update_kernel<PREC_SINGLE><<<blas_grid(n), 256, 0, st>>>(n, m, w, s, j, wj, r, feat);
  return cudaGetLastError();
}
cudaError_t launch_gcr_init(GcrState* s, double rr, double target, double d2, int limit,
                            cudaStream_t st) {
  gcr_init_kernel<<<1, 64, 0, st>>>(s, rr, target, d2, limit);
  return cudaGetLastError();
}
cudaError_t launch_gcr_coef(GcrState* s, const double* g, int j, int m, int second,
                            cudaStream_t st) {
  gcr_coef_kernel<<<1, 1, 0, st>>>(s, g, j, m, second);
  return cudaGetLastError();
}
__global__ void fill_int_kernel(int* p, int v) { *p = v; }
cudaError_t launch_fill_int(int* p, int v, cudaStream_t st) {
  fill_int_kernel<<<1, 1, 0, st>>>(p, v);
  return cudaGetLastError();
}
cudaError_t launch_gcr_gamma(GcrState* s, cudaStream_t st) {
  gcr_gamma_kernel<<<1, 32, 0, st>>>(s);
  return cudaGetLastError();
}

}  // namespace iro

// =====================================================================================
// Host side: the network object, training gradients and flexible GCR.
// =====================================================================================
#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>
#include <string>

namespace iro {
namespace host {
int apply(iro_ctx* c, int op, double mass, double csw, bool dag, const DevField& in, DevField& out,
          const Reduce* red, int red_mask, const int* skip);
DevField* workspace(iro_ctx* c, int subset, int prec, int nrhs, int slot, int* rc);
void* pinned(iro_ctx* c);
void* scratch(iro_ctx* c, size_t bytes, int* rc);
int import_field(iro_ctx* c, const double* host, bool full, DevField& f);
int export_field(iro_ctx* c, const DevField& f, bool full, double* host);
int norms(iro_ctx* c, const DevField& v, const DevField* w, std::vector<double>& nv,
          std::vector<double>* nw);
int axpby(iro_ctx* c, double a, const DevField& x, double b, const DevField& y, DevField& v);
int convert(iro_ctx* c, const DevField& in, DevField& out);
int set_error(iro_ctx* c, int code, const std::string& msg);
int cuda_error(iro_ctx* c, cudaError_t e, const char* where);
cudaStream_t stream(iro_ctx* c);
int device(iro_ctx* c);
DevField* field_dev(iro_field* f);
const Geom& geom(iro_ctx* c);
GaugePtr gauge_single(iro_ctx* c);
bool gauge_su3(iro_ctx* c);
int64_t volume(iro_ctx* c);
}  // namespace host
}  // namespace iro

// CG on device fields (solvers.cu), the fallback of the preconditioned solve
int cg_any_dev(iro_ctx* c, int op, double mass, double csw, const iro_cg_params* prm,
               const iro::DevField* B, iro::DevField* X, int nrhs, iro_solver_out* out);

using namespace iro;
using namespace iro::host;

#define LCK(call)                                            \
  do {                                                       \
    cudaError_t e__ = (call);                                \
    if (e__ != cudaSuccess) return cuda_error(c, e__, #call); \
  } while (0)
#define LRC(call)                  \
  do {                             \
    int r__ = (call);              \
    if (r__ != IRO_OK) return r__; \
  } while (0)

struct iro_ptc {
  iro_ctx* ctx = nullptr;
  int dev = 0;  // device of the buffers (iro_ptc_destroy does not touch the context)
  int nl = 0;
  std::vector<int> w;                 // widths, nl+1 entries
  std::vector<std::vector<float>> W;  // host weights, complex [9][cout][cin] (re,im)
  std::vector<void*> bop, bopT;       // device BF16 packed weights per layer
  std::vector<float2*> act;           // act[l]: input of layer l (act[nl]: output)
  float2* g0 = nullptr;               // gradient ping-pong buffers
  float2* g1 = nullptr;
  float* da = nullptr;
  float* partial = nullptr;
  std::vector<float*> db;
  int* err = nullptr;
  double* lpart = nullptr;
  size_t maxc = 0;
};

namespace {

void pack_bop(int cin, int cout, const std::vector<float>& W, std::vector<__nv_bfloat16>& bop,
              std::vector<__nv_bfloat16>& bopT) {
  int kf, kp, nf, np;
  ptc_dims(cin, cout, &kf, &kp, &nf, &np);
  std::vector<float> B(size_t(np) * kp, 0.f);
  for (int d = 0; d < 9; ++d)
    for (int o = 0; o < cout; ++o)
      for (int i = 0; i < cin; ++i) {
        const size_t w = ((size_t(d) * cout + o) * cin + i) * 2;
        const float wr = W[w], wi = W[w + 1];
        const int kre = (2 * d) * cin + i, kim = (2 * d + 1) * cin + i;
        B[size_t(2 * o) * kp + kre] = wr;
        B[size_t(2 * o) * kp + kim] = -wi;
        B[size_t(2 * o + 1) * kp + kre] = wi;
        B[size_t(2 * o + 1) * kp + kim] = wr;
      }
  bop.resize(B.size());
  bopT.resize(B.size());
  for (int n = 0; n < np; ++n)
    for (int k = 0; k < kp; ++k) {
      bop[size_t(n) * kp + k] = __float2bfloat16_rn(B[size_t(n) * kp + k]);
      bopT[size_t(k) * np + n] = __float2bfloat16_rn(B[size_t(n) * kp + k]);
    }
}

// dL/dB (NF x KF, real) -> dL/dW (complex [9][cout][cin])
void unpack_grad(int cin, int cout, const std::vector<float>& dB, float* g) {
  int kf, kp, nf, np;
  ptc_dims(cin, cout, &kf, &kp, &nf, &np);
  for (int d = 0; d < 9; ++d)
    for (int o = 0; o < cout; ++o)
      for (int i = 0; i < cin; ++i) {
        const int kre = (2 * d) * cin + i, kim = (2 * d + 1) * cin + i;
        const float rr = dB[size_t(2 * o) * kf + kre], ri = dB[size_t(2 * o) * kf + kim];
        const float ir = dB[size_t(2 * o + 1) * kf + kre], ii = dB[size_t(2 * o + 1) * kf + kim];
        const size_t w = ((size_t(d) * cout + o) * cin + i) * 2;
        g[w] = rr + ii;
        g[w + 1] = -ri + ir;
      }
}

PtcGeo make_geo(iro_ctx* c, int* err) {
  PtcGeo G;
  G.g = geom(c);
  G.gauge = gauge_single(c);
  G.V = int(volume(c));
  G.err = err;
  G.skip = nullptr;
  return G;
}

// features of a full-lattice spinor field (FP32 or FP64; converted to FP32);
// `skip` (FP32 fields only) as the forward pass's
int field_to_feat(iro_ctx* c, const DevField& f, float2* feat, const int* skip = nullptr) {
  const DevField* src = &f;
  int rc = IRO_OK;
  if (f.prec != PREC_SINGLE) {
    DevField* t = workspace(c, 2, PREC_SINGLE, 1, 70, &rc);
    if (!t) return rc;
    LRC(convert(c, f, *t));
    src = t;
  }
  LCK(launch_spinor_to_feat(int(src->Vh), src->half(0), src->half(1), feat, stream(c),
                            f.prec == PREC_SINGLE ? skip : nullptr));
  return IRO_OK;
}

int feat_to_field(iro_ctx* c, const float2* feat, DevField& f, const int* skip = nullptr) {
  if (f.prec == PREC_SINGLE || f.prec == PREC_HALF) {
    LCK(launch_feat_to_spinor(int(f.Vh), feat, f.half(0), f.half(1), stream(c), skip, f.prec));
    return IRO_OK;
  }
  int rc = IRO_OK;
  DevField* t = workspace(c, 2, PREC_SINGLE, 1, 71, &rc);
  if (!t) return rc;
  LCK(launch_feat_to_spinor(int(t->Vh), feat, t->half(0), t->half(1), stream(c)));
  return convert(c, *t, f);
}

int check_err(iro_ctx* c, iro_ptc* n) {
  int e = 0;
  LCK(cudaMemcpyAsync(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost, stream(c)));
  LCK(cudaStreamSynchronize(stream(c)));
  if (e) return set_error(c, IRO_TIMEOUT, "tensor-core wait timed out in the network kernels");
  return IRO_OK;
}

// act[0] must hold the input features; runs every layer
// the network's layers on n->act[0]; nothing when `skip` is set and nonzero
int forward(iro_ctx* c, iro_ptc* n, const int* skip = nullptr) {
  PtcGeo G = make_geo(c, n->err);
  G.skip = skip;
  for (int l = 0; l < n->nl; ++l)
    LCK(launch_ptc_fwd(n->w[l], n->w[l + 1], G, n->act[l], n->act[l + 1], n->bop[l], stream(c)));
  return IRO_OK;
}

}  // namespace

extern "C" {

int iro_ptc_create(iro_ctx* c, int nlayers, const int* widths, iro_ptc** out) {
  if (!c || !widths || !out || nlayers < 1 || nlayers > 8)
    return set_error(c, IRO_BAD_ARG, "bad network arguments");
  if (widths[0] != 4 || widths[nlayers] != 4)
    return set_error(c, IRO_BAD_ARG, "network input and output must be 4 channels (a spinor)");
  for (int l = 0; l < nlayers; ++l)
    if (!ptc_shape_ok(widths[l], widths[l + 1]))
      return set_error(c, IRO_BAD_ARG, "layer widths must be 4, 8 or 16 channels");
  LCK(cudaSetDevice(device(c)));
  std::unique_ptr<iro_ptc> n(new iro_ptc());
  n->ctx = c;
  n->dev = device(c);
  n->nl = nlayers;
  n->w.assign(widths, widths + nlayers + 1);
  const size_t V = size_t(volume(c));
  size_t maxc = 0;
  for (int w : n->w) maxc = std::max(maxc, size_t(w));
  n->maxc = maxc;
  n->W.resize(nlayers);
  n->bop.resize(nlayers);
  n->bopT.resize(nlayers);
  n->db.resize(nlayers);
  n->act.resize(nlayers + 1);
  int maxkp = 0, maxtiles = int((V + kTileSites - 1) / kTileSites), maxnk = 0;
  for (int l = 0; l < nlayers; ++l) {
    int kf, kp, nf, np;
    ptc_dims(n->w[l], n->w[l + 1], &kf, &kp, &nf, &np);
    maxkp = std::max(maxkp, kp);
    maxnk = std::max(maxnk, nf * kf);
    n->W[l].assign(size_t(9) * n->w[l + 1] * n->w[l] * 2, 0.f);
    LCK(cudaMalloc(&n->bop[l], size_t(np) * kp * 2));
    LCK(cudaMalloc(&n->bopT[l], size_t(np) * kp * 2));
    LCK(cudaMemset(n->bop[l], 0, size_t(np) * kp * 2));
    LCK(cudaMemset(n->bopT[l], 0, size_t(np) * kp * 2));
    LCK(cudaMalloc(&n->db[l], size_t(nf) * kf * sizeof(float)));
  }
  for (int l = 0; l <= nlayers; ++l) LCK(cudaMalloc(&n->act[l], V * n->w[l] * 3 * sizeof(float2)));
  LCK(cudaMalloc(&n->g0, V * maxc * 3 * sizeof(float2)));
  LCK(cudaMalloc(&n->g1, V * maxc * 3 * sizeof(float2)));
  LCK(cudaMalloc(&n->da, V * 3 * maxkp * sizeof(float)));
  LCK(cudaMalloc(&n->partial, size_t(maxtiles) * maxnk * sizeof(float)));
  LCK(cudaMalloc(&n->err, sizeof(int)));
  LCK(cudaMemset(n->err, 0, sizeof(int)));
  LCK(cudaMalloc(&n->lpart, sizeof(double) * 2 * loss_blocks()));
  *out = n.release();
  return IRO_OK;
}

int iro_ptc_destroy(iro_ptc* n) {
  if (!n) return IRO_BAD_ARG;
  // cudaFree waits for the device's work on these buffers; the context may be gone
  cudaSetDevice(n->dev);
  for (void* p : n->bop) cudaFree(p);
  for (void* p : n->bopT) cudaFree(p);
  for (float* p : n->db) cudaFree(p);
  for (float2* p : n->act) cudaFree(p);
  void* ps[] = {n->g0, n->g1, n->da, n->partial, n->err, n->lpart};
  for (void* p : ps)
    if (p) cudaFree(p);
  delete n;
  return IRO_OK;
}

int iro_ptc_set_weights(iro_ptc* n, int layer, const float* w) {
  if (!n || !w || layer < 0 || layer >= n->nl) return IRO_BAD_ARG;
  iro_ctx* c = n->ctx;
  LCK(cudaSetDevice(device(c)));
  const int cin = n->w[layer], cout = n->w[layer + 1];
  n->W[layer].assign(w, w + size_t(9) * cout * cin * 2);
  std::vector<__nv_bfloat16> b, bt;
  pack_bop(cin, cout, n->W[layer], b, bt);
  LCK(cudaMemcpyAsync(n->bop[layer], b.data(), b.size() * 2, cudaMemcpyHostToDevice, stream(c)));
  LCK(cudaMemcpyAsync(n->bopT[layer], bt.data(), bt.size() * 2, cudaMemcpyHostToDevice, stream(c)));
  LCK(cudaStreamSynchronize(stream(c)));
  return IRO_OK;
}

static bool same_lattice(iro_ctx* c, const iro_ptc* n) {
  return volume(c) == volume(n->ctx) && geom(c).L[0] == geom(n->ctx).L[0] &&
         geom(c).L[1] == geom(n->ctx).L[1] && geom(c).L[2] == geom(n->ctx).L[2];
}

int iro_ptc_apply_field(iro_ctx* c, iro_ptc* n, const iro_field* in, iro_field* out) {
  if (!c || !n || !in || !out) return IRO_BAD_ARG;
  if (!same_lattice(c, n)) return set_error(c, IRO_BAD_ARG, "network built for another lattice");
  const DevField* fi = field_dev(const_cast<iro_field*>(in));
  DevField* fo = field_dev(out);
  if (fi->subset != 2 || fo->subset != 2 || fi->nrhs != 1 || fo->nrhs != 1 || fi->prec == PREC_HALF ||
      fo->prec == PREC_HALF)
    return set_error(c, IRO_BAD_ARG, "network fields must be full-lattice FP32/FP64, one rhs");
  if (!gauge_su3(c)) return set_error(c, IRO_NO_GAUGE, "network needs an SU(3) gauge field");
  LCK(cudaSetDevice(device(c)));
  LRC(field_to_feat(c, *fi, n->act[0]));
  LRC(forward(c, n));
  LRC(feat_to_field(c, n->act[n->nl], *fo));
  return check_err(c, n);
}

int iro_ptc_apply(iro_ctx* c, iro_ptc* n, const double* in, double* out) {
  if (!c || !n || !in || !out) return IRO_BAD_ARG;
  if (!same_lattice(c, n)) return set_error(c, IRO_BAD_ARG, "network built for another lattice");
  if (!gauge_su3(c)) return set_error(c, IRO_NO_GAUGE, "network needs an SU(3) gauge field");
  LCK(cudaSetDevice(device(c)));
  int rc = IRO_OK;
  DevField* a = workspace(c, 2, PREC_DOUBLE, 1, 72, &rc);
  if (!a) return rc;
  DevField* b = workspace(c, 2, PREC_DOUBLE, 1, 73, &rc);
  if (!b) return rc;
  LRC(import_field(c, in, true, *a));
  LRC(field_to_feat(c, *a, n->act[0]));
  LRC(forward(c, n));
  LRC(check_err(c, n));
  LRC(feat_to_field(c, n->act[n->nl], *b));
  return export_field(c, *b, true, out);
}

int iro_ptc_loss_grad(iro_ctx* c, iro_ptc* n, const iro_field* in, const iro_field* target,
                      double* loss, float* grad) {
  if (!c || !n || !in || !target || !loss) return IRO_BAD_ARG;
  if (!same_lattice(c, n)) return set_error(c, IRO_BAD_ARG, "network built for another lattice");
  const DevField* fi = field_dev(const_cast<iro_field*>(in));
  const DevField* ft = field_dev(const_cast<iro_field*>(target));
  if (fi->subset != 2 || ft->subset != 2 || fi->nrhs != 1 || ft->nrhs != 1)
    return set_error(c, IRO_BAD_ARG, "training fields must be full-lattice, one rhs");
  if (!gauge_su3(c)) return set_error(c, IRO_NO_GAUGE, "network needs an SU(3) gauge field");
  LCK(cudaSetDevice(device(c)));
  cudaStream_t st = stream(c);
  const int V = int(volume(c));
  LRC(field_to_feat(c, *fi, n->act[0]));
  LRC(forward(c, n));
  // target features into g1, loss and dL/dy into g0
  LRC(field_to_feat(c, *ft, n->g1));
  const int nel = V * 12;
  LCK(launch_loss_partials(nel, n->act[n->nl], n->g1, n->lpart, st));
  std::vector<double> part(2 * loss_blocks());
  LCK(cudaMemcpyAsync(part.data(), n->lpart, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st));
  LCK(cudaStreamSynchronize(st));
  double dd = 0.0, tt = 0.0;
  for (int b = 0; b < loss_blocks(); ++b) {
    dd += part[2 * b];
    tt += part[2 * b + 1];
  }
  *loss = dd / tt;
  if (!grad) return check_err(c, n);
  LCK(launch_loss_grad(nel, n->act[n->nl], n->g1, float(2.0 / tt), n->g0, st));
  PtcGeo G = make_geo(c, n->err);
  float2* dy = n->g0;
  float2* dx = n->g1;
  std::vector<size_t> goff(n->nl + 1, 0);
  for (int l = 0; l < n->nl; ++l) goff[l + 1] = goff[l] + size_t(9) * n->w[l + 1] * n->w[l] * 2;
  for (int l = n->nl - 1; l >= 0; --l) {
    const int cin = n->w[l], cout = n->w[l + 1];
    LCK(launch_ptc_bwd(cin, cout, G, n->act[l], dy, n->da, l > 0 ? dx : nullptr, n->bopT[l],
                       n->partial, n->db[l], st));
    int kf, kp, nf, np;
    ptc_dims(cin, cout, &kf, &kp, &nf, &np);
    std::vector<float> dB(size_t(nf) * kf);
    LCK(cudaMemcpyAsync(dB.data(), n->db[l], dB.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
    LCK(cudaStreamSynchronize(st));
    unpack_grad(cin, cout, dB, grad + goff[l]);
    std::swap(dy, dx);
  }
  return check_err(c, n);
}

// ---- flexible GCR on A = D^dag D with the network as right preconditioner ---------------
int iro_gcr_solve_field(iro_ctx* c, int op, double mass, double csw, const iro_ptc* net,
                        const iro_gcr_params* prm, const iro_field* b, iro_field* x, iro_gcr_out* out) {
  const DevField* B = field_dev(const_cast<iro_field*>(b));
  DevField* X = field_dev(x);
  if (!c || !prm || !B || !X || !out || (op != IRO_OP_WILSON_FULL && op != IRO_OP_CLOVER_FULL) ||
      B->subset != 2 || X->subset != 2 || B->prec != PREC_DOUBLE || X->prec != PREC_DOUBLE ||
      B->nrhs != 1 || X->nrhs != 1 || prm->nkrylov < 1 || prm->nkrylov > kMaxVec ||
      !(prm->precision > 0.0))
    return set_error(c, IRO_BAD_ARG, "bad GCR arguments");
  if (net && !same_lattice(c, net)) return set_error(c, IRO_BAD_ARG, "network built for another lattice");
  LCK(cudaSetDevice(device(c)));
  auto t0 = std::chrono::steady_clock::now();
  cudaStream_t st = stream(c);
  const int m = prm->nkrylov;
  int rc = IRO_OK;
  DevField* R = workspace(c, 2, PREC_DOUBLE, 1, 80, &rc); if (!R) return rc;
  DevField* Q = workspace(c, 2, PREC_DOUBLE, 1, 81, &rc); if (!Q) return rc;
  DevField* S = workspace(c, 2, PREC_DOUBLE, 1, 82, &rc); if (!S) return rc;
  DevField* r32 = workspace(c, 2, PREC_SINGLE, 1, 83, &rc); if (!r32) return rc;
  DevField* e32 = workspace(c, 2, PREC_SINGLE, 1, 84, &rc); if (!e32) return rc;
  // the Krylov fields z_j, w_j (and D z_j) in FP32 or FP16
  const int kp = prm->krylov_half ? PREC_HALF : PREC_SINGLE;
  DevField* tk = workspace(c, 2, kp, 1, 85, &rc); if (!tk) return rc;
  std::vector<DevField*> Z(m), W(m);
  for (int j = 0; j < m; ++j) {
    Z[j] = workspace(c, 2, kp, 1, 90 + j, &rc); if (!Z[j]) return rc;
    W[j] = workspace(c, 2, kp, 1, 90 + kMaxVec + j, &rc); if (!W[j]) return rc;
  }
  const int64_t nel = R->sites();
  const int blocks = 148 * 8;  // inner-product partials: 8 blocks of 128 threads per SM
  // block partials, the first and second passes' sums, then the cycle state
  const size_t sum_off = size_t(blocks) * 2 * kMaxList;
  const size_t state_off = sum_off + 4 * kMaxList;
  // (the context's solver scratch: a solve allocates nothing)
  const size_t mask_off = sizeof(double) * state_off + (sizeof(GcrState) + 15) / 16 * 16;
  char* scr = static_cast<char*>(scratch(c, mask_off + 16, &rc));
  if (!scr) return rc;
  double* part = reinterpret_cast<double*>(scr);
  double* dsum = part + sum_off;
  double* dsum2 = dsum + 2 * kMaxList;
  GcrState* gs = reinterpret_cast<GcrState*>(part + state_off);
  int* dmask = reinterpret_cast<int*>(scr + mask_off);
  // the cycle's iteration count comes back through the context's pinned host
  // buffer (the solvers use its first bytes for their flags; GCR does not run
  // beside them)
  int* hjdone = reinterpret_cast<int*>(static_cast<char*>(pinned(c)) + 2048);
  // x = 0, r = b
  LRC(axpby(c, 0.0, *B, 0.0, *B, *X));
  LRC(axpby(c, 1.0, *B, 0.0, *B, *R));
  std::vector<double> bn;
  LRC(norms(c, *B, nullptr, bn, nullptr));
  const double target = prm->precision * bn[0];
  double rr = bn[0];
  const double delta = prm->delta > 0.0 ? prm->delta : 0.1;
  int iters = 0, restarts = 0, fallback = 0, pcapplies = 0, stalls = 0;
  bool converged = rr < target || rr == 0.0;  // b = 0: x = 0 is the solution
  LCK(launch_fill_int(dmask, 1, st));
  while (!converged && iters < prm->max_iter) {
    // One restart cycle, enqueued whole: the coefficients of every iteration
    // are formed on the device (gcr_coef_kernel), and the iterations after
    // the one that meets the restart test (|r|^2 below delta^2 of its value
    // at the cycle start, or the target) return at once.  The z_j are kept as
    // the network produced them; the orthogonalised directions are z'_j =
    // sum_i T[i][j] z_i (T unit upper triangular, from the Gram-Schmidt
    // coefficients of the w_j), and the correction of the cycle e = sum_j
    // alpha_j z'_j = sum_i gamma_i z_i is formed once at its end.
    const int cyc = std::min(m, prm->max_iter - iters);
    LRC(convert(c, *R, *r32));
    LRC(axpby(c, 0.0, *r32, 0.0, *r32, *e32));
    LCK(launch_gcr_init(gs, rr, target, delta * delta, cyc, st));
    for (int j = 0; j < cyc; ++j) {
      const int* skip = &gs->skip[j];
      // z_j = N(r) (or r without a network), w_j = A z_j
      if (net) {
        // the features of r: the previous iteration's update wrote them
        // unless it took the second pass (plain[j - 1] = 0)
        LRC(field_to_feat(c, *r32, net->act[0], j == 0 ? skip : &gs->plain[j - 1]));
        LRC(forward(c, const_cast<iro_ptc*>(net), skip));
        LRC(feat_to_field(c, net->act[net->nl], *Z[j], skip));
      } else if (kp == PREC_SINGLE) {
        LRC(axpby(c, 1.0, *r32, 0.0, *r32, *Z[j]));
      } else {
        LRC(convert(c, *r32, *Z[j]));
      }
      LRC(apply(c, op, mass, csw, false, *Z[j], *tk, nullptr, 0, skip));
      LRC(apply(c, op, mass, csw, true, *tk, *W[j], nullptr, 0, skip));
      // one pass forms <w_q, w_j> (q < j), |w_j|^2 and <r, w_j>; the
      // coefficient kernel turns them into beta_q, |w'_j|^2 and alpha, and a
      // second pass orthogonalises w_j and updates r -= alpha w'_j
      CFieldList L{};
      for (int q = 0; q <= j; ++q) L.f[q] = W[q]->all();
      L.f[j + 1] = r32->all();
      LCK(launch_cdot(nel, j + 2, L, W[j]->all(), part, blocks, dsum, skip, kp, st));
      LCK(launch_gcr_coef(gs, dsum, j, m, 0, st));
      LCK(launch_gcr_update(nel, j, L, kp, gs, j, W[j]->all(), r32->all(),
                            net ? net->act[0] : nullptr, st));
      // w_j nearly in the span of the w_q (plain[j] = 0): |w'_j|^2 and
      // <r, w'_j> from the orthogonalised vector, then r -= alpha w'_j
      const int* single = &gs->plain[j];
      CFieldList L2{};
      L2.f[0] = W[j]->all();
      L2.f[1] = r32->all();
      LCK(launch_cdot(nel, 2, L2, W[j]->all(), part, blocks, dsum2, single, kp, st));
      LCK(launch_gcr_coef(gs, dsum2, j, m, 1, st));
      LCK(launch_caxpy_dev(nel, 1, L2, kp, gs, nullptr, -1.f, r32->all(), single, st));
    }
    // e = sum_i gamma_i z_i, gamma = T alpha over the iterations done
    {
      LCK(launch_gcr_gamma(gs, st));
      CFieldList L{};
      for (int i = 0; i < cyc; ++i) L.f[i] = Z[i]->all();
      LCK(launch_caxpy_dev(nel, cyc, L, kp, gs, &gs->jdone, 1.f, e32->all(), nullptr, st));
      LCK(cudaMemcpyAsync(hjdone, &gs->jdone, sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    // x += e, r = b - A x in FP64
    LCK(launch_mx_merge(PREC_SINGLE, X->sites(), 1, X->all(), e32->all(), dmask, st));
    LRC(apply(c, op, mass, csw, false, *X, *Q, nullptr, 0, nullptr));
    LRC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, nullptr));
    LRC(axpby(c, 1.0, *B, -1.0, *S, *R));
    std::vector<double> rnorm;
    LRC(norms(c, *R, nullptr, rnorm, nullptr));
    const int jd = *hjdone;  // copied before the norms, which synchronise the stream
    iters += jd;
    if (net) pcapplies += jd;
    ++restarts;
    stalls = (rnorm[0] > 0.25 * rr) ? stalls + 1 : 0;
    rr = rnorm[0];
    converged = rr < target;
    if (!std::isfinite(rr)) break;
    if (!converged && stalls >= 2) {
      // the preconditioned iteration stalls: finish with mixed-precision CG on
      // the correction A e = r, then x += e
      iro_cg_params cp{prm->precision * bn[0] / rr, prm->max_iter, IRO_PREC_SINGLE, 0.1, 1};
      DevField* E = workspace(c, 2, PREC_DOUBLE, 1, 86, &rc); if (!E) return rc;
      iro_solver_out co;
      const int crc = cg_any_dev(c, op, mass, csw, &cp, R, E, 1, &co);
      if (crc != IRO_OK && crc != IRO_NOT_CONVERGED) return crc;
      LRC(axpby(c, 1.0, *X, 1.0, *E, *X));
      LRC(apply(c, op, mass, csw, false, *X, *Q, nullptr, 0, nullptr));
      LRC(apply(c, op, mass, csw, true, *Q, *S, nullptr, 0, nullptr));
      LRC(axpby(c, 1.0, *B, -1.0, *S, *R));
      LRC(norms(c, *R, nullptr, rnorm, nullptr));
      rr = rnorm[0];
      converged = rr < target;
      iters += co.iterations > 0 ? co.iterations : 0;
      fallback = 1;
      break;
    }
  }
  auto t1 = std::chrono::steady_clock::now();
  out->diff = bn[0] > 0.0 ? std::sqrt(rr / bn[0]) : 0.0;
  out->iterations = converged ? iters : -1;
  out->timing_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  out->restarts = restarts;
  out->fallback = fallback;
  out->precond_applies = pcapplies;
  if (net) {
    int e = check_err(c, const_cast<iro_ptc*>(net));
    if (e) return e;
  }
  if (!converged) return set_error(c, IRO_NOT_CONVERGED, "GCR not converged");
  return IRO_OK;
}

int iro_selftest_bounded_wait(iro_ctx* c, double limit_ms, double* waited_ms) {
  if (!c || !waited_ms || !(limit_ms > 0.0) || limit_ms > 1000.0) return IRO_BAD_ARG;
  LCK(cudaSetDevice(device(c)));
  cudaStream_t st = stream(c);
  int* err = nullptr;
  unsigned long long* ns = nullptr;
  LCK(cudaMalloc(reinterpret_cast<void**>(&err), sizeof(int)));
  const cudaError_t e0 = cudaMalloc(reinterpret_cast<void**>(&ns), sizeof(unsigned long long));
  if (e0 != cudaSuccess) {
    cudaFree(err);
    return cuda_error(c, e0, "cudaMalloc");
  }
  int herr = 0;
  unsigned long long hns = 0;
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), st);
  if (e == cudaSuccess) e = launch_bounded_wait_probe(uint64_t(limit_ms * 1e6), err, ns, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hns, ns, sizeof(hns), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(err);
  cudaFree(ns);
  if (e != cudaSuccess) return cuda_error(c, e, "bounded-wait self-test");
  *waited_ms = double(hns) * 1e-6;
  if (herr) return set_error(c, IRO_TIMEOUT, "bounded wait ran out (self-test)");
  return IRO_OK;
}

}  // extern "C"
