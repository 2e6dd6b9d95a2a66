// The two-right-hand-sides-per-thread stencil with its neighbour data staged
// through shared memory by cp.async, three half-directions ahead of use.
//
// hop_pair_kernel waits on every link and neighbour load where it is used:
// at the occupancy its 128 registers allow (15 warps per SM) the stencil
// stalls on load latency most of the time.  Here each thread copies the data
// of a half-direction (the link and the neighbour pair of one of the 8
// hops) into a private shared-memory slot with cp.async and computes on the
// slot filled three steps earlier, so four half-directions are in flight per
// thread without holding registers.  The 8 half-directions of a site are a
// static sequence: a thread issues items 3..7 of its site and then items 0..2
// of its next site (grid stride) while it computes items 0..7, so every
// stage index and neighbour lookup is known at compile time.
//
// Shared memory per thread and stage, in 16-byte slots laid out
// [thread][stage][slot], each thread's block padded by 16 bytes so that the
// 8 threads of a quarter warp start on different bank groups (no conflicts
// for 16-byte accesses); slot offsets within a thread are compile-time
// constants:
//   FP16: 6 spinor slots (3 chunks x 2 elements), the link's first 16 bytes,
//         and (norm pair, link's last 8 bytes);
//   FP32: 12 spinor slots (6 chunks x 2 elements) and 3 link slots.
// A thread only reads its own slots after cp.async.wait_group, which makes its
// own copies visible to it: no block barrier is needed.
#pragma once

#include "dslash_pair.cuh"

namespace iro {

constexpr int kStages = 4;  // 3 half-directions ahead of the one computed

__device__ __forceinline__ uint32_t smem_u32_generic(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

template <int SP>
struct StageSlots;
template <>
struct StageSlots<PREC_HALF> {
  static constexpr int N = 8;
};
template <>
struct StageSlots<PREC_SINGLE> {
  static constexpr int N = 15;
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// bytes of one thread's stages (padded by one slot)
template <int SP>
__host__ __device__ constexpr int stage_bytes() {
  return (kStages * StageSlots<SP>::N + 1) * 16;
}

// byte address of slot k of stage s, from this thread's first slot
__device__ __forceinline__ uint32_t slot_addr(uint32_t tbase, int s, int k, int nslots) {
  return tbase + uint32_t((s * nslots + k) * 16);
}

// Issues the copies of half-direction HD (mu = HD/2, backward if HD odd) of
// output site hs (parity p, neighbours nb) into stage S.
template <int SP, int HD, int S>
__device__ __forceinline__ void stage_issue(const GaugePtr& gauge, const SpinorPtr& in, int p,
                                            int hs, const int nb[8], int nrhs, int r0,
                                            uint32_t base) {
  constexpr int MU = HD >> 1;
  constexpr bool BWD = HD & 1;
  constexpr int NS = StageSlots<SP>::N;
  const int n = nb[HD];
  const int lp = BWD ? 1 - p : p;
  const int ls = BWD ? n : hs;
  const int64_t e0 = int64_t(n) * nrhs + r0;
  if constexpr (SP == PREC_HALF) {
    const uint4* sp = chunk0<3>(static_cast<const uint4*>(in.data), e0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      cp_async16(slot_addr(base, S, 2 * k, NS), sp + 32 * k);
      cp_async16(slot_addr(base, S, 2 * k + 1, NS), sp + 32 * k + 1);
    }
    const int64_t j = int64_t(lp * 4 + MU) * gauge.Vh + ls;
    cp_async16(slot_addr(base, S, 6, NS), static_cast<const uint4*>(gauge.a) + j);
    cp_async8(slot_addr(base, S, 7, NS), in.norm + uint32_t(e0));
    cp_async8(slot_addr(base, S, 7, NS) + 8, static_cast<const uint2*>(gauge.b) + j);
  } else {
    const float4* sp = chunk0<6>(static_cast<const float4*>(in.data), e0);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      cp_async16(slot_addr(base, S, 2 * k, NS), sp + 32 * k);
      cp_async16(slot_addr(base, S, 2 * k + 1, NS), sp + 32 * k + 1);
    }
    const float4* q = link_chunk0<3>(static_cast<const float4*>(gauge.a), gauge.Vh, lp, MU, ls);
#pragma unroll
    for (int k = 0; k < 3; ++k) cp_async16(slot_addr(base, S, 12 + k, NS), q + 32 * k);
  }
}

// Computes half-direction HD from stage S into acc: raw pair chunks, the
// FP16 norms, and the link read back from the thread's slots, then decoded
// one colour at a time.
template <int SP, int HD, int S, bool DAG>
__device__ __forceinline__ void stage_compute(const uint4* sm, Cp acc[12]) {
  constexpr int MU = HD >> 1;
  constexpr bool BWD = HD & 1;
  // forward hop: projector (1 - g_mu) [dagger (1 + g_mu)], U; backward: the opposite, U^dag
  constexpr int SG = (BWD ? -1 : 1) * (DAG ? -1 : 1);
  constexpr int NS = StageSlots<SP>::N;
  // plain shared-memory loads (ordered after the copies by cp_wait's clobber)
  auto lds = [&](int k) { return sm[S * NS + k]; };
  RawPair<SP> raw;
  float2 w;
  Su3<float> U;
  if constexpr (SP == PREC_HALF) {
#pragma unroll
    for (int k = 0; k < 6; ++k) raw.v[k] = lds(k);
    const uint4 la = lds(6), nl = lds(7);
    w = make_float2(__uint_as_float(nl.x), __uint_as_float(nl.y));
    float2 t;
    t = unpack_h2(la.x); U.e[0][0] = {t.x, t.y};
    t = unpack_h2(la.y); U.e[0][1] = {t.x, t.y};
    t = unpack_h2(la.z); U.e[0][2] = {t.x, t.y};
    t = unpack_h2(la.w); U.e[1][0] = {t.x, t.y};
    t = unpack_h2(nl.z); U.e[1][1] = {t.x, t.y};
    t = unpack_h2(nl.w); U.e[1][2] = {t.x, t.y};
  } else {
#pragma unroll
    for (int k = 0; k < 12; ++k) raw.v[k] = lds(k);
    const uint4 a = lds(12), b = lds(13), c = lds(14);
    U.e[0][0] = {__uint_as_float(a.x), __uint_as_float(a.y)};
    U.e[0][1] = {__uint_as_float(a.z), __uint_as_float(a.w)};
    U.e[0][2] = {__uint_as_float(b.x), __uint_as_float(b.y)};
    U.e[1][0] = {__uint_as_float(b.z), __uint_as_float(b.w)};
    U.e[1][1] = {__uint_as_float(c.x), __uint_as_float(c.y)};
    U.e[1][2] = {__uint_as_float(c.z), __uint_as_float(c.w)};
    w = bc(1.f);
  }
  reconstruct_row2(U);
  half_dir_raw<SP, MU, SG, BWD>(raw, w, U, acc);
}

// One pipeline step: issue item HD+3 (of this site, or of the next site for
// HD >= 5), wait for item HD, compute it.
template <int SP, int HD, bool DAG>
__device__ __forceinline__ void stage_step(const HopParams& P, int yi, int p, int hs, int nb[8],
                                           int nhs, bool has_next, int r0, uint32_t base,
                                           const uint4* sm, Cp acc[12]) {
  constexpr int NXT = HD + kStages - 1;  // item index issued at this step
  if (NXT < 8) {
    stage_issue<SP, NXT & 7, NXT % kStages>(P.gauge, P.in[yi], p, hs, nb, P.nrhs, r0, base);
  } else {
    if (NXT == 8 && has_next) {
      // the current site's neighbours are no longer needed: switch to the next site
      const Coord c = coord_of(P.g, nhs, p);
      neighbours(P.g, c, nhs, nb);
    }
    if (has_next)
      stage_issue<SP, NXT & 7, NXT % kStages>(P.gauge, P.in[yi], p, nhs, nb, P.nrhs, r0, base);
  }
  cp_commit();
  cp_wait<kStages - 1>();
  stage_compute<SP, HD, HD % kStages, DAG>(sm, acc);
}

template <int SP, bool DAG, int EPI, int VAR>
__global__ void __launch_bounds__(256, (VAR & 1) ? 2 : 1) hop_stage_kernel(HopParams P) {
  extern __shared__ __align__(16) unsigned char stage_smem[];
  // this thread's slots
  const uint32_t base = smem_u32_generic(stage_smem) + threadIdx.x * stage_bytes<SP>();
  const uint4* sm = reinterpret_cast<const uint4*>(stage_smem + threadIdx.x * stage_bytes<SP>());
  const int yi = blockIdx.y;
  const int p = P.p0 ^ yi;
  const int nrhs = P.nrhs;
  const int lanes = nrhs >> 1;
  const int nthreads = P.g.Vh * lanes;  // < 2^31, checked at context creation
  const int stride = gridDim.x * blockDim.x;
  double red[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const int q = (lanes == 1) ? 0 : int((blockIdx.x * blockDim.x + threadIdx.x) % unsigned(lanes));
  const int r0 = 2 * q;
  const bool idle = P.skip && P.skip[r0] && P.skip[r0 + 1];
  int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (!idle && tid < nthreads) {
    int hs = (lanes == 1) ? tid : int(unsigned(tid) / unsigned(lanes));
    int nb[8];
    {
      const Coord c = coord_of(P.g, hs, p);
      neighbours(P.g, c, hs, nb);
    }
    // prologue: items 0..2 of the first site
    stage_issue<SP, 0, 0>(P.gauge, P.in[yi], p, hs, nb, nrhs, r0, base);
    cp_commit();
    stage_issue<SP, 1, 1>(P.gauge, P.in[yi], p, hs, nb, nrhs, r0, base);
    cp_commit();
    stage_issue<SP, 2, 2>(P.gauge, P.in[yi], p, hs, nb, nrhs, r0, base);
    cp_commit();
    for (;;) {
      const int ntid = tid + stride;
      const bool has_next = ntid < nthreads;
      const int nhs = (lanes == 1) ? ntid : int(unsigned(ntid) / unsigned(lanes));
      Cp acc[12];
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[k] = {bc(0.f), bc(0.f)};
      stage_step<SP, 0, DAG>(P, yi, p, hs, nb, nhs, has_next, r0, base, sm, acc);
      stage_step<SP, 1, DAG>(P, yi, p, hs, nb, nhs, has_next, r0, base, sm, acc);
      stage_step<SP, 2, DAG>(P, yi, p, hs, nb, nhs, has_next, r0, base, sm, acc);
      stage_step<SP, 3, DAG>(P, yi, p, hs, nb, nhs, has_next, r0, base, sm, acc);
      stage_step<SP, 4, DAG>(P, yi, p, hs, nb, nhs, has_next, r0, base, sm, acc);
      stage_step<SP, 5, DAG>(P, yi, p, hs, nb, nhs, has_next, r0, base, sm, acc);
      stage_step<SP, 6, DAG>(P, yi, p, hs, nb, nhs, has_next, r0, base, sm, acc);
      stage_step<SP, 7, DAG>(P, yi, p, hs, nb, nhs, has_next, r0, base, sm, acc);
      pair_epilogue<SP, EPI>(P, yi, hs, int64_t(hs) * nrhs + r0, r0, acc, red);
      if (!has_next) break;
      tid = ntid;
      hs = nhs;
    }
    cp_wait<0>();
  }
  if (P.red_mask || P.cg)
    block_reduce_finish<3, 2>(P.red, red, nrhs, blockIdx.y * gridDim.x + blockIdx.x,
                              gridDim.x * gridDim.y);
}

}  // namespace iro
