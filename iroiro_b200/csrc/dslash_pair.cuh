// The FP32/FP16 hopping stencil with two right-hand sides per thread, in the
// packed FP32x2 arithmetic of sm_100 (__ffma2_rn, __fadd2_rn, __fmul2_rn).
//
// For an even number of right-hand sides, lane q of a site computes
// right-hand sides 2q and 2q+1.  Both run through one instruction stream with
// their values in the two halves of a float2 ("pair"), so
//   * every link (load, FP16 conversion, reconstruction of row 2) and every
//     neighbour index serves two right-hand sides, and
//   * each FP32 add or multiply-add of projection, SU(3) product and
//     reconstruction is one instruction for both.
// The spin algebra is that of hop_kernel (Dirac_Wilson::mult_offdiag,
// lib/Dirac_ops/dirac_wilson.cpp:107-113, per-direction projection as in
// lib/Dirac_ops/dirac_wilson_improved.code:5-648).  Arithmetic stays FP32;
// only the association of the sums differs from hop_kernel, so results agree
// with it to FP32 rounding, not bit for bit.  The two elements of a pair are
// adjacent in the warp-blocked layout (elements hs*nrhs + 2q and +1, never
// split across a 32-element block since 2q is even), so a pair is two
// neighbouring 16-byte chunks per chunk index.
#pragma once

#include "dslash.cuh"

namespace iro {

// one complex number of each of two right-hand sides
struct Cp {
  float2 re, im;
};

__device__ __forceinline__ float2 bc(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __ffma2_rn(b, bc(-1.f), a); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }

__device__ __forceinline__ Cp cadd(Cp a, Cp b) { return {padd(a.re, b.re), padd(a.im, b.im)}; }
__device__ __forceinline__ Cp csub(Cp a, Cp b) { return {psub(a.re, b.re), psub(a.im, b.im)}; }
// a + i b, a - i b
__device__ __forceinline__ Cp cadd_i(Cp a, Cp b) { return {psub(a.re, b.im), padd(a.im, b.re)}; }
__device__ __forceinline__ Cp csub_i(Cp a, Cp b) { return {padd(a.re, b.im), psub(a.im, b.re)}; }

// ---- pair storage access -------------------------------------------------------------
template <int SP>
struct PairIO;

template <>
struct PairIO<PREC_SINGLE> {
  // elements i0, i0+1 (i0 even); w = (1, 1)
  __device__ __forceinline__ static void load(const SpinorPtr& s, int64_t i0, Cp f[12], float2& w) {
    const float4* p = chunk0<6>(static_cast<const float4*>(s.data), i0);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const float4 a = __ldg(p + 32 * k), b = __ldg(p + 32 * k + 1);
      f[2 * k] = {make_float2(a.x, b.x), make_float2(a.y, b.y)};
      f[2 * k + 1] = {make_float2(a.z, b.z), make_float2(a.w, b.w)};
    }
    w = bc(1.f);
  }
  __device__ __forceinline__ static void load_scaled(const SpinorPtr& s, int64_t i0, Cp f[12]) {
    float2 w;
    load(s, i0, f, w);
  }
  __device__ __forceinline__ static void store(const SpinorPtr& s, int64_t i0, const Cp v[12]) {
    float4* p = chunk0<6>(static_cast<float4*>(s.data), i0);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const Cp a = v[2 * k], b = v[2 * k + 1];
      p[32 * k] = make_float4(a.re.x, a.im.x, b.re.x, b.im.x);
      p[32 * k + 1] = make_float4(a.re.y, a.im.y, b.re.y, b.im.y);
    }
  }
};

template <>
struct PairIO<PREC_HALF> {
  // the stored (normalised) values of elements i0, i0+1 and their norms w
  __device__ __forceinline__ static void load(const SpinorPtr& s, int64_t i0, Cp f[12], float2& w) {
    const uint4* p = chunk0<3>(static_cast<const uint4*>(s.data), i0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const uint4 a = __ldg(p + 32 * k), b = __ldg(p + 32 * k + 1);
      const uint32_t av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const float2 x = unpack_h2(av[m]), y = unpack_h2(bv[m]);
        f[4 * k + m] = {make_float2(x.x, y.x), make_float2(x.y, y.y)};
      }
    }
    w = __ldg(reinterpret_cast<const float2*>(s.norm + uint32_t(i0)));
  }
  __device__ __forceinline__ static void load_scaled(const SpinorPtr& s, int64_t i0, Cp f[12]) {
    float2 w;
    load(s, i0, f, w);
#pragma unroll
    for (int k = 0; k < 12; ++k) f[k] = {pmul(f[k].re, w), pmul(f[k].im, w)};
  }
  __device__ __forceinline__ static void store(const SpinorPtr& s, int64_t i0, const Cp v[12]) {
    float m0 = 0.f, m1 = 0.f;
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      m0 = fmaxf(m0, fmaxf(fabsf(v[k].re.x), fabsf(v[k].im.x)));
      m1 = fmaxf(m1, fmaxf(fabsf(v[k].re.y), fabsf(v[k].im.y)));
    }
    // the same subnormal flush as SpinorIO<PREC_HALF>::store
    if (!(m0 >= 1e-37f)) m0 = 0.f;
    if (!(m1 >= 1e-37f)) m1 = 0.f;
    const float2 inv = make_float2(m0 > 0.f ? 1.0f / m0 : 0.f, m1 > 0.f ? 1.0f / m1 : 0.f);
    uint4* p = chunk0<3>(static_cast<uint4*>(s.data), i0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      uint32_t a[4], b[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const float2 re = pmul(v[4 * k + m].re, inv), im = pmul(v[4 * k + m].im, inv);
        a[m] = pack_h2(re.x, im.x);
        b[m] = pack_h2(re.y, im.y);
      }
      p[32 * k] = make_uint4(a[0], a[1], a[2], a[3]);
      p[32 * k + 1] = make_uint4(b[0], b[1], b[2], b[3]);
    }
    *reinterpret_cast<float2*>(s.norm + uint32_t(i0)) = make_float2(m0, m1);
  }
};

// one right-hand side of a pair <-> a plain complex array (for the clover epilogue)
__device__ __forceinline__ void pair_get(const Cp v[12], int j, Cx<float> o[12]) {
#pragma unroll
  for (int k = 0; k < 12; ++k) o[k] = j ? Cx<float>{v[k].re.y, v[k].im.y} : Cx<float>{v[k].re.x, v[k].im.x};
}
__device__ __forceinline__ void pair_set(Cp v[12], int j, const Cx<float> o[12]) {
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    if (j) {
      v[k].re.y = o[k].re;
      v[k].im.y = o[k].im;
    } else {
      v[k].re.x = o[k].re;
      v[k].im.x = o[k].im;
    }
  }
}

// ---- spin projection / reconstruction (same gammas as project/reconstruct) -------------
// For the t direction the projector's factor 2 is left to the reconstruction
// weight, so the projection is a plain selection.
template <int MU, int S>
__device__ __forceinline__ void project_col(const Cp f0, const Cp f1, const Cp f2, const Cp f3, Cp& h0,
                                            Cp& h1) {
  if (MU == 0) {  // h0 = f0 + S i f3, h1 = f1 + S i f2
    h0 = (S > 0) ? cadd_i(f0, f3) : csub_i(f0, f3);
    h1 = (S > 0) ? cadd_i(f1, f2) : csub_i(f1, f2);
  } else if (MU == 1) {  // h0 = f0 + S f3, h1 = f1 - S f2
    h0 = (S > 0) ? cadd(f0, f3) : csub(f0, f3);
    h1 = (S > 0) ? csub(f1, f2) : cadd(f1, f2);
  } else if (MU == 2) {  // h0 = f0 + S i f2, h1 = f1 - S i f3
    h0 = (S > 0) ? cadd_i(f0, f2) : csub_i(f0, f2);
    h1 = (S > 0) ? csub_i(f1, f3) : cadd_i(f1, f3);
  } else {  // t: (2 f2, 2 f3) for S=+1, (2 f0, 2 f1) for S=-1; the 2 goes to the weight
    h0 = (S > 0) ? f2 : f0;
    h1 = (S > 0) ? f3 : f1;
  }
}

template <int MU, int S>
__device__ __forceinline__ void project_pair(const Cp f[12], Cp h[6]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) project_col<MU, S>(f[c], f[3 + c], f[6 + c], f[9 + c], h[c], h[3 + c]);
}

// a += w b, a += w (i b), a += w (-i b), with nw = -w
__device__ __forceinline__ void acc_w(Cp& a, float2 w, const Cp& b) {
  a.re = pfma(w, b.re, a.re);
  a.im = pfma(w, b.im, a.im);
}
__device__ __forceinline__ void acc_wi(Cp& a, float2 w, float2 nw, const Cp& b) {
  a.re = pfma(nw, b.im, a.re);
  a.im = pfma(w, b.re, a.im);
}
__device__ __forceinline__ void acc_wmi(Cp& a, float2 w, float2 nw, const Cp& b) {
  a.re = pfma(w, b.im, a.re);
  a.im = pfma(nw, b.re, a.im);
}

// acc (colour c) += w * (1 - S gamma_mu) reconstructed from g0 = g[c], g1 = g[3+c]
template <int MU, int S>
__device__ __forceinline__ void reconstruct_col(Cp acc[12], int c, const Cp g0, const Cp g1, float2 w,
                                                float2 nw) {
  if (MU == 3) {
    if (S > 0) {
      acc_w(acc[6 + c], w, g0);
      acc_w(acc[9 + c], w, g1);
    } else {
      acc_w(acc[c], w, g0);
      acc_w(acc[3 + c], w, g1);
    }
    return;
  }
  acc_w(acc[c], w, g0);
  acc_w(acc[3 + c], w, g1);
  if (MU == 0) {  // [h0, h1, -S i h1, -S i h0]
    if (S > 0) {
      acc_wmi(acc[6 + c], w, nw, g1);
      acc_wmi(acc[9 + c], w, nw, g0);
    } else {
      acc_wi(acc[6 + c], w, nw, g1);
      acc_wi(acc[9 + c], w, nw, g0);
    }
  } else if (MU == 1) {  // [h0, h1, -S h1, S h0]
    if (S > 0) {
      acc_w(acc[6 + c], nw, g1);
      acc_w(acc[9 + c], w, g0);
    } else {
      acc_w(acc[6 + c], w, g1);
      acc_w(acc[9 + c], nw, g0);
    }
  } else {  // MU==2: [h0, h1, -S i h0, S i h1]
    if (S > 0) {
      acc_wmi(acc[6 + c], w, nw, g0);
      acc_wi(acc[9 + c], w, nw, g1);
    } else {
      acc_wi(acc[6 + c], w, nw, g0);
      acc_wmi(acc[9 + c], w, nw, g1);
    }
  }
}

template <int MU, int S>
__device__ __forceinline__ void reconstruct_pair(Cp acc[12], const Cp g[6], float2 w) {
  const float2 nw = pmul(w, bc(-1.f));
#pragma unroll
  for (int c = 0; c < 3; ++c) reconstruct_col<MU, S>(acc, c, g[c], g[3 + c], w, nw);
}

// row a of g = U h (ADJ false) or U^dag h (ADJ true), for the colour vector
// h[0..2] of the pair; the link elements are broadcast to both lanes
template <bool ADJ>
__device__ __forceinline__ Cp su3_row(const Su3<float>& U, int a, const Cp h0, const Cp h1, const Cp h2) {
  const Cx<float> u0 = ADJ ? U.e[0][a] : U.e[a][0];
  const Cx<float> u1 = ADJ ? U.e[1][a] : U.e[a][1];
  const Cx<float> u2 = ADJ ? U.e[2][a] : U.e[a][2];
  float2 s1, s2, s3;
  if (!ADJ) {
    // re = sum ur h.re - sum ui h.im,  im = sum ur h.im + ui h.re
    s1 = pmul(bc(u0.re), h0.re);
    s1 = pfma(bc(u1.re), h1.re, s1);
    s1 = pfma(bc(u2.re), h2.re, s1);
    s2 = pmul(bc(u0.im), h0.im);
    s2 = pfma(bc(u1.im), h1.im, s2);
    s2 = pfma(bc(u2.im), h2.im, s2);
    s3 = pmul(bc(u0.re), h0.im);
    s3 = pfma(bc(u0.im), h0.re, s3);
    s3 = pfma(bc(u1.re), h1.im, s3);
    s3 = pfma(bc(u1.im), h1.re, s3);
    s3 = pfma(bc(u2.re), h2.im, s3);
    s3 = pfma(bc(u2.im), h2.re, s3);
    return {psub(s1, s2), s3};
  }
  // conj(u): re = sum ur h.re + ui h.im,  im = sum ur h.im - sum ui h.re
  s3 = pmul(bc(u0.re), h0.re);
  s3 = pfma(bc(u0.im), h0.im, s3);
  s3 = pfma(bc(u1.re), h1.re, s3);
  s3 = pfma(bc(u1.im), h1.im, s3);
  s3 = pfma(bc(u2.re), h2.re, s3);
  s3 = pfma(bc(u2.im), h2.im, s3);
  s1 = pmul(bc(u0.re), h0.im);
  s1 = pfma(bc(u1.re), h1.im, s1);
  s1 = pfma(bc(u2.re), h2.im, s1);
  s2 = pmul(bc(u0.im), h0.re);
  s2 = pfma(bc(u1.im), h1.re, s2);
  s2 = pfma(bc(u2.im), h2.re, s2);
  return {s3, psub(s1, s2)};
}

template <bool ADJ>
__device__ __forceinline__ void su3_pair(const Su3<float>& U, const Cp h[6], Cp g[6]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    g[a] = su3_row<ADJ>(U, a, h[0], h[1], h[2]);
    g[3 + a] = su3_row<ADJ>(U, a, h[3], h[4], h[5]);
  }
}

// ---- one half-direction from raw (undecoded) pair data -------------------------------
// raw[2k + j] is 16-byte chunk k of right-hand side j: FP16 holds complexes
// 4k..4k+3 of the element, FP32 complexes 2k, 2k+1 (complex i = 3*spin + colour).
template <int SP>
struct RawPair {
  uint4 v[SP == PREC_HALF ? 6 : 12];
};

template <int SP>
__device__ __forceinline__ Cp raw_get(const RawPair<SP>& r, int i) {
  if constexpr (SP == PREC_HALF) {
    const int k = i >> 2, m = i & 3;
    const uint4 a = r.v[2 * k], b = r.v[2 * k + 1];
    const uint32_t wa = m == 0 ? a.x : m == 1 ? a.y : m == 2 ? a.z : a.w;
    const uint32_t wb = m == 0 ? b.x : m == 1 ? b.y : m == 2 ? b.z : b.w;
    const float2 x = unpack_h2(wa), y = unpack_h2(wb);
    return {make_float2(x.x, y.x), make_float2(x.y, y.y)};
  } else {
    const int k = i >> 1;
    const uint4 a = r.v[2 * k], b = r.v[2 * k + 1];
    if (i & 1)
      return {make_float2(__uint_as_float(a.z), __uint_as_float(b.z)),
              make_float2(__uint_as_float(a.w), __uint_as_float(b.w))};
    return {make_float2(__uint_as_float(a.x), __uint_as_float(b.x)),
            make_float2(__uint_as_float(a.y), __uint_as_float(b.y))};
  }
}

// acc += w (1 - S gamma_mu) [U or U^dag] (1 - S gamma_mu)-projection of the
// neighbour pair, decoding one colour at a time (short live ranges)
template <int SP, int MU, int S, bool ADJ>
__device__ __forceinline__ void half_dir_raw(const RawPair<SP>& raw, float2 w, const Su3<float>& U,
                                             Cp acc[12]) {
  Cp h[6];
#pragma unroll
  for (int c = 0; c < 3; ++c)
    project_col<MU, S>(raw_get<SP>(raw, c), raw_get<SP>(raw, 3 + c), raw_get<SP>(raw, 6 + c),
                       raw_get<SP>(raw, 9 + c), h[c], h[3 + c]);
  if (MU == 3) w = pmul(w, bc(2.f));
  const float2 nw = pmul(w, bc(-1.f));
#pragma unroll
  for (int a = 0; a < 3; ++a)
    reconstruct_col<MU, S>(acc, a, su3_row<ADJ>(U, a, h[0], h[1], h[2]),
                           su3_row<ADJ>(U, a, h[3], h[4], h[5]), w, nw);
}

template <int SP>
__device__ __forceinline__ void load_raw_pair(const SpinorPtr& s, int64_t i0, RawPair<SP>& r,
                                              float2& w) {
  constexpr int NC = SP == PREC_HALF ? 3 : 6;
  const uint4* p = chunk0<NC>(static_cast<const uint4*>(s.data), i0);
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    r.v[2 * k] = __ldg(p + 32 * k);
    r.v[2 * k + 1] = __ldg(p + 32 * k + 1);
  }
  if constexpr (SP == PREC_HALF)
    w = __ldg(reinterpret_cast<const float2*>(s.norm + uint32_t(i0)));
  else
    w = bc(1.f);
}

// Forward and backward contributions of direction MU for the pair at
// element e0 (= site * nrhs + 2q) of every neighbour.
template <int MU, bool DAG, int SP>
__device__ __forceinline__ void hop_dir_pair(const GaugePtr& gauge, const SpinorPtr& in, int p,
                                             int hs, const int nb[8], int nrhs, int r0,
                                             Cp acc[12]) {
  {
    Su3<float> U;
    GaugeIO<SP, 12>::load(gauge, p, MU, hs, U);
    RawPair<SP> raw;
    float2 w;
    load_raw_pair<SP>(in, int64_t(nb[2 * MU]) * nrhs + r0, raw, w);
    half_dir_raw<SP, MU, DAG ? -1 : 1, false>(raw, w, U, acc);
  }
  {
    Su3<float> U;
    GaugeIO<SP, 12>::load(gauge, 1 - p, MU, nb[2 * MU + 1], U);
    RawPair<SP> raw;
    float2 w;
    load_raw_pair<SP>(in, int64_t(nb[2 * MU + 1]) * nrhs + r0, raw, w);
    half_dir_raw<SP, MU, DAG ? 1 : -1, true>(raw, w, U, acc);
  }
}

// Epilogue of one site for a pair: scale / clover / x + a*y, store, and the
// per-site FP32 sums of the reductions added to red[] in FP64.
template <int SP, int EPI>
__device__ __forceinline__ void pair_epilogue(const HopParams& P, int yi, int hs, int64_t e0,
                                              int r0, Cp acc[12], double red[6]) {
  const float2 sc = bc(float(P.scale));
  Cp xv[12];
  if (EPI == EPI_SCALE || EPI == EPI_SCALE_CLOV) {
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = {pmul(sc, acc[k].re), pmul(sc, acc[k].im)};
    if (EPI == EPI_SCALE_CLOV) {
      CloverBlock<float> B[2];
      CloverIO<SP>::load(P.clov[yi], hs, B);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        Cx<float> v[12];
        pair_get(acc, j, v);
        clover_apply(B, v);
        pair_set(acc, j, v);
      }
    }
  } else {
    PairIO<SP>::load_scaled(P.xin[yi], e0, xv);
    Cp ax[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) ax[k] = xv[k];
    if (EPI == EPI_XPAY_CLOV) {
      CloverBlock<float> B[2];
      CloverIO<SP>::load(P.clov[yi], hs, B);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        Cx<float> v[12];
        pair_get(ax, j, v);
        clover_apply(B, v);
        pair_set(ax, j, v);
      }
    }
#pragma unroll
    for (int k = 0; k < 12; ++k)
      acc[k] = {pfma(sc, acc[k].re, ax[k].re), pfma(sc, acc[k].im, ax[k].im)};
  }
  if (P.cg) {
    // r -= alpha s; |r|^2.  A lane whose right-hand side has left the
    // iteration gets alpha = 0 (its residual is re-stored unchanged).
    const float2 na = make_float2(P.skip && P.skip[r0] ? 0.f : -float(P.cst[r0].alpha),
                                  P.skip && P.skip[r0 + 1] ? 0.f : -float(P.cst[r0 + 1].alpha));
    Cp rv[12];
    PairIO<SP>::load_scaled(P.cr[yi], e0, rv);
    float2 rr = bc(0.f);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      rv[k] = {pfma(na, acc[k].re, rv[k].re), pfma(na, acc[k].im, rv[k].im)};
      rr = pfma(rv[k].re, rv[k].re, rr);
      rr = pfma(rv[k].im, rv[k].im, rr);
    }
    PairIO<SP>::store(P.cr[yi], e0, rv);
    red[0] += rr.x;
    red[3] += rr.y;
    return;
  }
  PairIO<SP>::store(P.out[yi], e0, acc);
  if (P.red_mask) {
    float2 o2 = bc(0.f), x2 = bc(0.f), xo = bc(0.f);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      o2 = pfma(acc[k].re, acc[k].re, o2);
      o2 = pfma(acc[k].im, acc[k].im, o2);
      if (EPI == EPI_XPAY || EPI == EPI_XPAY_CLOV) {
        x2 = pfma(xv[k].re, xv[k].re, x2);
        x2 = pfma(xv[k].im, xv[k].im, x2);
        xo = pfma(xv[k].re, acc[k].re, xo);
        xo = pfma(xv[k].im, acc[k].im, xo);
      }
    }
    red[0] += o2.x;
    red[1] += x2.x;
    red[2] += xo.x;
    red[3] += o2.y;
    red[4] += x2.y;
    red[5] += xo.y;
  }
}

// The stencil over pairs; same parameters, epilogues and reductions as
// hop_kernel.  A pair is skipped only when both its right-hand sides are
// flagged converged; a pair with one converged member still writes it (its
// outputs are scratch, and the solvers' stage updates ignore its sums).
// Per-site sums of the reductions are formed in FP32 and accumulated in FP64.
// VAR selects the register cap: none, 128, 152 or 168 registers per thread
// (the autotuner trades ILP against resident warps).
template <int VAR>
struct PairCap {
  static constexpr int regs = VAR == 1 ? 128 : (VAR == 2 ? 152 : (VAR == 3 ? 168 : 255));
};

template <int SP, bool DAG, int EPI, int VAR>
__global__ void __launch_bounds__(256) __maxnreg__(PairCap<VAR>::regs) hop_pair_kernel(HopParams P) {
  const int yi = blockIdx.y;
  const int p = P.p0 ^ yi;
  const int nrhs = P.nrhs;
  const int lanes = nrhs >> 1;
  const int nthreads = P.g.Vh * lanes;  // < 2^31, checked at context creation
  double red[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  // the grid stride is a multiple of lanes, so each thread keeps one pair
  const int q = (lanes == 1) ? 0 : int((blockIdx.x * blockDim.x + threadIdx.x) % unsigned(lanes));
  const int r0 = 2 * q;
  const bool idle = P.skip && P.skip[r0] && P.skip[r0 + 1];
  for (int tid = blockIdx.x * blockDim.x + threadIdx.x; tid < nthreads && !idle;
       tid += gridDim.x * blockDim.x) {
    const int hs = (lanes == 1) ? tid : int(unsigned(tid) / unsigned(lanes));
    const Coord c = coord_of(P.g, hs, p);
    int nb[8];
    neighbours(P.g, c, hs, nb);
    Cp acc[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = {bc(0.f), bc(0.f)};
    hop_dir_pair<0, DAG, SP>(P.gauge, P.in[yi], p, hs, nb, nrhs, r0, acc);
    hop_dir_pair<1, DAG, SP>(P.gauge, P.in[yi], p, hs, nb, nrhs, r0, acc);
    hop_dir_pair<2, DAG, SP>(P.gauge, P.in[yi], p, hs, nb, nrhs, r0, acc);
    hop_dir_pair<3, DAG, SP>(P.gauge, P.in[yi], p, hs, nb, nrhs, r0, acc);
    pair_epilogue<SP, EPI>(P, yi, hs, int64_t(hs) * nrhs + r0, r0, acc, red);
  }
  if (P.red_mask || P.cg)
    block_reduce_finish<3, 2>(P.red, red, nrhs, blockIdx.y * gridDim.x + blockIdx.x,
                              gridDim.x * gridDim.y);
}

}  // namespace iro
