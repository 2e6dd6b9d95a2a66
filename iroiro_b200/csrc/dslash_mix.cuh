// The FP16 hopping term in mixed precision, one right-hand side per thread:
// no FP16 -> FP32 conversions.
//
// sm_100 executes `fma.rn.f32.f16 d, a, b, c` (d = a * b + c with FP16 a, b
// and FP32 c, d) at the full FFMA rate, and the product of two FP16 numbers is
// exact in FP32, so the SU(3) product of an FP16 link with an FP16 half spinor
// can accumulate in FP32 straight from the stored halves.  The neighbour is
// projected in packed FP16 (one HADD2/HFMA2 per complex; the only rounding
// this path adds to the FP16 storage's), the links are the FP16 copies with
// all three rows stored (GaugeIO<PREC_HALF, 18> layout: no reconstruction)
// or with two (row 2 rebuilt per link, 12 bytes fewer per link), and the
// element norm joins the reconstruction's FP32 FMAs as a weight.
// The spin algebra is hop_kernel's (project / reconstruct above; Dirac_Wilson
// mult_offdiag, lib/Dirac_ops/dirac_wilson.cpp:107-113).
#pragma once

#include "common.cuh"

namespace iro {

// a.{lo,hi} * b.{lo,hi} + c with a, b pairs of FP16 in one 32-bit word
#define IRO_MFMA(NAME, A, B)                                                             \
  __device__ __forceinline__ float NAME(uint32_t a, uint32_t b, float c) {              \
    float d;                                                                             \
    asm("{\n\t.reg .f16 a0, a1, b0, b1;\n\tmov.b32 {a0, a1}, %1;\n\tmov.b32 {b0, b1}, %2;\n\t" \
        "fma.rn.f32.f16 %0, " A ", " B ", %3;\n\t}"                                      \
        : "=f"(d)                                                                        \
        : "r"(a), "r"(b), "f"(c));                                                       \
    return d;                                                                            \
  }
IRO_MFMA(mfma_ll, "a0", "b0")
IRO_MFMA(mfma_lh, "a0", "b1")
IRO_MFMA(mfma_hl, "a1", "b0")
IRO_MFMA(mfma_hh, "a1", "b1")
#undef IRO_MFMA

// -(a.{lo,hi} * b.{lo,hi}) + c, negating the FP16 operand
#define IRO_MFMA_NEG(NAME, A, B)                                                         \
  __device__ __forceinline__ float NAME(uint32_t a, uint32_t b, float c) {              \
    float d;                                                                             \
    asm("{\n\t.reg .f16 a0, a1, b0, b1, n;\n\tmov.b32 {a0, a1}, %1;\n\tmov.b32 {b0, b1}, %2;\n\t" \
        "neg.f16 n, " B ";\n\tfma.rn.f32.f16 %0, " A ", n, %3;\n\t}"                   \
        : "=f"(d)                                                                        \
        : "r"(a), "r"(b), "f"(c));                                                       \
    return d;                                                                            \
  }
IRO_MFMA_NEG(mfma_nhh, "a1", "b1")
IRO_MFMA_NEG(mfma_nhl, "a1", "b0")
#undef IRO_MFMA_NEG

__device__ __forceinline__ __half2 as_h2(uint32_t w) { return *reinterpret_cast<__half2*>(&w); }
__device__ __forceinline__ uint32_t as_w(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

// complex words (re in the low half): a + b, a - b, a + i b, a - i b
__device__ __forceinline__ uint32_t w_add(uint32_t a, uint32_t b) { return as_w(__hadd2(as_h2(a), as_h2(b))); }
__device__ __forceinline__ uint32_t w_sub(uint32_t a, uint32_t b) { return as_w(__hsub2(as_h2(a), as_h2(b))); }
__device__ __forceinline__ uint32_t w_add_i(uint32_t a, uint32_t b) {
  // (a.re - b.im, a.im + b.re)
  return as_w(__hfma2(__lowhigh2highlow(as_h2(b)), __floats2half2_rn(-1.f, 1.f), as_h2(a)));
}
__device__ __forceinline__ uint32_t w_sub_i(uint32_t a, uint32_t b) {
  // (a.re + b.im, a.im - b.re)
  return as_w(__hfma2(__lowhigh2highlow(as_h2(b)), __floats2half2_rn(1.f, -1.f), as_h2(a)));
}

// projector (1 - S gamma_mu) on stored FP16 words (complex 3*spin + colour);
// for t the factor 2 is left to the weight
template <int MU, int S>
__device__ __forceinline__ void project_w(const uint32_t f[12], uint32_t h[6]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const uint32_t f0 = f[c], f1 = f[3 + c], f2 = f[6 + c], f3 = f[9 + c];
    if (MU == 0) {  // h0 = f0 + S i f3, h1 = f1 + S i f2
      h[c] = (S > 0) ? w_add_i(f0, f3) : w_sub_i(f0, f3);
      h[3 + c] = (S > 0) ? w_add_i(f1, f2) : w_sub_i(f1, f2);
    } else if (MU == 1) {  // h0 = f0 + S f3, h1 = f1 - S f2
      h[c] = (S > 0) ? w_add(f0, f3) : w_sub(f0, f3);
      h[3 + c] = (S > 0) ? w_sub(f1, f2) : w_add(f1, f2);
    } else if (MU == 2) {  // h0 = f0 + S i f2, h1 = f1 - S i f3
      h[c] = (S > 0) ? w_add_i(f0, f2) : w_sub_i(f0, f2);
      h[3 + c] = (S > 0) ? w_sub_i(f1, f3) : w_add_i(f1, f3);
    } else {  // t: (f2, f3) for S = +1, (f0, f1) for S = -1
      h[c] = (S > 0) ? f2 : f0;
      h[3 + c] = (S > 0) ? f3 : f1;
    }
  }
}

// g = U h (ADJ false) or U^dag h (ADJ true), FP32 results from FP16 words.
// The minus signs are negated FP16 operands of the FMAs (U h: -Im u Im h in
// Re g; U^dag h: -Im u Re h in Im g).  Measured against flipping the half
// spinor's sign bits once per word first: 4.7 % less time per 12-RHS Schur
// application at 32^3x64, the same results to the bit.
template <bool ADJ>
__device__ __forceinline__ void su3_w(const uint32_t u[9], const uint32_t h[6], Cx<float> g[6]) {
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      float re = 0.f, im = 0.f;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const uint32_t hb = h[3 * s + b];
        if (!ADJ) {  // u_ab h_b: re = u.re h.re - u.im h.im, im = u.re h.im + u.im h.re
          const uint32_t w = u[3 * a + b];
          re = mfma_ll(w, hb, re);
          re = mfma_nhh(w, hb, re);
          im = mfma_lh(w, hb, im);
          im = mfma_hl(w, hb, im);
        } else {  // conj(u_ba) h_b: re = u.re h.re + u.im h.im, im = u.re h.im - u.im h.re
          const uint32_t w = u[3 * b + a];
          re = mfma_ll(w, hb, re);
          re = mfma_hh(w, hb, re);
          im = mfma_lh(w, hb, im);
          im = mfma_nhl(w, hb, im);
        }
      }
      g[3 * s + a] = {re, im};
    }
}

// acc += w (1 - S gamma_mu) reconstructed from g (as reconstruct<MU, S>)
template <int MU, int S>
__device__ __forceinline__ void reconstruct_w(Cx<float> acc[12], const Cx<float> g[6], float w) {
  auto add = [&](Cx<float>& a, Cx<float> v, float s) {  // a += s w v
    a.re = fmaf(s * w, v.re, a.re);
    a.im = fmaf(s * w, v.im, a.im);
  };
  auto add_i = [&](Cx<float>& a, Cx<float> v, float s) {  // a += s w (i v)
    a.re = fmaf(-s * w, v.im, a.re);
    a.im = fmaf(s * w, v.re, a.im);
  };
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const Cx<float> g0 = g[c], g1 = g[3 + c];
    if (MU == 3) {
      if (S > 0) {
        add(acc[6 + c], g0, 1.f);
        add(acc[9 + c], g1, 1.f);
      } else {
        add(acc[c], g0, 1.f);
        add(acc[3 + c], g1, 1.f);
      }
      continue;
    }
    add(acc[c], g0, 1.f);
    add(acc[3 + c], g1, 1.f);
    if (MU == 0) {  // [h0, h1, -S i h1, -S i h0]
      add_i(acc[6 + c], g1, S > 0 ? -1.f : 1.f);
      add_i(acc[9 + c], g0, S > 0 ? -1.f : 1.f);
    } else if (MU == 1) {  // [h0, h1, -S h1, S h0]
      add(acc[6 + c], g1, S > 0 ? -1.f : 1.f);
      add(acc[9 + c], g0, S > 0 ? 1.f : -1.f);
    } else {  // MU == 2: [h0, h1, -S i h0, S i h1]
      add_i(acc[6 + c], g0, S > 0 ? -1.f : 1.f);
      add_i(acc[9 + c], g1, S > 0 ? 1.f : -1.f);
    }
  }
}

// Addresses.  A context holds fewer than 2^31 elements (half-sites times
// right-hand sides) and fewer than 2^30 links, so element and link indices
// are formed in 32-bit arithmetic and widened only in the multiply that
// scales them to bytes.

// FP16 links with the three rows stored (GaugeIO<PREC_HALF, 18>), as words;
// j = (parity * 4 + mu) * Vh + half-site
__device__ __forceinline__ void load_link_w(const GaugePtr& g, uint32_t j, uint32_t u[9]) {
  const uint4* pa = static_cast<const uint4*>(g.a) + 2 * size_t(j);
  const uint4 a = __ldg(pa);
  const uint4 b = __ldg(pa + 1);
  u[0] = a.x; u[1] = a.y; u[2] = a.z; u[3] = a.w;
  u[4] = b.x; u[5] = b.y; u[6] = b.z; u[7] = b.w;
  u[8] = __ldg(static_cast<const uint32_t*>(g.b) + j);
}

// FP16 links with two stored rows (GaugeIO<PREC_HALF, 12>: 24 bytes instead
// of 36), as words: row 2 = conj(row 0 x row 1) is formed in FP32 from the
// stored rows and rounded to FP16 words, so the product below runs as on the
// three-row links (whose row 2 is the FP64 row rounded to FP16)
__device__ __forceinline__ void load_link_w12(const GaugePtr& g, uint32_t j, uint32_t u[9]) {
  const uint4 a = __ldg(static_cast<const uint4*>(g.a) + j);
  const uint2 b = __ldg(static_cast<const uint2*>(g.b) + j);
  u[0] = a.x; u[1] = a.y; u[2] = a.z; u[3] = a.w; u[4] = b.x; u[5] = b.y;
  float2 x[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) x[k] = __half22float2(as_h2(u[k]));
  // (p q - r s)^* of complex p, q, r, s
  auto cross = [](float2 p, float2 q, float2 r, float2 s) {
    const float re = fmaf(p.x, q.x, fmaf(-p.y, q.y, fmaf(-r.x, s.x, r.y * s.y)));
    const float im = fmaf(p.x, q.y, fmaf(p.y, q.x, fmaf(-r.x, s.y, -r.y * s.x)));
    return as_w(__floats2half2_rn(re, -im));
  };
  u[6] = cross(x[1], x[5], x[2], x[4]);  // (u01 u12 - u02 u11)^*
  u[7] = cross(x[2], x[3], x[0], x[5]);  // (u02 u10 - u00 u12)^*
  u[8] = cross(x[0], x[4], x[1], x[3]);  // (u00 u11 - u01 u10)^*
}

template <int RECON>
__device__ __forceinline__ void load_link_mix(const GaugePtr& g, uint32_t j, uint32_t u[9]) {
  if constexpr (RECON == 12)
    load_link_w12(g, j, u);
  else
    load_link_w(g, j, u);
}

// the stored words and norm of FP16 element i: chunk 0 of a warp block of 32
// elements sits at 16-byte unit (i / 32) * 96 + i % 32, i.e. at byte
// 32 * (i & ~31) + 16 * i
__device__ __forceinline__ float load_raw_w(const SpinorPtr& s, uint32_t i, uint32_t f[12]) {
  const char* base = static_cast<const char*>(s.data);
  const uint4* p = reinterpret_cast<const uint4*>(base + size_t(i & ~31u) * 32u + size_t(i) * 16u);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const uint4 d = __ldg(p + 32 * k);
    f[4 * k] = d.x;
    f[4 * k + 1] = d.y;
    f[4 * k + 2] = d.z;
    f[4 * k + 3] = d.w;
  }
  return __ldg(s.norm + i);
}

// forward and backward contributions of direction MU (as hop_dir); lown and
// lnb are the link indices of direction 0 at parity p and 1 - p
// ((p * 4) * Vh and ((1 - p) * 4) * Vh)
template <int MU, bool DAG, int RECON>
__device__ __forceinline__ void hop_dir_mix(const GaugePtr& gauge, const SpinorPtr& in, uint32_t lown,
                                            uint32_t lnb, uint32_t vh, int hs, const int nb[8],
                                            int nrhs, int r, Cx<float> acc[12]) {
  uint32_t u[9], f[12], h[6];
  Cx<float> g[6];
  {
    constexpr int S = DAG ? -1 : 1;
    load_link_mix<RECON>(gauge, lown + MU * vh + uint32_t(hs), u);
    const float n = load_raw_w(in, uint32_t(nb[2 * MU]) * uint32_t(nrhs) + uint32_t(r), f);
    project_w<MU, S>(f, h);
    su3_w<false>(u, h, g);
    reconstruct_w<MU, S>(acc, g, MU == 3 ? 2.f * n : n);
  }
  {
    constexpr int S = DAG ? 1 : -1;
    load_link_mix<RECON>(gauge, lnb + MU * vh + uint32_t(nb[2 * MU + 1]), u);
    const float n = load_raw_w(in, uint32_t(nb[2 * MU + 1]) * uint32_t(nrhs) + uint32_t(r), f);
    project_w<MU, S>(f, h);
    su3_w<true>(u, h, g);
    reconstruct_w<MU, S>(acc, g, MU == 3 ? 2.f * n : n);
  }
}

}  // namespace iro
