// Device-side building blocks shared by every kernel: complex arithmetic,
// lattice geometry of the even/odd-ordered half lattices, and the storage
// formats of spinors, links and clover blocks in HBM.
//
// Every field is stored warp-blocked ("array of structures of arrays"): the
// element index i (a half-lattice site, or site*nrhs + rhs for several
// right-hand sides) is split into a block of 32 (i >> 5) and a lane (i & 31),
// and 16-byte chunk k of element i lives at
//     ((i >> 5) * NCHUNK + k) * 32 + (i & 31)            [in 16-byte units]
// so that a warp reading chunk k of 32 consecutive elements reads 512
// contiguous bytes, and the chunks of one element sit at compile-time
// offsets (k * 512 bytes) from one base address.
//
//  spinor (12 complex, k = c + 3*s, the Format_F order of include/format_F.h:36-42):
//    FP64: 12 chunks of double2; FP32: 6 chunks of float4 (complexes 2j, 2j+1);
//    FP16: 3 chunks of 8 halves + one FP32 norm per element (values are
//          stored divided by the element's largest real component)
//  links U_mu(x) of the sites x of parity p, element = site:
//    [p][mu][blocked element]; rows 0 and 1 only (reconstruct-12: row 2 =
//    conj(row0 x row1)) or all three rows (FP64, for non-SU(3) input)
//    FP64: 6 (or 9) double2 chunks; FP32: 3 float4 chunks;
//    FP16: one 8-half chunk + one 4-half chunk (two plain arrays)
//  clover, parity p, element = site: two Hermitian 6x6 blocks acting on
//    phi+ = (psi0+psi2, psi1+psi3) and phi- = (psi0-psi2, psi1-psi3), the
//    gamma5 eigenbasis of the Dirac-Pauli basis used by the reference
//    (lib/Dirac_ops/wilsonLikeUtils.cpp:42-49); per block 6 real diagonal
//    entries and 15 complex upper-triangle entries = 36 reals
//    FP64: 36 double2 chunks, FP32: 18 float4, FP16: 9 chunks of 8 halves
// The element count of every array is a multiple of 32 (the context
// requires the lattice volume to be a multiple of 64).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace iro {

// ---- complex ---------------------------------------------------------------
template <typename R>
struct Cx {
  R re, im;
};

template <typename R>
__device__ __forceinline__ Cx<R> cx(R a, R b) {
  return Cx<R>{a, b};
}
template <typename R>
__device__ __forceinline__ Cx<R> operator+(Cx<R> a, Cx<R> b) {
  return {a.re + b.re, a.im + b.im};
}
template <typename R>
__device__ __forceinline__ Cx<R> operator-(Cx<R> a, Cx<R> b) {
  return {a.re - b.re, a.im - b.im};
}
template <typename R>
__device__ __forceinline__ Cx<R> operator*(Cx<R> a, Cx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R>
__device__ __forceinline__ Cx<R> operator*(R s, Cx<R> a) {
  return {s * a.re, s * a.im};
}
template <typename R>
__device__ __forceinline__ Cx<R> conjx(Cx<R> a) {
  return {a.re, -a.im};
}
// a * conj(b)
template <typename R>
__device__ __forceinline__ Cx<R> mul_cj(Cx<R> a, Cx<R> b) {
  return {a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im};
}
// conj(a) * b
template <typename R>
__device__ __forceinline__ Cx<R> cj_mul(Cx<R> a, Cx<R> b) {
  return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}
// i * a
template <typename R>
__device__ __forceinline__ Cx<R> mul_i(Cx<R> a) {
  return {-a.im, a.re};
}
// -i * a
template <typename R>
__device__ __forceinline__ Cx<R> mul_mi(Cx<R> a) {
  return {a.im, -a.re};
}

// ---- geometry ------------------------------------------------------------------
// n / d for 0 <= n < 2^31 by multiply-high (Granlund & Montgomery, "Division by
// invariant integers using multiplication", PLDI 1994): l = ceil(log2 d),
// m = floor(2^32 (2^l - d) / d) + 1, q = (mulhi(n, m) + n) >> l.
struct FastDiv {
  uint32_t d, m, l;
};

inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f{d, 0u, 0u};
  if (d > 1) {
    uint32_t l = 0;
    while ((1ull << l) < d) ++l;
    f.l = l;
    f.m = uint32_t((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
  }
  return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
  return f.d == 1 ? n : (__umulhi(n, f.m) + n) >> f.l;
}

struct Geom {
  int L[4];  // Lx, Ly, Lz, Lt (all even)
  int Lxh;   // Lx/2
  int Vh;    // half volume
  int sy, sz, st;  // half-site strides of y, z, t: Lxh, Lxh*Ly, Lxh*Ly*Lz
  FastDiv dxh, dy, dz;  // division by Lxh, Ly, Lz
};

// Coordinates of half-site hs of parity p; the lexicographic site is
// x + Lx*(y + Ly*(z + Lz*t)) = 2*hs + ((y+z+t+p)&1), which is how
// SiteIndex_EvenOdd orders esec/osec (lib/Geometry/siteIndex_EvenOdd.hpp:69-76).
struct Coord {
  int x, y, z, t, row;
};

__device__ __forceinline__ Coord coord_of(const Geom& g, int hs, int p) {
  Coord c;
  c.row = int(fdiv(uint32_t(hs), g.dxh));
  const int xh = hs - c.row * g.Lxh;
  const int yz = int(fdiv(uint32_t(c.row), g.dy));
  c.y = c.row - yz * g.L[1];
  c.t = int(fdiv(uint32_t(yz), g.dz));
  c.z = yz - c.t * g.L[2];
  c.x = 2 * xh + ((c.y + c.z + c.t + p) & 1);
  return c;
}

// Half-site indices of the 8 neighbours (in the opposite parity) of a site,
// periodic in every direction.  Order: x+, x-, y+, y-, z+, z-, t+, t-.
__device__ __forceinline__ void neighbours(const Geom& g, const Coord& c, int hs, int nb[8]) {
  const int xp = (c.x + 1 == g.L[0]) ? 0 : c.x + 1;
  const int xm = (c.x == 0) ? g.L[0] - 1 : c.x - 1;
  const int rowbase = c.row * g.Lxh;
  nb[0] = rowbase + (xp >> 1);
  nb[1] = rowbase + (xm >> 1);
  nb[2] = (c.y + 1 == g.L[1]) ? hs - (g.L[1] - 1) * g.sy : hs + g.sy;
  nb[3] = (c.y == 0) ? hs + (g.L[1] - 1) * g.sy : hs - g.sy;
  nb[4] = (c.z + 1 == g.L[2]) ? hs - (g.L[2] - 1) * g.sz : hs + g.sz;
  nb[5] = (c.z == 0) ? hs + (g.L[2] - 1) * g.sz : hs - g.sz;
  nb[6] = (c.t + 1 == g.L[3]) ? hs - (g.L[3] - 1) * g.st : hs + g.st;
  nb[7] = (c.t == 0) ? hs + (g.L[3] - 1) * g.st : hs - g.st;
}

// ---- stencil epilogues and reductions --------------------------------------------
enum Epilogue {
  EPI_SCALE = 0,       // out = scale * H in
  EPI_SCALE_CLOV = 1,  // out = C_p (scale * H in)            (C = clover inverse)
  EPI_XPAY = 2,        // out = xin + scale * H in
  EPI_XPAY_CLOV = 3    // out = C_p xin + scale * H in         (C = clover term)
};

enum RedBits { RED_OUT2 = 1, RED_X2 = 2, RED_XOUT = 4 };

// ---- warp-blocked addressing -------------------------------------------------------
// offset (in 16-byte units) of chunk 0 of element i in an array of NCHUNK chunks
template <int NCHUNK>
__host__ __device__ __forceinline__ int64_t blk0(int64_t i) {
  return (i >> 5) * (NCHUNK * 32) + (i & 31);
}

// Device address of chunk 0 of element i of a blocked array of 16-byte
// chunks, NCHUNK per element: unit (i & ~31) * NCHUNK + (i & 31) =
// (i & ~31) * (NCHUNK - 1) + i, as blk0.  Element indices on the device stay
// below 2^32 (a context holds fewer than 2^31 elements per parity), so the
// index arithmetic is 32-bit and only the byte offset is widened.
template <int NCHUNK, typename T>
__device__ __forceinline__ T* chunk0(T* base, int64_t i) {
  static_assert(sizeof(T) == 16, "16-byte chunks");
  const uint32_t e = uint32_t(i);
  const size_t off = size_t(e & ~31u) * (16u * (NCHUNK - 1)) + size_t(e) * 16u;
  return reinterpret_cast<T*>(reinterpret_cast<uintptr_t>(base) + off);
}

// ---- spinor storage ------------------------------------------------------------
enum Prec { PREC_DOUBLE = 0, PREC_SINGLE = 1, PREC_HALF = 2 };

struct SpinorPtr {
  void* data;   // blocked chunk array
  float* norm;  // FP16 only: one norm per element
};

template <int P>
struct SpinorIO;

template <>
struct SpinorIO<PREC_DOUBLE> {
  using Real = double;
  static constexpr int NCHUNK = 12;
  static constexpr int BYTES = 192;
  __device__ __forceinline__ static void load(const SpinorPtr& s, int64_t i, Cx<double> v[12]) {
    const double2* p = chunk0<12>(static_cast<const double2*>(s.data), i);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      double2 d = __ldg(p + 32 * k);
      v[k] = {d.x, d.y};
    }
  }
  __device__ __forceinline__ static void store(const SpinorPtr& s, int64_t i, const Cx<double> v[12]) {
    double2* p = chunk0<12>(static_cast<double2*>(s.data), i);
#pragma unroll
    for (int k = 0; k < 12; ++k) p[32 * k] = make_double2(v[k].re, v[k].im);
  }
};

template <>
struct SpinorIO<PREC_SINGLE> {
  using Real = float;
  static constexpr int NCHUNK = 6;
  static constexpr int BYTES = 96;
  __device__ __forceinline__ static void load(const SpinorPtr& s, int64_t i, Cx<float> v[12]) {
    const float4* p = chunk0<6>(static_cast<const float4*>(s.data), i);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      float4 d = __ldg(p + 32 * k);
      v[2 * k] = {d.x, d.y};
      v[2 * k + 1] = {d.z, d.w};
    }
  }
  __device__ __forceinline__ static void store(const SpinorPtr& s, int64_t i, const Cx<float> v[12]) {
    float4* p = chunk0<6>(static_cast<float4*>(s.data), i);
#pragma unroll
    for (int k = 0; k < 6; ++k)
      p[32 * k] = make_float4(v[2 * k].re, v[2 * k].im, v[2 * k + 1].re, v[2 * k + 1].im);
  }
};

__device__ __forceinline__ uint32_t pack_h2(float a, float b) {
  __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ float2 unpack_h2(uint32_t u) {
  __half2 h = *reinterpret_cast<__half2*>(&u);
  return __half22float2(h);
}

template <>
struct SpinorIO<PREC_HALF> {
  using Real = float;
  static constexpr int NCHUNK = 3;
  static constexpr int BYTES = 52;  // 48 bytes of FP16 + 4-byte norm
  // the stored (normalised) values and the element's norm
  __device__ __forceinline__ static float load_raw(const SpinorPtr& s, int64_t i, Cx<float> v[12]) {
    const uint4* p = chunk0<3>(static_cast<const uint4*>(s.data), i);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      uint4 d = __ldg(p + 32 * k);
      float2 a = unpack_h2(d.x), b = unpack_h2(d.y), c = unpack_h2(d.z), e = unpack_h2(d.w);
      v[4 * k + 0] = {a.x, a.y};
      v[4 * k + 1] = {b.x, b.y};
      v[4 * k + 2] = {c.x, c.y};
      v[4 * k + 3] = {e.x, e.y};
    }
    return __ldg(s.norm + uint32_t(i));
  }
  __device__ __forceinline__ static void load(const SpinorPtr& s, int64_t i, Cx<float> v[12]) {
    const float n = load_raw(s, i, v);
#pragma unroll
    for (int k = 0; k < 12; ++k) v[k] = n * v[k];
  }
  __device__ __forceinline__ static void store(const SpinorPtr& s, int64_t i, const Cx<float> v[12]) {
    store_scaled(s, i, v, 1.f);
  }
  // stores sc * v: the words are v / max|v| with the sign of sc, the norm
  // |sc| max|v|
  __device__ __forceinline__ static void store_scaled(const SpinorPtr& s, int64_t i, const Cx<float> v[12],
                                                      float sc) {
    float m = 0.f;
#pragma unroll
    for (int k = 0; k < 12; ++k) m = fmaxf(m, fmaxf(fabsf(v[k].re), fabsf(v[k].im)));
    float n = m * fabsf(sc);
    // elements whose largest component is below the normal FP32 range are
    // stored as zero: 1/m would overflow (0 * inf = NaN), and such values are
    // far below FP16 resolution relative to any field they belong to
    if (!(n >= 1e-37f) || !(m >= 1e-37f)) m = n = 0.f;
    const float inv = (m > 0.f) ? copysignf(1.0f / m, sc) : 0.f;
    uint4* p = chunk0<3>(static_cast<uint4*>(s.data), i);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      uint4 d;
      d.x = pack_h2(v[4 * k + 0].re * inv, v[4 * k + 0].im * inv);
      d.y = pack_h2(v[4 * k + 1].re * inv, v[4 * k + 1].im * inv);
      d.z = pack_h2(v[4 * k + 2].re * inv, v[4 * k + 2].im * inv);
      d.w = pack_h2(v[4 * k + 3].re * inv, v[4 * k + 3].im * inv);
      p[32 * k] = d;
    }
    s.norm[uint32_t(i)] = n;
  }
};

// ---- link storage -------------------------------------------------------------------
struct GaugePtr {
  const void* a;  // main chunk array  [p][mu][blocked site]
  const void* b;  // FP16 second array [p][mu][site] (4 halves)
  int64_t Vh;
};

template <typename R>
struct Su3 {
  Cx<R> e[3][3];
};

template <typename R>
__device__ __forceinline__ void reconstruct_row2(Su3<R>& U) {
  U.e[2][0] = conjx(U.e[0][1] * U.e[1][2] - U.e[0][2] * U.e[1][1]);
  U.e[2][1] = conjx(U.e[0][2] * U.e[1][0] - U.e[0][0] * U.e[1][2]);
  U.e[2][2] = conjx(U.e[0][0] * U.e[1][1] - U.e[0][1] * U.e[1][0]);
}

// offset (16-byte units) of chunk 0 of the link of site i, direction mu, parity p
template <int NCHUNK>
__host__ __device__ __forceinline__ int64_t link0(int64_t Vh, int p, int mu, int64_t i) {
  return int64_t(p * 4 + mu) * Vh * NCHUNK + blk0<NCHUNK>(i);
}

// device address of chunk 0 of the link of half-site i, direction mu, parity
// p (as link0; the parity/direction offset is uniform across a block)
template <int NCHUNK, typename T>
__device__ __forceinline__ T* link_chunk0(T* base, int64_t Vh, int p, int mu, int64_t i) {
  const size_t pm = size_t(p * 4 + mu) * size_t(Vh) * (16u * NCHUNK);
  return chunk0<NCHUNK>(reinterpret_cast<T*>(reinterpret_cast<uintptr_t>(base) + pm), i);
}

template <int P, int RECON>
struct GaugeIO;

template <int RECON>
struct GaugeIO<PREC_DOUBLE, RECON> {
  using Real = double;
  static constexpr int NCHUNK = RECON / 2;
  static constexpr int BYTES = RECON * 8;
  __device__ __forceinline__ static void load(const GaugePtr& g, int p, int mu, int64_t i, Su3<double>& U) {
    const double2* q = link_chunk0<NCHUNK>(static_cast<const double2*>(g.a), g.Vh, p, mu, i);
#pragma unroll
    for (int k = 0; k < NCHUNK; ++k) {
      double2 d = __ldg(q + 32 * k);
      U.e[k / 3][k % 3] = {d.x, d.y};
    }
    if (RECON == 12) reconstruct_row2(U);
  }
};

template <>
struct GaugeIO<PREC_SINGLE, 12> {
  using Real = float;
  static constexpr int NCHUNK = 3;
  static constexpr int BYTES = 48;
  __device__ __forceinline__ static void load(const GaugePtr& g, int p, int mu, int64_t i, Su3<float>& U) {
    const float4* q = link_chunk0<3>(static_cast<const float4*>(g.a), g.Vh, p, mu, i);
    float4 a = __ldg(q), b = __ldg(q + 32), c = __ldg(q + 64);
    U.e[0][0] = {a.x, a.y};
    U.e[0][1] = {a.z, a.w};
    U.e[0][2] = {b.x, b.y};
    U.e[1][0] = {b.z, b.w};
    U.e[1][1] = {c.x, c.y};
    U.e[1][2] = {c.z, c.w};
    reconstruct_row2(U);
  }
};

template <>
struct GaugeIO<PREC_HALF, 12> {
  using Real = float;
  static constexpr int NCHUNK = 1;
  static constexpr int BYTES = 24;
  __device__ __forceinline__ static void load(const GaugePtr& g, int p, int mu, int64_t i, Su3<float>& U) {
    const uint32_t j = uint32_t(p * 4 + mu) * uint32_t(g.Vh) + uint32_t(i);
    uint4 a = __ldg(static_cast<const uint4*>(g.a) + j);
    uint2 b = __ldg(static_cast<const uint2*>(g.b) + j);
    float2 t;
    t = unpack_h2(a.x); U.e[0][0] = {t.x, t.y};
    t = unpack_h2(a.y); U.e[0][1] = {t.x, t.y};
    t = unpack_h2(a.z); U.e[0][2] = {t.x, t.y};
    t = unpack_h2(a.w); U.e[1][0] = {t.x, t.y};
    t = unpack_h2(b.x); U.e[1][1] = {t.x, t.y};
    t = unpack_h2(b.y); U.e[1][2] = {t.x, t.y};
    reconstruct_row2(U);
  }
};

// ---- clover storage -------------------------------------------------------------------
// Per block: d[6] (real diagonal), o[15] (complex, upper triangle, row major).
template <typename R>
struct CloverBlock {
  R d[6];
  Cx<R> o[15];
};

struct CloverPtr {
  const void* data;  // blocked chunk array of one parity
  int64_t Vh;
};

template <int P>
struct CloverIO;

template <>
struct CloverIO<PREC_DOUBLE> {
  using Real = double;
  static constexpr int BYTES = 576;
  __device__ __forceinline__ static void load(const CloverPtr& c, int64_t i, CloverBlock<double> B[2]) {
    const double2* q = chunk0<36>(static_cast<const double2*>(c.data), i);
#pragma unroll
    for (int b = 0; b < 2; ++b) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        double2 d = __ldg(q + 32 * (b * 18 + k));
        B[b].d[2 * k] = d.x;
        B[b].d[2 * k + 1] = d.y;
      }
#pragma unroll
      for (int k = 0; k < 15; ++k) {
        double2 d = __ldg(q + 32 * (b * 18 + 3 + k));
        B[b].o[k] = {d.x, d.y};
      }
    }
  }
};

template <>
struct CloverIO<PREC_SINGLE> {
  using Real = float;
  static constexpr int BYTES = 288;
  __device__ __forceinline__ static void load(const CloverPtr& c, int64_t i, CloverBlock<float> B[2]) {
    const float4* q = chunk0<18>(static_cast<const float4*>(c.data), i);
    float v[72];
#pragma unroll
    for (int k = 0; k < 18; ++k) {
      float4 d = __ldg(q + 32 * k);
      v[4 * k] = d.x;
      v[4 * k + 1] = d.y;
      v[4 * k + 2] = d.z;
      v[4 * k + 3] = d.w;
    }
#pragma unroll
    for (int b = 0; b < 2; ++b) {
#pragma unroll
      for (int k = 0; k < 6; ++k) B[b].d[k] = v[36 * b + k];
#pragma unroll
      for (int k = 0; k < 15; ++k) B[b].o[k] = {v[36 * b + 6 + 2 * k], v[36 * b + 7 + 2 * k]};
    }
  }
};

template <>
struct CloverIO<PREC_HALF> {
  using Real = float;
  static constexpr int BYTES = 144;
  __device__ __forceinline__ static void load(const CloverPtr& c, int64_t i, CloverBlock<float> B[2]) {
    const uint4* q = chunk0<9>(static_cast<const uint4*>(c.data), i);
    float v[72];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      uint4 d = __ldg(q + 32 * k);
      float2 a = unpack_h2(d.x), b = unpack_h2(d.y), e = unpack_h2(d.z), f = unpack_h2(d.w);
      v[8 * k] = a.x; v[8 * k + 1] = a.y; v[8 * k + 2] = b.x; v[8 * k + 3] = b.y;
      v[8 * k + 4] = e.x; v[8 * k + 5] = e.y; v[8 * k + 6] = f.x; v[8 * k + 7] = f.y;
    }
#pragma unroll
    for (int b = 0; b < 2; ++b) {
#pragma unroll
      for (int k = 0; k < 6; ++k) B[b].d[k] = v[36 * b + k];
#pragma unroll
      for (int k = 0; k < 15; ++k) B[b].o[k] = {v[36 * b + 6 + 2 * k], v[36 * b + 7 + 2 * k]};
    }
  }
};

// index of the upper-triangle element (i<j) of a 6x6 matrix
__host__ __device__ constexpr int tri(int i, int j) { return i * 6 - i * (i + 1) / 2 + (j - i - 1); }

// y = B x for a Hermitian 6x6 block
template <typename R>
__device__ __forceinline__ void herm6(const CloverBlock<R>& B, const Cx<R> x[6], Cx<R> y[6]) {
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    Cx<R> acc = B.d[i] * x[i];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      if (j > i) acc = acc + B.o[tri(i, j)] * x[j];
      if (j < i) acc = acc + cj_mul(B.o[tri(j, i)], x[j]);
    }
    y[i] = acc;
  }
}

// psi -> A psi with A = P^-1 diag(B+, B-) P, P: phi+- = (psi0 +- psi2, psi1 +- psi3)
template <typename R>
__device__ __forceinline__ void clover_apply(const CloverBlock<R> B[2], Cx<R> v[12]) {
  Cx<R> pp[6], pm[6], qp[6], qm[6];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    pp[c] = v[c] + v[6 + c];
    pp[3 + c] = v[3 + c] + v[9 + c];
    pm[c] = v[c] - v[6 + c];
    pm[3 + c] = v[3 + c] - v[9 + c];
  }
  herm6(B[0], pp, qp);
  herm6(B[1], pm, qm);
  const R h = R(0.5);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    v[c] = h * (qp[c] + qm[c]);
    v[6 + c] = h * (qp[c] - qm[c]);
    v[3 + c] = h * (qp[3 + c] + qm[3 + c]);
    v[9 + c] = h * (qp[3 + c] - qm[3 + c]);
  }
}

// ---- block reductions ---------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace iro
