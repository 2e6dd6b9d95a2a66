// Gauge-configuration files <-> Format_G host arrays.
//
// The file formats are those of IroIro's readers and writers (lib/IO/ and
// GaugeConf_*::init_conf, lib/Main/gaugeConf.cpp); the byte layouts, header
// keys and checksums must match them to exchange files, so they do.  The
// code is host-only: a read fills the caller's Format_G array
// u[18 * (site + V * mu) + 2 * (3 a + b) + re/im], site = x + Lx (y + Ly (z +
// Lz t)), which iro_gauge_upload then converts once for the device.
//
// File orders (s = lexicographic site, fastest index last):
//   Binary       [s][mu][18]        big-endian doubles in, host order out
//   JLQCDLegacy  4-byte record word, [mu][s][18] host-order doubles
//   NERSC        text header, [s][mu][12 | 18] big-endian float | double
//   csdt         4-byte record word, [t][mu][z][y][x][a][b][re, im] big-endian
//   text         [t][z][y][x][mu][a][b] "re im"
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "iroiro_b200.h"

namespace {

thread_local std::string g_io_err;

int io_fail(int code, const std::string& msg) {
  g_io_err = msg;
  return code;
}

struct Lat {
  int L[4];
  int64_t V;
  int64_t site(int x, int y, int z, int t) const {
    return x + int64_t(L[0]) * (y + int64_t(L[1]) * (z + int64_t(L[2]) * t));
  }
};

bool host_little_endian() {
  const uint16_t one = 1;
  unsigned char b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}

template <int N>
void swap_bytes(void* p, size_t count) {
  unsigned char* c = static_cast<unsigned char*>(p);
  for (size_t i = 0; i < count; ++i, c += N)
    for (int k = 0; k < N / 2; ++k) std::swap(c[k], c[N - 1 - k]);
}

// big-endian <-> host order, in place
template <int N>
void from_big_endian(void* p, size_t count) {
  if (host_little_endian()) swap_bytes<N>(p, count);
}

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

int read_exact(FILE* f, void* dst, size_t bytes, const char* path) {
  if (std::fread(dst, 1, bytes, f) != bytes)
    return io_fail(IRO_IO_ERROR, std::string("short read from ") + path);
  return IRO_OK;
}

double* link(double* u, const Lat& g, int64_t s, int mu) { return u + 18 * (s + g.V * mu); }
const double* link(const double* u, const Lat& g, int64_t s, int mu) {
  return u + 18 * (s + g.V * mu);
}

// row 2 = conj(row 0 x row 1) of a matrix whose first 12 reals are rows 0, 1
void third_row(double* m) {
  auto re = [&](int a, int b) { return m[2 * (3 * a + b)]; };
  auto im = [&](int a, int b) { return m[2 * (3 * a + b) + 1]; };
  for (int b = 0; b < 3; ++b) {
    const int c = (b + 1) % 3, d = (b + 2) % 3;
    // (u0c u1d - u0d u1c)^*
    const double pr = re(0, c) * re(1, d) - im(0, c) * im(1, d) - (re(0, d) * re(1, c) - im(0, d) * im(1, c));
    const double pi = re(0, c) * im(1, d) + im(0, c) * re(1, d) - (re(0, d) * im(1, c) + im(0, d) * re(1, c));
    m[2 * (6 + b)] = pr;
    m[2 * (6 + b) + 1] = -pi;
  }
}

// ---- Staples::plaquette / link_trace ------------------------------------------
struct M3 {
  double r[3][3], i[3][3];
};

M3 load(const double* p) {
  M3 m;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      m.r[a][b] = p[2 * (3 * a + b)];
      m.i[a][b] = p[2 * (3 * a + b) + 1];
    }
  return m;
}

// A B (DB false) or A B^dagger (DB true)
M3 mul(const M3& A, const M3& B, bool DB) {
  M3 C;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double sr = 0.0, si = 0.0;
      for (int c = 0; c < 3; ++c) {
        const double br = DB ? B.r[b][c] : B.r[c][b];
        const double bi = DB ? -B.i[b][c] : B.i[c][b];
        sr += A.r[a][c] * br - A.i[a][c] * bi;
        si += A.r[a][c] * bi + A.i[a][c] * br;
      }
      C.r[a][b] = sr;
      C.i[a][b] = si;
    }
  return C;
}

int64_t shift(const Lat& g, int64_t s, int mu) {
  int c[4];
  int64_t r = s;
  for (int d = 0; d < 4; ++d) {
    c[d] = int(r % g.L[d]);
    r /= g.L[d];
  }
  c[mu] = (c[mu] + 1) % g.L[mu];
  return g.site(c[0], c[1], c[2], c[3]);
}

// per time slice, then summed in slice order: the same bits for any thread count
void plaquette(const Lat& g, const double* u, double* plaq, double* trace) {
  const int T = g.L[3];
  const int64_t slice = g.V / T;
  std::vector<double> ps(T, 0.0), ts(T, 0.0);
#pragma omp parallel for schedule(static)
  for (int t = 0; t < T; ++t) {
    double p = 0.0, tr = 0.0;
    for (int64_t k = 0; k < slice; ++k) {
      const int64_t s = int64_t(t) * slice + k;
      for (int mu = 0; mu < 4; ++mu) {
        const M3 Um = load(link(u, g, s, mu));
        tr += Um.r[0][0] + Um.r[1][1] + Um.r[2][2];
        const int64_t sm = shift(g, s, mu);
        for (int nu = mu + 1; nu < 4; ++nu) {
          const int64_t sn = shift(g, s, nu);
          // U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
          const M3 A = mul(Um, load(link(u, g, sm, nu)), false);
          const M3 B = mul(A, load(link(u, g, sn, mu)), true);
          const M3 P = mul(B, load(link(u, g, s, nu)), true);
          p += P.r[0][0] + P.r[1][1] + P.r[2][2];
        }
      }
    }
    ps[t] = p;
    ts[t] = tr;
  }
  double p = 0.0, tr = 0.0;
  for (int t = 0; t < T; ++t) {
    p += ps[t];
    tr += ts[t];
  }
  *plaq = p / (double(g.V) * 3.0 * 6.0);
  *trace = tr / (double(g.V) * 3.0 * 4.0);
}

// NERSC checksum of a field as NERSCWriter::checksum (NERSC_writer.cpp:18-43)
// forms it: each 18-double matrix in big-endian byte order, summed as 32-bit
// words in host order
uint32_t nersc_checksum(const Lat& g, const double* u) {
  uint32_t sum = 0;
  double m[18];
  for (int64_t s = 0; s < g.V; ++s)
    for (int mu = 0; mu < 4; ++mu) {
      std::memcpy(m, link(u, g, s, mu), sizeof(m));
      if (host_little_endian()) swap_bytes<8>(m, 18);
      uint32_t w[36];
      std::memcpy(w, m, sizeof(m));
      for (int k = 0; k < 36; ++k) sum += w[k];
    }
  return sum;
}

// ---- readers ----------------------------------------------------------------------
int read_binary(FILE* f, const Lat& g, double* u, const char* path) {
  std::vector<double> row(size_t(18) * 4 * g.L[0]);
  for (int64_t r = 0; r < g.V / g.L[0]; ++r) {
    if (int rc = read_exact(f, row.data(), row.size() * sizeof(double), path)) return rc;
    from_big_endian<8>(row.data(), row.size());
    for (int x = 0; x < g.L[0]; ++x)
      for (int mu = 0; mu < 4; ++mu)
        std::memcpy(link(u, g, r * g.L[0] + x, mu), &row[18 * (mu + 4 * size_t(x))], 18 * sizeof(double));
  }
  return IRO_OK;
}

int read_jlqcd_legacy(FILE* f, const Lat& g, double* u, const char* path) {
  return read_exact(f, u, size_t(18) * 4 * g.V * sizeof(double), path);
}

int read_csdt(FILE* f, const Lat& g, double* u, const char* path) {
  std::vector<double> row(size_t(18) * g.L[0]);
  for (int t = 0; t < g.L[3]; ++t)
    for (int mu = 0; mu < 4; ++mu)
      for (int z = 0; z < g.L[2]; ++z)
        for (int y = 0; y < g.L[1]; ++y) {
          if (int rc = read_exact(f, row.data(), row.size() * sizeof(double), path)) return rc;
          from_big_endian<8>(row.data(), row.size());
          for (int x = 0; x < g.L[0]; ++x)
            std::memcpy(link(u, g, g.site(x, y, z, t), mu), &row[18 * size_t(x)], 18 * sizeof(double));
        }
  return IRO_OK;
}

int read_text(FILE* f, const Lat& g, double* u, const char* path) {
  for (int t = 0; t < g.L[3]; ++t)
    for (int z = 0; z < g.L[2]; ++z)
      for (int y = 0; y < g.L[1]; ++y)
        for (int x = 0; x < g.L[0]; ++x)
          for (int mu = 0; mu < 4; ++mu) {
            double* m = link(u, g, g.site(x, y, z, t), mu);
            for (int k = 0; k < 18; ++k)
              if (std::fscanf(f, "%lf", &m[k]) != 1)
                return io_fail(IRO_IO_ERROR, std::string("text configuration too short: ") + path);
          }
  return IRO_OK;
}

// NERSC: "KEY = value" lines between BEGIN_HEADER and END_HEADER
// (NERSCReader::header, NERSC_reader.cpp:47-175)
int read_nersc(FILE* f, const Lat& g, double* u, const char* path, iro_gauge_info* info) {
  char line[1024];
  if (!std::fgets(line, sizeof(line), f) || std::strcmp(line, "BEGIN_HEADER\n") != 0)
    return io_fail(IRO_FORMAT_ERROR, std::string("NERSC type header not found: ") + path);
  std::map<std::string, std::string> kv;
  for (;;) {
    if (!std::fgets(line, sizeof(line), f))
      return io_fail(IRO_FORMAT_ERROR, std::string("NERSC header without END_HEADER: ") + path);
    if (std::strcmp(line, "END_HEADER\n") == 0) break;
    std::string s(line);
    if (!s.empty() && s.back() == '\n') s.pop_back();
    const size_t eq = s.find('=');
    if (eq == std::string::npos) continue;
    auto trim = [](std::string v) {
      const size_t a = v.find_first_not_of(" \t"), b = v.find_last_not_of(" \t\r");
      return a == std::string::npos ? std::string() : v.substr(a, b - a + 1);
    };
    kv[trim(s.substr(0, eq))] = trim(s.substr(eq + 1));
  }
  const std::string dt = kv["DATATYPE"], fp = kv["FLOATING_POINT"];
  int is3x2;
  if (dt == "4D_SU3_GAUGE") is3x2 = 1;
  else if (dt == "4D_SU3_GAUGE_3x3") is3x2 = 0;
  else return io_fail(IRO_FORMAT_ERROR, "NERSC DATATYPE not supported: " + dt);
  int bits;
  if (fp == "IEEE32" || fp == "IEEE32BIG") bits = 32;
  else if (fp == "IEEE64BIG") bits = 64;
  else return io_fail(IRO_FORMAT_ERROR, "NERSC FLOATING_POINT not supported: " + fp);
  const char* dimkey[4] = {"DIMENSION_1", "DIMENSION_2", "DIMENSION_3", "DIMENSION_4"};
  for (int d = 0; d < 4; ++d)
    if (std::atoi(kv[dimkey[d]].c_str()) != g.L[d])
      return io_fail(IRO_FORMAT_ERROR, std::string("NERSC file dimension ") + dimkey[d] +
                                           " does not match the lattice");
  const int nm = is3x2 ? 12 : 18;
  const size_t n = size_t(nm) * 4 * g.V;
  const size_t bytes = n * (bits / 8);
  std::vector<unsigned char> raw(bytes);
  if (int rc = read_exact(f, raw.data(), bytes, path)) return rc;
  // checksum over the data words as stored (NERSC_reader.cpp:126-153)
  uint32_t chk = 0;
  for (size_t k = 0; k + 4 <= bytes; k += 4) {
    uint32_t w;
    std::memcpy(&w, &raw[k], 4);
    chk += w;
  }
  std::vector<double> vals(n);
  if (bits == 32) {
    from_big_endian<4>(raw.data(), n);
    const float* fv = reinterpret_cast<const float*>(raw.data());
    for (size_t k = 0; k < n; ++k) vals[k] = fv[k];
  } else {
    from_big_endian<8>(raw.data(), n);
    std::memcpy(vals.data(), raw.data(), bytes);
  }
  for (int64_t s = 0; s < g.V; ++s)
    for (int mu = 0; mu < 4; ++mu) {
      double* m = link(u, g, s, mu);
      std::memcpy(m, &vals[size_t(nm) * (mu + 4 * size_t(s))], nm * sizeof(double));
      if (is3x2) third_row(m);
    }
  if (info) {
    info->stored_plaquette = std::atof(kv["PLAQUETTE"].c_str());
    info->stored_link_trace = std::atof(kv["LINK_TRACE"].c_str());
    info->stored_checksum = uint32_t(std::strtoul(kv["CHECKSUM"].c_str(), nullptr, 16));
    info->checksum = chk;
    info->is3x2 = is3x2;
    info->bits = bits;
  }
  return IRO_OK;
}

// ---- writers ----------------------------------------------------------------------
int write_binary(FILE* f, const Lat& g, const double* u, const char* path, bool big_endian) {
  std::vector<double> row(size_t(18) * 4 * g.L[0]);
  for (int64_t r = 0; r < g.V / g.L[0]; ++r) {
    for (int x = 0; x < g.L[0]; ++x)
      for (int mu = 0; mu < 4; ++mu)
        std::memcpy(&row[18 * (mu + 4 * size_t(x))], link(u, g, r * g.L[0] + x, mu), 18 * sizeof(double));
    if (big_endian && host_little_endian()) swap_bytes<8>(row.data(), row.size());
    if (std::fwrite(row.data(), sizeof(double), row.size(), f) != row.size())
      return io_fail(IRO_IO_ERROR, std::string("write failed: ") + path);
  }
  return IRO_OK;
}

// NERSCWriter::header (NERSC_writer.cpp:49-66): the same keys, order and formats
int write_nersc(FILE* f, const Lat& g, const double* u, const char* path) {
  double plaq, trace;
  plaquette(g, u, &plaq, &trace);
  const uint32_t chk = nersc_checksum(g, u);
  std::fprintf(f, "BEGIN_HEADER\n");
  std::fprintf(f, "HDR_VERSION = 1.0\n");
  std::fprintf(f, "DATATYPE = 4D_SU3_GAUGE_3x3\n");
  std::fprintf(f, "STORAGE_FORMAT = 1.0\n");
  for (int d = 0; d < 4; ++d) std::fprintf(f, "DIMENSION_%d = %d\n", d + 1, g.L[d]);
  std::fprintf(f, "LINK_TRACE = %1.15g\n", trace);
  std::fprintf(f, "PLAQUETTE = %1.15g\n", plaq);
  std::fprintf(f, "CHECKSUM = %x\n", chk);
  std::fprintf(f, "ENSEMBLE_ID = %s\n", "JLQCD_null");
  std::fprintf(f, "SEQUENCE_NUMBER = %d\n", 0);
  std::fprintf(f, "FLOATING_POINT = IEEE64BIG\n");
  std::fprintf(f, "END_HEADER\n");
  return write_binary(f, g, u, path, true);
}

int lattice(const int L[4], Lat& g) {
  if (!L) return io_fail(IRO_BAD_ARG, "null lattice");
  g.V = 1;
  for (int d = 0; d < 4; ++d) {
    if (L[d] < 1) return io_fail(IRO_BAD_ARG, "bad lattice extent");
    g.L[d] = L[d];
    g.V *= L[d];
  }
  return IRO_OK;
}

}  // namespace

extern "C" const char* iro_io_last_error(void) { return g_io_err.c_str(); }

extern "C" int iro_gauge_plaquette(const int L[4], const double* u, double* plaq, double* trace) {
  Lat g;
  if (int rc = lattice(L, g)) return rc;
  if (!u || !plaq || !trace) return io_fail(IRO_BAD_ARG, "null argument");
  plaquette(g, u, plaq, trace);
  return IRO_OK;
}

extern "C" int iro_gauge_read(const char* path, int format, const int L[4], int64_t offset,
                              double* u, iro_gauge_info* info) {
  Lat g;
  if (int rc = lattice(L, g)) return rc;
  if (!u || offset < 0) return io_fail(IRO_BAD_ARG, "bad argument");
  if (info) std::memset(info, 0, sizeof(*info));
  int rc = IRO_OK;
  if (format == IRO_GAUGE_UNIT) {
    std::memset(u, 0, size_t(18) * 4 * g.V * sizeof(double));
    for (int64_t k = 0; k < 4 * g.V; ++k)
      for (int a = 0; a < 3; ++a) u[18 * k + 2 * (3 * a + a)] = 1.0;
  } else if (format == IRO_GAUGE_ILDG || format == IRO_GAUGE_ILDG_FORTRAN) {
    return io_fail(IRO_UNSUPPORTED, "ILDG files need the lime library, which is not available");
  } else if (format >= IRO_GAUGE_BINARY && format <= IRO_GAUGE_TEXT) {
    if (!path) return io_fail(IRO_BAD_ARG, "null path");
    File fh;
    fh.f = std::fopen(path, format == IRO_GAUGE_TEXT ? "r" : "rb");
    if (!fh.f) return io_fail(IRO_IO_ERROR, std::string("cannot open ") + path + ": " + std::strerror(errno));
    // GaugeConf_JLQCDLegacy and GaugeConf_csdt skip one Fortran record word
    // (FORTRAN_CONTROL_WORDS, fields_io.hpp:25) on top of the caller's offset
    const int64_t skip = offset + ((format == IRO_GAUGE_JLQCD_LEGACY || format == IRO_GAUGE_CSDT) ? 4 : 0);
    if (skip && std::fseek(fh.f, long(skip), SEEK_SET) != 0)
      return io_fail(IRO_IO_ERROR, std::string("cannot seek in ") + path);
    switch (format) {
      case IRO_GAUGE_BINARY: rc = read_binary(fh.f, g, u, path); break;
      case IRO_GAUGE_JLQCD_LEGACY: rc = read_jlqcd_legacy(fh.f, g, u, path); break;
      case IRO_GAUGE_NERSC: rc = read_nersc(fh.f, g, u, path, info); break;
      case IRO_GAUGE_CSDT: rc = read_csdt(fh.f, g, u, path); break;
      default: rc = read_text(fh.f, g, u, path); break;
    }
  } else {
    return io_fail(IRO_BAD_ARG, "unknown gauge format");
  }
  if (rc == IRO_OK && info) plaquette(g, u, &info->plaquette, &info->link_trace);
  return rc;
}

extern "C" int iro_gauge_write(const char* path, int format, const int L[4], const double* u,
                               int append) {
  Lat g;
  if (int rc = lattice(L, g)) return rc;
  if (!path || !u) return io_fail(IRO_BAD_ARG, "null argument");
  if (format == IRO_GAUGE_ILDG || format == IRO_GAUGE_ILDG_FORTRAN)
    return io_fail(IRO_UNSUPPORTED, "ILDG files need the lime library, which is not available");
  if (format != IRO_GAUGE_BINARY && format != IRO_GAUGE_NERSC)
    return io_fail(IRO_BAD_ARG, "the reference writes Binary and NERSC configurations only");
  File fh;
  fh.f = std::fopen(path, append ? "ab" : "wb");
  if (!fh.f) return io_fail(IRO_IO_ERROR, std::string("cannot open ") + path + ": " + std::strerror(errno));
  // BinaryWriter::write stores host byte order (binary_writer.cpp:18-21)
  const int rc = format == IRO_GAUGE_NERSC ? write_nersc(fh.f, g, u, path)
                                           : write_binary(fh.f, g, u, path, false);
  if (rc) return rc;
  if (std::fflush(fh.f) != 0) return io_fail(IRO_IO_ERROR, std::string("write failed: ") + path);
  return IRO_OK;
}
