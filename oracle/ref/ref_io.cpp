// Test-infrastructure driver around the reference's gauge-configuration
// readers and writers (lib/IO/, lib/Main/gaugeConf.cpp) and Staples'
// plaquette, for the golden fixtures of the gauge-file readers.
//
// Compiled with the reference's IO sources at -O0 without unreachable traps by
// oracle/Makefile (those sources have int functions without a return,
// harmless only so) and
// linked into oracle/_ref/libiroiro_ref.so next to ref_driver.cpp, whose
// ref_init() sets up the lattice singletons these calls use.  Like the other
// reference calls, each runs on a worker thread with a large stack.
#include <pthread.h>
#include <cstring>
#include <functional>
#include <iostream>
#include <streambuf>
#include <string>

#include "include/commonPrms.hpp"
#include "include/field.h"
#include "include/format_G.h"
#include "IO/fields_io.hpp"
#include "Main/gaugeConf.hpp"
#include "Measurements/GaugeM/staples.hpp"

// CCIO::getReader / getWriter live in lib/IO/fields_io.cpp next to the ILDG
// classes, which need the absent lime library; the factories for the formats
// that do build are defined here instead (same contract: a new object per call).
namespace CCIO {
GeneralReader* getReader(const std::string id, int vol, int nin, int nex) {
  if (id == "Binary") return new BinaryReader(vol, nin, nex);
  if (id == "NERSC") return new NERSCReader(vol, nin, nex);
  if (id == "JLQCDLegacy") return new JLQCDLegacyReader(vol, nin, nex);
  return nullptr;
}
GeneralWriter* getWriter(const std::string id, int vol, int nin, int nex, const Field& U) {
  if (id == "Binary") return new BinaryWriter(vol, nin, nex);
  if (id == "NERSC") return new NERSCWriter(vol, nin, nex, U);
  return nullptr;
}
GeneralWriter* getWriter(const std::string id, int vol, int nin, int nex) {
  if (id == "Binary") return new BinaryWriter(vol, nin, nex);
  return nullptr;
}
}  // namespace CCIO

extern "C" int ref_ready(void);  // ref_driver.cpp: ref_init() has run

namespace {

struct NullBuf : std::streambuf {
  int overflow(int c) override { return c; }
};
NullBuf g_null;

// silences the readers' and writers' progress output
struct Quiet {
  std::streambuf* old;
  Quiet() : old(std::cout.rdbuf(&g_null)) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

struct Job {
  std::function<int()> fn;
  int rc;
};

void* job_entry(void* p) {
  Job* j = static_cast<Job*>(p);
  try {
    j->rc = j->fn();
  } catch (...) {
    j->rc = 3;
  }
  return nullptr;
}

int on_big_stack(std::function<int()> fn) {
  Job job{std::move(fn), -1};
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, size_t(256) << 20);
  pthread_t th;
  if (pthread_create(&th, &attr, job_entry, &job) != 0) return 4;
  pthread_join(th, nullptr);
  pthread_attr_destroy(&attr);
  return job.rc;
}

bool ready() { return ref_ready() != 0; }

size_t gsize() { return size_t(18) * 4 * CommonPrms::instance()->Nvol(); }

}  // namespace

extern "C" {

// CCIO::SaveOnDisk<Format_G>(u, path, false, writer) (lib/IO/fields_io.hpp:48-139);
// writer 0 = "Binary", 2 = "NERSC".
int ref_gauge_save(const double* u, const char* path, int writer) {
  if (!ready()) return 1;
  if (writer != 0 && writer != 2) return 2;
  const std::string file(path);
  return on_big_stack([=]() {
    Quiet q;
    Field f(std::valarray<double>(u, gsize()));
    return CCIO::SaveOnDisk<Format::Format_G>(f, file.c_str(), false,
                                              writer == 0 ? "Binary" : "NERSC");
  });
}

// GaugeConf_*::init_conf (lib/Main/gaugeConf.cpp:23-228): kind 0 = bin, 2 = NERSC,
// 5 = csdt, 6 = txt, 7 = unit.  JLQCDLegacy is not offered: its reader
// indexes past its row buffer for directions > 0 (JLQCDLegacy_reader.cpp:16-43).
int ref_gauge_load(const char* path, int kind, double* u) {
  if (!ready()) return 1;
  if (kind != 0 && kind != 2 && kind != 5 && kind != 6 && kind != 7) return 2;
  const std::string file(path ? path : "");
  return on_big_stack([=]() {
    Quiet q;
    Format::Format_G fg(CommonPrms::instance()->Nvol());
    Field f(fg.size());
    switch (kind) {
      case 0: GaugeConf_bin(fg, file).init_conf(f); break;
      case 2: GaugeConf_NERSC(fg, file).init_conf(f); break;
      case 5: GaugeConf_csdt(fg, file).init_conf(f); break;
      case 6: GaugeConf_txt(fg, file).init_conf(f); break;
      default: GaugeConf_unit(fg).init_conf(f); break;
    }
    const std::valarray<double>& va = f.getva();
    std::memcpy(u, &va[0], sizeof(double) * va.size());
    return 0;
  });
}

// Staples::plaquette and Staples::link_trace
// (lib/Measurements/GaugeM/staples.cpp:24-38).
int ref_plaquette(const double* u, double* plaq, double* trace) {
  if (!ready()) return 1;
  return on_big_stack([=]() {
    Quiet q;
    Field f(std::valarray<double>(u, gsize()));
    GaugeField U(f);
    Staples st;
    *plaq = st.plaquette(U);
    *trace = st.link_trace(U);
    return 0;
  });
}

}  // extern "C"
