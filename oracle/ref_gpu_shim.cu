/*
 * ref_gpu_shim.cu -- a C entry point over the reference's own GPU init
 * engine, SmpInitEngine3 ("Smp-Init-Gpu", include/smp/smp_init_3.h).
 *
 * STUDY INFRASTRUCTURE ONLY.  Compiled by `make -C oracle ref-gpu` from the
 * reference's unmodified headers into oracle/_ref/libsmpref_gpu.so, and used
 * by `bench.py --init-study` to time the reference's rank-matrix (and
 * PR-matrix) initialisation beside this library's inversion on the same
 * B200, as the reference's benchmark/figure_5.cu does through
 * SmpInitEngineExecutor (benchmark/smp_init_engine_exec.h:7-37).  The
 * engine reports its own figures through PrintProfilingInfo
 * (smp_init_3.h:36-66); they are read back from that output.
 */
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>
#include <thrust/device_vector.h>
#include <thrust/host_vector.h>

#include "utils/utils.h"
#include "utils/types.h"
#include "smp/smp_init.h"
#include "utils/dev_array.h"
#include "utils/stream.h"
#include "utils/launcher.h"
// The engine keeps the rank matrix it copied back in a private member; the
// parity test reads it, so this one header is compiled with its members open
// (every header it relies on is already included above).
#define private public
#include "smp/smp_init_3.h"
#undef private

namespace {

// "<name> <label>: <value> ms" from the engine's report, or -1.
double field(const std::string &text, const std::string &label) {
  const size_t at = text.find(label);
  if (at == std::string::npos) return -1.0;
  return std::stod(text.substr(at + label.size()));
}

}  // namespace

extern "C" {

// Runs SmpInitEngine3 on the lists (host, n x n int32).  Returns the engine's
// kernel, host-device transfer and total init times in ms.
int ref_gpu_init(const int32_t *pref_m, const int32_t *pref_w, int32_t n, int init_pr, double *kernel_ms,
                 double *transfer_ms, double *total_ms) {
  const size_t nn = static_cast<size_t>(n) * n;
  FlatPreferenceList m(pref_m, pref_m + nn), w(pref_w, pref_w + nn);
  auto smp = bamboosmp::SmpObjInit::CreateFromFlatLists(m, w, n);
  bamboosmp::SmpInitEngine3 engine(*smp, static_cast<size_t>(n), init_pr != 0);
  engine.Init();
  std::stringstream out;
  std::streambuf *old = std::cout.rdbuf(out.rdbuf());
  engine.PrintProfilingInfo();
  std::cout.rdbuf(old);
  const std::string text = out.str();
  *kernel_ms = field(text, "Kernel Time: ");
  *transfer_ms = field(text, "Host-Device Transfer Time: ");
  *total_ms = field(text, "Total Init Time: ");
  return *kernel_ms < 0 ? -1 : 0;
}

// The rank matrix SmpInitEngine3 computes on the GPU (InitRankMatrix,
// include/smp/smp_init_3.h:68-95) and copies back: rank_out[w*n + m] =
// position of m in w's list (n x n int32).  Returns 0.
int ref_gpu_rank(const int32_t *pref_m, const int32_t *pref_w, int32_t n, int32_t *rank_out) {
  const size_t nn = static_cast<size_t>(n) * n;
  FlatPreferenceList m(pref_m, pref_m + nn), w(pref_w, pref_w + nn);
  auto smp = bamboosmp::SmpObjInit::CreateFromFlatLists(m, w, n);
  bamboosmp::SmpInitEngine3 engine(*smp, static_cast<size_t>(n), false);
  engine.Init();
  if (engine.host_rank_mtx_w_.size() != nn) return -1;
  std::memcpy(rank_out, thrust::raw_pointer_cast(engine.host_rank_mtx_w_.data()), sizeof(int32_t) * nn);
  return 0;
}

}  // extern "C"
