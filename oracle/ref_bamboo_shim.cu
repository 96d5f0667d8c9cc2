/*
 * ref_bamboo_shim.cu -- a C entry point over the reference's own GPU engine,
 * SmpEngineBamboo ("BambooSMP", src/smp/smp_engine_bamboo.cu:6-306).
 *
 * STUDY INFRASTRUCTURE ONLY.  `make -C oracle ref-bamboo` compiles it with
 * the reference's unmodified sources (src/smp/smp.cu,
 * src/smp/smp_engine_bamboo.cu, src/smp/kernel.cu) into
 * oracle/_ref/libsmpref_bamboo.so (the reference's release flags, whose
 * ptxas level is -O0) and oracle/_ref/libsmpref_bamboo_o3.so (ptxas -O3).
 * `bench.py --bamboo-study` uses it to time the reference's GPU path beside
 * this library's solve on the same B200 and inputs, driving the engine the
 * way SmpEngineExecutor does (benchmark/smp_engine_exec.h:6-32).
 *
 * Two things about the engine shape this file:
 *  - CoreProc detaches the thread that launched La3F9CoreKernel
 *    (smp_engine_bamboo.cu:108-112); that thread still calls the engine's
 *    stream Sync after the kernel.  The device is synchronised, and the
 *    thread given time to return, before the engine is destroyed.
 *  - The engine prints progress lines on stdout; they go to stderr here, so
 *    a caller's stdout keeps only its own output.
 */
#include <cuda_runtime.h>
#include <unistd.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <memory>
#include <thread>

#include "smp/smp.h"
#include "smp/smp_engine_bamboo.h"

namespace {

// AbsSmpEngine keeps the phase timings protected; a subclass reads them.
struct TimedBamboo : bamboosmp::SmpEngineBamboo {
  using bamboosmp::SmpEngineBamboo::SmpEngineBamboo;
  double precheck() const { return this->precheck_time_; }
  double init() const { return this->init_time_; }
  double core() const { return this->core_time_; }
};

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// stdout -> stderr for the engine's prints, restored on scope exit.
struct StdoutToStderr {
  int saved = -1;
  StdoutToStderr() {
    std::cout.flush();
    std::fflush(stdout);
    saved = dup(1);
    if (saved >= 0) dup2(2, 1);
  }
  ~StdoutToStderr() {
    std::cout.flush();
    std::fflush(stdout);
    if (saved >= 0) {
      dup2(saved, 1);
      close(saved);
    }
  }
};

}  // namespace

extern "C" {

/* Solves one instance with SmpEngineBamboo.  ms6 (optional) receives the
 * engine's own precheck / init / core milliseconds (AbsSmpEngine's timed
 * phases), then the wall milliseconds of the constructor (the lists' copy to
 * the device), of FindStableMatching (which adds the untimed BambooTransfer,
 * a 8n^2-byte copy of the PR matrix to the host, and PostProc) and of the
 * whole call.  Returns 0, -1 on bad arguments, -2 if n is outside the range
 * the engine's int index arithmetic covers (n * n < 2^31). */
int ref_bamboo_solve(const int32_t *pref_m, const int32_t *pref_w, int32_t n, int32_t *match, double *ms6) {
  if (n <= 0 || !pref_m || !pref_w || !match) return -1;
  if (static_cast<int64_t>(n) * n >= (int64_t{1} << 31)) return -2;
  const auto t_call = std::chrono::steady_clock::now();
  const size_t nn = static_cast<size_t>(n) * n;
  auto smp = bamboosmp::SmpObj::CreateFromFlatLists(FlatPreferenceList(pref_m, pref_m + nn),
                                                    FlatPreferenceList(pref_w, pref_w + nn), n);
  double times[6] = {0, 0, 0, 0, 0, 0};
  {
    StdoutToStderr quiet;
    const auto t_ctor = std::chrono::steady_clock::now();
    std::unique_ptr<TimedBamboo> engine(new TimedBamboo(*smp, static_cast<size_t>(n)));
    times[3] = ms_since(t_ctor);
    const auto t_find = std::chrono::steady_clock::now();
    Matching m = engine->FindStableMatching();
    times[4] = ms_since(t_find);
    times[0] = engine->precheck();
    times[1] = engine->init();
    times[2] = engine->core();
    if (static_cast<int32_t>(m.size()) == n) std::memcpy(match, m.data(), sizeof(int32_t) * static_cast<size_t>(n));
    // the detached kernel thread: its kernel ends, then its stream Sync returns
    cudaDeviceSynchronize();
    std::this_thread::sleep_for(std::chrono::milliseconds(200));
    engine.reset();
    if (static_cast<int32_t>(m.size()) != n) return -1;
  }
  times[5] = ms_since(t_call);
  if (ms6)
    for (int i = 0; i < 6; ++i) ms6[i] = times[i];
  return 0;
}

}  // extern "C"
