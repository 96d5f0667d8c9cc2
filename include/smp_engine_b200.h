// smp_engine_b200.h -- C++ drop-in engine over the C ABI of smp_b200.h.
//
// SmpEngineB200 has the shape the reference's executor template expects of
// an engine (victorliu-sq/PACTAE, benchmark/smp_engine_exec.h:6-32):
//
//     SmpEngineB200 engine(smp, n);           // smp: bamboosmp::SmpObj
//     Matching m = engine.FindStableMatching();
//     engine.PrintProfilingInfo();
//     engine.GetEngineName();
//
// Built inside the reference tree (define SMP_B200_WITH_REFERENCE_API and
// put the reference's include/ on the include path) it derives from the
// reference's AbsSmpEngine (include/smp/smp_engine_abs.h:6-74), so the
// template method FindStableMatching, its precheck/init/core stopwatches and
// PrintProfilingInfo are the reference's own.  Built standalone it derives
// from smp_b200::EngineBase below, a restatement of the same template method
// (the phase order and the timing of precheck, init and core are kept alike
// so the reference's log parsers read this engine's output unchanged).
//
// Phase mapping (SmpEngineBamboo, src/smp/smp_engine_bamboo.cu):
//   constructor   copy both lists to the device        (:6-31, H2D :28-29)
//   IsPerfect     distinct first choices, on the GPU   (smp_engine_bamboo.h:25-33)
//   InitProc      rank inversion / prefix build         (:33-106)
//   CoreProc      proposals + the tail, all on the GPU (:108-287)
//   PostProc      match[m] = w, copied to the host      (:289-306)
//
// Errors: a non-OK status from the library throws smp_b200::Error (the
// reference terminates the process instead, include/utils/utils.h:38-47).
#ifndef SMP_ENGINE_B200_H
#define SMP_ENGINE_B200_H

#include <chrono>
#include <cstddef>
#include <cstdint>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "smp_b200.h"

#ifdef SMP_B200_WITH_REFERENCE_API
#include "smp/smp.h"
#include "smp/smp_engine_abs.h"
#endif

namespace smp_b200 {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string &where)
      : std::runtime_error(where + ": " + smp_b200_strerror(status)), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void check(int status, const char *where) {
  if (status != SMP_OK) throw Error(status, where);
}

#ifndef SMP_B200_WITH_REFERENCE_API
// Standalone stand-ins for the reference's types (include/utils/types.h:33,
// :44; include/smp/smp.h:8-16): the engine only reads the two flat lists.
using Matching = std::vector<int>;
using String = std::string;

struct SmpObj {
  std::vector<int> flatten_pref_lists_m_vec;
  std::vector<int> flatten_pref_lists_w_vec;
  int *flatten_pref_lists_m = nullptr;
  int *flatten_pref_lists_w = nullptr;

  static SmpObj FromFlatLists(std::vector<int> m, std::vector<int> w) {
    SmpObj o;
    o.flatten_pref_lists_m_vec = std::move(m);
    o.flatten_pref_lists_w_vec = std::move(w);
    o.flatten_pref_lists_m = o.flatten_pref_lists_m_vec.data();
    o.flatten_pref_lists_w = o.flatten_pref_lists_w_vec.data();
    return o;
  }
};

// The template method of the reference's engine base: precheck, then (unless
// the first choices are distinct) init and core, each timed by the wall
// clock, then post-processing.
class EngineBase {
 public:
  virtual ~EngineBase() = default;

  Matching FindStableMatching() {
    auto t0 = Clock::now();
    const bool perfect = IsPerfect();
    precheck_time_ = Ms(t0);
    if (!perfect) {
      t0 = Clock::now();
      InitProc();
      init_time_ = Ms(t0);
      t0 = Clock::now();
      CoreProc();
      core_time_ = Ms(t0);
    } else {
      std::cout << "Perfect matching identified; skipping execution steps." << std::endl;
    }
    return PostProc();
  }

  virtual void PrintProfilingInfo() {
    const String name = GetEngineName();
    std::cout << name << " Profiling Info:" << std::endl;
    std::cout << name << " Precheck Time: " << precheck_time_ << " ms" << std::endl;
    std::cout << name << " Init Time: " << init_time_ << " ms" << std::endl;
    std::cout << name << " Core Time: " << core_time_ << " ms" << std::endl;
    std::cout << name << " Total Time: " << precheck_time_ + init_time_ + core_time_ << " ms" << std::endl;
    std::cout << "==================================================================" << std::endl;
  }

  virtual String GetEngineName() const = 0;

 protected:
  virtual bool IsPerfect() const = 0;
  virtual void InitProc() = 0;
  virtual void CoreProc() = 0;
  virtual Matching PostProc() = 0;

  double precheck_time_ = 0;
  double init_time_ = 0;
  double core_time_ = 0;

 private:
  using Clock = std::chrono::steady_clock;
  static double Ms(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  }
};
using SmpObjType = SmpObj;
using Base = EngineBase;
#else
using Matching = ::Matching;
using String = ::String;
using SmpObjType = bamboosmp::SmpObj;
using Base = ::AbsSmpEngine;
#endif

// The engine: one library context per engine; the two lists are borrowed
// from the SmpObj (which must outlive the engine) and copied to the device
// in the constructor, as the reference's GPU engines do.
class SmpEngineB200 : public Base {
 public:
  SmpEngineB200(const SmpObjType &smp, size_t n, int device = 0) : n_(static_cast<int32_t>(n)) {
    smp_cfg cfg = {};
    cfg.device = device;
    check(smp_b200_create(&ctx_, &cfg), "smp_b200_create");
    try {
      check(smp_b200_stage(ctx_, smp.flatten_pref_lists_m, smp.flatten_pref_lists_w, n_, 0), "smp_b200_stage");
    } catch (...) {
      smp_b200_destroy(ctx_);
      throw;
    }
  }
  ~SmpEngineB200() override { smp_b200_destroy(ctx_); }
  SmpEngineB200(const SmpEngineB200 &) = delete;
  SmpEngineB200 &operator=(const SmpEngineB200 &) = delete;

  auto GetEngineName() const -> String override { return "B200-GS"; }

  // Device-side statistics of the last run (proposals, per-phase GPU time).
  smp_stats Stats() const {
    smp_stats st = {};
    smp_b200_stats(ctx_, &st);
    return st;
  }

 protected:
  auto IsPerfect() const -> bool override {
    int32_t perfect = 0;
    check(smp_b200_precheck(ctx_, &perfect), "smp_b200_precheck");
    return perfect != 0;
  }
  void InitProc() override { check(smp_b200_init(ctx_), "smp_b200_init"); }
  void CoreProc() override { check(smp_b200_core(ctx_), "smp_b200_core"); }
  auto PostProc() -> Matching override {
    Matching match(static_cast<size_t>(n_));
    check(smp_b200_post(ctx_, match.data(), 0), "smp_b200_post");
    return match;
  }

 private:
  smp_ctx *ctx_ = nullptr;
  int32_t n_;
};

}  // namespace smp_b200

#endif  // SMP_ENGINE_B200_H
