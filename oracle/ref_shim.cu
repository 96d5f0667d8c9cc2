/*
 * ref_shim.cu -- a C entry point over the reference's own CPU engines.
 *
 * TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile together with the
 * reference's unmodified sources (src/smp/smp.cu and
 * src/smp/smp_engine_{gs_1,mw_1,gs_2,mw_2}.cu) into oracle/_ref/libsmpref.so.
 * It is how the tests pin the oracle to the reference, and how bench.py's
 * reference arm times the reference's CPU path.  It drives the engines the
 * way the reference's SmpEngineExecutor does (benchmark/smp_engine_exec.h:6-32):
 * SmpObj::CreateFromFlatLists, Engine(smp, n), FindStableMatching(), and
 * reads the phase timings that AbsSmpEngine records (smp_engine_abs.h:10-36).
 */
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>

#include "smp/smp.h"
#include "smp/smp_engine_gs_1.h"
#include "smp/smp_engine_gs_2.h"
#include "smp/smp_engine_mw_1.h"
#include "smp/smp_engine_mw_2.h"
#include "utils/generate_workloads_flat.h"

namespace {

// AbsSmpEngine keeps the phase timings protected; a subclass reads them.
template <class Engine>
struct Timed : Engine {
  using Engine::Engine;
  double precheck() const { return this->precheck_time_; }
  double init() const { return this->init_time_; }
  double core() const { return this->core_time_; }
};

template <class Engine>
int run(const bamboosmp::SmpObj &smp, int32_t n, int32_t *match, double *ms3) {
  Timed<Engine> engine(smp, static_cast<size_t>(n));
  Matching m = engine.FindStableMatching();
  if (static_cast<int32_t>(m.size()) != n) return -1;
  std::memcpy(match, m.data(), sizeof(int32_t) * static_cast<size_t>(n));
  if (ms3) {
    ms3[0] = engine.precheck();
    ms3[1] = engine.init();
    ms3[2] = engine.core();
  }
  return 0;
}

int hw_threads() {
  unsigned hw = std::thread::hardware_concurrency();
  return static_cast<int>(hw < 96u ? hw : 96u);
}

// The reference's row split for the rank init (smp_engine_mw_1.cu:18-24,
// smp_engine_mw_2.cu:17-23, smp_engine_gs_2.cu:19-25) gives thread t the rows
// [t*R, (t+1)*R) with R = ceil(n/T), except the last thread, which ends at n.
// A thread t < T-1 whose range starts below n but ends above it writes past
// the rank matrix, so those engines are only run when (T-1)*R <= n.  Gs-Par
// also pops from per-thread queues that are empty when n < T
// (smp_engine_gs_2.cu:47-59), so it needs n >= T as well.
bool engine_safe(int engine, int32_t n) {
  if (engine == 0) return true;
  const long t = hw_threads();
  const long r = (static_cast<long>(n) + t - 1) / t;
  if ((t - 1) * r > n) return false;
  if (engine == 2 && n < t) return false;
  return true;
}

}  // namespace

extern "C" {

/* engine: 0 Gs-Seq-CPU, 1 Mw-Seq-CPU, 2 Gs-Par-Cpu, 3 Mw-Par-Cpu.
 * ms3 (optional) receives the precheck / init / core milliseconds.
 * Returns 0, -1 on bad arguments, -2 if the engine is unsafe at this n. */
int ref_solve(int engine, const int32_t *pref_m, const int32_t *pref_w,
              int32_t n, int32_t *match, double *ms3) {
  if (n <= 0 || !pref_m || !pref_w || !match) return -1;
  if (!engine_safe(engine, n)) return -2;
  const size_t nn = static_cast<size_t>(n) * static_cast<size_t>(n);
  std::unique_ptr<bamboosmp::SmpObj> smp;
  {
    FlatPreferenceList fm(pref_m, pref_m + nn), fw(pref_w, pref_w + nn);
    smp = bamboosmp::SmpObj::CreateFromFlatLists(fm, fw, n);
  }
  switch (engine) {
    case 0: return run<bamboosmp::SmpEngineGs>(*smp, n, match, ms3);
    case 1: return run<bamboosmp::SmpEngineMw>(*smp, n, match, ms3);
    case 2: return run<bamboosmp::SmpEngineGs2>(*smp, n, match, ms3);
    case 3: return run<bamboosmp::SmpEngineMw2>(*smp, n, match, ms3);
    default: return -1;
  }
}

/* A problem object kept across solves, so repeated timed runs do not copy
 * the n x n lists again (SmpObj::CreateFromFlatLists copies them). */
void *ref_obj_create(const int32_t *pref_m, const int32_t *pref_w, int32_t n) {
  if (n <= 0 || !pref_m || !pref_w) return nullptr;
  const size_t nn = static_cast<size_t>(n) * static_cast<size_t>(n);
  FlatPreferenceList fm(pref_m, pref_m + nn), fw(pref_w, pref_w + nn);
  return bamboosmp::SmpObj::CreateFromFlatLists(fm, fw, n).release();
}

void ref_obj_destroy(void *obj) { delete static_cast<bamboosmp::SmpObj *>(obj); }

/* Construct the engine on the kept object and run FindStableMatching once. */
int ref_obj_solve(void *obj, int engine, int32_t n, int32_t *match, double *ms3) {
  if (!obj || !match || n <= 0) return -1;
  if (!engine_safe(engine, n)) return -2;
  const auto &smp = *static_cast<bamboosmp::SmpObj *>(obj);
  switch (engine) {
    case 0: return run<bamboosmp::SmpEngineGs>(smp, n, match, ms3);
    case 1: return run<bamboosmp::SmpEngineMw>(smp, n, match, ms3);
    case 2: return run<bamboosmp::SmpEngineGs2>(smp, n, match, ms3);
    case 3: return run<bamboosmp::SmpEngineMw2>(smp, n, match, ms3);
    default: return -1;
  }
}

/* Threads the multithreaded engines use: min(hardware_concurrency, 96)
 * (smp_engine_gs_2.cu:8, smp_engine_mw_2.cu:7). */
int ref_threads(void) { return hw_threads(); }

/* 1 if the engine can run at this n without the out-of-range writes above. */
int ref_engine_safe(int engine, int32_t n) { return engine_safe(engine, n) ? 1 : 0; }

// The reference's workload cache (generate_workloads_flat.h:283-376).  Both
// prepend "data/workloads/" to the file name, relative to the working
// directory, as the reference does.
int ref_workload_save(const char *filename, const int32_t *pref_m, const int32_t *pref_w, int32_t n) {
  const size_t nn = static_cast<size_t>(n) * n;
  FlatPreferenceList m(pref_m, pref_m + nn), w(pref_w, pref_w + nn);
  SaveSmpWorkload(filename, m, w, n);
  return 0;
}
int ref_workload_load(const char *filename, int32_t n, int32_t *pref_m, int32_t *pref_w) {
  FlatPreferenceList m, w;
  int n_file = 0;
  LoadSmpWorkload(filename, m, w, n_file);
  if (n_file != n) return -1;
  std::memcpy(pref_m, m.data(), sizeof(int32_t) * m.size());
  std::memcpy(pref_w, w.data(), sizeof(int32_t) * w.size());
  return 0;
}
int ref_workload_filename(int type, int32_t n, int32_t group_size, char *buf, int32_t len) {
  const String name = GetWorkloadFilename(static_cast<WorkloadType>(type), static_cast<size_t>(n),
                                          static_cast<size_t>(group_size));
  if (static_cast<int32_t>(name.size()) + 1 > len) return -1;
  std::memcpy(buf, name.c_str(), name.size() + 1);
  return 0;
}

}  // extern "C"
