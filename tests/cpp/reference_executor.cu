// The reference's own engine API driving SmpEngineB200.
//
// Built inside the reference's include tree (SMP_B200_WITH_REFERENCE_API),
// SmpEngineB200 derives from the reference's AbsSmpEngine
// (include/smp/smp_engine_abs.h:6-74), so FindStableMatching, its phase
// stopwatches and PrintProfilingInfo below are the reference's own code.  The
// SmpObj is the reference's bamboosmp::SmpObj (include/smp/smp.h:8-52, with
// src/smp/smp.cu linked in), made the way its executor makes one
// (benchmark/smp_engine_exec.h:13-15).  The executor template itself also
// instantiates with this engine (run_b200_like_figure_9); it is not called,
// because its GenerateWorkloadCached draws unseeded lists.
//
// Usage: reference_executor <in.bin> <out.bin>
//   in.bin:  int32 n, then pref_m (n*n int32), then pref_w (n*n int32)
//   out.bin: int32 match[n] as FindStableMatching returned it
#define SMP_B200_WITH_REFERENCE_API
#include <cstdio>
#include <vector>

#include "smp_engine_exec.h"
#include "smp_engine_b200.h"

void run_b200_like_figure_9() { SmpEngineExecutor<smp_b200::SmpEngineB200>(RANDOM, 30000); }

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s <in.bin> <out.bin>\n", argv[0]);
    return 2;
  }
  std::FILE *in = std::fopen(argv[1], "rb");
  if (!in) return 2;
  int n = 0;
  if (std::fread(&n, sizeof(int), 1, in) != 1 || n <= 0) return 2;
  const size_t nn = static_cast<size_t>(n) * n;
  FlatPreferenceList plM(nn), plW(nn);
  if (std::fread(plM.data(), sizeof(int), nn, in) != nn || std::fread(plW.data(), sizeof(int), nn, in) != nn) return 2;
  std::fclose(in);

  auto smp = bamboosmp::SmpObj::CreateFromFlatLists(plM, plW, n);
  Matching match;
  try {
    smp_b200::SmpEngineB200 engine(*smp, static_cast<size_t>(n));
    match = engine.FindStableMatching();
    engine.PrintProfilingInfo();
  } catch (const smp_b200::Error &e) {
    std::fprintf(stderr, "engine error: %s\n", e.what());
    return 1;
  }
  std::FILE *out = std::fopen(argv[2], "wb");
  if (!out || std::fwrite(match.data(), sizeof(int), match.size(), out) != match.size()) return 2;
  std::fclose(out);
  std::printf("REFERENCE_API_OK n=%d\n", n);
  return 0;
}
