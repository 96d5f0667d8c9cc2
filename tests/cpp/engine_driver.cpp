// Drives smp_b200::SmpEngineB200 the way the reference's executor does
// (construct on an SmpObj, FindStableMatching, PrintProfilingInfo) and checks
// the matching against smp_b200_solve with the GPU stability checker.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "smp_engine_b200.h"

int main(int argc, char **argv) {
  const int n = argc > 1 ? std::atoi(argv[1]) : 500;
  const int kind = argc > 2 ? std::atoi(argv[2]) : SMP_GEN_UNIFORM;
  std::vector<int> m(static_cast<size_t>(n) * n), w(static_cast<size_t>(n) * n);
  smp_ctx *ctx = nullptr;
  smp_b200::check(smp_b200_create(&ctx, nullptr), "smp_b200_create");
  smp_b200::check(smp_b200_generate(ctx, kind, n, 7, 0, kind == SMP_GEN_CORRELATED ? 500 : 0, m.data(), w.data(), 0),
                  "smp_b200_generate");
  const auto smp = smp_b200::SmpObj::FromFlatLists(m, w);
  std::vector<int> match;
  {
    smp_b200::SmpEngineB200 engine(smp, static_cast<size_t>(n));
    match = engine.FindStableMatching();
    engine.PrintProfilingInfo();
  }
  std::vector<int32_t> ref(static_cast<size_t>(n));
  smp_stats st = {};
  smp_b200::check(smp_b200_solve(ctx, m.data(), w.data(), n, ref.data(), SMP_F_CHECK, &st), "smp_b200_solve");
  smp_b200_destroy(ctx);
  if (match != std::vector<int>(ref.begin(), ref.end()) || st.blocking_pairs != 0) {
    std::printf("ENGINE_MISMATCH\n");
    return 1;
  }
  std::printf("ENGINE_OK n=%d proposals=%lld\n", n, static_cast<long long>(st.proposals));
  return 0;
}
