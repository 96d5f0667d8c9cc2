// Compile-only check: the reference's own executor template
// (benchmark/smp_engine_exec.h:6-32) instantiates with SmpEngineB200 derived
// from the reference's AbsSmpEngine.
#define SMP_B200_WITH_REFERENCE_API
#include "smp_engine_exec.h"
#include "smp_engine_b200.h"

void run_b200_like_figure_9() { SmpEngineExecutor<smp_b200::SmpEngineB200>(RANDOM, 30000); }
