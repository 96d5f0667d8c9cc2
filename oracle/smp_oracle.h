/*
 * smp_oracle.h -- CPU oracle for the Gale-Shapley stable-marriage path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs may load it.  The product library
 * (pactae_b200/libsmp_b200.so) never links, loads or calls it.
 *
 * What it restates (reference = victorliu-sq/PACTAE, paths relative to that
 * project):
 *   oracle_gs_seq     src/smp/smp_engine_gs_1.cu:16-98   (Gs-Seq-CPU: rank init,
 *                     FIFO free-men queue, CoreProc loop, PostProc)
 *   oracle_mw_seq     src/smp/smp_engine_mw_1.cu:45-91   (Mw-Seq-CPU chain
 *                     following; cross-check only)
 *   oracle_invert     src/smp/kernel.cu:672-686 / smp_engine_gs_1.cu:18-36
 *                     (rank[w][pref_w[w][r]] = r)
 *   oracle_is_perfect include/smp/smp_engine_bamboo.h:25-33 (distinct first
 *                     choices)
 *   oracle_generate   seeded restatement of the workload families in
 *                     include/utils/generate_workloads_flat.h:14-280, plus the
 *                     uniform / congested / correlated distributions of the
 *                     B200 build (the reference generators are unseeded, so
 *                     these are new, fully specified, counter-based streams).
 *
 * Parity pin: the reference's own CPU engines are compiled from their sources
 * by oracle/Makefile into oracle/_ref/ and run on the same seeded inputs by
 * tests/golden/make_golden.py; the matchings they return are committed as
 * fixtures and this oracle is tested against them.
 */
#ifndef SMP_ORACLE_H
#define SMP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Workload kinds; identical numbering to SMP_GEN_* in include/smp_b200.h. */
enum {
  ORACLE_GEN_UNIFORM = 0,       /* both sides: independent uniform permutations   */
  ORACLE_GEN_CONGESTED = 1,     /* men: one shared uniform row; women: uniform    */
  ORACLE_GEN_CORRELATED = 2,    /* score + Irwin-Hall noise, sigma in 1e-4 units  */
  ORACLE_GEN_PERFECT = 3,       /* reference PERFECT: distinct first choices      */
  ORACLE_GEN_REF_CONGESTED = 4, /* reference CONGESTED: every row identical       */
  ORACLE_GEN_GROUPED = 5,       /* reference RANDOM(group): in-group shuffles     */
  ORACLE_GEN_SOLO = 6           /* reference SOLO                                 */
};

/* Philox4x32-10 (Salmon et al., SC'11), the counter-based generator every
 * workload stream is drawn from. */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2],
                          uint32_t out[4]);

/* Fill one side (side 0 = men, 1 = women) of an instance: pref[i*n + r] is the
 * r-th choice of row i.  salt separates instances of a batch (0 for single
 * instances).  param: sigma*1e4 for CORRELATED, group size for GROUPED.
 * Returns 0, or -1 on invalid arguments. */
int oracle_generate_side(int kind, int side, int32_t n, uint64_t seed,
                         uint32_t salt, int32_t param, int32_t *pref);

/* Both sides.  Returns 0 or -1. */
int oracle_generate(int kind, int32_t n, uint64_t seed, uint32_t salt,
                    int32_t param, int32_t *pref_m, int32_t *pref_w);

/* rank[w*n + pref_w[w*n + r]] = r.  Returns 0, or -1 if a row of pref_w is
 * not a permutation of 0..n-1. */
int oracle_invert(const int32_t *pref_w, int32_t n, int32_t *rank);

/* 1 if every man's first choice is distinct, else 0. */
int oracle_is_perfect(const int32_t *pref_m, int32_t n);

/* Sequential Gale-Shapley with a FIFO queue of free men (Gs-Seq-CPU).
 * match[m] = w.  *proposals receives the number of proposals made.
 * Returns 0, or -1 on invalid input (non-permutation rows). */
int oracle_gs_seq(const int32_t *pref_m, const int32_t *pref_w, int32_t n,
                  int32_t *match, int64_t *proposals);

/* Sequential McVitie-Wilson chain following (Mw-Seq-CPU). */
int oracle_mw_seq(const int32_t *pref_m, const int32_t *pref_w, int32_t n,
                  int32_t *match, int64_t *proposals);

/* Stability check.  Returns the number of blocking pairs (>= 0), or -1 if
 * match is not a perfect matching (a permutation of 0..n-1) or the input is
 * invalid.  *proposals (if non-null) receives sum_m (position of match[m] in
 * m's list + 1), which equals the proposal count of every Gale-Shapley
 * execution on this instance. */
int64_t oracle_check(const int32_t *pref_m, const int32_t *pref_w, int32_t n,
                     const int32_t *match, int64_t *proposals);

/* Batch recipe shared by the oracle and the product: instance b of a batch
 * drawn with (seed, n_lo, n_hi) has size n = floor(n_lo * (n_hi/n_lo)^u) and
 * kind uniform/congested/correlated chosen from the same Philox stream. */
void oracle_batch_instance(uint64_t seed, uint32_t b, int32_t n_lo,
                           int32_t n_hi, int32_t *n_out, int32_t *kind_out);

#ifdef __cplusplus
}
#endif

#endif /* SMP_ORACLE_H */
