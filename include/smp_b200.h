/*
 * smp_b200.h -- C ABI of the B200 (sm_100a) Gale-Shapley stable-marriage
 * solver.
 *
 * The reference (victorliu-sq/PACTAE, BambooSMP) has no C or FFI layer; its
 * public surface is the C++ engine API.  Every entry point below replaces one
 * piece of that API, cited by file:line within the reference project:
 *
 *   smp_b200_create / smp_b200_destroy
 *       SmpEngineBamboo::SmpEngineBamboo (src/smp/smp_engine_bamboo.cu:6-31),
 *       which allocates the engine's device arrays, and its destructor
 *       (include/smp/smp_engine_bamboo.h:19-20).
 *   smp_b200_stage
 *       the H2D copy of both preference lists in the engine constructor
 *       (smp_engine_bamboo.cu:28-29), over the flat row-major lists of
 *       SmpObj (include/smp/smp.h:8-16).
 *   smp_b200_precheck    SmpEngineBamboo::IsPerfect (smp_engine_bamboo.h:25-33)
 *   smp_b200_init        SmpEngineBamboo::InitProc  (smp_engine_bamboo.cu:33-106)
 *   smp_b200_core        SmpEngineBamboo::CoreProc  (smp_engine_bamboo.cu:108-287),
 *                        including the host monitor / LAProcedure tail that
 *                        this library runs on the GPU instead.
 *   smp_b200_post        SmpEngineBamboo::PostProc  (smp_engine_bamboo.cu:289-306)
 *   smp_b200_solve       AbsSmpEngine::FindStableMatching
 *                        (include/smp/smp_engine_abs.h:10-36) in one call.
 *   smp_b200_stats       the phase timings AbsSmpEngine keeps
 *                        (smp_engine_abs.h:38-52, :68-70).
 *   smp_b200_invert      F9RankMatrixInitKernel (src/smp/kernel.cu:672-686) /
 *                        SmpInitEngine3::InitRankMatrix
 *                        (include/smp/smp_init_3.h:68-95).
 *   smp_b200_check       no counterpart (the reference has no stability
 *                        checker); verifies a Matching as returned by
 *                        FindStableMatching (include/utils/types.h:44).
 *   smp_b200_generate    GenerateWorkload (include/utils/generate_workloads_flat.h:250-280),
 *                        seeded.
 *   smp_b200_batch_*     many SmpEngineExecutor runs
 *   smp_b200_solve_batch (benchmark/smp_engine_exec.h:6-32) in one launch.
 *   smp_b200_server_*, smp_b200_submit / smp_b200_poll
 *                        no counterpart (serving loop on top of the solver).
 *
 * Conventions.
 *   - Preference lists are row-major int32 n x n: pref_m[m*n + r] is man m's
 *     r-th choice, pref_w[w*n + r] is woman w's r-th choice (SmpObj,
 *     smp.h:14-15).  The result is match[m] = w (Matching, types.h:44).
 *   - Every call returns an smp_status; none terminates the process (the
 *     reference's CUDA_CHECK calls std::terminate, include/utils/utils.h:38-47).
 *   - A context is not thread-safe; use one context per host thread.  All
 *     calls except smp_b200_submit are synchronous: when they return, the
 *     GPU work they started has finished.
 *   - Pointers are host pointers unless SMP_F_DEVICE_PTRS is given, in which
 *     case they are device pointers on the context's device, ready for use
 *     (the library runs on its own stream and does not wait on the caller's).
 */
#ifndef SMP_B200_H
#define SMP_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__) || defined(__clang__)
#define SMP_B200_API __attribute__((visibility("default")))
#else
#define SMP_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum smp_status {
  SMP_OK = 0,
  SMP_ERR_INVALID_ARG = 1,   /* null pointer, bad flag, n out of range       */
  SMP_ERR_INVALID_INPUT = 2, /* a preference row is not a permutation       */
  SMP_ERR_OOM = 3,           /* device or pinned allocation failed          */
  SMP_ERR_CUDA = 4,          /* a CUDA call failed                          */
  SMP_ERR_TIMEOUT = 5,       /* reserved: no call waits on the device with a */
                             /* time limit, so none returns it              */
  SMP_ERR_BUSY = 6,          /* serving: no slot or HBM budget free          */
  SMP_ERR_NOT_READY = 7,     /* serving: the ticket has not finished         */
  SMP_ERR_UNSUPPORTED = 8,   /* request outside this build's limits          */
  SMP_ERR_IO = 9             /* a workload file could not be read or written */
} smp_status;

/* Largest n accepted by any entry point (rank indices, men and positions are
 * packed into 21-bit fields). */
#define SMP_B200_MAX_N 1048575

/* Flags (bitwise OR). */
#define SMP_F_DEVICE_PTRS 0x1u  /* pref_m / pref_w / match are device pointers  */
#define SMP_F_CHECK 0x2u        /* run the GPU stability checker after solving  */
#define SMP_F_VALIDATE 0x4u     /* also check every man's row is a permutation   */
#define SMP_F_NO_PRECHECK 0x8u  /* skip the distinct-first-choices shortcut      */

/* Workload kinds for smp_b200_generate. */
#define SMP_GEN_UNIFORM 0       /* independent uniform permutations, both sides  */
#define SMP_GEN_CONGESTED 1     /* all men share one uniform row; women uniform  */
#define SMP_GEN_CORRELATED 2    /* common score + noise; param = sigma * 1e4     */
#define SMP_GEN_PERFECT 3       /* reference PERFECT (generate_workloads_flat.h:50-82)  */
#define SMP_GEN_REF_CONGESTED 4 /* reference CONGESTED (:14-47), both sides      */
#define SMP_GEN_GROUPED 5       /* reference RANDOM(g) (:85-137); param = g      */
#define SMP_GEN_SOLO 6          /* reference SOLO (:140-247); n >= 3             */

typedef struct smp_ctx smp_ctx;

typedef struct smp_cfg {
  int32_t device;          /* CUDA device ordinal                                   */
  int32_t prefix_k;        /* width of the per-man (woman, rank) prefix; 0 = auto,  */
                           /* -1 = none                                             */
  int32_t tail_threshold;  /* free men at which the single-CTA tail takes over;     */
                           /* 0 = auto, -1 = never                                  */
  int32_t bulk_window;     /* widest look-ahead of the all-SM kernel, in choices    */
                           /* per warp step (32, 64, 128, 256); 0 = auto            */
  uint64_t hbm_budget;     /* bytes the batch / serving paths may hold resident;    */
                           /* 0 = 64 GiB                                            */
  int32_t tail_window;     /* the same for the tail kernel; 0 = auto                */
  int32_t mode;            /* 0 = auto, 1 = the men's rank-matrix mode only         */
  int32_t rank_bytes;      /* bytes per rank-matrix entry: 0 = auto (2 up to        */
                           /* n = 65535, else 4), 4 = int32 ranks at any n (the     */
                           /* layout every n above 65535 uses)                      */
  int32_t reserved32;
  uint64_t reserved[2];
} smp_cfg;

typedef struct smp_stats {
  int64_t proposals;       /* Gale-Shapley proposals (equal for every execution)    */
  int64_t blocking_pairs;  /* from smp_b200_check / SMP_F_CHECK; -1 if not run     */
  int64_t tail_proposals;  /* the share of proposals settled by the tail kernel     */
  int32_t n;
  int32_t perfect;         /* 1 if the precheck short-circuited the solve          */
  int32_t tail_men;        /* free men handed to the tail kernel                   */
  int32_t rank_bytes;      /* bytes per rank-matrix entry (2 or 4)                  */
  int32_t kernel_launches; /* kernels the call launched                            */
  int32_t bulk_hops;       /* accepted proposals in the all-SM kernel              */
  int32_t tail_hops;       /* accepted proposals in the tail kernel                */
  int32_t mode;            /* 0 rank-matrix mode, 1 query mode, 2 query then rank, */
                           /* 3 the men share one list and the women proposed      */
  float stage_ms;          /* host->device copy of the inputs                       */
  float precheck_ms;       /* device time of each phase (CUDA events)              */
  float init_ms;
  float core_ms;
  float post_ms;
  float check_ms;
  float total_ms;          /* precheck + init + core + post                        */
  float invert_ms;         /* rank inversion / prefix query kernels (part of init) */
  float bulk_ms;           /* all-SM proposal kernel (part of core)                */
  float tail_ms;           /* single-CTA tail kernel (part of core)                */
  float reserved[2];
} smp_stats;

/* Context lifetime.  cfg may be NULL (device 0, defaults). */
SMP_B200_API int smp_b200_create(smp_ctx **out, const smp_cfg *cfg);
SMP_B200_API void smp_b200_destroy(smp_ctx *ctx);
SMP_B200_API const char *smp_b200_strerror(int status);
/* The message of the context's last failed call (which step, and the CUDA
 * error text where there is one); "" if none.  Valid until the next call on
 * the context. */
SMP_B200_API const char *smp_b200_last_error(const smp_ctx *ctx);
SMP_B200_API const char *smp_b200_version(void);

/* Phase API (AbsSmpEngine's template method, one call per phase). */
SMP_B200_API int smp_b200_stage(smp_ctx *ctx, const int32_t *pref_m, const int32_t *pref_w,
                   int32_t n, uint32_t flags);
SMP_B200_API int smp_b200_precheck(smp_ctx *ctx, int32_t *is_perfect);
SMP_B200_API int smp_b200_init(smp_ctx *ctx);
SMP_B200_API int smp_b200_core(smp_ctx *ctx);
SMP_B200_API int smp_b200_post(smp_ctx *ctx, int32_t *match_out, uint32_t flags);
SMP_B200_API int smp_b200_stats(const smp_ctx *ctx, smp_stats *st);

/* Whole solve: stage + precheck + init + core + post (+ check).  st may be
 * NULL. */
SMP_B200_API int smp_b200_solve(smp_ctx *ctx, const int32_t *pref_m, const int32_t *pref_w,
                   int32_t n, int32_t *match_out, uint32_t flags,
                   smp_stats *st);

/* Rank matrix rank[w*n + pref_w[w*n + r]] = r as int32. */
SMP_B200_API int smp_b200_invert(smp_ctx *ctx, const int32_t *pref_w, int32_t n,
                    int32_t *rank_out, uint32_t flags);

/* Stability checker: counts blocking pairs of match (SMP_ERR_INVALID_INPUT
 * if match is not a permutation) and the proposal count sum_m (position of
 * match[m] in m's list + 1). */
SMP_B200_API int smp_b200_check(smp_ctx *ctx, const int32_t *pref_m, const int32_t *pref_w,
                   int32_t n, const int32_t *match, uint32_t flags,
                   int64_t *blocking_pairs, int64_t *proposals);

/* ------------------------------------------------------------------------ */
/* Batches: many independent instances in one persistent launch.            */
/* ------------------------------------------------------------------------ */

/* One instance of a batch.  All pointers are device pointers on the
 * context's device; status and proposals are filled in by a run. */
typedef struct smp_instance {
  const int32_t *pref_m;   /* n*n int32, row-major                          */
  const int32_t *pref_w;   /* n*n int32, row-major                          */
  int32_t *match;          /* n int32: match[m] = w                          */
  int32_t n;               /* 1 .. SMP_B200_BATCH_MAX_N                      */
  int32_t status;          /* out: smp_status of this instance               */
  int64_t proposals;       /* out: Gale-Shapley proposals                    */
} smp_instance;

/* Largest instance a batch accepts (each CTA keeps one instance's bids and
 * positions in shared memory). */
#define SMP_B200_BATCH_MAX_N 16384

typedef struct smp_batch_cfg {
  int32_t block_threads;   /* threads per CTA (64..512); 0 = auto            */
  int32_t ctas_per_sm;     /* resident CTAs per SM (1..4); 0 = auto          */
  int32_t window;          /* look-ahead choices per warp step; 0 = auto     */
  int32_t use_graph;       /* 1 (default, also 0 here) = replay a captured   */
                           /* CUDA graph; -1 = plain stream launch           */
  int32_t rank_smem_kb;    /* shared memory per CTA for the rank matrix of   */
                           /* small instances (those with 2 n^2 bytes that  */
                           /* fit stay on chip); 0 = auto, -1 = none         */
  int32_t tune;            /* 0 = the autotuner picks every auto field on a  */
                           /* sample of the batch (cached per device, n and  */
                           /* batch size); -1 = fixed defaults               */
  int32_t threshold_n;     /* instances with n above it run the all-SM       */
                           /* single-instance pipeline, on side streams     */
                           /* beside the persistent kernel; 0 = auto (the    */
                           /* autotuner times none and the largest 8, 32 and */
                           /* 128; with tune = -1: none), -1 = none          */
  int32_t reserved;
} smp_batch_cfg;

typedef struct smp_batch_stats {
  int32_t instances;       /* instances in the batch                         */
  int32_t failed;          /* instances whose status is not SMP_OK           */
  int64_t proposals;       /* sum over the instances                         */
  float ms;                /* device time of the run (CUDA events)           */
  int32_t launches;        /* kernel launches the run made                   */
} smp_batch_stats;

typedef struct smp_batch smp_batch;

/* Prepares a batch: uploads the instance table (sorted largest first for
 * the work queue), sizes per-CTA scratch for the largest n and captures the
 * batched step as a CUDA graph.  The table is copied; the device buffers it
 * points to must stay valid while the batch is used.  cfg may be NULL. */
SMP_B200_API int smp_b200_batch_create(smp_ctx *ctx, const smp_instance *inst, int32_t count,
                                       const smp_batch_cfg *cfg, smp_batch **out);
/* One batched run: every instance solved by the persistent kernel.
 * results (may be NULL) receives the table with status and proposals. */
SMP_B200_API int smp_b200_batch_run(smp_batch *batch, smp_instance *results, smp_batch_stats *st);
/* The same kernel launched once per instance (the per-instance baseline). */
SMP_B200_API int smp_b200_batch_run_plain(smp_batch *batch, smp_instance *results, smp_batch_stats *st);
SMP_B200_API void smp_b200_batch_destroy(smp_batch *batch);
/* The shape a batch runs with (after tuning): block_threads, ctas_per_sm,
 * window, use_graph, rank_smem_kb (-1: none), tune (1: chosen by the
 * autotuner, -1: fixed) and threshold_n (-1: no instance is routed to the
 * all-SM pipeline). */
SMP_B200_API int smp_b200_batch_config(const smp_batch *batch, smp_batch_cfg *out);
/* create + run + destroy; the status and proposals of inst[] are filled in. */
SMP_B200_API int smp_b200_solve_batch(smp_ctx *ctx, smp_instance *inst, int32_t count, const smp_batch_cfg *cfg,
                                      smp_batch_stats *st);
/* Size and kind of instance b of a seeded mix: n = floor(n_lo * (n_hi/n_lo)^u)
 * (log-uniform) and kind uniform / congested / correlated, from the same
 * Philox stream as smp_b200_generate.  Host only. */
SMP_B200_API void smp_b200_batch_instance(uint64_t seed, uint32_t b, int32_t n_lo, int32_t n_hi, int32_t *n_out,
                                          int32_t *kind_out);

/* ------------------------------------------------------------------------ */
/* The reference's workload text cache (include/utils/generate_workloads_  */
/* flat.h:283-376, SaveSmpWorkload / LoadSmpWorkload / GetWorkloadFilename): */
/* "n\n", then the n rows of pref_m and the n rows of pref_w, each row     */
/* "v v ... v \n".  Host memory, every host thread.                        */
/* ------------------------------------------------------------------------ */

/* n from a workload file's first line. */
SMP_B200_API int smp_b200_workload_read_n(const char *path, int32_t *n_out);
/* Both lists of an n x n workload file into caller buffers (n*n int32 each).
 * Values are not checked (the solver validates); a short or malformed file
 * is SMP_ERR_INVALID_INPUT, an unreadable one SMP_ERR_IO.  Replaces
 * LoadSmpWorkload. */
SMP_B200_API int smp_b200_workload_read(const char *path, int32_t n, int32_t *pref_m, int32_t *pref_w);
/* Writes both lists in the same format (replaces SaveSmpWorkload). */
SMP_B200_API int smp_b200_workload_write(const char *path, const int32_t *pref_m, const int32_t *pref_w,
                                         int32_t n);
/* The file name the reference gives a workload of this kind
 * (SMP_GEN_GROUPED = RANDOM(group_size), SMP_GEN_SOLO, SMP_GEN_REF_CONGESTED,
 * SMP_GEN_PERFECT), e.g. "smp_workload_random_30000_5.txt".  Replaces
 * GetWorkloadFilename. */
SMP_B200_API int smp_b200_workload_filename(int32_t kind, int32_t n, int32_t group_size, char *buf, size_t len);

/* ------------------------------------------------------------------------ */
/* Serving: a request loop with continuous batching and HBM admission.      */
/* ------------------------------------------------------------------------ */

typedef struct smp_server smp_server;

typedef struct smp_server_cfg {
  int32_t device;          /* CUDA device ordinal                                    */
  int32_t max_wave;        /* most requests one batched launch takes; 0 = 256        */
  int32_t route_n;         /* requests with n above this use the all-SM pipeline;    */
                           /* 0 = 1024                                               */
  int32_t waves;           /* batched launches in flight at once; 0 = 2              */
  uint64_t hbm_budget;     /* bytes of admitted requests' preference and rank        */
                           /* matrices (10 n^2 per request); 0 = 64 GiB              */
  int32_t block_threads;   /* threads per CTA of the batched launches; 0 = 512       */
  int32_t ctas_per_sm;     /* CTAs per SM of a batched launch; 0 = 2                 */
  uint64_t large_slots;    /* requests above route_n solved at once, each on its own */
                           /* context and stream; 0 = 4 (at most 16)                 */
  uint64_t reserved[2];
} smp_server_cfg;

typedef struct smp_result {
  int32_t status;          /* smp_status of the request                              */
  int32_t n;
  int64_t proposals;
  double queue_ms;         /* submission to launch                                   */
  double latency_ms;       /* submission to completion                               */
} smp_result;

typedef struct smp_server_stats {
  int64_t submitted;
  int64_t completed;
  int64_t waves;           /* batched launches made                                  */
  int64_t large;           /* requests solved by the all-SM pipeline                 */
  int64_t admitted_bytes;  /* budget in use now                                      */
  int64_t peak_bytes;      /* most budget ever in use                                */
} smp_server_stats;

/* Starts the serving loop (its own host thread and CUDA streams). */
SMP_B200_API int smp_b200_server_create(const smp_server_cfg *cfg, smp_server **out);
/* Queues one request and returns at once with its ticket.  With
 * SMP_F_DEVICE_PTRS the lists and match_out are device pointers that must
 * stay valid until the request completes; otherwise they are host pointers
 * (copied in when the request is admitted, the matching copied back when it
 * completes).  A request whose matrices alone exceed the budget is refused
 * with SMP_ERR_BUSY. */
SMP_B200_API int smp_b200_submit(smp_server *srv, const int32_t *pref_m, const int32_t *pref_w, int32_t n,
                                 int32_t *match_out, uint32_t flags, int64_t *ticket);
/* Waits up to wait_ms (negative = forever) for a request.  SMP_OK: *result
 * holds its outcome (and the ticket is released); SMP_ERR_NOT_READY: still
 * running; SMP_ERR_INVALID_ARG: unknown ticket. */
SMP_B200_API int smp_b200_poll(smp_server *srv, int64_t ticket, int32_t wait_ms, smp_result *result);
SMP_B200_API int smp_b200_server_stats(smp_server *srv, smp_server_stats *st);
/* Finishes every submitted request, then stops the loop. */
SMP_B200_API void smp_b200_server_destroy(smp_server *srv);

/* Largest n smp_b200_solve_static accepts. */
#define SMP_B200_STATIC_MAX_N 1024

/* A whole solve that allocates nothing.  No counterpart in the reference:
 * it exists for callers that cannot allocate device memory when they need a
 * matching -- an application whose device memory is already held by its own
 * caching allocator, a process under a per-process device-memory limit, or a
 * loop that must not stall on cudaMalloc/cudaFree.  pref_m, pref_w and
 * match_out are device pointers on the current device; stream is a
 * cudaStream_t (NULL = the legacy default stream); proposals may be NULL.
 * All scratch lives in one file-scope device array of 2 MiB + 256 bytes that
 * every GPU loading the library keeps until exit, so n is limited to
 * SMP_B200_STATIC_MAX_N (larger n returns SMP_ERR_UNSUPPORTED before
 * anything runs).  The call is synchronous: it waits on the stream for the
 * result header, so it cannot be made on a stream under capture (that would
 * invalidate the capture) or captured into a graph.  Every call shares the
 * array: calls that overlap on the GPU race, so order them on one stream. */
SMP_B200_API int smp_b200_solve_static(const int32_t *pref_m, const int32_t *pref_w, int32_t n,
                                       int32_t *match_out, int64_t *proposals, void *stream);

/* Seeded workload generator.  salt separates instances of a batch; param is
 * sigma*1e4 (CORRELATED) or the group size (GROUPED).  Writes both lists,
 * drawn from counter-based Philox4x32-10 streams (pactae_b200/csrc/generate.cu
 * states the recipe), so the same (kind, n, seed, salt, param) always gives
 * the same lists. */
SMP_B200_API int smp_b200_generate(smp_ctx *ctx, int32_t kind, int32_t n, uint64_t seed,
                      uint32_t salt, int32_t param, int32_t *pref_m,
                      int32_t *pref_w, uint32_t flags);

#ifdef __cplusplus
}
#endif

#endif /* SMP_B200_H */
