/*
 * smp_oracle.c -- CPU oracle for the Gale-Shapley stable-marriage path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the thing measured or
 * shipped).  See smp_oracle.h for the reference functions each entry point
 * restates and for how the oracle is pinned.
 */
#include "smp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Philox4x32-10: published algorithm (Salmon, Moraes, Dror, Shaw, "Parallel */
/* random numbers: as easy as 1, 2, 3", SC'11).                              */
/* ------------------------------------------------------------------------ */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2],
                          uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; ++round) {
    uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
    uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += PHILOX_W0;
    k1 += PHILOX_W1;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static uint32_t draw(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2,
                     uint32_t c3, int lane) {
  uint32_t ctr[4] = {c0, c1, c2, c3};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t out[4];
  oracle_philox4x32_10(ctr, key, out);
  return out[lane];
}

/* Stream tags (third counter word = side << 8 | tag). */
enum {
  TAG_UNIFORM = 0,
  TAG_SCORE = 1,
  TAG_NOISE = 2, /* 2, 3, 4: three draws of four words = 12 uniforms */
  TAG_SHARED_ROW = 5,
  TAG_PERFECT_FIRST = 6,
  TAG_PERFECT_TAIL = 7,
  TAG_GROUP_IDS = 8,
  TAG_GROUP_ROW = 9,
  TAG_SOLO = 10,
  TAG_REF_CONGESTED = 11,
  TAG_BATCH = 12
};
#define ROW_SHARED 0xFFFFFFFFu

/* ------------------------------------------------------------------------ */
/* Row sort: every generator builds one u64 key per column with the column  */
/* index in the low bits (so keys are unique), sorts ascending, and keeps    */
/* the low bits.  LSD radix sort, 16-bit digits.                             */
/* ------------------------------------------------------------------------ */
typedef struct {
  uint64_t *k;
  uint64_t *tmp;
  size_t *cnt; /* 65536 digit counters */
} workspace;

static int ws_init(workspace *ws, int32_t n) {
  ws->k = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
  ws->tmp = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
  ws->cnt = (size_t *)malloc(65536 * sizeof(size_t));
  return (ws->k && ws->tmp && ws->cnt) ? 0 : -1;
}

static void ws_free(workspace *ws) {
  free(ws->k);
  free(ws->tmp);
  free(ws->cnt);
}

static void radix_sort_u64(uint64_t *a, workspace *ws, int32_t n, int bits) {
  size_t *cnt = ws->cnt;
  uint64_t *tmp = ws->tmp;
  for (int shift = 0; shift < bits; shift += 16) {
    memset(cnt, 0, 65536 * sizeof(size_t));
    for (int32_t i = 0; i < n; ++i) cnt[(a[i] >> shift) & 0xFFFF]++;
    size_t sum = 0;
    for (int d = 0; d < 65536; ++d) {
      size_t c = cnt[d];
      cnt[d] = sum;
      sum += c;
    }
    for (int32_t i = 0; i < n; ++i) tmp[cnt[(a[i] >> shift) & 0xFFFF]++] = a[i];
    memcpy(a, tmp, (size_t)n * sizeof(uint64_t));
  }
}

#define LOW20 0xFFFFFu

/* Sort the n keys in ws->k and write their low 20 bits (column indices) to
 * out[0..n). */
static void sort_emit(workspace *ws, int32_t n, int bits, int32_t *out) {
  radix_sort_u64(ws->k, ws, n, bits);
  for (int32_t j = 0; j < n; ++j) out[j] = (int32_t)(ws->k[j] & LOW20);
}

/* Uniform permutation of 0..n-1 for (side, tag, row): columns ordered by a
 * 32-bit Philox key, ties by column index. */
static void uniform_row(uint64_t seed, uint32_t salt, int side, int tag,
                        uint32_t row, int32_t n, int32_t *out, workspace *ws) {
  for (int32_t j = 0; j < n; ++j) {
    uint32_t r = draw(seed, (uint32_t)j, row, ((uint32_t)side << 8) | tag, salt, 0);
    ws->k[j] = ((uint64_t)r << 20) | (uint64_t)j;
  }
  sort_emit(ws, n, 52, out);
}

/* Correlated row: row i ranks column j by score[j] + noise(i, j), higher
 * first, ties by index.  Scores are u32 fixed point (2^32 = 1.0); noise is an
 * Irwin-Hall(12) sum centred and scaled to sigma (sigma_e4 / 1e4) in the same
 * fixed point, in exact integer arithmetic (C division truncates toward 0). */
static void correlated_row(uint64_t seed, uint32_t salt, int side, uint32_t row,
                           int32_t n, int32_t sigma_e4, const uint32_t *score,
                           int32_t *out, workspace *ws) {
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int32_t j = 0; j < n; ++j) {
    int64_t ih = 0;
    for (int t = 0; t < 3; ++t) {
      uint32_t ctr[4] = {(uint32_t)j, row, ((uint32_t)side << 8) | (uint32_t)(TAG_NOISE + t), salt};
      uint32_t o[4];
      oracle_philox4x32_10(ctr, key, o);
      ih += (int64_t)(o[0] >> 8) + (o[1] >> 8) + (o[2] >> 8) + (o[3] >> 8);
    }
    int64_t z = ih - 6 * ((int64_t)1 << 24);
    int64_t noise = (z * 256 * (int64_t)sigma_e4) / 10000;
    int64_t total = (int64_t)score[j] + noise;
    uint64_t inv = (uint64_t)(((int64_t)1 << 36) - total);
    ws->k[j] = (inv << 20) | (uint64_t)j;
  }
  sort_emit(ws, n, 60, out);
}

/* Shared per-side data computed once before the rows. */
typedef struct {
  int32_t *aux; /* first choices / group ids / scores */
} side_ctx;

static void gen_row(int kind, int side, int32_t n, uint64_t seed, uint32_t salt,
                    int32_t param, const side_ctx *sc, int32_t i, int32_t *row,
                    workspace *ws) {
  uint32_t sidebits = (uint32_t)side << 8;
  switch (kind) {
    case ORACLE_GEN_UNIFORM:
      uniform_row(seed, salt, side, TAG_UNIFORM, (uint32_t)i, n, row, ws);
      break;
    case ORACLE_GEN_CONGESTED: /* women's rows; the men's shared row is copied */
      uniform_row(seed, salt, side, TAG_UNIFORM, (uint32_t)i, n, row, ws);
      break;
    case ORACLE_GEN_CORRELATED:
      correlated_row(seed, salt, side, (uint32_t)i, n, param, (const uint32_t *)sc->aux, row, ws);
      break;
    case ORACLE_GEN_PERFECT: {
      /* generate_workloads_flat.h:50-82: distinct first choices (a shuffled
       * permutation), the other n-1 entries of the row in random order. */
      int32_t first = sc->aux[i];
      for (int32_t j = 0; j < n; ++j) {
        uint32_t r = draw(seed, (uint32_t)j, (uint32_t)i, sidebits | TAG_PERFECT_TAIL, salt, 0);
        uint64_t hi = (j == first) ? 0 : ((uint64_t)(r >> 1) + 1);
        ws->k[j] = (hi << 20) | (uint64_t)j;
      }
      sort_emit(ws, n, 52, row);
      break;
    }
    case ORACLE_GEN_GROUPED: {
      /* generate_workloads_flat.h:85-137: a global shuffle of ids, then each
       * row shuffles the ids inside consecutive groups of size g. */
      int32_t g = param;
      for (int32_t p = 0; p < n; ++p) {
        uint32_t r = draw(seed, (uint32_t)p, (uint32_t)i, sidebits | TAG_GROUP_ROW, salt, 0);
        uint64_t grp = (uint64_t)(p / g);
        ws->k[p] = (grp << 44) | ((uint64_t)(r >> 8) << 20) | (uint64_t)p;
      }
      radix_sort_u64(ws->k, ws, n, 64);
      for (int32_t p = 0; p < n; ++p) row[p] = sc->aux[ws->k[p] & LOW20];
      break;
    }
    case ORACLE_GEN_SOLO: {
      /* generate_workloads_flat.h:140-247 (n >= 3).  Men: slot 0 = m', slot
       * n-2 = (m'-1) mod (n-1), slot n-1 = n-1 with m' = min(m, n-2), the rest
       * shuffled in between.  Women w < n-1: slots 0, 1 = (w+1) mod (n-1) and
       * the man before it, the rest shuffled; woman n-1: a uniform row. */
      int32_t a0 = -1, a1 = -1, a2 = -1, lo = 0;
      if (side == 0) {
        int32_t m = (i == n - 1) ? n - 2 : i;
        a0 = m;
        a1 = (m - 1 + n - 1) % (n - 1);
        a2 = n - 1;
        row[0] = a0; row[n - 2] = a1; row[n - 1] = a2;
        lo = 1;
      } else if (i < n - 1) {
        a0 = (i + 1) % (n - 1);
        a1 = (a0 + n - 1) % n;
        row[0] = a0; row[1] = a1;
        lo = 2;
      }
      int32_t cnt = 0;
      for (int32_t j = 0; j < n; ++j) {
        if (j == a0 || j == a1 || j == a2) continue;
        uint32_t r = draw(seed, (uint32_t)j, (uint32_t)i, sidebits | TAG_SOLO, salt, 0);
        ws->k[cnt++] = ((uint64_t)r << 20) | (uint64_t)j;
      }
      sort_emit(ws, cnt, 52, row + lo);
      break;
    }
    default:
      break;
  }
}

int oracle_generate_side(int kind, int side, int32_t n, uint64_t seed,
                         uint32_t salt, int32_t param, int32_t *pref) {
  if (n <= 0 || n > (1 << 20) || pref == NULL || (side != 0 && side != 1)) return -1;
  if (kind < ORACLE_GEN_UNIFORM || kind > ORACLE_GEN_SOLO) return -1;
  if (kind == ORACLE_GEN_CORRELATED && (param < 0 || param > 10000)) return -1;
  if (kind == ORACLE_GEN_GROUPED && param <= 0) return -1;
  if (kind == ORACLE_GEN_SOLO && n < 3) return -1;
  size_t nn = (size_t)n;
  uint32_t sidebits = (uint32_t)side << 8;
  side_ctx sc;
  sc.aux = (int32_t *)malloc(nn * sizeof(int32_t));
  workspace ws0 = {NULL, NULL, NULL};
  if (!sc.aux || ws_init(&ws0, n) != 0) { free(sc.aux); ws_free(&ws0); return -1; }

  /* Rows that are one shared row copied n times. */
  int shared_tag = -1;
  if (kind == ORACLE_GEN_CONGESTED && side == 0) shared_tag = TAG_SHARED_ROW;
  if (kind == ORACLE_GEN_REF_CONGESTED) shared_tag = TAG_REF_CONGESTED; /* :14-47 */
  if (shared_tag >= 0) {
    uniform_row(seed, salt, side, shared_tag, ROW_SHARED, n, pref, &ws0);
    for (int32_t i = 1; i < n; ++i) memcpy(pref + i * nn, pref, nn * sizeof(int32_t));
    free(sc.aux);
    ws_free(&ws0);
    return 0;
  }
  if (kind == ORACLE_GEN_CORRELATED) {
    uint32_t *score = (uint32_t *)sc.aux;
    for (int32_t j = 0; j < n; ++j)
      score[j] = draw(seed, (uint32_t)j, ROW_SHARED, sidebits | TAG_SCORE, salt, 0);
  } else if (kind == ORACLE_GEN_PERFECT) {
    uniform_row(seed, salt, side, TAG_PERFECT_FIRST, ROW_SHARED, n, sc.aux, &ws0);
  } else if (kind == ORACLE_GEN_GROUPED) {
    uniform_row(seed, salt, side, TAG_GROUP_IDS, ROW_SHARED, n, sc.aux, &ws0);
  }
  ws_free(&ws0);

  int failed = 0;
#pragma omp parallel reduction(| : failed)
  {
    workspace ws = {NULL, NULL, NULL};
    int ok = ws_init(&ws, n) == 0;
    if (!ok) failed = 1;
    /* every thread reaches the worksharing loop, even without a workspace */
#pragma omp for schedule(dynamic, 8)
    for (int32_t i = 0; i < n; ++i)
      if (ok) gen_row(kind, side, n, seed, salt, param, &sc, i, pref + i * nn, &ws);
    ws_free(&ws);
  }
  free(sc.aux);
  return failed ? -1 : 0;
}

int oracle_generate(int kind, int32_t n, uint64_t seed, uint32_t salt,
                    int32_t param, int32_t *pref_m, int32_t *pref_w) {
  if (oracle_generate_side(kind, 0, n, seed, salt, param, pref_m) != 0) return -1;
  if (oracle_generate_side(kind, 1, n, seed, salt, param, pref_w) != 0) return -1;
  return 0;
}

void oracle_batch_instance(uint64_t seed, uint32_t b, int32_t n_lo, int32_t n_hi,
                           int32_t *n_out, int32_t *kind_out) {
  uint32_t ctr[4] = {b, ROW_SHARED, TAG_BATCH, 0};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  oracle_philox4x32_10(ctr, key, o);
  double u = (double)o[0] * (1.0 / 4294967296.0);
  double v = (double)n_lo * exp2(u * log2((double)n_hi / (double)n_lo));
  int32_t n = (int32_t)floor(v);
  if (n < n_lo) n = n_lo;
  if (n > n_hi) n = n_hi;
  *n_out = n;
  *kind_out = (int32_t)(o[1] % 3u);
}

/* ------------------------------------------------------------------------ */
/* Rank inversion and the two sequential engines.                            */
/* ------------------------------------------------------------------------ */
int oracle_invert(const int32_t *pref_w, int32_t n, int32_t *rank) {
  size_t nn = (size_t)n;
  for (int32_t w = 0; w < n; ++w) {
    int32_t *row = rank + w * nn;
    for (int32_t m = 0; m < n; ++m) row[m] = -1;
    for (int32_t r = 0; r < n; ++r) {
      int32_t m = pref_w[w * nn + r];
      if (m < 0 || m >= n || row[m] != -1) return -1;
      row[m] = r;
    }
  }
  return 0;
}

int oracle_is_perfect(const int32_t *pref_m, int32_t n) {
  unsigned char *seen = (unsigned char *)calloc((size_t)n, 1);
  int perfect = 1;
  for (int32_t m = 0; m < n && perfect; ++m) {
    int32_t w = pref_m[(size_t)m * n];
    if (w < 0 || w >= n || seen[w]) perfect = 0;
    else seen[w] = 1;
  }
  free(seen);
  return perfect;
}

static int rows_are_permutations(const int32_t *pref, int32_t n) {
  unsigned char *seen = (unsigned char *)malloc((size_t)n);
  int ok = 1;
  for (int32_t i = 0; i < n && ok; ++i) {
    memset(seen, 0, (size_t)n);
    for (int32_t r = 0; r < n; ++r) {
      int32_t v = pref[(size_t)i * n + r];
      if (v < 0 || v >= n || seen[v]) { ok = 0; break; }
      seen[v] = 1;
    }
  }
  free(seen);
  return ok;
}

/* smp_engine_gs_1.cu:16-98.  FIFO queue of free men; the popped man keeps
 * proposing down his list until accepted; a displaced man is queued. */
int oracle_gs_seq(const int32_t *pref_m, const int32_t *pref_w, int32_t n,
                  int32_t *match, int64_t *proposals) {
  if (n <= 0 || !rows_are_permutations(pref_m, n)) return -1;
  size_t nn = (size_t)n;
  int32_t *rank = (int32_t *)malloc(nn * nn * sizeof(int32_t));
  int32_t *queue = (int32_t *)malloc(nn * sizeof(int32_t)); /* ring of size n */
  int32_t *next = (int32_t *)calloc(nn, sizeof(int32_t));
  int32_t *partner_rank = (int32_t *)malloc(nn * sizeof(int32_t));
  if (!rank || !queue || !next || !partner_rank || oracle_invert(pref_w, n, rank) != 0) {
    free(rank); free(queue); free(next); free(partner_rank);
    return -1;
  }
  int32_t head = 0, count = n;
  for (int32_t i = 0; i < n; ++i) { queue[i] = i; partner_rank[i] = n; }
  int64_t props = 0;
  int32_t m = queue[head]; head = (head + 1) % n; count--;
  int32_t pos = 0;
  for (;;) {
    int32_t w = pref_m[m * nn + pos];
    int32_t r = rank[w * nn + m];
    pos++;
    props++;
    int32_t p = partner_rank[w];
    if (r < p) {
      partner_rank[w] = r;
      if (p != n) { /* displaced man re-enters the queue */
        queue[(head + count) % n] = pref_w[w * nn + p];
        count++;
      }
      next[m] = pos;
      if (count == 0) break;
      m = queue[head]; head = (head + 1) % n; count--;
      pos = next[m];
    }
  }
  for (int32_t w = 0; w < n; ++w) match[pref_w[w * nn + partner_rank[w]]] = w;
  if (proposals) *proposals = props;
  free(rank); free(queue); free(next); free(partner_rank);
  return 0;
}

/* smp_engine_mw_1.cu:45-91.  Each man in index order follows his displacement
 * chain until someone lands on a free woman. */
int oracle_mw_seq(const int32_t *pref_m, const int32_t *pref_w, int32_t n,
                  int32_t *match, int64_t *proposals) {
  if (n <= 0 || !rows_are_permutations(pref_m, n)) return -1;
  size_t nn = (size_t)n;
  int32_t *rank = (int32_t *)malloc(nn * nn * sizeof(int32_t));
  int32_t *next = (int32_t *)calloc(nn, sizeof(int32_t));
  int32_t *partner_rank = (int32_t *)malloc(nn * sizeof(int32_t));
  if (!rank || !next || !partner_rank || oracle_invert(pref_w, n, rank) != 0) {
    free(rank); free(next); free(partner_rank);
    return -1;
  }
  for (int32_t i = 0; i < n; ++i) partner_rank[i] = n;
  int64_t props = 0;
  for (int32_t start = 0; start < n; ++start) {
    int32_t m = start, pos = next[m];
    for (;;) {
      int32_t w = pref_m[m * nn + pos];
      int32_t r = rank[w * nn + m];
      pos++;
      props++;
      int32_t p = partner_rank[w];
      if (p == n) { next[m] = pos; partner_rank[w] = r; break; }
      if (p > r) {
        next[m] = pos;
        partner_rank[w] = r;
        m = pref_w[w * nn + p];
        pos = next[m];
      }
    }
  }
  for (int32_t w = 0; w < n; ++w) match[pref_w[w * nn + partner_rank[w]]] = w;
  if (proposals) *proposals = props;
  free(rank); free(next); free(partner_rank);
  return 0;
}

int64_t oracle_check(const int32_t *pref_m, const int32_t *pref_w, int32_t n,
                     const int32_t *match, int64_t *proposals) {
  if (n <= 0 || !rows_are_permutations(pref_m, n)) return -1;
  size_t nn = (size_t)n;
  int32_t *rank = (int32_t *)malloc(nn * nn * sizeof(int32_t));
  int32_t *husband = (int32_t *)malloc(nn * sizeof(int32_t));
  if (!rank || !husband || oracle_invert(pref_w, n, rank) != 0) {
    free(rank); free(husband);
    return -1;
  }
  for (int32_t w = 0; w < n; ++w) husband[w] = -1;
  for (int32_t m = 0; m < n; ++m) {
    int32_t w = match[m];
    if (w < 0 || w >= n || husband[w] != -1) { free(rank); free(husband); return -1; }
    husband[w] = m;
  }
  int64_t blocking = 0, props = 0;
  for (int32_t m = 0; m < n; ++m) {
    /* every woman m ranks above his wife must prefer her own husband */
    for (int32_t r = 0; r < n; ++r) {
      int32_t w = pref_m[m * nn + r];
      props++;
      if (w == match[m]) break;
      if (rank[w * nn + m] < rank[w * nn + husband[w]]) blocking++;
    }
  }
  if (proposals) *proposals = props;
  free(rank); free(husband);
  return blocking;
}
