// workload_io.cpp -- the reference's workload text cache, read and written
// natively (include/utils/generate_workloads_flat.h:283-376: SaveSmpWorkload,
// LoadSmpWorkload, GetWorkloadFilename).  A file is "n\n", then the n rows of
// the men's lists and the n rows of the women's, each row written as
// "v v ... v \n".  At n = 30000 that is about 10 GB of text, so both
// directions use every host thread:
//   read:  the file is mapped; threads count the newlines in their byte
//          ranges, a prefix sum numbers the lines, and each thread parses
//          the rows that start in its range.  A file that is not one row per
//          line (the reference's reader only needs whitespace) is parsed by
//          a single-threaded tokenizer instead.
//   write: threads measure their rows' text, a prefix sum gives each row its
//          file offset, and each thread formats and writes its rows there.
// Host code only; no CUDA.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "smp_b200.h"

namespace {

int host_threads() {
  const unsigned t = std::thread::hardware_concurrency();
  return static_cast<int>(std::max(1u, std::min(t, 64u)));
}

template <typename F>
void parallel(int threads, F f) {
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; ++t) pool.emplace_back(f, t);
  f(0);
  for (auto &th : pool) th.join();
}

struct Mapped {
  const char *p = nullptr;
  size_t size = 0;
  int fd = -1;
  ~Mapped() {
    if (p && size) munmap(const_cast<char *>(p), size);
    if (fd >= 0) close(fd);
  }
};

int map_file(const char *path, Mapped &m) {
  m.fd = open(path, O_RDONLY);
  if (m.fd < 0) return SMP_ERR_IO;
  struct stat st;
  if (fstat(m.fd, &st) != 0 || st.st_size <= 0) return SMP_ERR_INVALID_INPUT;
  m.size = static_cast<size_t>(st.st_size);
  void *p = mmap(nullptr, m.size, PROT_READ, MAP_PRIVATE, m.fd, 0);
  if (p == MAP_FAILED) {
    m.size = 0;
    return SMP_ERR_OOM;
  }
  m.p = static_cast<const char *>(p);
  madvise(p, m.size, MADV_SEQUENTIAL);
  return SMP_OK;
}

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f'; }

// One decimal int32 (optional sign) after optional whitespace; nullptr if
// none or out of range.
inline const char *parse_int(const char *p, const char *end, int32_t &v) {
  while (p < end && is_space(*p)) ++p;
  if (p == end) return nullptr;
  bool neg = false;
  if (*p == '-' || *p == '+') {
    neg = *p == '-';
    ++p;
  }
  if (p == end || *p < '0' || *p > '9') return nullptr;
  int64_t x = 0;
  while (p < end && *p >= '0' && *p <= '9') {
    x = x * 10 + (*p - '0');
    if (x > 2147483648ll) return nullptr;
    ++p;
  }
  if (neg) x = -x;
  if (x > INT32_MAX || x < INT32_MIN) return nullptr;
  v = static_cast<int32_t>(x);
  return p;
}

// The header: n, then the rest of its line.  Returns the body start.
const char *parse_header(const char *p, const char *end, int32_t &n) {
  p = parse_int(p, end, n);
  if (!p || n <= 0) return nullptr;
  while (p < end && *p != '\n') {
    if (!is_space(*p)) return nullptr;
    ++p;
  }
  return p < end ? p + 1 : p;
}

// Row-per-line parse on every thread.  False if the file is not laid out
// that way (the caller then tokenizes it).
bool parse_lines(const char *body, const char *end, int32_t n, int32_t *pm, int32_t *pw) {
  const size_t len = static_cast<size_t>(end - body);
  const int T = static_cast<int>(std::min<size_t>(host_threads(), std::max<size_t>(1, len >> 20)));
  std::vector<size_t> lo(T + 1), nl(T + 1, 0);
  for (int t = 0; t <= T; ++t) lo[t] = len * t / T;
  parallel(T, [&](int t) {
    size_t c = 0;
    for (const char *q = body + lo[t], *e = body + lo[t + 1];; ++q) {
      q = static_cast<const char *>(std::memchr(q, '\n', static_cast<size_t>(e - q)));
      if (!q) break;
      ++c;
    }
    nl[t + 1] = c;
  });
  for (int t = 0; t < T; ++t) nl[t + 1] += nl[t];  // newlines before each range
  std::atomic<bool> ok{true};
  std::atomic<int64_t> rows{0};
  const int64_t nrows = 2ll * n;
  parallel(T, [&](int t) {
    int64_t line = static_cast<int64_t>(nl[t]);
    const char *e = body + lo[t + 1];
    const char *s = body + lo[t];
    // the first line start at or after s
    if (s != body && s[-1] != '\n') {
      const char *q = static_cast<const char *>(std::memchr(s, '\n', static_cast<size_t>(end - s)));
      if (!q || q >= e) return;  // no line starts in this range
      s = q + 1;
      ++line;
    }
    int64_t done = 0;
    while (s < e && ok.load(std::memory_order_relaxed)) {
      const char *eol = static_cast<const char *>(std::memchr(s, '\n', static_cast<size_t>(end - s)));
      const char *stop = eol ? eol : end;
      if (line < nrows) {
        int32_t *dst = (line < n ? pm : pw) + static_cast<size_t>(line % n) * n;
        const char *q = s;
        for (int32_t c = 0; c < n; ++c) {
          q = parse_int(q, stop, dst[c]);
          if (!q) {
            ok = false;
            return;
          }
        }
        for (; q < stop; ++q)
          if (!is_space(*q)) {
            ok = false;
            return;
          }
        ++done;
      } else {
        for (const char *q = s; q < stop; ++q)
          if (!is_space(*q)) {
            ok = false;
            return;
          }
      }
      if (!eol) break;
      s = eol + 1;
      ++line;
    }
    rows += done;
  });
  return ok && rows.load() == nrows;
}

// The reference reader's semantics: 2 n^2 integers separated by any
// whitespace.
bool parse_tokens(const char *body, const char *end, int32_t n, int32_t *pm, int32_t *pw) {
  const size_t nn = static_cast<size_t>(n) * n;
  const char *q = body;
  for (size_t i = 0; i < nn; ++i)
    if (!(q = parse_int(q, end, pm[i]))) return false;
  for (size_t i = 0; i < nn; ++i)
    if (!(q = parse_int(q, end, pw[i]))) return false;
  return true;
}

inline int digits(int32_t v) {
  uint32_t u = v < 0 ? static_cast<uint32_t>(-static_cast<int64_t>(v)) : static_cast<uint32_t>(v);
  int d = 1;
  while (u >= 10) {
    u /= 10;
    ++d;
  }
  return d + (v < 0 ? 1 : 0);
}

inline char *put_int(char *p, int32_t v) {
  char tmp[12];
  int k = 0;
  int64_t x = v;
  const bool neg = x < 0;
  if (neg) x = -x;
  do {
    tmp[k++] = static_cast<char>('0' + x % 10);
    x /= 10;
  } while (x);
  if (neg) *p++ = '-';
  while (k) *p++ = tmp[--k];
  return p;
}

}  // namespace

extern "C" {

int smp_b200_workload_read_n(const char *path, int32_t *n_out) {
  if (!path || !n_out) return SMP_ERR_INVALID_ARG;
  FILE *f = std::fopen(path, "rb");
  if (!f) return SMP_ERR_IO;
  char buf[64] = {};
  const size_t got = std::fread(buf, 1, sizeof(buf) - 1, f);
  std::fclose(f);
  int32_t n = 0;
  if (!parse_int(buf, buf + got, n) || n <= 0 || n > SMP_B200_MAX_N) return SMP_ERR_INVALID_INPUT;
  *n_out = n;
  return SMP_OK;
}

int smp_b200_workload_read(const char *path, int32_t n, int32_t *pref_m, int32_t *pref_w) {
  if (!path || !pref_m || !pref_w || n <= 0 || n > SMP_B200_MAX_N) return SMP_ERR_INVALID_ARG;
  Mapped m;
  int rc = map_file(path, m);
  if (rc) return rc;
  const char *end = m.p + m.size;
  int32_t fn = 0;
  const char *body = parse_header(m.p, end, fn);
  if (!body || fn != n) return SMP_ERR_INVALID_INPUT;
  if (parse_lines(body, end, n, pref_m, pref_w)) return SMP_OK;
  return parse_tokens(body, end, n, pref_m, pref_w) ? SMP_OK : SMP_ERR_INVALID_INPUT;
}

int smp_b200_workload_write(const char *path, const int32_t *pref_m, const int32_t *pref_w, int32_t n) {
  if (!path || !pref_m || !pref_w || n <= 0 || n > SMP_B200_MAX_N) return SMP_ERR_INVALID_ARG;
  const int64_t nrows = 2ll * n;
  const auto row = [&](int64_t r) { return (r < n ? pref_m : pref_w) + static_cast<size_t>(r % n) * n; };
  std::vector<uint64_t> off(static_cast<size_t>(nrows) + 1, 0);
  const int T = static_cast<int>(std::min<int64_t>(host_threads(), nrows));
  parallel(T, [&](int t) {
    for (int64_t r = t; r < nrows; r += T) {
      const int32_t *v = row(r);
      uint64_t len = 1;  // '\n'
      for (int32_t c = 0; c < n; ++c) len += static_cast<uint64_t>(digits(v[c])) + 1;
      off[static_cast<size_t>(r) + 1] = len;
    }
  });
  char head[32];
  const int hl = std::snprintf(head, sizeof(head), "%d\n", n);
  off[0] = static_cast<uint64_t>(hl);
  for (int64_t r = 0; r < nrows; ++r) off[static_cast<size_t>(r) + 1] += off[static_cast<size_t>(r)];
  const int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (fd < 0) return SMP_ERR_IO;
  std::atomic<bool> ok{pwrite(fd, head, static_cast<size_t>(hl), 0) == hl};
  if (ok && ftruncate(fd, static_cast<off_t>(off[static_cast<size_t>(nrows)])) != 0) ok = false;
  parallel(T, [&](int t) {
    std::vector<char> buf(static_cast<size_t>(n) * 12 + 2);
    for (int64_t r = t; r < nrows && ok.load(std::memory_order_relaxed); r += T) {
      const int32_t *v = row(r);
      char *p = buf.data();
      for (int32_t c = 0; c < n; ++c) {
        p = put_int(p, v[c]);
        *p++ = ' ';
      }
      *p++ = '\n';
      const size_t len = static_cast<size_t>(p - buf.data());
      size_t put = 0;
      while (put < len) {
        const ssize_t w = pwrite(fd, buf.data() + put, len - put, static_cast<off_t>(off[static_cast<size_t>(r)] + put));
        if (w <= 0) {
          ok = false;
          break;
        }
        put += static_cast<size_t>(w);
      }
    }
  });
  if (close(fd) != 0) ok = false;
  return ok ? SMP_OK : SMP_ERR_IO;
}

int smp_b200_workload_filename(int32_t kind, int32_t n, int32_t group_size, char *buf, size_t len) {
  if (!buf || len == 0 || n <= 0) return SMP_ERR_INVALID_ARG;
  int w;
  switch (kind) {
    case SMP_GEN_GROUPED: w = std::snprintf(buf, len, "smp_workload_random_%d_%d.txt", n, group_size); break;
    case SMP_GEN_SOLO: w = std::snprintf(buf, len, "smp_workload_solo_%d.txt", n); break;
    case SMP_GEN_REF_CONGESTED: w = std::snprintf(buf, len, "smp_workload_congested_%d.txt", n); break;
    case SMP_GEN_PERFECT: w = std::snprintf(buf, len, "smp_workload_perfect_%d.txt", n); break;
    default: return SMP_ERR_INVALID_ARG;
  }
  return (w > 0 && static_cast<size_t>(w) < len) ? SMP_OK : SMP_ERR_INVALID_ARG;
}

}  // extern "C"
