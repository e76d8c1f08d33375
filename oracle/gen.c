/*
 * Seeded synthetic graphs for the CPU side of the benchmark -- TEST
 * INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the library's host generators (R-MAT, 2-D grid with
 * deletions and shortcuts, Chung-Lu, symmetric edge weights, source picking).
 * It exists so that the reference arm of the benchmark, which times the
 * reference's own CPU traversal, builds the very same CSR without loading the
 * product library.  A CPU test checks that every array it produces equals the
 * library's bit for bit.
 *
 * Every random draw is a counter-based hash of (seed, stream, index): the
 * splitmix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom
 * number generators", OOPSLA 2014) applied twice.  R-MAT follows Chakrabarti,
 * Zhan, Faloutsos (SDM 2004); Chung-Lu follows Chung and Lu (2002) with
 * expected degrees proportional to (i + 1)^(-1/(gamma - 1)).
 *
 * CSR contract (the reference loader's, puercgp/examples/mtx_loader.hxx:160-177):
 * rows by source, each row sorted by destination; symmetrisation inserts both
 * directions, self loops are dropped and duplicate entries removed.
 */
#include "gen.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

static uint64_t draw(uint64_t seed, uint64_t stream, uint64_t index) {
  return mix64(mix64(seed ^ (stream * 0xD1B54A32D192ED03ULL)) ^ index);
}

static double unit01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

/* Bijection on [0, 2^bits): four rounds of odd multiply-add and xor-shift. */
static uint64_t permute_id(uint64_t x, int bits, uint64_t seed) {
  const uint64_t mask = bits >= 64 ? ~0ULL : ((1ULL << bits) - 1);
  const int shift = bits > 1 ? bits / 2 : 1;
  for (int r = 0; r < 4; ++r) {
    uint64_t mul = draw(seed, 1000 + (uint64_t)r, 0) | 1ULL;
    uint64_t add = draw(seed, 2000 + (uint64_t)r, 0);
    x = (x * mul + add) & mask;
    x ^= x >> shift;
  }
  return x & mask;
}

static void sort_i32(int32_t* a, int64_t n);

static void isort(int32_t* a, int64_t n) {
  for (int64_t i = 1; i < n; ++i) {
    int32_t x = a[i];
    int64_t j = i - 1;
    while (j >= 0 && a[j] > x) {
      a[j + 1] = a[j];
      --j;
    }
    a[j + 1] = x;
  }
}

/* In-place LSD radix sort (8-bit digits) of non-negative ints through a
 * scratch buffer; insertion sort for short runs. */
static void sort_i32(int32_t* a, int64_t n) {
  if (n <= 48) {
    isort(a, n);
    return;
  }
  int32_t* tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  if (!tmp) { /* fall back to insertion sort rather than fail */
    isort(a, n);
    return;
  }
  int32_t* src = a;
  int32_t* dst = tmp;
  for (int sh = 0; sh < 32; sh += 8) {
    int64_t cnt[257];
    memset(cnt, 0, sizeof(cnt));
    for (int64_t i = 0; i < n; ++i) cnt[((uint32_t)src[i] >> sh & 0xffu) + 1]++;
    for (int k = 0; k < 256; ++k) cnt[k + 1] += cnt[k];
    for (int64_t i = 0; i < n; ++i) dst[cnt[(uint32_t)src[i] >> sh & 0xffu]++] = src[i];
    int32_t* t = src;
    src = dst;
    dst = t;
  }
  /* four passes: the result is back in `a` */
  free(tmp);
}

void oracle_csr_free(oracle_csr* g) {
  if (!g) return;
  free(g->row);
  free(g->col);
  free(g->w);
  memset(g, 0, sizeof(*g));
}

/* Edge list -> CSR (symmetrize != 0 inserts both directions). */
int oracle_csr_from_edges(int64_t V, int64_t M, const int32_t* src, const int32_t* dst,
                          int32_t symmetrize, oracle_csr* out) {
  memset(out, 0, sizeof(*out));
  if (V <= 0 || V > INT32_MAX) return 1;
  int64_t* start = (int64_t*)calloc((size_t)V + 1, sizeof(int64_t));
  if (!start) return 2;
  for (int64_t i = 0; i < M; ++i) {
    int32_t u = src[i], v = dst[i];
    if (u < 0 || v < 0 || u >= V || v >= V) {
      free(start);
      return 1;
    }
    if (u == v) continue;
    start[u + 1]++;
    if (symmetrize) start[v + 1]++;
  }
  for (int64_t v = 0; v < V; ++v) start[v + 1] += start[v];
  const int64_t raw = start[V];
  int32_t* adj = (int32_t*)malloc(sizeof(int32_t) * (size_t)(raw > 0 ? raw : 1));
  int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)V);
  if (!adj || !cur) {
    free(start);
    free(adj);
    free(cur);
    return 2;
  }
  memcpy(cur, start, sizeof(int64_t) * (size_t)V);
  for (int64_t i = 0; i < M; ++i) {
    int32_t u = src[i], v = dst[i];
    if (u == v) continue;
    adj[cur[u]++] = v;
    if (symmetrize) adj[cur[v]++] = u;
  }
  /* sort and deduplicate every row; cur[v] becomes the unique count */
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < V; ++v) {
    int32_t* b = adj + start[v];
    const int64_t n = start[v + 1] - start[v];
    sort_i32(b, n);
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i)
      if (k == 0 || b[i] != b[k - 1]) b[k++] = b[i];
    cur[v] = k;
  }
  out->V = V;
  out->row = (int64_t*)malloc(sizeof(int64_t) * ((size_t)V + 1));
  if (!out->row) {
    free(start);
    free(adj);
    free(cur);
    return 2;
  }
  out->row[0] = 0;
  for (int64_t v = 0; v < V; ++v) out->row[v + 1] = out->row[v] + cur[v];
  out->E = out->row[V];
  out->col = (int32_t*)malloc(sizeof(int32_t) * (size_t)(out->E > 0 ? out->E : 1));
  if (!out->col) {
    free(start);
    free(adj);
    free(cur);
    free(out->row);
    memset(out, 0, sizeof(*out));
    return 2;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < V; ++v)
    memcpy(out->col + out->row[v], adj + start[v], sizeof(int32_t) * (size_t)cur[v]);
  free(start);
  free(adj);
  free(cur);
  return 0;
}

int oracle_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                    uint64_t seed, int32_t permute, oracle_csr* out) {
  memset(out, 0, sizeof(*out));
  if (scale < 1 || scale > 30 || edge_factor < 1) return 1;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return 1;
  const int64_t V = (int64_t)1 << scale;
  const int64_t M = (int64_t)edge_factor * V;
  int32_t* s = (int32_t*)malloc(sizeof(int32_t) * (size_t)M);
  int32_t* d = (int32_t*)malloc(sizeof(int32_t) * (size_t)M);
  if (!s || !d) {
    free(s);
    free(d);
    return 2;
  }
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    uint64_t u = 0, v = 0;
    for (int l = 0; l < scale; ++l) {
      double r = unit01(draw(seed, 1 + (uint64_t)l, (uint64_t)i));
      uint64_t bu = r >= ab ? 1 : 0;
      uint64_t bv = ((r >= a && r < ab) || r >= abc) ? 1 : 0;
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    if (permute) {
      u = permute_id(u, scale, seed);
      v = permute_id(v, scale, seed);
    }
    s[i] = (int32_t)u;
    d[i] = (int32_t)v;
  }
  int rc = oracle_csr_from_edges(V, M, s, d, 1, out);
  free(s);
  free(d);
  return rc;
}

int oracle_gen_grid(int32_t rows, int32_t cols, double delete_frac, double shortcut_frac,
                    uint64_t seed, oracle_csr* out) {
  memset(out, 0, sizeof(*out));
  if (rows < 1 || cols < 1) return 1;
  const int64_t V = (int64_t)rows * cols;
  if (V > INT32_MAX) return 1;
  const int64_t cap = 2 * V + (int64_t)(shortcut_frac * 2.0 * (double)V) + 16;
  int32_t* s = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
  int32_t* d = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
  if (!s || !d) {
    free(s);
    free(d);
    return 2;
  }
  int64_t n = 0;
  for (int64_t v = 0; v < V; ++v) {
    const int64_t r = v / cols, cc = v % cols;
    if (cc + 1 < cols && unit01(draw(seed, 11, 2 * (uint64_t)v)) >= delete_frac) {
      s[n] = (int32_t)v;
      d[n++] = (int32_t)(v + 1);
    }
    if (r + 1 < rows && unit01(draw(seed, 11, 2 * (uint64_t)v + 1)) >= delete_frac) {
      s[n] = (int32_t)v;
      d[n++] = (int32_t)(v + cols);
    }
  }
  const int64_t kept = n;
  const int64_t shortcuts = (int64_t)llround(shortcut_frac * (double)kept);
  if (kept + shortcuts > cap) {
    free(s);
    free(d);
    return 1;
  }
  for (int64_t i = 0; i < shortcuts; ++i) {
    s[n] = (int32_t)(draw(seed, 12, (uint64_t)i) % (uint64_t)V);
    d[n++] = (int32_t)(draw(seed, 13, (uint64_t)i) % (uint64_t)V);
  }
  int rc = oracle_csr_from_edges(V, n, s, d, 1, out);
  free(s);
  free(d);
  return rc;
}

int oracle_gen_chung_lu(int64_t V, double exponent, double mean_degree, uint64_t seed,
                        oracle_csr* out) {
  memset(out, 0, sizeof(*out));
  if (V < 2 || V > INT32_MAX || exponent <= 1.0 || mean_degree <= 0) return 1;
  const double alpha = 1.0 / (exponent - 1.0);
  double* cdf = (double*)malloc(sizeof(double) * (size_t)V);
  if (!cdf) return 2;
  double total = 0;
  for (int64_t i = 0; i < V; ++i) {
    total += pow((double)(i + 1), -alpha);
    cdf[i] = total;
  }
  const int64_t M = (int64_t)llround(mean_degree * (double)V / 2.0);
  int32_t* s = (int32_t*)malloc(sizeof(int32_t) * (size_t)(M > 0 ? M : 1));
  int32_t* d = (int32_t*)malloc(sizeof(int32_t) * (size_t)(M > 0 ? M : 1));
  if (!s || !d) {
    free(cdf);
    free(s);
    free(d);
    return 2;
  }
  int bits = 1;
  while (((int64_t)1 << bits) < V) ++bits;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    for (int side = 0; side < 2; ++side) {
      const double r = unit01(draw(seed, 21 + (uint64_t)side, (uint64_t)i)) * total;
      /* first k with cdf[k] > r */
      int64_t lo = 0, hi = V;
      while (lo < hi) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (cdf[mid] > r) hi = mid;
        else lo = mid + 1;
      }
      int64_t k = lo >= V ? V - 1 : lo;
      uint64_t x = (uint64_t)k;
      do {
        x = permute_id(x, bits, seed);
      } while (x >= (uint64_t)V);
      (side == 0 ? s : d)[i] = (int32_t)x;
    }
  }
  free(cdf);
  int rc = oracle_csr_from_edges(V, M, s, d, 1, out);
  free(s);
  free(d);
  return rc;
}

int oracle_gen_weights(oracle_csr* g, int32_t kind, double p0, double p1, int32_t lognormal,
                       uint64_t seed) {
  if (!g || !g->row || (kind != ORACLE_W_U32 && kind != ORACLE_W_F32)) return 1;
  if (kind == ORACLE_W_U32 && (p0 < 0 || p1 < p0 || p1 > 4294967294.0)) return 1;
  free(g->w);
  g->w = malloc(4 * (size_t)(g->E > 0 ? g->E : 1));
  if (!g->w) return 2;
  g->weight_kind = kind;
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t u = 0; u < g->V; ++u) {
    for (int64_t e = g->row[u]; e < g->row[u + 1]; ++e) {
      const uint64_t v = (uint64_t)g->col[e];
      const uint64_t lo = (uint64_t)u < v ? (uint64_t)u : v;
      const uint64_t hi = (uint64_t)u < v ? v : (uint64_t)u;
      const uint64_t key = (lo << 32) | hi;
      const uint64_t h = draw(seed, 31, key);
      if (kind == ORACLE_W_U32) {
        const uint64_t span = (uint64_t)(p1 - p0) + 1;
        ((uint32_t*)g->w)[e] = (uint32_t)p0 + (uint32_t)(h % span);
      } else if (!lognormal) {
        ((float*)g->w)[e] = (float)(p0 + (p1 - p0) * unit01(h));
      } else {
        const double u1 = unit01(h), u2 = unit01(draw(seed, 32, key));
        const double z = sqrt(-2.0 * log(1.0 - u1)) * cos(6.283185307179586 * u2);
        ((float*)g->w)[e] = (float)exp(p0 + p1 * z);
      }
    }
  }
  return 0;
}

int oracle_pick_sources(const oracle_csr* g, int32_t count, int32_t min_degree,
                        const uint8_t* allowed, uint64_t seed, int32_t* sources) {
  if (!g || !sources || count < 0) return 1;
  int32_t* cand = (int32_t*)malloc(sizeof(int32_t) * (size_t)(g->V > 0 ? g->V : 1));
  if (!cand) return 2;
  int64_t n = 0;
  for (int64_t v = 0; v < g->V; ++v)
    if (g->row[v + 1] - g->row[v] >= min_degree && (allowed == NULL || allowed[v] != 0))
      cand[n++] = (int32_t)v;
  if (n == 0) {
    free(cand);
    return 1;
  }
  for (int32_t i = 0; i < count; ++i)
    sources[i] = cand[draw(seed, 41, (uint64_t)i) % (uint64_t)n];
  free(cand);
  return 0;
}
