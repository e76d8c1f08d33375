// Synthetic graph generators and host CSR construction.
//
// The reference benchmarks real SNAP graphs loaded from Matrix Market or
// binary CSR directories (puercgp/examples/mtx_loader.hxx:99-260).  Those
// datasets are not available here, so the workloads are seeded synthetic
// graphs with the same shapes: R-MAT (Chakrabarti, Zhan, Faloutsos 2004),
// a 2-D 4-neighbour grid with deletions and shortcuts, and a Chung-Lu
// power-law graph.  Every random draw comes from a counter-based hash
// (splitmix64 finaliser) of (seed, stream, index), so generation is parallel
// and reproducible bit for bit on any host and thread count.
//
// CSR construction follows the loader's contract (mtx_loader.hxx:160-177):
// rows sorted by source, each row sorted by destination.  Symmetrisation adds
// both directions, self loops are dropped and duplicate entries removed.
#include "cgp_b200_internal.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <omp.h>

namespace cgp {

uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

static inline uint64_t draw(uint64_t seed, uint64_t stream, uint64_t index) {
  return mix64(mix64(seed ^ (stream * 0xD1B54A32D192ED03ULL)) ^ index);
}

static inline double unit01(uint64_t h) {  // [0, 1) with 53 random bits
  return static_cast<double>(h >> 11) * (1.0 / 9007199254740992.0);
}

// Bijection on [0, 2^bits): alternating odd multiply-add and xor-shift rounds.
static inline uint64_t permute_id(uint64_t x, int bits, uint64_t seed) {
  const uint64_t mask = bits >= 64 ? ~0ULL : ((1ULL << bits) - 1);
  const int shift = bits > 1 ? bits / 2 : 1;
  for (int r = 0; r < 4; ++r) {
    uint64_t mul = draw(seed, 1000 + r, 0) | 1ULL;
    uint64_t add = draw(seed, 2000 + r, 0);
    x = (x * mul + add) & mask;
    x ^= x >> shift;
  }
  return x & mask;
}

}  // namespace cgp

using cgp::draw;
using cgp::unit01;

namespace {

void csr_reset(cgp_host_csr* g) { std::memset(g, 0, sizeof(*g)); }

// Builds a CSR from an edge list.  symmetrize != 0 inserts both directions.
int build_csr(int64_t V, int64_t M, const int32_t* src, const int32_t* dst,
              int symmetrize, cgp_host_csr* out) {
  csr_reset(out);
  if (V <= 0 || V > INT32_MAX) return CGP_ERR_INVALID_ARG;
  std::vector<std::atomic<int64_t>> deg(static_cast<std::size_t>(V));
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < V; ++v) deg[v].store(0, std::memory_order_relaxed);
  bool bad = false;
#pragma omp parallel for schedule(static) reduction(|| : bad)
  for (int64_t i = 0; i < M; ++i) {
    int32_t u = src[i], v = dst[i];
    if (u < 0 || v < 0 || u >= V || v >= V) {
      bad = true;
      continue;
    }
    if (u == v) continue;
    deg[u].fetch_add(1, std::memory_order_relaxed);
    if (symmetrize) deg[v].fetch_add(1, std::memory_order_relaxed);
  }
  if (bad) return CGP_ERR_INVALID_ARG;
  std::vector<int64_t> start(static_cast<std::size_t>(V) + 1);
  start[0] = 0;
  for (int64_t v = 0; v < V; ++v) start[v + 1] = start[v] + deg[v].load();
  const int64_t raw = start[V];
  std::vector<int32_t> adj(static_cast<std::size_t>(raw));
  std::vector<std::atomic<int64_t>>& cursor = deg;
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < V; ++v) cursor[v].store(start[v], std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    int32_t u = src[i], v = dst[i];
    if (u == v) continue;
    adj[cursor[u].fetch_add(1, std::memory_order_relaxed)] = v;
    if (symmetrize) adj[cursor[v].fetch_add(1, std::memory_order_relaxed)] = u;
  }
  std::vector<int64_t> uniq(static_cast<std::size_t>(V));
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < V; ++v) {
    int32_t* b = adj.data() + start[v];
    int32_t* e = adj.data() + start[v + 1];
    std::sort(b, e);
    uniq[v] = std::unique(b, e) - b;
  }
  out->num_vertices = V;
  out->row_offsets = static_cast<int64_t*>(std::malloc(sizeof(int64_t) * (V + 1)));
  if (!out->row_offsets) return CGP_ERR_OOM;
  out->row_offsets[0] = 0;
  for (int64_t v = 0; v < V; ++v) out->row_offsets[v + 1] = out->row_offsets[v] + uniq[v];
  const int64_t E = out->row_offsets[V];
  out->num_edges = E;
  out->col_indices = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (E > 0 ? E : 1)));
  if (!out->col_indices) {
    std::free(out->row_offsets);
    csr_reset(out);
    return CGP_ERR_OOM;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < V; ++v) {
    std::memcpy(out->col_indices + out->row_offsets[v], adj.data() + start[v],
                sizeof(int32_t) * uniq[v]);
  }
  return CGP_OK;
}

}  // namespace

extern "C" {

void cgp_host_csr_free(cgp_host_csr* g) {
  if (!g) return;
  std::free(g->row_offsets);
  std::free(g->col_indices);
  std::free(g->weights);
  csr_reset(g);
}

int cgp_csr_from_edges(int64_t num_vertices, int64_t num_pairs,
                       const int32_t* src, const int32_t* dst, int32_t symmetrize,
                       cgp_host_csr* out) {
  if (!out || (num_pairs > 0 && (!src || !dst))) return CGP_ERR_INVALID_ARG;
  return build_csr(num_vertices, num_pairs, src, dst, symmetrize, out);
}

// R-MAT: each of edge_factor * 2^scale undirected edges descends `scale`
// quadrant levels with probabilities (a, b, c, 1-a-b-c); vertex ids are then
// relabelled by a seeded bijection so that degree is not correlated with id.
int cgp_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b,
                 double c, uint64_t seed, int32_t permute, cgp_host_csr* out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 1) return CGP_ERR_INVALID_ARG;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return CGP_ERR_INVALID_ARG;
  const int64_t V = 1LL << scale;
  const int64_t M = static_cast<int64_t>(edge_factor) * V;
  std::vector<int32_t> s(static_cast<std::size_t>(M)), d(static_cast<std::size_t>(M));
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    uint64_t u = 0, v = 0;
    for (int l = 0; l < scale; ++l) {
      double r = unit01(draw(seed, 1 + static_cast<uint64_t>(l), static_cast<uint64_t>(i)));
      uint64_t bu = r >= ab ? 1 : 0;
      uint64_t bv = (r >= a && r < ab) || r >= abc ? 1 : 0;
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    if (permute) {
      u = cgp::permute_id(u, scale, seed);
      v = cgp::permute_id(v, scale, seed);
    }
    s[i] = static_cast<int32_t>(u);
    d[i] = static_cast<int32_t>(v);
  }
  return build_csr(V, M, s.data(), d.data(), 1, out);
}

// rows x cols grid with right and down neighbours, each edge deleted with
// probability delete_frac, plus round(shortcut_frac * kept edges) random
// long-range pairs; symmetrised.
int cgp_gen_grid(int32_t rows, int32_t cols, double delete_frac,
                 double shortcut_frac, uint64_t seed, cgp_host_csr* out) {
  if (!out || rows < 1 || cols < 1) return CGP_ERR_INVALID_ARG;
  const int64_t V = static_cast<int64_t>(rows) * cols;
  if (V > INT32_MAX) return CGP_ERR_INVALID_ARG;
  const int64_t slots = 2 * V;  // right + down candidate per vertex
  std::vector<int32_t> s, d;
  s.reserve(static_cast<std::size_t>(slots));
  d.reserve(static_cast<std::size_t>(slots));
  for (int64_t v = 0; v < V; ++v) {
    int64_t r = v / cols, cc = v % cols;
    if (cc + 1 < cols && unit01(draw(seed, 11, 2 * v)) >= delete_frac) {
      s.push_back(static_cast<int32_t>(v));
      d.push_back(static_cast<int32_t>(v + 1));
    }
    if (r + 1 < rows && unit01(draw(seed, 11, 2 * v + 1)) >= delete_frac) {
      s.push_back(static_cast<int32_t>(v));
      d.push_back(static_cast<int32_t>(v + cols));
    }
  }
  const int64_t kept = static_cast<int64_t>(s.size());
  const int64_t shortcuts = static_cast<int64_t>(std::llround(shortcut_frac * kept));
  for (int64_t i = 0; i < shortcuts; ++i) {
    s.push_back(static_cast<int32_t>(draw(seed, 12, i) % static_cast<uint64_t>(V)));
    d.push_back(static_cast<int32_t>(draw(seed, 13, i) % static_cast<uint64_t>(V)));
  }
  return build_csr(V, static_cast<int64_t>(s.size()), s.data(), d.data(), 1, out);
}

// Chung-Lu: expected degree of vertex i proportional to (i + i0)^(-1/(gamma-1)),
// scaled to `mean_degree`; V*mean_degree/2 edges, each endpoint drawn from
// the weight distribution by inverse-CDF binary search; ids relabelled.
int cgp_gen_chung_lu(int64_t num_vertices, double exponent, double mean_degree,
                     uint64_t seed, cgp_host_csr* out) {
  if (!out || num_vertices < 2 || num_vertices > INT32_MAX || exponent <= 1.0 ||
      mean_degree <= 0)
    return CGP_ERR_INVALID_ARG;
  const int64_t V = num_vertices;
  const double alpha = 1.0 / (exponent - 1.0);
  std::vector<double> cdf(static_cast<std::size_t>(V));
  double total = 0;
  for (int64_t i = 0; i < V; ++i) {
    total += std::pow(static_cast<double>(i + 1), -alpha);
    cdf[i] = total;
  }
  const int64_t M = static_cast<int64_t>(std::llround(mean_degree * V / 2.0));
  std::vector<int32_t> s(static_cast<std::size_t>(M)), d(static_cast<std::size_t>(M));
  int bits = 1;
  while ((1LL << bits) < V) ++bits;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    for (int side = 0; side < 2; ++side) {
      double r = unit01(draw(seed, 21 + side, static_cast<uint64_t>(i))) * total;
      int64_t k = std::upper_bound(cdf.begin(), cdf.end(), r) - cdf.begin();
      if (k >= V) k = V - 1;
      // relabel by cycle-walking a bijection on [0, 2^bits) until inside [0, V)
      uint64_t x = static_cast<uint64_t>(k);
      do {
        x = cgp::permute_id(x, bits, seed);
      } while (x >= static_cast<uint64_t>(V));
      (side == 0 ? s : d)[i] = static_cast<int32_t>(x);
    }
  }
  return build_csr(V, M, s.data(), d.data(), 1, out);
}

// Attaches symmetric edge weights: w(u,v) = w(v,u) drawn from a hash of the
// unordered pair.  kind: CGP_WEIGHT_U32 uniform integers in [p0, p1];
// CGP_WEIGHT_F32 with p1 >= p0 >= 0: uniform reals in [p0, p1) rounded to
// fp32; CGP_WEIGHT_F32 with lognormal != 0: exp(p0 + p1 * N(0,1)).
int cgp_gen_weights(cgp_host_csr* g, int32_t kind, double p0, double p1,
                    int32_t lognormal, uint64_t seed) {
  if (!g || !g->row_offsets || (kind != CGP_WEIGHT_U32 && kind != CGP_WEIGHT_F32))
    return CGP_ERR_INVALID_ARG;
  if (kind == CGP_WEIGHT_U32 && (p0 < 0 || p1 < p0 || p1 > 4294967294.0))
    return CGP_ERR_INVALID_ARG;
  std::free(g->weights);
  const int64_t E = g->num_edges;
  g->weights = std::malloc(4 * static_cast<std::size_t>(E > 0 ? E : 1));
  if (!g->weights) return CGP_ERR_OOM;
  g->weight_kind = kind;
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t u = 0; u < g->num_vertices; ++u) {
    for (int64_t e = g->row_offsets[u]; e < g->row_offsets[u + 1]; ++e) {
      uint64_t v = static_cast<uint64_t>(g->col_indices[e]);
      uint64_t lo = std::min<uint64_t>(u, v), hi = std::max<uint64_t>(u, v);
      uint64_t key = (lo << 32) | hi;
      uint64_t h = draw(seed, 31, key);
      if (kind == CGP_WEIGHT_U32) {
        uint64_t span = static_cast<uint64_t>(p1 - p0) + 1;
        static_cast<uint32_t*>(g->weights)[e] = static_cast<uint32_t>(p0) + static_cast<uint32_t>(h % span);
      } else if (!lognormal) {
        static_cast<float*>(g->weights)[e] = static_cast<float>(p0 + (p1 - p0) * unit01(h));
      } else {
        double u1 = unit01(h), u2 = unit01(draw(seed, 32, key));
        double z = std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(6.283185307179586 * u2);
        static_cast<float*>(g->weights)[e] = static_cast<float>(std::exp(p0 + p1 * z));
      }
    }
  }
  return CGP_OK;
}

// Picks `count` query sources with a seeded hash, uniformly among vertices
// whose out-degree is at least min_degree (min_degree 1 = non-isolated) and,
// if `allowed` is given, with allowed[v] != 0.
// Returns CGP_ERR_INVALID_ARG if no vertex qualifies.
int cgp_pick_sources(const cgp_host_csr* g, int32_t count, int32_t min_degree,
                     const uint8_t* allowed, uint64_t seed, int32_t* sources) {
  if (!g || !sources || count < 0) return CGP_ERR_INVALID_ARG;
  std::vector<int32_t> cand;
  for (int64_t v = 0; v < g->num_vertices; ++v)
    if (g->row_offsets[v + 1] - g->row_offsets[v] >= min_degree &&
        (allowed == nullptr || allowed[v] != 0))
      cand.push_back(static_cast<int32_t>(v));
  if (cand.empty()) return CGP_ERR_INVALID_ARG;
  for (int32_t i = 0; i < count; ++i)
    sources[i] = cand[draw(seed, 41, static_cast<uint64_t>(i)) % cand.size()];
  return CGP_OK;
}

}  // extern "C"
