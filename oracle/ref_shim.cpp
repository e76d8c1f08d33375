// C entry points over the reference's own CPU traversals.
//
// TEST INFRASTRUCTURE ONLY.  This file holds no traversal code: it includes
// the reference's puercgp/examples/mtx_loader.hxx straight from the reference
// tree (see oracle/Makefile) and exposes its cpu_bfs / cpu_sssp / cpu_wcc /
// load_matrix_market behind plain C signatures, so the tests can pin the C
// restatement in oracle.c against the reference itself, and bench.py can time
// the reference's CPU path as the reference arm.  The build writes only into
// oracle/_ref/.
#include "mtx_loader.hxx"

#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

puercgp_examples::host_csr_graph make_graph(int64_t V, const int64_t* row,
                                            const int32_t* col,
                                            const float* w) {
  puercgp_examples::host_csr_graph g;
  g.vertices = static_cast<int>(V);
  g.edges = static_cast<int>(row[V]);
  g.row_offsets.assign(row, row + V + 1);
  g.column_indices.assign(col, col + row[V]);
  if (w != nullptr) {
    g.edge_weights.assign(w, w + row[V]);
  } else {
    g.edge_weights.assign(static_cast<std::size_t>(row[V]), 1.0f);
  }
  return g;
}

}  // namespace

extern "C" {

// cpu_bfs (mtx_loader.hxx:269-290): depth per vertex, INT_MAX = unreached.
int ref_cpu_bfs(int64_t V, const int64_t* row, const int32_t* col,
                int32_t source, int32_t* depth) {
  auto g = make_graph(V, row, col, nullptr);
  auto d = puercgp_examples::cpu_bfs(g, source);
  std::memcpy(depth, d.data(), sizeof(int32_t) * static_cast<std::size_t>(V));
  return 0;
}

// cpu_sssp (mtx_loader.hxx:292-319): float Dijkstra, +inf = unreached.
int ref_cpu_sssp(int64_t V, const int64_t* row, const int32_t* col,
                 const float* w, int32_t source, float* dist) {
  auto g = make_graph(V, row, col, w);
  auto d = puercgp_examples::cpu_sssp(g, source);
  std::memcpy(dist, d.data(), sizeof(float) * static_cast<std::size_t>(V));
  return 0;
}

// cpu_wcc (mtx_loader.hxx:328-356): float labels (exact below 2^24).
int ref_cpu_wcc(int64_t V, const int64_t* row, const int32_t* col,
                int32_t max_iterations, float* label) {
  auto g = make_graph(V, row, col, nullptr);
  auto l = puercgp_examples::cpu_wcc(g, max_iterations);
  std::memcpy(label, l.data(), sizeof(float) * static_cast<std::size_t>(V));
  return 0;
}

// load_matrix_market (mtx_loader.hxx:99-187).  First call with row == NULL to
// get V and E; second call fills row[V+1], col[E], w[E].
int ref_load_matrix_market(const char* path, int64_t* V, int64_t* E,
                           int64_t* row, int32_t* col, float* w) {
  try {
    auto g = puercgp_examples::load_matrix_market(path);
    *V = g.vertices;
    *E = g.edges;
    if (row != nullptr) {
      for (int i = 0; i <= g.vertices; ++i) row[i] = g.row_offsets[i];
      std::memcpy(col, g.column_indices.data(), sizeof(int32_t) * g.edges);
      std::memcpy(w, g.edge_weights.data(), sizeof(float) * g.edges);
    }
    return 0;
  } catch (...) {
    return 1;
  }
}

// Runs `nq` independent reference queries over `threads` host threads and
// writes query-major out[q*V+v].  kind 0 = cpu_bfs (int32 out), 2 = cpu_sssp
// (float out).  The graph is built once and shared read-only.
int ref_batch(int32_t kind, int64_t V, const int64_t* row, const int32_t* col,
              const float* w, const int32_t* sources, int32_t nq,
              int32_t threads, void* out) {
  auto g = make_graph(V, row, col, w);
  std::atomic<int32_t> next{0};
  auto worker = [&]() {
    for (;;) {
      int32_t q = next.fetch_add(1);
      if (q >= nq) break;
      std::size_t off = static_cast<std::size_t>(q) * static_cast<std::size_t>(V);
      if (kind == 0) {
        auto d = puercgp_examples::cpu_bfs(g, sources[q]);
        std::memcpy(static_cast<int32_t*>(out) + off, d.data(),
                    sizeof(int32_t) * static_cast<std::size_t>(V));
      } else {
        auto d = puercgp_examples::cpu_sssp(g, sources[q]);
        std::memcpy(static_cast<float*>(out) + off, d.data(),
                    sizeof(float) * static_cast<std::size_t>(V));
      }
    }
  };
  if (threads < 1) threads = 1;
  std::vector<std::thread> pool;
  for (int32_t t = 0; t < threads; ++t) pool.emplace_back(worker);
  for (auto& t : pool) t.join();
  return 0;
}

}  // extern "C"
