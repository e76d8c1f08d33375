// Known-answer checks through the C++ host API (include/cgp_b200.hpp), written
// the way the reference's example validators use puercgp:
//   validate_hybrid.cu:41-106, validate_wcc.cu:33-72, validate_replenish.cu:33-112,
//   smoke_hybrid_push.cu:117-173 (one push level through the operator surface).
// Prints [PASS]/[FAIL] lines and exits non-zero on any failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <vector>

#include "cgp_b200.hpp"

static int failures = 0;
static void check(const char* name, bool cond) {
  std::printf("  [%s] %s\n", cond ? "PASS" : "FAIL", name);
  if (!cond) ++failures;
}

int main() {
  using cgp::algo_kind_t;
  const int INF = std::numeric_limits<int>::max();
  const float FINF = std::numeric_limits<float>::infinity();
  cgp::execution_context ctx(0);
  // toy graph 0->1 (w=2), 0->2 (w=5), 1->3 (w=1)
  std::vector<int64_t> row = {0, 2, 3, 3, 3};
  std::vector<int32_t> col = {1, 2, 3};
  {
    cgp::csr_graph g(row, col, std::vector<float>{2.0f, 5.0f, 1.0f});
    cgp::hybrid_query_batch batch({{0, algo_kind_t::bfs}, {0, algo_kind_t::sssp},
                                   {0, algo_kind_t::wcc}});
    cgp::run_options opts;
    opts.traversal_mode = cgp::traversal_mode_t::push;
    auto r = cgp::run_heterogeneous(g, batch, ctx, opts);
    const int Q = 3;
    std::printf("run_heterogeneous [BFS 0, SSSP 0, WCC]:\n");
    check("BFS [0,1,1,2]", r.value<int>(0 * Q + 0) == 0 && r.value<int>(1 * Q + 0) == 1 &&
                               r.value<int>(2 * Q + 0) == 1 && r.value<int>(3 * Q + 0) == 2);
    check("SSSP [0,2,5,3]", r.value<float>(0 * Q + 1) == 0.0f && r.value<float>(1 * Q + 1) == 2.0f &&
                                r.value<float>(2 * Q + 1) == 5.0f && r.value<float>(3 * Q + 1) == 3.0f);
    check("WCC [0,0,0,0]", r.value<uint32_t>(0 * Q + 2) == 0 && r.value<uint32_t>(1 * Q + 2) == 0 &&
                               r.value<uint32_t>(2 * Q + 2) == 0 && r.value<uint32_t>(3 * Q + 2) == 0);
  }
  {
    cgp::csr_graph g(row, col);
    auto r = cgp::run<cgp::wcc_policy>(g, cgp::query_batch<int>({0}), ctx);
    std::printf("run<wcc_policy> on the directed toy:\n");
    bool all0 = true;
    for (int v = 0; v < 4; ++v) all0 &= r.value<uint32_t>(v) == 0;
    check("labels all 0", all0);
    auto b = cgp::run<cgp::bfs_policy>(g, cgp::query_batch<int>({0, 1, 2, 3}), ctx);
    check("BFS from 1 reaches 3 at depth 1", b.value<int>(3 * 4 + 1) == 1 && b.value<int>(0 * 4 + 1) == INF);
  }
  {
    cgp::csr_graph g(row, col, std::vector<float>{2.0f, 5.0f, 3.0f});
    std::vector<cgp::query_descriptor_t> all = {{0, algo_kind_t::bfs}, {0, algo_kind_t::sssp},
                                                {1, algo_kind_t::bfs}, {1, algo_kind_t::sssp}};
    cgp::run_options opts;
    opts.enable_replenishment = true;
    opts.traversal_mode = cgp::traversal_mode_t::push;
    opts.slots = 2;
    auto r = cgp::run_replenish_pipeline(g, all, ctx, opts);
    const int V = 4;
    std::printf("run_replenish_pipeline N=4 through 2 slots:\n");
    check("q0 BFS [0,1,1,2]", r.value<int>(0 * V + 3) == 2 && r.value<int>(0 * V + 1) == 1);
    check("q1 SSSP [0,2,5,5]", r.value<float>(1 * V + 3) == 5.0f && r.value<float>(1 * V + 2) == 5.0f);
    check("q2 BFS [INF,0,INF,1]", r.value<int>(2 * V + 0) == INF && r.value<int>(2 * V + 3) == 1);
    check("q3 SSSP [INF,0,INF,3]", r.value<float>(3 * V + 0) == FINF && r.value<float>(3 * V + 3) == 3.0f);
    bool done = true;
    for (auto& q : r.queries) done &= q.completion_level > 0;
    check("all completed", done && r.queries.size() == 4);
  }
  {
    cgp::csr_graph g(row, col, std::vector<float>{2.0f, 5.0f, 1.0f});
    cgp::run_options opts;
    opts.traversal_mode = cgp::traversal_mode_t::push;
    cgp::problem_t p(g, {{0, algo_kind_t::bfs}, {0, algo_kind_t::sssp}}, opts);
    cgp::enactor_t e(&p);
    e.prepare_frontier();
    int64_t next = cgp::operators::advance_filter(p, cgp::traversal_mode_t::push);
    auto v = p.values();
    std::printf("one push level (operator surface):\n");
    check("next frontier {1,2}", next == 2);
    check("BFS [0,1,1,INF]", v[0 * 2] == 0 && v[1 * 2] == 1 && v[2 * 2] == 1 &&
                                 v[3 * 2] == static_cast<uint32_t>(INF));
    float d1, d2;
    std::memcpy(&d1, &v[1 * 2 + 1], 4);
    std::memcpy(&d2, &v[2 * 2 + 1], 4);
    check("SSSP [0,2,5,INF]", d1 == 2.0f && d2 == 5.0f);
    while (!e.is_converged()) e.loop();
    auto f = p.values();
    check("converged BFS depth 2 at vertex 3", f[3 * 2] == 2);
    e.enact();
    check("enact reproduces", p.values() == f);
  }
  {
    std::printf("argument errors:\n");
    bool threw = false;
    try {
      cgp::csr_graph g(row, col);
      cgp::run<cgp::bfs_policy>(g, cgp::query_batch<int>({7}), ctx);
    } catch (const std::invalid_argument&) {
      threw = true;
    }
    check("out-of-range source throws invalid_argument", threw);
  }
  if (failures == 0) {
    std::printf("\nvalidate_facade: ALL PASS\n");
    return EXIT_SUCCESS;
  }
  std::printf("\nvalidate_facade: %d FAILURES\n", failures);
  return EXIT_FAILURE;
}
