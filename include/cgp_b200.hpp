// Header-only C++ host API over the C ABI of cgp_b200.h.
//
// Re-creates the reference's host surface so that a caller of puercgp /
// the cgp Gunrock fork can switch with minimal edits:
//   cgp::run<bfs_policy|sssp_policy|wcc_policy>(graph, query_batch, ctx, opts)
//                                          <- puercgp::run (puercgp/include/puercgp/run.hxx:11-23)
//   cgp::run_heterogeneous(graph, hybrid_query_batch, ctx, opts)
//                                          <- hybrid_engine.hxx:1144-1150
//   cgp::run_replenish_pipeline(graph, descriptors, ctx, opts)
//                                          <- replenish_engine.hxx:559-573
//   cgp::problem_t / cgp::enactor_t / cgp::operators::advance_filter
//                                          <- cgp/include/gunrock/framework/{problem,enactor}.hxx
// Errors surface as std::invalid_argument (CGP_ERR_INVALID_ARG) or
// std::runtime_error (everything else), as in the reference.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cgp_b200.h"

namespace cgp {

inline void throw_if_error(cgp_status s, const char* what) {
  if (s == CGP_OK) return;
  char buf[1024];
  cgp_last_error(buf, sizeof(buf));
  std::string msg = std::string(what) + ": " + cgp_status_name(s) + ": " + buf;
  if (s == CGP_ERR_INVALID_ARG) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

enum class traversal_mode_t { push = CGP_MODE_PUSH, pull = CGP_MODE_PULL, hybrid = CGP_MODE_HYBRID };
enum class algo_kind_t : int32_t { bfs = CGP_KIND_BFS, sssp = CGP_KIND_SSSP, wcc = CGP_KIND_WCC, khop = CGP_KIND_KHOP };

// run_options (puercgp/include/puercgp/core/types.hxx:26-46).
struct run_options {
  traversal_mode_t traversal_mode = traversal_mode_t::hybrid;
  double pull_frontier_ratio = 0.15;
  double pull_edge_ratio = 0.20;
  bool profile_iterations = false;
  int max_iterations = 0;
  std::size_t max_queries = 0;
  bool enable_replenishment = false;
  bool discard_results = false;
  int slots = 64;  // slot count of the replenishment pipeline

  cgp_options to_c() const {
    cgp_options o;
    cgp_options_init(&o);
    o.traversal_mode = static_cast<int32_t>(traversal_mode);
    o.pull_frontier_ratio = pull_frontier_ratio;
    o.pull_edge_ratio = pull_edge_ratio;
    o.profile_iterations = profile_iterations ? 1 : 0;
    o.max_iterations = max_iterations;
    o.max_queries = static_cast<int32_t>(max_queries);
    o.discard_results = discard_results ? 1 : 0;
    return o;
  }
};

// execution_context (backend/graph_adapter.hxx:43-97): the device and an
// optional stream handle (cudaStream_t) the work is enqueued on.
class execution_context {
 public:
  explicit execution_context(int device = 0, void* stream = nullptr)
      : device_(device), stream_(stream) {
    throw_if_error(cgp_set_device(device), "cgp_set_device");
  }
  void* stream() const noexcept { return stream_; }
  int device() const noexcept { return device_; }

 private:
  int device_;
  void* stream_;
};

// Device CSR graph (csr_graph_storage, backend/csr_graph.hxx:42-75).
class csr_graph {
 public:
  csr_graph(const std::vector<int64_t>& row_offsets, const std::vector<int32_t>& col_indices,
            const std::vector<float>& weights = {}) {
    throw_if_error(cgp_graph_create(row_offsets.data(), 8, col_indices.data(),
                                    weights.empty() ? nullptr : weights.data(),
                                    weights.empty() ? CGP_WEIGHT_NONE : CGP_WEIGHT_F32,
                                    static_cast<int64_t>(row_offsets.size()) - 1,
                                    static_cast<int64_t>(col_indices.size()), 0, &g_),
                   "cgp_graph_create");
  }
  csr_graph(const std::vector<int64_t>& row_offsets, const std::vector<int32_t>& col_indices,
            const std::vector<uint32_t>& weights) {
    throw_if_error(cgp_graph_create(row_offsets.data(), 8, col_indices.data(), weights.data(),
                                    CGP_WEIGHT_U32, static_cast<int64_t>(row_offsets.size()) - 1,
                                    static_cast<int64_t>(col_indices.size()), 0, &g_),
                   "cgp_graph_create");
  }
  csr_graph(const csr_graph&) = delete;
  csr_graph& operator=(const csr_graph&) = delete;
  ~csr_graph() { cgp_graph_destroy(g_); }
  cgp_graph* handle() const noexcept { return g_; }
  int64_t get_number_of_vertices() const {
    int64_t v = 0;
    cgp_graph_info(g_, &v, nullptr, nullptr, nullptr);
    return v;
  }
  int64_t get_number_of_edges() const {
    int64_t e = 0;
    cgp_graph_info(g_, nullptr, &e, nullptr, nullptr);
    return e;
  }

 private:
  cgp_graph* g_ = nullptr;
};

// query_descriptor_t (core/query_descriptor.hxx:19-24) + hop bound.
struct query_descriptor_t {
  int source = 0;
  algo_kind_t kind = algo_kind_t::bfs;
  int k = 0;
};

// hybrid_query_batch (core/query_descriptor.hxx:28-145), without the 64 cap.
class hybrid_query_batch {
 public:
  hybrid_query_batch() = default;
  explicit hybrid_query_batch(std::vector<query_descriptor_t> d) : descs_(std::move(d)) {}
  std::size_t size() const noexcept { return descs_.size(); }
  const std::vector<query_descriptor_t>& descriptors() const { return descs_; }
  void validate(std::size_t max_queries = 0) const {
    if (descs_.empty()) throw std::invalid_argument("hybrid_query_batch must be non-empty");
    if (max_queries != 0 && descs_.size() > max_queries)
      throw std::invalid_argument("hybrid_query_batch exceeds max_queries");
    for (const auto& d : descs_)
      if (d.source < 0) throw std::invalid_argument("query source must be non-negative");
  }

 private:
  std::vector<query_descriptor_t> descs_;
};

template <typename vertex_t = int>
class query_batch {  // core/query_batch.hxx
 public:
  query_batch(std::initializer_list<vertex_t> s) : sources_(s) {}
  explicit query_batch(std::vector<vertex_t> s) : sources_(std::move(s)) {}
  std::size_t size() const noexcept { return sources_.size(); }
  const std::vector<vertex_t>& sources() const noexcept { return sources_; }
  void validate(std::size_t max_queries) const {
    if (sources_.empty()) throw std::invalid_argument("query_batch must contain at least one source");
    if (max_queries != 0 && sources_.size() > max_queries)
      throw std::invalid_argument("query_batch exceeds max_queries");
    for (auto s : sources_)
      if (s < 0) throw std::invalid_argument("query_batch sources must be non-negative");
  }

 private:
  std::vector<vertex_t> sources_;
};

struct bfs_policy {
  using value_type = int32_t;
  static constexpr algo_kind_t kind = algo_kind_t::bfs;
  static constexpr value_type infinity() { return std::numeric_limits<int32_t>::max(); }
};
struct sssp_policy {  // float distances on float-weighted graphs, uint32 otherwise
  using value_type = uint32_t;
  static constexpr algo_kind_t kind = algo_kind_t::sssp;
};
struct wcc_policy {
  using value_type = uint32_t;
  static constexpr algo_kind_t kind = algo_kind_t::wcc;
};

// query_result_t (core/result.hxx:13-19).
struct query_result_t {
  int query_id = 0;
  int source = 0;
  int completion_level = 0;
  float completion_wall_time_ms = 0.0f;
};

// run_result_t (core/result.hxx:49-66); values are 4-byte words, vertex-major
// values[v*Q + q] for run/run_heterogeneous, row-major [N][V] for the
// replenishment pipeline.
struct run_result_t {
  std::vector<uint32_t> values;
  std::vector<query_result_t> queries;
  std::vector<cgp_level_profile> iteration_profiles;
  int effective_query_dim = 0;
  int iterations = 0;
  float gpu_time_ms = 0.0f;
  float wall_time_ms = 0.0f;
  template <typename T>
  T value(std::size_t i) const {
    T t;
    static_assert(sizeof(T) == 4, "values are 4-byte words");
    std::memcpy(&t, &values[i], 4);
    return t;
  }
};

namespace detail {
inline run_result_t run_descs(const csr_graph& g, const std::vector<query_descriptor_t>& d,
                              const execution_context& ctx, const run_options& opts,
                              int layout) {
  std::vector<cgp_query> q(d.size());
  for (std::size_t i = 0; i < d.size(); ++i)
    q[i] = cgp_query{d[i].source, static_cast<int32_t>(d[i].kind), d[i].k, 0};
  cgp_options o = opts.to_c();
  o.stream = ctx.stream();
  run_result_t r;
  r.values.resize(static_cast<std::size_t>(g.get_number_of_vertices()) * d.size());
  cgp_stats st;
  throw_if_error(cgp_batch_run(g.handle(), q.data(), static_cast<int32_t>(q.size()), &o,
                               r.values.data(), layout, 0, &st),
                 "cgp_batch_run");
  r.effective_query_dim = static_cast<int>(d.size());
  r.iterations = st.iterations;
  r.gpu_time_ms = st.gpu_time_ms;
  r.wall_time_ms = st.wall_time_ms;
  if (opts.profile_iterations) {
    int32_t n = 0;
    cgp_last_profiles(nullptr, 0, &n);
    r.iteration_profiles.resize(n);
    cgp_last_profiles(r.iteration_profiles.data(), n, &n);
  }
  for (std::size_t i = 0; i < d.size(); ++i)
    r.queries.push_back({static_cast<int>(i), d[i].source, st.iterations, st.wall_time_ms});
  return r;
}
}  // namespace detail

template <typename Policy>
run_result_t run(const csr_graph& g, const query_batch<int>& queries,
                 const execution_context& ctx, const run_options& opts = {}) {
  queries.validate(opts.max_queries);
  std::vector<query_descriptor_t> d;
  for (int s : queries.sources()) d.push_back({s, Policy::kind, 0});
  return detail::run_descs(g, d, ctx, opts, CGP_LAYOUT_VERTEX_MAJOR);
}

inline run_result_t run_heterogeneous(const csr_graph& g, const hybrid_query_batch& batch,
                                      const execution_context& ctx,
                                      const run_options& opts = {}) {
  batch.validate(opts.max_queries);
  return detail::run_descs(g, batch.descriptors(), ctx, opts, CGP_LAYOUT_VERTEX_MAJOR);
}

// All queries through `opts.slots` bitmask slots reused as queries converge;
// values row-major [N][V].
inline run_result_t run_replenish_pipeline(const csr_graph& g,
                                           const std::vector<query_descriptor_t>& all,
                                           const execution_context& ctx,
                                           const run_options& opts = {}) {
  if (all.empty()) throw std::invalid_argument("replenish: query list must be non-empty");
  if (!opts.enable_replenishment)
    return detail::run_descs(g, all, ctx, opts, CGP_LAYOUT_QUERY_MAJOR);
  const std::size_t V = static_cast<std::size_t>(g.get_number_of_vertices());
  run_result_t r;
  r.values.resize(all.size() * V);
  cgp_options o = opts.to_c();
  cgp_server* s = nullptr;
  const int slots = static_cast<int>(std::min<std::size_t>(all.size(), opts.slots));
  throw_if_error(cgp_server_create(g.handle(), slots, &o, 0, &s), "cgp_server_create");
  std::unique_ptr<cgp_server, cgp_status (*)(cgp_server*)> guard(s, cgp_server_destroy);
  std::vector<uint64_t> tickets(all.size());
  for (std::size_t i = 0; i < all.size(); ++i) {
    cgp_query q{all[i].source, static_cast<int32_t>(all[i].kind), all[i].k, 0};
    throw_if_error(cgp_server_submit(s, &q, opts.discard_results ? nullptr : &r.values[i * V], 0,
                                     &tickets[i]),
                   "cgp_server_submit");
  }
  throw_if_error(cgp_server_drain(s, -1), "cgp_server_drain");
  for (std::size_t i = 0; i < all.size(); ++i) {
    cgp_request_info info;
    throw_if_error(cgp_server_wait(s, tickets[i], -1, &info), "cgp_server_wait");
    r.queries.push_back({static_cast<int>(i), all[i].source, info.completion_level,
                         static_cast<float>(info.finish_time_ms - info.submit_time_ms)});
    r.iterations = std::max(r.iterations, info.admit_level + info.completion_level);
  }
  r.effective_query_dim = static_cast<int>(all.size());
  return r;
}

// ---------------------------------------------------------- operator surface
// problem_t (cgp/include/gunrock/framework/problem.hxx:28-58): the queries of
// one traversal group on one graph.
struct problem_t {
  const csr_graph& graph;
  std::vector<query_descriptor_t> queries;
  cgp_enactor* e = nullptr;
  problem_t(const csr_graph& g, std::vector<query_descriptor_t> q, const run_options& opts = {})
      : graph(g), queries(std::move(q)) {
    std::vector<cgp_query> cq;
    for (auto& d : queries) cq.push_back({d.source, static_cast<int32_t>(d.kind), d.k, 0});
    cgp_options o = opts.to_c();
    throw_if_error(cgp_enactor_create(g.handle(), cq.data(), static_cast<int32_t>(cq.size()), &o, &e),
                   "cgp_enactor_create");
  }
  problem_t(const problem_t&) = delete;
  problem_t& operator=(const problem_t&) = delete;
  ~problem_t() { cgp_enactor_destroy(e); }
  void init() {}
  void reset() { throw_if_error(cgp_enactor_prepare_frontier(e), "reset"); }
  std::vector<uint32_t> values(int layout = CGP_LAYOUT_VERTEX_MAJOR) const {
    std::vector<uint32_t> v(static_cast<std::size_t>(graph.get_number_of_vertices()) * queries.size());
    throw_if_error(cgp_enactor_read_values(e, v.data(), layout, 0), "read_values");
    return v;
  }
};

namespace operators {
// advance over the query-bitmask frontier fused with the filter that builds
// the next unique frontier (operators::advance::execute_runtime +
// operators::filter::execute_runtime, advance.hxx:244-270, filter.hxx:187-203).
inline int64_t advance_filter(problem_t& p, traversal_mode_t direction) {
  int64_t n = 0;
  throw_if_error(cgp_advance_filter_level(p.e, static_cast<int32_t>(direction), &n),
                 "advance_filter");
  return n;
}
}  // namespace operators

// enactor_t (cgp/include/gunrock/framework/enactor.hxx:78-344).
struct enactor_t {
  problem_t* problem;
  int iteration = 0;
  explicit enactor_t(problem_t* p) : problem(p) {}
  virtual ~enactor_t() = default;
  virtual void prepare_frontier() { problem->reset(); }
  virtual void loop() { operators::advance_filter(*problem, traversal_mode_t::hybrid); }
  virtual bool is_converged() {
    int32_t c = 0;
    throw_if_error(cgp_enactor_is_converged(problem->e, &c), "is_converged");
    return c != 0;
  }
  virtual void finalize() {}
  // Runs prepare_frontier, loop until converged, finalize; returns GPU ms.
  float enact() {
    iteration = 0;
    prepare_frontier();
    cgp_stats st;
    throw_if_error(cgp_enactor_enact(problem->e, &st), "enact");
    iteration = st.iterations;
    finalize();
    return st.gpu_time_ms;
  }
};

}  // namespace cgp
