// Operator-level surface: the Gunrock problem/enactor shape over one
// traversal group, with one fused advance+filter level per call.
//
// problem_t::init/reset (cgp/include/gunrock/framework/problem.hxx:48-49) and
// enactor_t::prepare_frontier / loop / is_converged / enact
// (cgp/include/gunrock/framework/enactor.hxx:243-330) map to
// cgp_enactor_prepare_frontier, cgp_advance_filter_level,
// cgp_enactor_is_converged and cgp_enactor_enact.
#include <cstring>

#include "engine.h"

using namespace cgp;
using namespace cgp::dev;

struct cgp_enactor {
  GraphImpl* g = nullptr;
  std::unique_ptr<Workspace> ws;
  GroupSpec spec;
  std::vector<int> wcc_slots;
  cgp_options opts;
  cudaStream_t stream = nullptr;
  bool prepared = false;
};

extern "C" {

cgp_status cgp_enactor_create(cgp_graph* graph, const cgp_query* queries, int32_t nq,
                              const cgp_options* opts, cgp_enactor** out) {
  clear_error();
  if (out == nullptr) return set_error(CGP_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (graph == nullptr) return set_error(CGP_ERR_INVALID_ARG, "graph is NULL");
  if (queries == nullptr || nq <= 0) return set_error(CGP_ERR_INVALID_ARG, "query batch must be non-empty");
  if (nq > kMaxWords * 64)
    return set_error(CGP_ERR_INVALID_ARG, "an enactor holds at most 1024 queries");
  GraphImpl* g = &graph->impl;
  for (int i = 0; i < nq; ++i) {
    if (queries[i].kind < CGP_KIND_BFS || queries[i].kind > CGP_KIND_KHOP)
      return set_error(CGP_ERR_INVALID_ARG, "unknown query kind");
    if (queries[i].kind != CGP_KIND_WCC && (queries[i].source < 0 || queries[i].source >= g->V))
      return set_error(CGP_ERR_INVALID_ARG, "query source out of range");
    if (queries[i].kind == CGP_KIND_KHOP && queries[i].k < 0)
      return set_error(CGP_ERR_INVALID_ARG, "k-hop bound must be non-negative");
  }
  auto* e = new (std::nothrow) cgp_enactor();
  if (!e) return set_error(CGP_ERR_OOM, "host allocation failed");
  try {
    ck(cudaSetDevice(g->device), "cudaSetDevice");
    e->g = g;
    if (opts) e->opts = *opts;
    else cgp_options_init(&e->opts);
    e->opts.use_cuda_graph = 0;  // single levels are launched directly
    e->ws = std::make_unique<Workspace>(g->device);
    e->stream = e->opts.stream ? static_cast<cudaStream_t>(e->opts.stream) : e->ws->stream;
    e->spec = make_group(queries, nq, choose_words(nq, e->opts.mask_words), e->opts.depth_mode);
    for (int i = 0; i < nq; ++i)
      if (queries[i].kind == CGP_KIND_WCC) e->wcc_slots.push_back(i);
    *out = e;
    return CGP_OK;
  } catch (...) {
    cgp_status st = translate_exception();
    delete e;
    return st;
  }
}

cgp_status cgp_enactor_destroy(cgp_enactor* e) {
  clear_error();
  if (e == nullptr) return CGP_OK;
  if (e->stream) cudaStreamSynchronize(e->stream);
  delete e;
  return CGP_OK;
}

cgp_status cgp_enactor_prepare_frontier(cgp_enactor* e) {
  clear_error();
  if (e == nullptr) return set_error(CGP_ERR_INVALID_ARG, "enactor is NULL");
  try {
    group_prepare(e->g, e->ws.get(), e->spec, e->opts, e->stream);
    ck(cudaStreamSynchronize(e->stream), "prepare");
    e->prepared = true;
    return CGP_OK;
  } catch (...) {
    return translate_exception();
  }
}

static LevelCtl read_ctl(cgp_enactor* e) {
  LevelCtl c;
  ck(cudaStreamSynchronize(e->stream), "sync");
  ck(cudaMemcpy(&c, e->ws->ctl.p, sizeof(LevelCtl), cudaMemcpyDeviceToHost), "read ctl");
  return c;
}

cgp_status cgp_advance_filter_level(cgp_enactor* e, int32_t direction, int64_t* next_size) {
  clear_error();
  if (e == nullptr) return set_error(CGP_ERR_INVALID_ARG, "enactor is NULL");
  if (!e->prepared) return set_error(CGP_ERR_INVALID_ARG, "prepare_frontier was not called");
  if (direction < CGP_MODE_PUSH || direction > CGP_MODE_HYBRID)
    return set_error(CGP_ERR_INVALID_ARG, "unknown direction");
  try {
    LevelCtl c = read_ctl(e);
    if (c.done == 1) {
      if (next_size) *next_size = 0;
      return CGP_OK;
    }
    if (direction == CGP_MODE_PULL && !e->g->can_gather())
      return set_error(CGP_ERR_INVALID_ARG, "pull needs a symmetric graph or its transpose");
    if (direction != CGP_MODE_HYBRID && e->spec.has_bfs) {
      int32_t dir = direction == CGP_MODE_PULL ? kDirPull : kDirPush;
      ck(cudaMemcpyAsync(reinterpret_cast<char*>(e->ws->ctl.p) + offsetof(LevelCtl, dir), &dir,
                         sizeof(dir), cudaMemcpyHostToDevice, e->stream), "set direction");
    }
    cgp_options o = e->opts;
    if (direction == CGP_MODE_PULL) o.traversal_mode = CGP_MODE_HYBRID;  // pull kernels enqueued
    GroupRun r;
    group_enact(e->g, e->ws.get(), e->spec, o, e->stream, &r, 1);
    LevelCtl after = read_ctl(e);
    if (next_size) *next_size = static_cast<int64_t>(after.count[after.level & 1]);
    if (after.done == 1 && next_size) *next_size = static_cast<int64_t>(after.count[after.level & 1]);
    return CGP_OK;
  } catch (...) {
    return translate_exception();
  }
}

cgp_status cgp_enactor_is_converged(cgp_enactor* e, int32_t* converged) {
  clear_error();
  if (e == nullptr || converged == nullptr) return set_error(CGP_ERR_INVALID_ARG, "NULL argument");
  try {
    LevelCtl c = read_ctl(e);
    *converged = c.done == 1 ? 1 : 0;
    return CGP_OK;
  } catch (...) {
    return translate_exception();
  }
}

cgp_status cgp_enactor_enact(cgp_enactor* e, cgp_stats* stats) {
  clear_error();
  if (e == nullptr) return set_error(CGP_ERR_INVALID_ARG, "enactor is NULL");
  try {
    if (!e->prepared) {
      group_prepare(e->g, e->ws.get(), e->spec, e->opts, e->stream);
      e->prepared = true;
    }
    cudaEvent_t t0, t1;
    ck(cudaEventCreate(&t0), "event");
    ck(cudaEventCreate(&t1), "event");
    ck(cudaEventRecord(t0, e->stream), "event");
    cgp_options o = e->opts;
    o.use_cuda_graph = 1;
    GroupRun r;
    group_enact(e->g, e->ws.get(), e->spec, o, e->stream, &r, 0);
    ck(cudaEventRecord(t1, e->stream), "event");
    ck(cudaEventSynchronize(t1), "event");
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (stats) {
      std::memset(stats, 0, sizeof(*stats));
      stats->iterations = r.iterations;
      stats->push_levels = r.push_levels;
      stats->pull_levels = r.pull_levels;
      stats->groups = 1;
      stats->gpu_time_ms = ms;
      stats->frontier_vertices = r.frontier_vertices;
      stats->frontier_edges = r.frontier_edges;
      stats->device_status = r.status;
      stats->mask_words = e->spec.W;
      stats->depth_mode = e->spec.depth_mode == kDepthPlanes ? CGP_DEPTH_PLANES : CGP_DEPTH_DIRECT;
    }
    return CGP_OK;
  } catch (...) {
    return translate_exception();
  }
}

cgp_status cgp_enactor_frontier(cgp_enactor* e, int32_t* vertices, uint64_t* masks, int64_t cap,
                                int64_t* count, int32_t* mask_words) {
  clear_error();
  if (e == nullptr || count == nullptr) return set_error(CGP_ERR_INVALID_ARG, "NULL argument");
  try {
    LevelCtl c = read_ctl(e);
    const int par = c.level & 1;
    const int64_t n = c.done == 1 ? 0 : static_cast<int64_t>(c.count[par]);
    *count = n;
    if (mask_words) *mask_words = e->spec.W;
    if (vertices == nullptr || n == 0) return CGP_OK;
    const int64_t m = std::min(n, cap);
    const int W = e->spec.W;
    std::vector<int32_t> list(m);
    ck(cudaMemcpy(list.data(), (par ? e->ws->list1 : e->ws->list0).p, m * 4, cudaMemcpyDeviceToHost),
       "read frontier");
    std::memcpy(vertices, list.data(), m * 4);
    if (masks) {
      const uint64_t* f = (par ? e->ws->fbuf1 : e->ws->fbuf0).as<uint64_t>();
      for (int64_t i = 0; i < m; ++i)
        ck(cudaMemcpy(masks + i * W, f + static_cast<size_t>(list[i]) * W, W * 8,
                      cudaMemcpyDeviceToHost), "read masks");
    }
    return CGP_OK;
  } catch (...) {
    return translate_exception();
  }
}

cgp_status cgp_enactor_read_values(cgp_enactor* e, void* out, int32_t out_layout, int32_t on_device) {
  clear_error();
  if (e == nullptr || out == nullptr) return set_error(CGP_ERR_INVALID_ARG, "NULL argument");
  if (out_layout != CGP_LAYOUT_VERTEX_MAJOR && out_layout != CGP_LAYOUT_QUERY_MAJOR)
    return set_error(CGP_ERR_INVALID_ARG, "unknown out_layout");
  if (!e->prepared) return set_error(CGP_ERR_INVALID_ARG, "prepare_frontier was not called");
  try {
    const int64_t V = e->g->V;
    const int nq = e->spec.Qg;
    const bool qmajor = out_layout == CGP_LAYOUT_QUERY_MAJOR;
    uint32_t* dout = static_cast<uint32_t*>(out);
    if (!on_device) {
      e->ws->stage.ensure(static_cast<size_t>(V) * nq * 4);
      dout = e->ws->stage.as<uint32_t>();
    }
    std::vector<int32_t> qmap(nq);
    for (int i = 0; i < nq; ++i) qmap[i] = i;
    e->ws->qmap.ensure(static_cast<size_t>(nq) * 4);
    ck(cudaMemcpyAsync(e->ws->qmap.p, qmap.data(), nq * 4, cudaMemcpyHostToDevice, e->stream),
       "upload query map");
    OutMap om;
    om.out = dout;
    om.sv = qmajor ? 1 : nq;
    om.sq = qmajor ? V : 1;
    om.qmap = e->ws->qmap.as<int32_t>();
    om.qmap_contiguous = 1;
    group_write_output(e->g, e->ws.get(), e->spec, om, qmajor, e->stream);
    if (!e->wcc_slots.empty()) {
      e->ws->wcc.ensure(static_cast<size_t>(V) * 4);
      wcc_labels(e->g, e->ws->wcc.as<uint32_t>(), e->stream);
      for (int i : e->wcc_slots) broadcast_labels(e->ws->wcc.as<uint32_t>(), V, om, i, e->stream);
    }
    if (!on_device)
      ck(cudaMemcpyAsync(out, dout, static_cast<size_t>(V) * nq * 4, cudaMemcpyDeviceToHost, e->stream),
         "copy out");
    ck(cudaStreamSynchronize(e->stream), "read values");
    return CGP_OK;
  } catch (...) {
    return translate_exception();
  }
}

}  // extern "C"
