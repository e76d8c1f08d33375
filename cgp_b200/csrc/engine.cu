// Multi-query traversal engine: graph upload, cached device workspaces, the
// device-driven level loop (replayed as CUDA graphs) and output writing.
//
// Replaces the host loops of frontier_engine::run
// (puercgp/include/puercgp/engine/frontier_engine.hxx:2203-3139) and
// hybrid_frontier_engine::run (hybrid_engine.hxx:793-1141).  The reference
// copies one or two counters to the host and synchronises after every level;
// here the direction decision, counter resets and convergence test run in a
// one-thread kernel at the end of each level, and the host only looks at the
// control block once per chunk of levels.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <numeric>

#include "engine.h"
#include "kernels.cuh"

namespace cgp {

using namespace dev;

// ------------------------------------------------------------- buffers
namespace {
// Fault-injection hook for tests: >= 0 counts down the device allocations
// still allowed before one fails as if the device were out of memory; -1 off.
std::atomic<int64_t> g_fail_alloc_countdown{-1};

bool injected_alloc_failure() {
  int64_t c = g_fail_alloc_countdown.load();
  while (c >= 0) {
    if (g_fail_alloc_countdown.compare_exchange_weak(c, c - 1)) return c == 0;
  }
  return false;
}
}  // namespace

DevBuf::~DevBuf() {
  if (p) cudaFree(p);
}

bool DevBuf::ensure(size_t need) {
  if (need <= bytes && p) return false;
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
  size_t alloc = std::max<size_t>(need, 256);
  if (injected_alloc_failure())
    throw ApiError{CGP_ERR_OOM, "cudaMalloc of " + std::to_string(alloc) +
                                    " bytes failed (injected by cgp_debug_fail_allocations)"};
  cudaError_t e = cudaMalloc(&p, alloc);
  if (e != cudaSuccess) {
    cudaGetLastError();
    p = nullptr;
    throw ApiError{CGP_ERR_OOM, "cudaMalloc of " + std::to_string(alloc) + " bytes failed"};
  }
  bytes = alloc;
  return true;
}

Workspace::Workspace(int dev) : device(dev) {
  ck(cudaHostAlloc(reinterpret_cast<void**>(&hctl), 2 * sizeof(LevelCtl), cudaHostAllocDefault),
     "cudaHostAlloc(ctl)");
  ck(cudaHostAlloc(reinterpret_cast<void**>(&hslots), kMaxWords * 64 * sizeof(SlotDev),
                   cudaHostAllocDefault),
     "cudaHostAlloc(slots)");
  ck(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaStreamCreateWithFlags(&capture, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaEventCreateWithFlags(&out_ready, cudaEventDisableTiming), "cudaEventCreate");
  for (auto& e : ev) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
  ctl.ensure(sizeof(LevelCtl));
  slots.ensure(kMaxWords * 64 * sizeof(SlotDev));
}

void Workspace::clear_graphs() {
  for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);
  graphs.clear();
}

Workspace::~Workspace() {
  clear_graphs();
  if (hctl) cudaFreeHost(hctl);
  if (hslots) cudaFreeHost(hslots);
  if (stream) cudaStreamDestroy(stream);
  if (capture) cudaStreamDestroy(capture);
  if (copy) cudaStreamDestroy(copy);
  if (out_ready) cudaEventDestroy(out_ready);
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
}

KernelTimer::KernelTimer() {
  for (auto& e : ev) ck(cudaEventCreate(&e), "cudaEventCreate");
}

KernelTimer::~KernelTimer() {
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
}

void KernelTimer::mark(int c, cudaStream_t s) {
  if (n == kMaxMarks) flush();
  ck(cudaEventRecord(ev[n], s), "timer event");
  cls[n] = c;
  ++n;
  if (c >= 0) ++count[c];
}

void KernelTimer::flush() {
  if (n == 0) return;
  ck(cudaEventSynchronize(ev[n - 1]), "timer sync");
  for (int i = 0; i + 1 < n; ++i) {
    if (cls[i] < 0) continue;
    float t = 0;
    ck(cudaEventElapsedTime(&t, ev[i], ev[i + 1]), "timer elapsed");
    ms[cls[i]] += t;
  }
  // keep the last mark open across flushes
  if (cls[n - 1] >= 0) {
    cudaEvent_t last = ev[n - 1];
    int lc = cls[n - 1];
    ev[n - 1] = ev[0];
    ev[0] = last;
    cls[0] = lc;
    n = 1;
  } else {
    n = 0;
  }
}

// --------------------------------------------------------------- graph
DevGraph GraphImpl::dev_graph(int64_t h) {
  const HeavyPair& hp = heavy_for(h);
  DevGraph d;
  d.row = row.p;
  d.col = col.as<int32_t>();
  d.w = w.p;
  d.prow = pull_row();
  d.pcol = pull_col();
  d.pw = pull_w();
  d.V = V;
  d.E = E;
  d.heavy = hp.heavy.vertices.as<int32_t>();
  d.heavy_chunk_start = hp.heavy.chunk_start.as<int64_t>();
  d.n_heavy = hp.heavy.n;
  d.heavy_chunks = hp.heavy.chunks;
  d.pheavy = hp.pheavy.vertices.as<int32_t>();
  d.pheavy_chunk_start = hp.pheavy.chunk_start.as<int64_t>();
  d.pheavy_ch = hp.pheavy.chunk_h.as<int32_t>();
  d.pheavy_cb = hp.pheavy.chunk_beg.as<int64_t>();
  d.pheavy_ce = hp.pheavy.chunk_end.as<int64_t>();
  d.n_pheavy = hp.pheavy.n;
  d.pheavy_chunks = hp.pheavy.chunks;
  d.plight = hp.plight.vertices.as<int32_t>();
  d.plight_chunk_start = hp.plight.chunk_start.as<int32_t>();
  d.plight_beg = hp.plight.beg.as<int64_t>();
  d.plight_pre = hp.plight.pre.as<int32_t>();
  d.n_plight_chunks = hp.plight.chunks;
  d.n_pmid = hp.plight.n_mid;
  d.heavy_degree = h;
  return d;
}

namespace {

// Host copies kept for table building.
struct HostCsr {
  std::vector<int64_t> row, trow;
};
std::mutex g_host_mu;
std::map<const GraphImpl*, HostCsr> g_host;

void build_heavy(const std::vector<int64_t>& row, int64_t V, int64_t h, HeavyTable& t) {
  std::vector<int32_t> vs;
  std::vector<int64_t> cs{0};
  for (int64_t v = 0; v < V; ++v) {
    int64_t d = row[v + 1] - row[v];
    if (d > h) {
      vs.push_back(static_cast<int32_t>(v));
      cs.push_back(cs.back() + (d + kHeavyChunk - 1) / kHeavyChunk);
    }
  }
  t.n = static_cast<int32_t>(vs.size());
  t.chunks = cs.back();
  // per chunk: its vertex's table index and its edge range, so that a CTA
  // finds its work with three independent loads instead of a binary search
  std::vector<int32_t> ch(static_cast<size_t>(t.chunks));
  std::vector<int64_t> cb(static_cast<size_t>(t.chunks)), ce(static_cast<size_t>(t.chunks));
  for (size_t i = 0; i < vs.size(); ++i) {
    const int64_t b = row[vs[i]], e = row[vs[i] + 1];
    for (int64_t c = cs[i]; c < cs[i + 1]; ++c) {
      ch[c] = static_cast<int32_t>(i);
      cb[c] = b + (c - cs[i]) * kHeavyChunk;
      ce[c] = std::min(e, cb[c] + kHeavyChunk);
    }
  }
  t.vertices.ensure(std::max<size_t>(vs.size(), 1) * sizeof(int32_t));
  t.chunk_start.ensure(cs.size() * sizeof(int64_t));
  t.chunk_h.ensure(std::max<size_t>(ch.size(), 1) * sizeof(int32_t));
  t.chunk_beg.ensure(std::max<size_t>(cb.size(), 1) * sizeof(int64_t));
  t.chunk_end.ensure(std::max<size_t>(ce.size(), 1) * sizeof(int64_t));
  if (!vs.empty()) {
    ck(cudaMemcpy(t.vertices.p, vs.data(), vs.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
       "upload heavy");
    ck(cudaMemcpy(t.chunk_h.p, ch.data(), ch.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
       "upload heavy chunk vertices");
    ck(cudaMemcpy(t.chunk_beg.p, cb.data(), cb.size() * sizeof(int64_t), cudaMemcpyHostToDevice),
       "upload heavy chunk starts");
    ck(cudaMemcpy(t.chunk_end.p, ce.data(), ce.size() * sizeof(int64_t), cudaMemcpyHostToDevice),
       "upload heavy chunk ends");
  }
  ck(cudaMemcpy(t.chunk_start.p, cs.data(), cs.size() * sizeof(int64_t), cudaMemcpyHostToDevice),
     "upload heavy chunks");
}

void build_light_chunks(const std::vector<int64_t>& row, int64_t V, int64_t h, LightChunks& t) {
  // light vertices by in-degree, largest first (ties by id): CTAs take chunks
  // roughly in this order, so within a gather level the better-connected
  // vertices settle first and the rest read their lowered distances
  std::vector<int32_t> order;
  for (int64_t v = 0; v < V; ++v) {
    const int64_t d = row[v + 1] - row[v];
    if (d > 0 && d <= h) order.push_back(static_cast<int32_t>(v));
  }
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    return row[a + 1] - row[a] > row[b + 1] - row[b];
  });
  std::vector<int32_t> vs;
  std::vector<int32_t> cs{0};
  int cur_v = 0;
  int64_t cur_e = 0;
  for (const int32_t v : order) {
    const int64_t d = row[v + 1] - row[v];
    if (cur_v > 0 && (cur_v == dev::kLightChunkVerts || cur_e + d > dev::kLightChunkEdges)) {
      cs.push_back(static_cast<int32_t>(vs.size()));
      cur_v = 0;
      cur_e = 0;
    }
    vs.push_back(static_cast<int32_t>(v));
    ++cur_v;
    cur_e += d;
  }
  if (cur_v > 0) cs.push_back(static_cast<int32_t>(vs.size()));
  t.n = static_cast<int32_t>(vs.size());
  t.chunks = static_cast<int32_t>(cs.size()) - 1;
  t.n_mid = 0;
  while (t.n_mid < t.n && row[vs[t.n_mid] + 1] - row[vs[t.n_mid]] > 32) ++t.n_mid;
  // per entry: its first in-edge and the chunk's in-edges up to and including
  // it, so that a chunk's header is three independent loads
  std::vector<int64_t> beg(vs.size());
  std::vector<int32_t> pre(vs.size());
  for (size_t c = 0; c + 1 < cs.size(); ++c) {
    int32_t acc = 0;
    for (int32_t i = cs[c]; i < cs[c + 1]; ++i) {
      const int32_t v = vs[i];
      beg[i] = row[v];
      acc += static_cast<int32_t>(row[v + 1] - row[v]);
      pre[i] = acc;
    }
  }
  t.vertices.ensure(std::max<size_t>(vs.size(), 1) * sizeof(int32_t));
  t.chunk_start.ensure(cs.size() * sizeof(int32_t));
  t.beg.ensure(std::max<size_t>(vs.size(), 1) * sizeof(int64_t));
  t.pre.ensure(std::max<size_t>(vs.size(), 1) * sizeof(int32_t));
  if (!vs.empty()) {
    ck(cudaMemcpy(t.vertices.p, vs.data(), vs.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
       "upload light vertices");
    ck(cudaMemcpy(t.beg.p, beg.data(), beg.size() * sizeof(int64_t), cudaMemcpyHostToDevice),
       "upload light offsets");
    ck(cudaMemcpy(t.pre.p, pre.data(), pre.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
       "upload light prefixes");
  }
  ck(cudaMemcpy(t.chunk_start.p, cs.data(), cs.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
     "upload light chunks");
}

}  // namespace

const HeavyPair& GraphImpl::heavy_for(int64_t h) {
  std::lock_guard<std::mutex> lk(heavy_mu);
  auto it = heavy_cache.find(h);
  if (it != heavy_cache.end()) return *it->second;
  auto hp = std::make_unique<HeavyPair>();
  {
    std::lock_guard<std::mutex> hl(g_host_mu);
    HostCsr& hc = g_host[this];
    build_heavy(hc.row, V, h, hp->heavy);
    build_heavy(hc.trow.empty() ? hc.row : hc.trow, V, h, hp->pheavy);
    build_light_chunks(hc.trow.empty() ? hc.row : hc.trow, V, h, hp->plight);
  }
  return *heavy_cache.emplace(h, std::move(hp)).first->second;
}

std::unique_ptr<Workspace> GraphImpl::acquire() {
  std::lock_guard<std::mutex> lk(mu);
  if (!pool.empty()) {
    auto ws = std::move(pool.back());
    pool.pop_back();
    return ws;
  }
  return std::make_unique<Workspace>(device);
}

void GraphImpl::release(std::unique_ptr<Workspace> ws) {
  std::lock_guard<std::mutex> lk(mu);
  pool.push_back(std::move(ws));
}

cgp_status translate_exception() {
  try {
    throw;
  } catch (const ApiError& e) {
    return set_error(e.code, e.msg);
  } catch (const CudaError& e) {
    cudaError_t c = e.code;
    return set_error(c == cudaErrorMemoryAllocation ? CGP_ERR_OOM : CGP_ERR_CUDA,
                     e.where + ": " + cudaGetErrorString(c));
  } catch (const std::bad_alloc&) {
    return set_error(CGP_ERR_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return set_error(CGP_ERR_INVALID_ARG, e.what());
  } catch (...) {
    return set_error(CGP_ERR_INVALID_ARG, "unknown error");
  }
}

// -------------------------------------------------------------- groups
int choose_words(int n, int requested) {
  if (requested > 0) {
    int w = 1;
    while (w < requested) w <<= 1;
    return std::min(w, kMaxWords);
  }
  int need = std::max(1, (n + 63) / 64);
  int w = 1;
  while (w < need) w <<= 1;
  return std::min(w, kMaxWords);
}

GroupSpec make_group(const cgp_query* q, int n, int W, int depth_mode) {
  GroupSpec g;
  g.W = W;
  g.Qg = n;
  g.slots.resize(n);
  for (int i = 0; i < n; ++i) {
    g.slots[i].kind = q[i].kind;
    g.slots[i].source = q[i].source;
    g.slots[i].k = q[i].k;
    g.slots[i].base = 0;
    if (q[i].kind == CGP_KIND_SSSP) g.has_sssp = true;
    if (q[i].kind == CGP_KIND_BFS || q[i].kind == CGP_KIND_KHOP) g.has_bfs = true;
  }
  if (depth_mode == CGP_DEPTH_PLANES && !g.has_sssp) g.depth_mode = kDepthPlanes;
  else if (depth_mode == CGP_DEPTH_DIRECT || g.has_sssp) g.depth_mode = kDepthDirect;
  else g.depth_mode = (n >= 16) ? kDepthPlanes : kDepthDirect;  // auto
  return g;
}

static constexpr int kInitialPlanes = 8;

int64_t group_state_bytes(const GraphImpl* g, int W, int Qg, int depth_mode) {
  const int64_t V = g->V;
  int64_t b = 3 * V * W * 8 + 3 * V * 4;
  if (depth_mode == kDepthPlanes) b += static_cast<int64_t>(kInitialPlanes) * V * W * 8;
  else b += V * static_cast<int64_t>(Qg) * 4;
  return b;
}

namespace {

struct Grids {
  int tile;   // tile kernels (grid-stride)
  int heavy;
  int clear;
  int dense;
  int dense2;
  int gather;
  int gather_heavy;
  int gather_vec;
  int gather_heavy_vec;
  int gather_chunked;
  int gather_heavy_vec2;
  int bfs_chunked;
  int bfs_mid;
};

struct LevelLaunch {
  GroupDev g{};
  DevGraph G;
  Grids gr;
  bool has_bfs;
  bool has_sssp;
  bool pull;
  bool spull;        // SSSP gather kernels are part of the level
  bool gvec;         // rows allow the vectorised gather (alignment, width)
  bool lchunks;      // light vertices gathered in CTA chunks (in 4-word slices above W = 4)
  int dense_unroll;  // edges per step of the dense SSSP kernel (1 or 2)
  KernelTimer* kt;   // per-class event timing (non-graph runs only)
  bool heavy_push = false;                // heavy-queue push kernels are part of a level
  bool bfs_chunked = false;               // chunked light-vertex BFS pull is part of a pull level
  bool chunk_dir = false;                 // census of per-chunk frontier edges
  bool device_loop = false;               // level end sets a WHILE node's condition
  cudaGraphConditionalHandle loop = 0;    // ... this one
  int32_t level_cap = 0;                  // ... and stops at this many levels
};

template <typename K>
int occupancy_grid(K kernel, int sms) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 2;
  }
  return std::max(1, per_sm) * sms;
}

// Enqueues one level; returns the number of kernels launched.
template <int W, typename OT, int DEPTH, int WK>
int enqueue_level_t(const LevelLaunch& L, cudaStream_t s) {
  const int t = L.gr.tile, h = L.gr.heavy, c = L.gr.clear;
  KernelTimer* kt = L.kt;
  int n = 0;
  if (kt) kt->mark(kClassClear, s);
  k_clear_next<W><<<c, kBlock, 0, s>>>(L.g, L.G.E);
  ++n;
  if (L.g.fsum != nullptr && (L.pull || L.spull)) {
    k_frontier_summary<W, OT><<<c, kBlock, 0, s>>>(L.g, L.G);
    ++n;
  }
  if (L.heavy_push) {
    k_heavy_queue<OT><<<c, kBlock, 0, s>>>(L.g, L.G);
    ++n;
  }
  if (L.has_bfs) {
    if (kt) kt->mark(kClassBfsPush, s);
    k_bfs_push<W, OT, DEPTH><<<t, kBlock, 0, s>>>(L.g, L.G);
    ++n;
    if (L.heavy_push) {
      k_bfs_push_heavy<W, OT, DEPTH><<<h, kBlock, 0, s>>>(L.g, L.G);
      ++n;
    }
    if (L.pull) {
      if (kt) kt->mark(kClassBfsPull, s);
      k_bfs_pull<W, OT, DEPTH><<<t, kBlock, 0, s>>>(L.g, L.G);
      ++n;
      if (L.G.n_pmid > 0) {  // in-degree 33 .. heavy_degree: warp per vertex
        k_bfs_pull_mid<W, OT, DEPTH><<<L.gr.bfs_mid, kBlock, 0, s>>>(L.g, L.G);
        ++n;
      }
      if (L.bfs_chunked) {  // each of the two forms returns at once on the other's levels
        k_bfs_pull_chunked<W, OT, DEPTH><<<L.gr.bfs_chunked, kBlock, 0, s>>>(L.g, L.G);
        ++n;
      }
      if (L.G.n_pheavy) {
        k_bfs_pull_heavy<W, OT><<<h, kBlock, 0, s>>>(L.g, L.G);
        k_bfs_pull_heavy_commit<W, OT, DEPTH><<<std::max(1, (L.G.n_pheavy + kBlock - 1) / kBlock), kBlock, 0, s>>>(L.g, L.G);
        n += 2;
      }
    }
  }
  if (L.has_sssp) {
    if (kt) kt->mark(kClassSsspPush, s);
    k_sssp_push<W, OT, WK><<<t, kBlock, 0, s>>>(L.g, L.G);
    if (kt) kt->mark(kClassSsspDense, s);
    if (L.dense_unroll == 2)
      k_sssp_dense<W, OT, WK, 2><<<L.gr.dense2, kBlock, 0, s>>>(L.g, L.G);
    else
      k_sssp_dense<W, OT, WK, 1><<<L.gr.dense, kBlock, 0, s>>>(L.g, L.G);
    n += 2;
    if (L.heavy_push) {
      if (kt) kt->mark(kClassSsspHeavy, s);
      k_sssp_push_heavy<W, OT, WK><<<h, kBlock, 0, s>>>(L.g, L.G);
      ++n;
    }
    if (L.spull) {
      if (kt) kt->mark(kClassSsspPull, s);
      // heavy vertices first: the light vertices' gathers of the same level
      // then read the hubs' lowered distances (the level is Gauss-Seidel)
      if (L.G.n_pheavy) {
        if (L.gvec && W <= 4) {
          // whole-row and chunk-skipping variants; each returns at once on the
          // other's levels
          k_sssp_pull_heavy_vec<W, OT, WK, 1><<<L.gr.gather_heavy_vec, kBlock, 0, s>>>(L.g, L.G);
          k_sssp_pull_heavy_vec<W, OT, WK, 2><<<L.gr.gather_heavy_vec2, kBlock, 0, s>>>(L.g, L.G);
          ++n;
        } else if (L.gvec) {
          k_sssp_pull_heavy_vec<W, OT, WK, 0><<<L.gr.gather_heavy_vec, kBlock, 0, s>>>(L.g, L.G);
        } else {
          k_sssp_pull_heavy<W, OT, WK><<<L.gr.gather_heavy, kBlock, 0, s>>>(L.g, L.G);
        }
        ++n;
      }
      if constexpr (W <= 4) {
        if (L.gvec && L.lchunks) {
          k_sssp_pull_chunked<W, OT, WK><<<L.gr.gather_chunked, kBlock, 0, s>>>(L.g, L.G);
        } else if (L.gvec) {
          k_sssp_pull_vec<W, OT, WK><<<L.gr.gather_vec, kBlock, 0, s>>>(L.g, L.G);
        } else {
          k_sssp_pull<W, OT, WK><<<L.gr.gather, kBlock, 0, s>>>(L.g, L.G);
        }
      } else if (L.gvec && L.lchunks) {
        k_sssp_pull_chunked<4, OT, WK, W><<<dim3(L.gr.gather_chunked, W / 4), kBlock, 0, s>>>(L.g, L.G);
      } else if (L.gvec) {
        k_sssp_pull_vec<W, OT, WK><<<L.gr.gather_vec, kBlock, 0, s>>>(L.g, L.G);
      } else {
        k_sssp_pull<W, OT, WK><<<L.gr.gather, kBlock, 0, s>>>(L.g, L.G);
      }
      ++n;
    }

  }
  if (kt) kt->mark(kClassLevelEnd, s);
  if (L.chunk_dir) {
    k_chunk_census<W, OT><<<c, kBlock, 0, s>>>(L.g, L.G);
    ++n;
  }
  if (L.device_loop) k_level_end_loop<W><<<1, 32, 0, s>>>(L.g, L.loop, L.level_cap);
  else k_level_end<W><<<1, 32, 0, s>>>(L.g);
  ++n;
  if (kt) kt->mark(-1, s);
  return n;
}

template <int W, typename OT, int DEPTH, int WK>
Grids grids_t(int sms) {
  static int tile = 0, heavy = 0, dense = 0, dense2 = 0, gather = 0, gather_heavy = 0;
  static int gather_vec = 0, gather_heavy_vec = 0, gather_chunked = 0, gather_heavy_vec2 = 0;
  static int bfs_chunked = 0, bfs_mid = 0;
  if (tile == 0) {
    bfs_chunked = occupancy_grid(k_bfs_pull_chunked<W, OT, DEPTH>, sms);
    bfs_mid = occupancy_grid(k_bfs_pull_mid<W, OT, DEPTH>, sms);
    if constexpr (W <= 4) {
      gather_chunked = occupancy_grid(k_sssp_pull_chunked<W, OT, WK>, sms);
    } else {
      // slices of 4 words, all resident at once: x blocks per slice
      gather_chunked = std::max(1, occupancy_grid(k_sssp_pull_chunked<4, OT, WK, W>, sms) / (W / 4));
    }
    gather_vec = occupancy_grid(k_sssp_pull_vec<W, OT, WK>, sms);
    gather_heavy_vec = occupancy_grid(k_sssp_pull_heavy_vec<W, OT, WK, (W <= 4 ? 1 : 0)>, sms);
    gather_heavy_vec2 = occupancy_grid(k_sssp_pull_heavy_vec<W, OT, WK, 2>, sms);
    gather = occupancy_grid(k_sssp_pull<W, OT, WK>, sms);
    gather_heavy = occupancy_grid(k_sssp_pull_heavy<W, OT, WK>, sms);
    dense = occupancy_grid(k_sssp_dense<W, OT, WK, 1>, sms);
    dense2 = occupancy_grid(k_sssp_dense<W, OT, WK, 2>, sms);
    int a = occupancy_grid(k_bfs_push<W, OT, DEPTH>, sms);
    int b = occupancy_grid(k_bfs_pull<W, OT, DEPTH>, sms);
    int c = occupancy_grid(k_sssp_push<W, OT, WK>, sms);
    tile = std::min(a, std::min(b, c));
    heavy = std::min(occupancy_grid(k_bfs_pull_heavy<W, OT>, sms),
                     occupancy_grid(k_sssp_push_heavy<W, OT, WK>, sms));
  }
  Grids g;
  g.tile = tile;
  g.heavy = heavy;
  g.clear = sms * 4;
  g.dense = dense;
  g.dense2 = dense2;
  g.gather = gather;
  g.gather_heavy = gather_heavy;
  g.gather_vec = gather_vec;
  g.gather_heavy_vec = gather_heavy_vec;
  g.gather_chunked = gather_chunked;
  g.gather_heavy_vec2 = gather_heavy_vec2;
  g.bfs_chunked = bfs_chunked;
  g.bfs_mid = bfs_mid;
  return g;
}

template <int W, typename OT>
void seed_t(const GroupDev& g, const DevGraph& G, cudaStream_t s) {
  k_seed<W, OT><<<1, kBlock, 0, s>>>(g, G);
}

using EnqueueFn = int (*)(const LevelLaunch&, cudaStream_t);
using GridsFn = Grids (*)(int);
using SeedFn = void (*)(const GroupDev&, const DevGraph&, cudaStream_t);

struct Dispatch {
  EnqueueFn enqueue;
  GridsFn grids;
  SeedFn seed;
};

template <int W, typename OT, int DEPTH>
Dispatch pick_wk(int wk) {
  switch (wk) {
    case kWeightU32: return {enqueue_level_t<W, OT, DEPTH, kWeightU32>, grids_t<W, OT, DEPTH, kWeightU32>, seed_t<W, OT>};
    case kWeightF32: return {enqueue_level_t<W, OT, DEPTH, kWeightF32>, grids_t<W, OT, DEPTH, kWeightF32>, seed_t<W, OT>};
    default: return {enqueue_level_t<W, OT, DEPTH, kWeightNone>, grids_t<W, OT, DEPTH, kWeightNone>, seed_t<W, OT>};
  }
}

template <int W, typename OT>
Dispatch pick_depth(int depth, int wk) {
  return depth == kDepthPlanes ? pick_wk<W, OT, kDepthPlanes>(wk) : pick_wk<W, OT, kDepthDirect>(wk);
}

template <int W>
Dispatch pick_ot(int ob, int depth, int wk) {
  return ob == 8 ? pick_depth<W, int64_t>(depth, wk) : pick_depth<W, int32_t>(depth, wk);
}

Dispatch dispatch(int W, int ob, int depth, int wk) {
  switch (W) {
    case 1: return pick_ot<1>(ob, depth, wk);
    case 2: return pick_ot<2>(ob, depth, wk);
    case 4: return pick_ot<4>(ob, depth, wk);
    case 8: return pick_ot<8>(ob, depth, wk);
    default: return pick_ot<16>(ob, depth, wk);
  }
}

GroupDev group_dev(Workspace* ws, const GroupSpec& spec, bool profiles) {
  GroupDev g{};
  g.visited = ws->visited.as<uint64_t>();
  g.fbuf0 = ws->fbuf0.as<uint64_t>();
  g.fbuf1 = ws->fbuf1.as<uint64_t>();
  g.list0 = ws->list0.as<int32_t>();
  g.list1 = ws->list1.as<int32_t>();
  g.stamp = ws->stamp.as<int32_t>();
  g.planes = spec.depth_mode == kDepthPlanes ? ws->planes.as<uint64_t>() : nullptr;
  g.values = spec.depth_mode == kDepthPlanes
                 ? nullptr
                 : (spec.external_values ? spec.external_values : ws->values.as<uint32_t>());
  g.hacc = ws->hacc.as<uint64_t>();
  g.fsum = ws->fsum.as<uint64_t>();
  g.dense_list = ws->dense.as<int32_t>();
  g.hq_vertex = ws->hq_vertex.as<int32_t>();
  g.hq_start = ws->hq_start.as<int64_t>();
  g.hq_cap = static_cast<int64_t>(ws->hq_start.bytes / sizeof(int64_t));
  g.ctl = ws->ctl.as<LevelCtl>();
  g.prof = profiles ? ws->prof.as<LevelProfile>() : nullptr;
  g.slots = ws->slots.as<SlotDev>();
  g.Qg = spec.Qg;
  return g;
}

constexpr int kProfileCap = 1 << 16;

// SSSP levels may gather (pull) when the pull CSR exists and the options
// allow it: always in pull mode, by frontier edges in hybrid mode.
bool sssp_gather_on(const GraphImpl* g, const cgp_options& o) {
  if (!g->can_gather() || o.traversal_mode == CGP_MODE_PUSH) return false;
  return o.traversal_mode == CGP_MODE_PULL || o.sssp_pull_edge_ratio > 0;
}

// SSSP direction per 32-slot chunk: asked for, or by default in serving
// groups (whose slots are in every phase of their traversals at once).
bool sssp_chunk_dir(const GroupSpec& spec, const cgp_options& o) {
  if (!spec.has_sssp || o.traversal_mode != CGP_MODE_HYBRID) return false;
  return o.sssp_chunk_direction > 0 || (o.sssp_chunk_direction == 0 && spec.serving);
}

}  // namespace

void group_prepare(GraphImpl* g, Workspace* ws, GroupSpec& spec, const cgp_options& o,
                   cudaStream_t s) {
  const int64_t V = g->V;
  const int W = spec.W;
  const int64_t hth = heavy_threshold(o);
  const HeavyPair& hp = g->heavy_for(hth);
  bool moved = false;
  const size_t mask_bytes = static_cast<size_t>(V) * W * 8;
  try {
    moved |= ws->visited.ensure(mask_bytes);
    moved |= ws->fbuf0.ensure(mask_bytes);
    moved |= ws->fbuf1.ensure(mask_bytes);
    moved |= ws->list0.ensure(static_cast<size_t>(V) * 4);
    moved |= ws->list1.ensure(static_cast<size_t>(V) * 4);
    moved |= ws->stamp.ensure(static_cast<size_t>(V) * 4);
    moved |= ws->hacc.ensure(static_cast<size_t>(std::max(1, hp.pheavy.n)) * W * 8);
    moved |= ws->fsum.ensure(static_cast<size_t>(V) * 8);
    // heavy-queue capacity: every heavy vertex, and every vertex of out-degree
    // > 32 (small or skewed frontiers queue those)
    const size_t hq_cap = std::max<size_t>(std::max<int64_t>(1, hp.heavy.n), g->n_deg32);
    moved |= ws->hq_vertex.ensure(hq_cap * 4);
    moved |= ws->hq_start.ensure(hq_cap * 8);
    if (spec.has_sssp) moved |= ws->dense.ensure(static_cast<size_t>(V) * 4);
    if (spec.depth_mode == kDepthPlanes) {
      moved |= ws->planes.ensure(static_cast<size_t>(kInitialPlanes) * mask_bytes);
    } else if (spec.external_values == nullptr) {
      moved |= ws->values.ensure(static_cast<size_t>(V) * spec.Qg * 4);
    }
    if (o.profile_iterations) moved |= ws->prof.ensure(kProfileCap * sizeof(LevelProfile));
  } catch (...) {
    // a failed ensure() has already freed its old block: graphs captured with
    // the old pointers must never be replayed
    ws->generation++;
    ws->clear_graphs();
    throw;
  }
  if (moved) {
    ws->generation++;
    ws->clear_graphs();
  }
  ck(cudaMemsetAsync(ws->visited.p, 0, mask_bytes, s), "memset visited");
  ck(cudaMemsetAsync(ws->fbuf0.p, 0, mask_bytes, s), "memset frontier");
  ck(cudaMemsetAsync(ws->fbuf1.p, 0, mask_bytes, s), "memset next frontier");
  ck(cudaMemsetAsync(ws->stamp.p, 0xff, static_cast<size_t>(V) * 4, s), "memset stamp");
  ck(cudaMemsetAsync(ws->hacc.p, 0, static_cast<size_t>(std::max(1, hp.pheavy.n)) * W * 8, s),
     "memset hacc");
  ck(cudaMemsetAsync(ws->fsum.p, 0, static_cast<size_t>(V) * 8, s), "memset fsum");
  if (spec.depth_mode == kDepthPlanes)
    ck(cudaMemsetAsync(ws->planes.p, 0, static_cast<size_t>(kInitialPlanes) * mask_bytes, s),
       "memset planes");

  // slots and control block
  ck(cudaStreamSynchronize(s), "sync before slot upload");  // hslots/hctl are reused
  std::memcpy(ws->hslots, spec.slots.data(), spec.slots.size() * sizeof(SlotDev));
  ck(cudaMemcpyAsync(ws->slots.p, ws->hslots, spec.slots.size() * sizeof(SlotDev),
                     cudaMemcpyHostToDevice, s),
     "upload slots");
  LevelCtl& c = ws->hctl[0];
  std::memset(&c, 0, sizeof(c));
  for (int q = 0; q < spec.Qg; ++q) {
    const int k = spec.slots[q].kind;
    if (k == CGP_KIND_BFS || k == CGP_KIND_KHOP) c.bfs_bits[q >> 6] |= 1ULL << (q & 63);
    if (k == CGP_KIND_SSSP) c.sssp_bits[q >> 6] |= 1ULL << (q & 63);
  }
  for (int i = 0; i < kMaxW; ++i) c.expand[i] = ~0ULL;
  c.forced_dir = -1;
  c.halt_level = -1;
  c.max_iterations = o.max_iterations;
  int mode = o.traversal_mode;
  if (!g->can_gather()) mode = CGP_MODE_PUSH;
  c.mode = mode;
  c.num_planes = spec.depth_mode == kDepthPlanes ? kInitialPlanes : 0;
  c.profile_cap = o.profile_iterations ? kProfileCap : 0;
  c.pull_vertex_threshold = static_cast<unsigned long long>(
      std::max(1.0, o.pull_frontier_ratio * static_cast<double>(V)));
  c.pull_edge_threshold = static_cast<unsigned long long>(
      std::max(1.0, o.pull_edge_ratio * static_cast<double>(g->E)));
  c.sssp_gather = sssp_gather_on(g, o) ? 1 : 0;
  c.chunk_dir = sssp_chunk_dir(spec, o) ? 1 : 0;
  c.bfs_chunked = (spec.has_bfs && (o.bfs_pull_form == 1 || o.bfs_pull_form == 2) &&
                   hp.plight.chunks > 0) ? o.bfs_pull_form : 0;
  c.prev_dir = kDirPush;
  c.sssp_pull_edge_threshold = static_cast<unsigned long long>(
      std::max(1.0, o.sssp_pull_edge_ratio * static_cast<double>(g->E)));
  c.sssp_pull_pair_unit = o.sssp_pull_pair_ratio > 0
                              ? static_cast<unsigned long long>(
                                    std::max(1.0, o.sssp_pull_pair_ratio * static_cast<double>(g->E)))
                              : 0ULL;
  ck(cudaMemcpyAsync(ws->ctl.p, &c, sizeof(LevelCtl), cudaMemcpyHostToDevice, s), "upload ctl");

  const uint32_t sssp_inf = g->weight_kind == CGP_WEIGHT_F32 ? 0x7f800000u : 0xffffffffu;
  if (spec.depth_mode != kDepthPlanes) {
    int blocks = g->num_sms * 8;
    k_fill_values<<<blocks, kBlock, 0, s>>>(group_dev(ws, spec, false).values,
                                            ws->slots.as<SlotDev>(), spec.Qg, V, sssp_inf,
                                            spec.uniform_inf);
    ck(cudaGetLastError(), "fill values");
    spec.launches++;
  }
  Dispatch d = dispatch(W, g->offset_bytes, spec.depth_mode, g->weight_kind);
  d.seed(group_dev(ws, spec, o.profile_iterations != 0), g->dev_graph(hth), s);
  ck(cudaGetLastError(), "seed");
  spec.launches++;
}

namespace {

// Enqueues `levels` levels either as a replayed CUDA graph or as plain
// launches; levels < 0: the whole traversal as one device-looped graph (a
// WHILE conditional node around one level, the condition set by the level's
// last kernel from the done flag).
int enqueue_levels(GraphImpl* g, Workspace* ws, const GroupSpec& spec, const cgp_options& o,
                   cudaStream_t s, int levels, KernelTimer* kt) {
  Dispatch d = dispatch(spec.W, g->offset_bytes, spec.depth_mode, g->weight_kind);
  LevelLaunch L;
  L.g = group_dev(ws, spec, o.profile_iterations != 0);
  L.G = g->dev_graph(heavy_threshold(o));
  L.gr = d.grids(g->num_sms);
  L.has_bfs = spec.has_bfs;
  L.has_sssp = spec.has_sssp;
  int mode = o.traversal_mode;
  if (!g->can_gather()) mode = CGP_MODE_PUSH;
  L.pull = mode != CGP_MODE_PUSH;
  L.heavy_push = L.G.n_heavy > 0 || g->max_degree > 32;
  L.bfs_chunked = L.pull && spec.has_bfs && L.G.n_plight_chunks > 0 && o.bfs_pull_form == 1;
  L.spull = spec.has_sssp && sssp_gather_on(g, o);
  {
    // vector gather: kElem-slot vectors must stay inside rows and be aligned
    const int elem = spec.W == 1 ? 2 : 4;
    L.gvec = L.g.values != nullptr && spec.Qg % elem == 0 &&
             reinterpret_cast<uintptr_t>(L.g.values) % (4 * elem) == 0;
    L.lchunks = o.light_chunks >= 0;
  }
  L.dense_unroll = o.dense_unroll == 2 ? 2 : 1;
  L.chunk_dir = L.spull && sssp_chunk_dir(spec, o);
  L.kt = kt;
  if (!o.use_cuda_graph || kt != nullptr) {
    int n = 0;
    for (int i = 0; i < levels; ++i) n += d.enqueue(L, s);
    ck(cudaGetLastError(), "level launch");
    return n;
  }
  L.kt = nullptr;
  const bool loop = levels < 0;
  auto key = std::make_tuple(spec.W, g->offset_bytes, spec.depth_mode, g->weight_kind,
                             (spec.has_bfs ? 1 : 0) | (spec.has_sssp ? 2 : 0) | (L.pull ? 4 : 0) |
                                 (o.profile_iterations ? 8 : 0) | (L.dense_unroll == 2 ? 16 : 0) |
                                 (L.spull ? 32 : 0) | (L.lchunks ? 64 : 0) | (loop ? 128 : 0) |
                                 (L.chunk_dir ? 256 : 0) | (L.bfs_chunked ? 512 : 0),
                             levels, spec.Qg, static_cast<int>(L.G.heavy_degree), ws->generation,
                             reinterpret_cast<uint64_t>(L.g.values));
  auto it = ws->graphs.find(key);
  if (it == ws->graphs.end()) {
    cudaGraph_t graph = nullptr;
    int n = 0;
    if (loop) {
      ck(cudaGraphCreate(&graph, 0), "graph create");
      try {
        cudaGraphConditionalHandle h = 0;
        ck(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault),
           "conditional handle");
        cudaGraphNodeParams p{};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        ck(cudaGraphAddNode(&node, graph, nullptr, 0, &p), "conditional node");
        cudaGraph_t body = p.conditional.phGraph_out[0];
        L.device_loop = true;
        L.loop = h;
        L.level_cap = static_cast<int32_t>(std::min<int64_t>(g->V + 2, INT32_MAX - 1));
        ck(cudaStreamBeginCaptureToGraph(ws->capture, body, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal),
           "begin capture");
        n = d.enqueue(L, ws->capture);
        cudaError_t le = cudaGetLastError();
        cudaError_t ce = cudaStreamEndCapture(ws->capture, &body);
        ck(le, "capture launch");
        ck(ce, "end capture");
      } catch (...) {
        cudaGraphDestroy(graph);
        throw;
      }
    } else {
      ck(cudaStreamBeginCapture(ws->capture, cudaStreamCaptureModeThreadLocal), "begin capture");
      for (int i = 0; i < levels; ++i) n += d.enqueue(L, ws->capture);
      cudaError_t le = cudaGetLastError();
      cudaError_t ce = cudaStreamEndCapture(ws->capture, &graph);
      ck(le, "capture launch");
      ck(ce, "end capture");
    }
    cudaGraphExec_t exec = nullptr;
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    ck(ie, "instantiate");
    it = ws->graphs.emplace(key, CachedGraph{exec, n}).first;
  }
  ck(cudaGraphLaunch(it->second.exec, s), "graph launch");
  return it->second.launches;
}

}  // namespace

void group_enact(GraphImpl* g, Workspace* ws, GroupSpec& spec, const cgp_options& o,
                 cudaStream_t s, GroupRun* out, int max_levels, KernelTimer* kt) {
  const int per_chunk = kt ? 1 : (o.levels_per_sync > 0 ? o.levels_per_sync : 8);
  int enqueued = 0;
  int chunk = 0;
  LevelCtl* snap = ws->hctl;
  // A run to convergence without per-level timing is one device-looped graph:
  // the host waits once.  (The launch count of such a run is that of one
  // level; the per-level count is reported with the level count below.)
  const bool device_loop = kt == nullptr && max_levels <= 0 && o.use_cuda_graph &&
                           o.level_loop == CGP_LOOP_DEVICE;
  if (device_loop) {
    const int per_level = enqueue_levels(g, ws, spec, o, s, -1, nullptr);
    ck(cudaStreamSynchronize(s), "device level loop");
    LevelCtl c;
    ck(cudaMemcpy(&c, ws->ctl.p, sizeof(LevelCtl), cudaMemcpyDeviceToHost), "read ctl");
    spec.launches += static_cast<uint64_t>(per_level) * static_cast<uint64_t>(std::max(1, c.level));
  }
  for (;;) {
    if (device_loop) break;
    int n = per_chunk;
    if (max_levels > 0) n = std::min(n, max_levels - enqueued);
    if (n <= 0) break;
    // level time = the level kernels' classes (the open init interval of the
    // group is charged to its own class when the first level's marks flush)
    auto level_sum = [](const KernelTimer* t) {
      double x = 0;
      for (int c = 0; c < kNumClasses; ++c)
        if (c != kClassInit && c != kClassOutput && c != kClassWcc) x += t->ms[c];
      return x;
    };
    const double before = kt ? level_sum(kt) : 0.0;
    spec.launches += enqueue_levels(g, ws, spec, o, s, n, kt);
    enqueued += n;
    ck(cudaMemcpyAsync(&snap[chunk & 1], ws->ctl.p, sizeof(LevelCtl), cudaMemcpyDeviceToHost, s),
       "read ctl");
    ck(cudaEventRecord(ws->ev[chunk & 1], s), "event");
    bool stop = false;
    if (kt) {
      kt->flush();
      ck(cudaEventSynchronize(ws->ev[chunk & 1]), "sync level");
      out->level_ms.push_back(static_cast<float>(level_sum(kt) - before));
      stop = snap[chunk & 1].done != 0;
    } else if (chunk > 0) {
      ck(cudaEventSynchronize(ws->ev[(chunk - 1) & 1]), "sync chunk");
      const LevelCtl& c = snap[(chunk - 1) & 1];
      stop = c.done != 0;
    }
    if (stop) break;
    ++chunk;
  }
  ck(cudaStreamSynchronize(s), "level loop");
  LevelCtl c;
  ck(cudaMemcpy(&c, ws->ctl.p, sizeof(LevelCtl), cudaMemcpyDeviceToHost), "read ctl");
  if (c.status & kStatusLevelCap)
    throw ApiError{CGP_ERR_DEVICE, "traversal did not converge within " +
                                       std::to_string(c.level) + " levels"};
  if (c.done == 2 && (c.status & kStatusPlanesExhausted)) {
    // Deeper than the depth planes can hold: grow them and resume.
    const size_t mask_bytes = static_cast<size_t>(g->V) * spec.W * 8;
    const int K = c.num_planes;
    const int K2 = std::min(kMaxPlanes, K + 8);
    if (K2 == K) throw ApiError{CGP_ERR_DEVICE, "BFS depth exceeds 2^24 levels"};
    DevBuf bigger;
    bigger.ensure(static_cast<size_t>(K2) * mask_bytes);
    ck(cudaMemcpyAsync(bigger.p, ws->planes.p, static_cast<size_t>(K) * mask_bytes,
                       cudaMemcpyDeviceToDevice, s), "grow planes");
    ck(cudaMemsetAsync(static_cast<char*>(bigger.p) + static_cast<size_t>(K) * mask_bytes, 0,
                       static_cast<size_t>(K2 - K) * mask_bytes, s), "zero planes");
    std::swap(ws->planes.p, bigger.p);
    std::swap(ws->planes.bytes, bigger.bytes);
    ck(cudaStreamSynchronize(s), "grow planes");
    ws->generation++;
    ws->clear_graphs();
    c.num_planes = K2;
    c.status &= ~kStatusPlanesExhausted;
    c.done = 0;
    ck(cudaMemcpy(ws->ctl.p, &c, sizeof(LevelCtl), cudaMemcpyHostToDevice), "resume");
    group_enact(g, ws, spec, o, s, out, max_levels > 0 ? max_levels - enqueued : 0, kt);
    return;
  }
  out->iterations = c.level;
  out->push_levels = c.push_levels;
  out->pull_levels = c.pull_levels;
  out->frontier_vertices = c.total_frontier;
  out->frontier_edges = c.total_edges;
  out->status = c.status;
  out->counters = c.total;
  if (o.profile_iterations) {
    int n = std::min(c.level, kProfileCap);
    out->profiles.resize(n);
    if (n > 0)
      ck(cudaMemcpy(out->profiles.data(), ws->prof.p, n * sizeof(LevelProfile),
                    cudaMemcpyDeviceToHost), "read profiles");
  }
}

void group_enqueue_levels(GraphImpl* g, Workspace* ws, GroupSpec& spec, const cgp_options& o,
                          cudaStream_t s, int levels) {
  spec.launches += enqueue_levels(g, ws, spec, o, s, levels, nullptr);
}

void group_write_output(GraphImpl* g, Workspace* ws, GroupSpec& spec, OutMap om,
                        int query_major, cudaStream_t s) {
  spec.launches++;
  const dim3 grid(g->num_sms * 8, query_major ? std::min(spec.Qg, 65535) : 1);
  if (spec.depth_mode == kDepthPlanes) {
    LevelCtl c;
    ck(cudaMemcpyAsync(&c, ws->ctl.p, sizeof(LevelCtl), cudaMemcpyDeviceToHost, s), "read ctl");
    ck(cudaStreamSynchronize(s), "read ctl");
    switch (spec.W) {
#define CGP_MAT(WW) case WW: k_materialize_planes<WW><<<grid, kBlock, 0, s>>>(ws->visited.as<uint64_t>(), ws->planes.as<uint64_t>(), c.num_planes, g->V, spec.Qg, om, query_major); break;
      CGP_MAT(1) CGP_MAT(2) CGP_MAT(4) CGP_MAT(8) CGP_MAT(16)
#undef CGP_MAT
    }
  } else {
    k_copy_values<<<grid, kBlock, 0, s>>>(group_dev(ws, spec, false).values, ws->slots.as<SlotDev>(),
                                          g->V, spec.Qg, om, query_major);
  }
  ck(cudaGetLastError(), "write output");
}

}  // namespace cgp

// ======================================================================
//                                C ABI
// ======================================================================
using namespace cgp;

namespace {

// Symmetry check on a host CSR with sorted rows.
bool csr_is_symmetric(const std::vector<int64_t>& row, const int32_t* col, int64_t V) {
  for (int64_t u = 0; u < V; ++u) {
    for (int64_t e = row[u]; e < row[u + 1]; ++e) {
      int32_t v = col[e];
      const int32_t* b = col + row[v];
      const int32_t* en = col + row[v + 1];
      bool sorted = std::is_sorted(b, en);
      bool found = sorted ? std::binary_search(b, en, static_cast<int32_t>(u))
                          : std::find(b, en, static_cast<int32_t>(u)) != en;
      if (!found) return false;
    }
  }
  return true;
}

thread_local std::vector<LevelProfile> t_profiles;
thread_local std::vector<float> t_level_ms;  // per-level kernel time (profile_kernels)
thread_local cgp_kernel_profile t_kernel_profile;

}  // namespace

extern "C" {

cgp_status cgp_graph_create(const void* row_offsets, int32_t offset_bytes,
                            const int32_t* col_indices, const void* weights,
                            int32_t weight_kind, int64_t num_vertices, int64_t num_edges,
                            int32_t flags, cgp_graph** out) {
  clear_error();
  if (out == nullptr) return set_error(CGP_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (row_offsets == nullptr || (num_edges > 0 && col_indices == nullptr))
    return set_error(CGP_ERR_INVALID_ARG, "row_offsets/col_indices is NULL");
  if (offset_bytes != 4 && offset_bytes != 8)
    return set_error(CGP_ERR_INVALID_ARG, "offset_bytes must be 4 or 8");
  if (num_vertices <= 0 || num_vertices >= INT32_MAX || num_edges < 0)
    return set_error(CGP_ERR_INVALID_ARG, "vertex count must be in [1, 2^31-1)");
  if (weight_kind != CGP_WEIGHT_NONE && weight_kind != CGP_WEIGHT_U32 && weight_kind != CGP_WEIGHT_F32)
    return set_error(CGP_ERR_INVALID_ARG, "unknown weight_kind");
  if (weight_kind != CGP_WEIGHT_NONE && weights == nullptr)
    return set_error(CGP_ERR_INVALID_ARG, "weights is NULL");
  auto* g = new (std::nothrow) cgp_graph();
  if (!g) return set_error(CGP_ERR_OOM, "host allocation failed");
  try {
    GraphImpl& G = g->impl;
    ck(cudaGetDevice(&G.device), "cudaGetDevice");
    ck(cudaDeviceGetAttribute(&G.num_sms, cudaDevAttrMultiProcessorCount, G.device), "attr");
    G.V = num_vertices;
    G.E = num_edges;
    G.weight_kind = weight_kind;
    const bool on_dev = (flags & CGP_GRAPH_DEVICE_POINTERS) != 0;
    const cudaMemcpyKind kind = on_dev ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
    // host copies: 64-bit offsets and (for validation / transpose) columns
    std::vector<int64_t> hrow(num_vertices + 1);
    if (offset_bytes == 8) {
      ck(cudaMemcpy(hrow.data(), row_offsets, (num_vertices + 1) * 8, kind), "read offsets");
    } else {
      std::vector<int32_t> r32(num_vertices + 1);
      ck(cudaMemcpy(r32.data(), row_offsets, (num_vertices + 1) * 4, kind), "read offsets");
      for (int64_t i = 0; i <= num_vertices; ++i) hrow[i] = r32[i];
    }
    if (hrow[0] != 0 || hrow[num_vertices] != num_edges)
      throw ApiError{CGP_ERR_INVALID_ARG, "row_offsets must start at 0 and end at num_edges"};
    for (int64_t v = 0; v < num_vertices; ++v) {
      if (hrow[v + 1] < hrow[v]) throw ApiError{CGP_ERR_INVALID_ARG, "row_offsets not monotone"};
      G.max_degree = std::max(G.max_degree, hrow[v + 1] - hrow[v]);
      G.n_deg32 += hrow[v + 1] - hrow[v] > 32 ? 1 : 0;
    }
    std::vector<int32_t> hcol(num_edges);
    if (num_edges > 0)
      ck(cudaMemcpy(hcol.data(), col_indices, num_edges * 4, kind), "read columns");
    for (int64_t e = 0; e < num_edges; ++e)
      if (hcol[e] < 0 || hcol[e] >= num_vertices)
        throw ApiError{CGP_ERR_INVALID_ARG, "column index out of range at edge " + std::to_string(e)};
    // device offsets: 32-bit unless asked for 64 or the edge count needs it
    const bool off64 = (flags & CGP_GRAPH_OFFSETS64) != 0 || num_edges >= INT32_MAX;
    G.offset_bytes = off64 ? 8 : 4;
    G.row.ensure((num_vertices + 1) * G.offset_bytes);
    if (off64) {
      ck(cudaMemcpy(G.row.p, hrow.data(), (num_vertices + 1) * 8, cudaMemcpyHostToDevice), "upload offsets");
    } else {
      std::vector<int32_t> r32(hrow.begin(), hrow.end());
      ck(cudaMemcpy(G.row.p, r32.data(), (num_vertices + 1) * 4, cudaMemcpyHostToDevice), "upload offsets");
    }
    G.col.ensure(std::max<int64_t>(num_edges, 1) * 4);
    if (num_edges > 0)
      ck(cudaMemcpy(G.col.p, hcol.data(), num_edges * 4, cudaMemcpyHostToDevice), "upload columns");
    if (weight_kind != CGP_WEIGHT_NONE) {
      G.w.ensure(std::max<int64_t>(num_edges, 1) * 4);
      if (num_edges > 0)
        ck(cudaMemcpy(G.w.p, weights, num_edges * 4,
                      on_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice), "upload weights");
    }
    G.symmetric = (flags & CGP_GRAPH_SYMMETRIC) != 0 || csr_is_symmetric(hrow, hcol.data(), num_vertices);
    // Pull CSR.  A directed graph needs its transpose.  A symmetric one can be
    // pulled over directly, except that an SSSP gather also needs, per entry
    // (v, u), the weight of u -> v: the transpose (counting sort by
    // destination, sources ascending) gives it, and when its columns equal
    // the CSR's (sorted lists, no multi-edge mismatch) only the weights are
    // kept, or nothing when they equal w.
    std::vector<int64_t> trow;
    const bool weighted = weight_kind != CGP_WEIGHT_NONE;
    if (!G.symmetric || weighted) {
      std::vector<uint32_t> hw;
      if (weighted) {
        hw.resize(num_edges);
        if (num_edges > 0)
          ck(cudaMemcpy(hw.data(), weights, num_edges * 4, kind), "read weights");
      }
      trow.assign(num_vertices + 1, 0);
      for (int64_t e = 0; e < num_edges; ++e) trow[hcol[e] + 1]++;
      for (int64_t v = 0; v < num_vertices; ++v) trow[v + 1] += trow[v];
      std::vector<int64_t> cur(trow.begin(), trow.end() - 1);
      std::vector<int32_t> tcol(num_edges);
      std::vector<uint32_t> tw(weighted ? num_edges : 0);
      for (int64_t u = 0; u < num_vertices; ++u)
        for (int64_t e = hrow[u]; e < hrow[u + 1]; ++e) {
          const int64_t p = cur[hcol[e]]++;
          tcol[p] = static_cast<int32_t>(u);
          if (weighted) tw[p] = hw[e];
        }
      const bool aligned = G.symmetric && trow == hrow && tcol == hcol;
      if (aligned) {
        trow.clear();
        if (tw != hw) {
          G.tw.ensure(std::max<int64_t>(num_edges, 1) * 4);
          ck(cudaMemcpy(G.tw.p, tw.data(), num_edges * 4, cudaMemcpyHostToDevice), "upload t-weights");
        }
      } else {
        G.trow.ensure((num_vertices + 1) * G.offset_bytes);
        if (off64) {
          ck(cudaMemcpy(G.trow.p, trow.data(), (num_vertices + 1) * 8, cudaMemcpyHostToDevice), "upload t-offsets");
        } else {
          std::vector<int32_t> r32(trow.begin(), trow.end());
          ck(cudaMemcpy(G.trow.p, r32.data(), (num_vertices + 1) * 4, cudaMemcpyHostToDevice), "upload t-offsets");
        }
        G.tcol.ensure(std::max<int64_t>(num_edges, 1) * 4);
        if (num_edges > 0)
          ck(cudaMemcpy(G.tcol.p, tcol.data(), num_edges * 4, cudaMemcpyHostToDevice), "upload t-columns");
        if (weighted) {
          G.tw.ensure(std::max<int64_t>(num_edges, 1) * 4);
          if (num_edges > 0)
            ck(cudaMemcpy(G.tw.p, tw.data(), num_edges * 4, cudaMemcpyHostToDevice), "upload t-weights");
        }
      }
    }
    {
      std::lock_guard<std::mutex> lk(g_host_mu);
      HostCsr& hc = g_host[&G];
      hc.row = std::move(hrow);
      hc.trow = std::move(trow);
    }
    *out = g;
    return CGP_OK;
  } catch (...) {
    cgp_status st = translate_exception();
    delete g;
    return st;
  }
}

cgp_status cgp_graph_destroy(cgp_graph* g) {
  clear_error();
  if (g == nullptr) return CGP_OK;
  {
    std::lock_guard<std::mutex> lk(g_host_mu);
    g_host.erase(&g->impl);
  }
  cudaDeviceSynchronize();
  delete g;
  return CGP_OK;
}

cgp_status cgp_graph_info(const cgp_graph* g, int64_t* V, int64_t* E, int32_t* wk, int32_t* sym) {
  if (g == nullptr) return set_error(CGP_ERR_INVALID_ARG, "graph is NULL");
  if (V) *V = g->impl.V;
  if (E) *E = g->impl.E;
  if (wk) *wk = g->impl.weight_kind;
  if (sym) *sym = g->impl.symmetric ? 1 : 0;
  return CGP_OK;
}

cgp_status cgp_last_profiles(cgp_level_profile* out, int32_t cap, int32_t* count) {
  if (count == nullptr) return set_error(CGP_ERR_INVALID_ARG, "count is NULL");
  int n = static_cast<int>(t_profiles.size());
  *count = n;
  if (out != nullptr) {
    for (int i = 0; i < std::min(n, cap); ++i) {
      out[i].iteration = t_profiles[i].level;
      out[i].mode = t_profiles[i].dir;
      out[i].frontier_size = t_profiles[i].frontier;
      out[i].frontier_edges = t_profiles[i].edges;
      out[i].next_size = t_profiles[i].next;
      out[i].query_convergence_mask = t_profiles[i].active0;
      out[i].new_pairs = t_profiles[i].new_pairs;
      out[i].pull_vertices = t_profiles[i].pull_vertices;
      out[i].pull_edges = t_profiles[i].pull_edges;
      out[i].sssp_pairs = t_profiles[i].sssp_pairs;
      out[i].sssp_active = t_profiles[i].sssp_active;
      out[i].improved = t_profiles[i].improved;
      out[i].sssp_pull_vertices = t_profiles[i].spull_vertices;
      out[i].sssp_pull_edges = t_profiles[i].spull_edges;
      out[i].sssp_mode = t_profiles[i].sdir;
      out[i].kernel_ms = i < static_cast<int>(t_level_ms.size()) ? t_level_ms[i] : 0.0f;
    }
  }
  return CGP_OK;
}

cgp_status cgp_debug_fail_allocations(int64_t after) {
  g_fail_alloc_countdown.store(after < 0 ? -1 : after);
  return CGP_OK;
}

cgp_status cgp_last_kernel_profile(cgp_kernel_profile* out) {
  if (out == nullptr) return set_error(CGP_ERR_INVALID_ARG, "out is NULL");
  *out = t_kernel_profile;
  return CGP_OK;
}

cgp_status cgp_batch_run(cgp_graph* graph, const cgp_query* queries, int32_t nq,
                         const cgp_options* opts, void* out, int32_t out_layout,
                         int32_t out_on_device, cgp_stats* stats) {
  clear_error();
  if (graph == nullptr) return set_error(CGP_ERR_INVALID_ARG, "graph is NULL");
  if (queries == nullptr || nq <= 0)
    return set_error(CGP_ERR_INVALID_ARG, "query batch must be non-empty");
  if (out == nullptr) return set_error(CGP_ERR_INVALID_ARG, "out is NULL");
  if (out_layout != CGP_LAYOUT_VERTEX_MAJOR && out_layout != CGP_LAYOUT_QUERY_MAJOR)
    return set_error(CGP_ERR_INVALID_ARG, "unknown out_layout");
  cgp_options o;
  if (opts) o = *opts;
  else cgp_options_init(&o);
  if (o.max_queries > 0 && nq > o.max_queries)
    return set_error(CGP_ERR_INVALID_ARG, "query batch exceeds max_queries");
  GraphImpl* g = &graph->impl;
  for (int i = 0; i < nq; ++i) {
    const cgp_query& q = queries[i];
    if (q.kind < CGP_KIND_BFS || q.kind > CGP_KIND_KHOP)
      return set_error(CGP_ERR_INVALID_ARG, "unknown query kind at index " + std::to_string(i));
    if (q.kind != CGP_KIND_WCC && (q.source < 0 || q.source >= g->V))
      return set_error(CGP_ERR_INVALID_ARG, "query source out of range at index " + std::to_string(i));
    if (q.kind == CGP_KIND_KHOP && q.k < 0)
      return set_error(CGP_ERR_INVALID_ARG, "k-hop bound must be non-negative");
  }
  std::unique_ptr<Workspace> ws;
  std::unique_ptr<KernelTimer> kt;
  try {
    ck(cudaSetDevice(g->device), "cudaSetDevice");
    ws = g->acquire();
    if (o.profile_kernels) kt = std::make_unique<KernelTimer>();
    cudaStream_t s = o.stream ? static_cast<cudaStream_t>(o.stream) : ws->stream;
    auto wall0 = std::chrono::steady_clock::now();
    cudaEvent_t t0, t1;
    ck(cudaEventCreate(&t0), "event");
    ck(cudaEventCreate(&t1), "event");
    ck(cudaEventRecord(t0, s), "event");
    const int64_t V = g->V;
    const bool qmajor = out_layout == CGP_LAYOUT_QUERY_MAJOR;
    // output target on the device
    uint32_t* dout = static_cast<uint32_t*>(out);
    if (!out_on_device) {
      ws->stage.ensure(static_cast<size_t>(V) * nq * 4);
      dout = ws->stage.as<uint32_t>();
    }
    OutMap om;
    om.out = dout;
    om.sv = qmajor ? 1 : nq;
    om.sq = qmajor ? V : 1;
    om.qmap = nullptr;
    om.qmap_contiguous = 0;
    // WCC queries: one union-find pass, labels broadcast to every WCC column
    std::vector<int> wcc_idx, trav_idx;
    for (int i = 0; i < nq; ++i) (queries[i].kind == CGP_KIND_WCC ? wcc_idx : trav_idx).push_back(i);
    GroupRun total;
    uint64_t launches = 0;
    int groups = 0;
    int W0 = 0, depth0 = 0;
    t_profiles.clear();
    t_level_ms.clear();
    if (!wcc_idx.empty()) {
      if (kt) kt->mark(kClassWcc, s);
      ws->wcc.ensure(static_cast<size_t>(V) * 4);
      wcc_labels(g, ws->wcc.as<uint32_t>(), s);
      for (int i : wcc_idx) broadcast_labels(ws->wcc.as<uint32_t>(), V, om, i, s);
      launches += 3 + wcc_idx.size();
      if (kt) kt->mark(-1, s);
    }
    // Traversal groups of up to 64*W queries, in submission order.  A batch
    // with many BFS-like and many SSSP queries is split by kind first (each
    // kind then gets its own groups): the kinds share no state, a pure BFS
    // group keeps its depths in bit-planes, and a pure SSSP group reads no
    // BFS slots in its gathers.  Small mixed batches share one group, as in
    // the reference's hybrid batch.
    std::vector<std::vector<int>> classes;
    {
      std::vector<int> bfs_like, sssp_q;
      for (int i : trav_idx) (queries[i].kind == CGP_KIND_SSSP ? sssp_q : bfs_like).push_back(i);
      if (bfs_like.size() >= 64 && sssp_q.size() >= 64) classes = {bfs_like, sssp_q};
      else if (!trav_idx.empty()) classes = {trav_idx};
    }
    struct GroupPlan {
      const std::vector<int>* cls;
      size_t begin;
      int n;
      int W;
    };
    std::vector<GroupPlan> plan;
    for (const auto& cls : classes) {
      const int Wc = choose_words(static_cast<int>(cls.size()), o.mask_words);
      const int per_group = 64 * Wc;
      for (size_t b = 0; b < cls.size(); b += per_group) {
        const int n = static_cast<int>(std::min<size_t>(per_group, cls.size() - b));
        plan.push_back(GroupPlan{&cls, b, n, choose_words(n, o.mask_words)});
      }
    }
    const bool single = plan.size() == 1;
    // Host output: each group's result block is copied to the host on the
    // copy stream as soon as it is written, overlapping the next group's
    // traversal, when its destination is one contiguous block (query-major
    // rows, or a run of vertex-major columns as a 2D copy).
    const bool host_out = !out_on_device && !o.discard_results;
    bool copied_all = host_out;
    std::vector<char> col_copied(host_out ? nq : 0, 0);
    for (const GroupPlan& gp : plan) {
      const int n = gp.n;
      std::vector<cgp_query> gq(n);
      for (int i = 0; i < n; ++i) gq[i] = queries[(*gp.cls)[gp.begin + i]];
      GroupSpec spec = make_group(gq.data(), n, gp.W, o.depth_mode);
      // A device vertex-major output holding exactly this group's columns is
      // used directly as the working value matrix (no copy at the end).
      const bool in_place = out_on_device && !qmajor && single && wcc_idx.empty() &&
                            spec.depth_mode != kDepthPlanes;
      if (in_place) spec.external_values = dout;
      if (kt) kt->mark(kClassInit, s);
      group_prepare(g, ws.get(), spec, o, s);
      GroupRun r;
      group_enact(g, ws.get(), spec, o, s, &r, 0, kt.get());
      if (r.status != 0) throw ApiError{CGP_ERR_DEVICE, "device status " + std::to_string(r.status)};
      if (!in_place) {
        if (kt) kt->mark(kClassOutput, s);
        std::vector<int32_t> qmap(n);
        for (int i = 0; i < n; ++i) qmap[i] = (*gp.cls)[gp.begin + i];
        ws->qmap.ensure(static_cast<size_t>(n) * 4);
        ck(cudaMemcpyAsync(ws->qmap.p, qmap.data(), static_cast<size_t>(n) * 4,
                           cudaMemcpyHostToDevice, s), "upload query map");
        OutMap m = om;
        m.qmap = ws->qmap.as<int32_t>();
        m.qmap_contiguous = 1;
        for (int i = 1; i < n; ++i) m.qmap_contiguous &= qmap[i] == qmap[0] + i ? 1 : 0;
        group_write_output(g, ws.get(), spec, m, qmajor, s);
        if (kt) kt->mark(-1, s);
        if (host_out && m.qmap_contiguous && wcc_idx.empty()) {
          ck(cudaEventRecord(ws->out_ready, s), "event");
          ck(cudaStreamWaitEvent(ws->copy, ws->out_ready, 0), "wait");
          const size_t q0 = static_cast<size_t>(qmap[0]);
          char* hbase = static_cast<char*>(out);
          const char* dbase = reinterpret_cast<const char*>(dout);
          if (qmajor) {
            const size_t off = q0 * static_cast<size_t>(V) * 4;
            ck(cudaMemcpyAsync(hbase + off, dbase + off, static_cast<size_t>(n) * V * 4,
                               cudaMemcpyDeviceToHost, ws->copy), "copy out");
          } else {
            ck(cudaMemcpy2DAsync(hbase + q0 * 4, static_cast<size_t>(nq) * 4, dbase + q0 * 4,
                                 static_cast<size_t>(nq) * 4, static_cast<size_t>(n) * 4, V,
                                 cudaMemcpyDeviceToHost, ws->copy), "copy out");
          }
          for (int i = 0; i < n; ++i) col_copied[qmap[i]] = 1;
        }
      }
      launches += spec.launches;
      total.iterations = std::max(total.iterations, r.iterations);
      total.push_levels += r.push_levels;
      total.pull_levels += r.pull_levels;
      total.frontier_vertices += r.frontier_vertices;
      total.frontier_edges += r.frontier_edges;
      total.counters.new_pairs += r.counters.new_pairs;
      total.counters.pull_vertices += r.counters.pull_vertices;
      total.counters.pull_edges += r.counters.pull_edges;
      total.counters.sssp_pairs += r.counters.sssp_pairs;
      total.counters.sssp_active += r.counters.sssp_active;
      total.counters.improved += r.counters.improved;
      total.counters.spull_vertices += r.counters.spull_vertices;
      total.counters.spull_edges += r.counters.spull_edges;
      if (groups == 0) {
        W0 = spec.W;
        depth0 = spec.depth_mode;
        t_profiles = r.profiles;
        t_level_ms = r.level_ms;
      }
      ++groups;
    }
    ck(cudaEventRecord(t1, s), "event");
    for (char c : col_copied) copied_all = copied_all && c;
    if (host_out && !copied_all)
      ck(cudaMemcpyAsync(out, dout, static_cast<size_t>(V) * nq * 4, cudaMemcpyDeviceToHost, s),
         "copy out");
    ck(cudaStreamSynchronize(s), "batch");
    if (host_out) ck(cudaStreamSynchronize(ws->copy), "copy out");
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (kt) {
      kt->flush();
      std::memset(&t_kernel_profile, 0, sizeof(t_kernel_profile));
      for (int c = 0; c < kNumClasses; ++c) {
        t_kernel_profile.ms[c] = kt->ms[c];
        t_kernel_profile.launches[c] = kt->count[c];
      }
    }
    if (stats) {
      std::memset(stats, 0, sizeof(*stats));
      stats->iterations = total.iterations;
      stats->push_levels = total.push_levels;
      stats->pull_levels = total.pull_levels;
      stats->groups = groups;
      stats->gpu_time_ms = ms;
      stats->wall_time_ms = std::chrono::duration<float, std::milli>(
                                std::chrono::steady_clock::now() - wall0).count();
      stats->frontier_vertices = total.frontier_vertices;
      stats->frontier_edges = total.frontier_edges;
      stats->mask_words = W0;
      stats->depth_mode = depth0 == kDepthPlanes ? CGP_DEPTH_PLANES : CGP_DEPTH_DIRECT;
      stats->kernel_launches = launches;
      stats->new_pairs = total.counters.new_pairs;
      stats->pull_vertices = total.counters.pull_vertices;
      stats->pull_edges = total.counters.pull_edges;
      stats->sssp_pairs = total.counters.sssp_pairs;
      stats->sssp_active = total.counters.sssp_active;
      stats->improved = total.counters.improved;
      stats->sssp_pull_vertices = total.counters.spull_vertices;
      stats->sssp_pull_edges = total.counters.spull_edges;
    }
    g->release(std::move(ws));
    return CGP_OK;
  } catch (...) {
    cgp_status st = translate_exception();
    if (ws) {
      cudaStreamSynchronize(ws->stream);
      g->release(std::move(ws));
    }
    return st;
  }
}

}  // extern "C"
