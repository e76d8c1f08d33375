// Host-side engine structures shared by the batch runner, the enactor
// surface and the serving loop.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "cgp_b200_internal.h"
#include "device_types.cuh"

namespace cgp {

// Throws CudaError; caught at the C boundary and turned into CGP_ERR_CUDA/OOM.
struct CudaError {
  cudaError_t code;
  std::string where;
};
struct ApiError {
  cgp_status code;
  std::string msg;
};

inline void ck(cudaError_t e, const char* where) {
  if (e != cudaSuccess) throw CudaError{e, where};
}

// One device allocation that only grows.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DevBuf();
  // Returns true when a new block was allocated (pointers changed).
  bool ensure(size_t need);
  template <typename T>
  T* as() const { return static_cast<T*>(p); }
};

struct HeavyTable {
  DevBuf vertices;     // int32 [n]
  DevBuf chunk_start;  // int64 [n + 1]
  DevBuf chunk_h;      // int32 [chunks] table index of each chunk's vertex
  DevBuf chunk_beg;    // int64 [chunks] first edge of each chunk
  DevBuf chunk_end;    // int64 [chunks] one past its last edge
  int32_t n = 0;
  int64_t chunks = 0;
};

// Heavy tables of the traversal CSR and of the pull CSR for one threshold.
// Chunks of light vertices of the pull CSR (in-degree in [1, threshold]),
// taken in order of decreasing in-degree: runs with at most kLightChunkVerts
// vertices and kLightChunkEdges in-edges (a single larger vertex forms its own
// chunk).
struct LightChunks {
  DevBuf vertices;     // int32 [n] light vertices, largest in-degree first
  DevBuf chunk_start;  // int32 [chunks + 1] positions in `vertices`
  DevBuf beg;          // int64 [n] first in-edge of each vertex in the pull CSR
  DevBuf pre;          // int32 [n] in-edges of the chunk up to and including the vertex
  int32_t n = 0;
  int32_t chunks = 0;
  int32_t n_mid = 0;   // the first n_mid have in-degree > 32
};

struct HeavyPair {
  HeavyTable heavy, pheavy;
  LightChunks plight;
};

// Degree above which adjacency lists are split into CTA work items.
inline int64_t heavy_threshold(const cgp_options& o) {
  if (o.heavy_degree > 0) return o.heavy_degree < (1 << 20) ? o.heavy_degree : (1 << 20);
  return 2048;
}

using LevelCtl = dev::LevelCtl;

struct CachedGraph {
  cudaGraphExec_t exec;
  int launches;  // kernels per replay
};

// Kernel classes timed by KernelTimer.
enum KernelClass {
  kClassClear = 0,
  kClassBfsPush,
  kClassBfsPull,
  kClassSsspPush,   // SSSP tile kernel (few active queries per vertex)
  kClassLevelEnd,
  kClassInit,
  kClassOutput,
  kClassWcc,
  kClassSsspDense,  // SSSP dense kernel (many active queries per vertex)
  kClassSsspHeavy,  // SSSP heavy-vertex chunks
  kClassSsspPull,   // SSSP gather levels (light and heavy vertices)
  kNumClasses
};

// CUDA-event timing per kernel class on the launching stream.  mark(c)
// closes the open interval and opens one of class c (c < 0: close only).
struct KernelTimer {
  static constexpr int kMaxMarks = 32;
  cudaEvent_t ev[kMaxMarks] = {};
  int cls[kMaxMarks] = {};
  int n = 0;
  double ms[kNumClasses] = {};
  long long count[kNumClasses] = {};
  KernelTimer();
  ~KernelTimer();
  void mark(int c, cudaStream_t s);
  void flush();  // waits for the recorded events and accumulates
};

// Everything that belongs to one traversal group's device state.  Reused
// across runs; `generation` changes whenever an allocation moves, which
// invalidates captured CUDA graphs.
struct Workspace {
  int device = 0;
  DevBuf visited, fbuf0, fbuf1, list0, list1, stamp, planes, values, hacc, dense, hq_vertex, hq_start;
  DevBuf fsum;  // frontier summary words (uint64 per vertex)
  DevBuf ctl, prof, slots, stage, wcc, qmap;
  LevelCtl* hctl = nullptr;  // pinned, 2 snapshots
  dev::SlotDev* hslots = nullptr;  // pinned, kMaxWords*64 entries
  cudaStream_t stream = nullptr;
  cudaStream_t capture = nullptr;
  cudaStream_t copy = nullptr;     // device->host result copies overlapping later groups
  cudaEvent_t out_ready = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  uint64_t generation = 1;
  std::map<std::tuple<int, int, int, int, int, int, int, int, uint64_t, uint64_t>, CachedGraph>
      graphs;
  Workspace(int dev);
  ~Workspace();
  void clear_graphs();
};

struct GraphImpl {
  int device = 0;
  int num_sms = 148;
  int64_t V = 0, E = 0;
  int64_t max_degree = 0;  // largest out-degree of the traversal CSR
  int64_t n_deg32 = 0;     // vertices of out-degree > 32 (heavy-queue capacity)
  int offset_bytes = 4;
  int weight_kind = CGP_WEIGHT_NONE;
  bool symmetric = false;
  DevBuf row, col, w;      // traversal CSR
  DevBuf trow, tcol;       // in-edge CSR for pull when the CSR itself cannot serve
  DevBuf tw;               // weights aligned with the pull CSR when they differ from w
  std::mutex mu;
  std::mutex heavy_mu;
  std::map<int64_t, std::unique_ptr<HeavyPair>> heavy_cache;  // built once per threshold
  std::vector<std::unique_ptr<Workspace>> pool;  // idle workspaces

  // Pull CSR: the CSR itself when it lists every vertex's in-edges in the
  // order of the transpose (symmetric, sorted), else the stored transpose.
  const void* pull_row() const { return trow.p ? trow.p : (symmetric ? row.p : nullptr); }
  const int32_t* pull_col() const {
    return trow.p ? tcol.as<int32_t>() : (symmetric ? col.as<int32_t>() : nullptr);
  }
  // pw[e] = weight of the edge pull_col()[e] -> v (the reverse edge's weight).
  const void* pull_w() const { return tw.p ? tw.p : w.p; }
  // SSSP gather levels need the pull CSR (and its weights on weighted graphs).
  bool can_gather() const { return pull_row() != nullptr; }
  // Heavy tables for threshold h (built on first use, then kept).
  const HeavyPair& heavy_for(int64_t h);
  dev::DevGraph dev_graph(int64_t h);
  std::unique_ptr<Workspace> acquire();
  void release(std::unique_ptr<Workspace> ws);
};

// A traversal group: up to 64*W slots sharing one set of vertex masks.
struct GroupSpec {
  int W = 1;
  int Qg = 0;
  std::vector<dev::SlotDev> slots;
  int depth_mode = dev::kDepthDirect;
  bool has_bfs = false;
  bool has_sssp = false;
  uint32_t* external_values = nullptr;  // caller's device buffer used as working values
  uint32_t uniform_inf = 0;             // nonzero: fill every value with it (serving)
  bool serving = false;                 // the group belongs to a serving loop
  uint64_t launches = 0;                // kernels enqueued for this group
};

struct GroupRun {
  int32_t iterations = 0;
  int32_t push_levels = 0;
  int32_t pull_levels = 0;
  uint64_t frontier_vertices = 0;
  uint64_t frontier_edges = 0;
  uint32_t status = 0;
  dev::LevelCounters counters{};
  std::vector<dev::LevelProfile> profiles;
  std::vector<float> level_ms;  // kernel time per level when kernel classes are timed
};

// Engine entry points (engine.cu).
GroupSpec make_group(const cgp_query* q, int n, int W, int depth_mode);
void group_prepare(GraphImpl* g, Workspace* ws, GroupSpec& spec, const cgp_options& o,
                   cudaStream_t s);
// Runs levels until convergence (done != 0) or, with max_levels > 0, that
// many levels.  With a KernelTimer, levels run one at a time without graphs.
void group_enact(GraphImpl* g, Workspace* ws, GroupSpec& spec, const cgp_options& o,
                 cudaStream_t s, GroupRun* out, int max_levels, KernelTimer* kt = nullptr);
// Enqueues `levels` levels on stream s without waiting for them (the serving
// loop overlaps several groups this way).
void group_enqueue_levels(GraphImpl* g, Workspace* ws, GroupSpec& spec, const cgp_options& o,
                          cudaStream_t s, int levels);
void group_write_output(GraphImpl* g, Workspace* ws, GroupSpec& spec,
                        dev::OutMap om, int query_major, cudaStream_t s);
int choose_words(int n, int requested);
int64_t group_state_bytes(const GraphImpl* g, int W, int Qg, int depth_mode);
// WCC: minimum vertex id of each weak component into `labels` (device).
void wcc_labels(GraphImpl* g, uint32_t* labels, cudaStream_t s);
// Writes labels[v] into global column `col` of the output mapping.
void broadcast_labels(const uint32_t* labels, int64_t V, dev::OutMap om, int col,
                      cudaStream_t s);

cgp_status translate_exception();

}  // namespace cgp

struct cgp_graph {
  cgp::GraphImpl impl;
};
