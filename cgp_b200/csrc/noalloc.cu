// Batched BFS for callers that must not allocate device memory.
//
// Some callers cannot call cudaMalloc at the point where they need a
// traversal: code that runs while another component owns the whole device
// memory pool (a framework allocator that reserved the free HBM up front, so
// a cudaMalloc would fail or fragment its pool), latency-critical request
// paths where a cudaMalloc/cudaFree would synchronise the device and stall
// every stream, and embedded or plug-in hosts that only hand over the buffers
// they own.  cgp_bfs_batch_noalloc serves them: it takes the CSR, the sources
// and the output buffer from the caller and keeps its working state (query
// masks, frontier lists, control block) in one fixed device array that is
// part of the loaded library.  It calls no cudaMalloc, cudaFree or other
// allocating routine, creates no events, graphs or streams, and launches the
// same level kernels as cgp_batch_run (push + pull, direct depth writes).
//
// The array is CGP_NOALLOC_SCRATCH_BYTES large (see cgp_b200.h) and lives on
// every GPU that loads the library until the process exits.  All calls on a
// device share it and it keeps the previous call's contents: each call clears
// what must start at zero before using it, and two calls that overlap on the
// GPU (different streams or threads on the same device) race on it, so such
// calls must be serialised by the caller.
#include <cstring>

#include "engine.h"
#include "kernels.cuh"

namespace cgp {
namespace {

using namespace dev;

constexpr size_t kScratchBytes = CGP_NOALLOC_SCRATCH_BYTES;

// The fixed working area.  In host code its name is only a host-side handle;
// the device address comes from cudaGetSymbolAddress (scratch_address below).
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of the scratch array on the current device.  Looked up on
// every call (the lookup is cheap), so that an address cached before a
// cudaDeviceReset or a re-created primary context is never handed to a kernel.
cgp_status scratch_address(void** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr) {
    cudaGetLastError();
    return set_error(CGP_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") +
                                       cudaGetErrorString(e));
  }
  *out = p;
  return CGP_OK;
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Marks *flag when the caller's CSR is malformed: row offsets not starting at
// 0, not ending at E or decreasing, or a column outside [0, V).  Runs before
// any traversal so that no kernel indexes the scratch array out of range.
template <typename OT>
__global__ void k_check_csr(const void* row, const int32_t* col, int64_t V, int64_t E,
                            uint32_t* flag) {
  const OT* r = static_cast<const OT*>(row);
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t0 == 0 && (r[0] != 0 || static_cast<int64_t>(r[V]) != E)) *flag = 1u;
  for (int64_t v = t0; v < V; v += stride)
    if (r[v + 1] < r[v]) *flag = 1u;
  for (int64_t e = t0; e < E; e += stride)
    if (col[e] < 0 || col[e] >= V) *flag = 1u;
}

// Byte size of the working state for V vertices and W mask words.
size_t scratch_need(int64_t V, int W) {
  size_t b = align256(sizeof(LevelCtl)) + align256(sizeof(SlotDev) * kMaxWords * 64);
  b += 3 * align256(static_cast<size_t>(V) * W * 8);  // visited, two frontier buffers
  b += 3 * align256(static_cast<size_t>(V) * 4);      // two lists, stamps
  return b;
}

template <int W, typename OT>
void run_levels(const GroupDev& g, const DevGraph& G, bool pull, int64_t V, int nq,
                uint32_t* out, cudaStream_t s) {
  const int blocks = 148 * 4;
  k_fill_values<<<blocks, kBlock, 0, s>>>(out, g.slots, nq, V, 0u, 0u);
  k_seed<W, OT><<<1, kBlock, 0, s>>>(g, G);
  // One level per iteration until the control block reports convergence;
  // the flag is read back every 4 levels.
  for (int chunk = 0;; ++chunk) {
    for (int i = 0; i < 4; ++i) {
      k_clear_next<W><<<blocks, kBlock, 0, s>>>(g, G.E);
      k_bfs_push<W, OT, kDepthDirect><<<blocks, kBlock, 0, s>>>(g, G);
      if (pull) k_bfs_pull<W, OT, kDepthDirect><<<blocks, kBlock, 0, s>>>(g, G);
      k_level_end<W><<<1, 32, 0, s>>>(g);
    }
    int32_t done = 0;
    ck(cudaMemcpyAsync(&done, reinterpret_cast<char*>(g.ctl) + offsetof(LevelCtl, done),
                       sizeof(done), cudaMemcpyDeviceToHost, s), "read done flag");
    ck(cudaStreamSynchronize(s), "level loop");
    if (done != 0) break;
  }
}

// The status word the level kernels raise (0 = clean), read after the loop.
uint32_t read_status(const GroupDev& g, cudaStream_t s) {
  uint32_t st = 0;
  ck(cudaMemcpyAsync(&st, reinterpret_cast<char*>(g.ctl) + offsetof(LevelCtl, status), sizeof(st),
                     cudaMemcpyDeviceToHost, s), "read status");
  ck(cudaStreamSynchronize(s), "read status");
  return st;
}

template <int W>
void run_w(const GroupDev& g, const DevGraph& G, bool pull, int64_t V, int nq, uint32_t* out,
           int offset_bytes, cudaStream_t s) {
  if (offset_bytes == 8) run_levels<W, int64_t>(g, G, pull, V, nq, out, s);
  else run_levels<W, int32_t>(g, G, pull, V, nq, out, s);
}

}  // namespace
}  // namespace cgp

using namespace cgp;
using namespace cgp::dev;

extern "C" cgp_status cgp_bfs_batch_noalloc(const void* row_offsets, int32_t offset_bytes,
                                           const int32_t* col_indices, int64_t num_vertices,
                                           int64_t num_edges, const int32_t* sources,
                                           int32_t nq, int32_t symmetric, int32_t* out,
                                           void* stream) {
  clear_error();
  if (row_offsets == nullptr || col_indices == nullptr || sources == nullptr || out == nullptr)
    return set_error(CGP_ERR_INVALID_ARG, "NULL argument");
  if (offset_bytes != 4 && offset_bytes != 8)
    return set_error(CGP_ERR_INVALID_ARG, "offset_bytes must be 4 or 8");
  if (nq <= 0 || nq > CGP_NOALLOC_MAX_QUERIES)
    return set_error(CGP_ERR_INVALID_ARG, "nq must be in [1, 256]");
  if (num_vertices <= 0 || num_vertices >= INT32_MAX || num_edges < 0)
    return set_error(CGP_ERR_INVALID_ARG, "bad graph size");
  for (int i = 0; i < nq; ++i)
    if (sources[i] < 0 || sources[i] >= num_vertices)
      return set_error(CGP_ERR_INVALID_ARG, "query source out of range at index " + std::to_string(i));
  const int W = choose_words(nq, 0);
  const size_t need = scratch_need(num_vertices, W);
  if (need > kScratchBytes)
    return set_error(CGP_ERR_INVALID_ARG,
                     "graph too large for the fixed scratch array: needs " + std::to_string(need) +
                         " bytes, the maximum is " + std::to_string(kScratchBytes) +
                         " (about 17 KiB plus 36, 60 or 108 bytes per vertex for up to 64, "
                         "128 or 256 queries)");
  try {
    void* base = nullptr;
    cgp_status st = scratch_address(&base);
    if (st != CGP_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t V = num_vertices;
    // carve the scratch array
    char* p = static_cast<char*>(base);
    GroupDev g{};
    g.ctl = reinterpret_cast<LevelCtl*>(p);
    p += align256(sizeof(LevelCtl));
    g.slots = reinterpret_cast<const SlotDev*>(p);
    SlotDev* slots_dev = reinterpret_cast<SlotDev*>(p);
    p += align256(sizeof(SlotDev) * kMaxWords * 64);
    const size_t mask_bytes = static_cast<size_t>(V) * W * 8;
    g.visited = reinterpret_cast<uint64_t*>(p);
    p += align256(mask_bytes);
    g.fbuf0 = reinterpret_cast<uint64_t*>(p);
    p += align256(mask_bytes);
    g.fbuf1 = reinterpret_cast<uint64_t*>(p);
    p += align256(mask_bytes);
    g.list0 = reinterpret_cast<int32_t*>(p);
    p += align256(static_cast<size_t>(V) * 4);
    g.list1 = reinterpret_cast<int32_t*>(p);
    p += align256(static_cast<size_t>(V) * 4);
    g.stamp = reinterpret_cast<int32_t*>(p);
    g.planes = nullptr;
    g.values = reinterpret_cast<uint32_t*>(out);
    g.hacc = nullptr;
    g.fsum = nullptr;
    g.dense_list = nullptr;
    g.prof = nullptr;
    g.Qg = nq;
    // what must start at zero (or -1) every call
    ck(cudaMemsetAsync(g.visited, 0, mask_bytes, s), "clear visited");
    ck(cudaMemsetAsync(g.fbuf0, 0, mask_bytes, s), "clear frontier");
    ck(cudaMemsetAsync(g.fbuf1, 0, mask_bytes, s), "clear next frontier");
    ck(cudaMemsetAsync(g.stamp, 0xff, static_cast<size_t>(V) * 4, s), "clear stamps");
    SlotDev hs[CGP_NOALLOC_MAX_QUERIES];
    for (int i = 0; i < nq; ++i) hs[i] = SlotDev{CGP_KIND_BFS, sources[i], 0, 0};
    ck(cudaMemcpyAsync(slots_dev, hs, sizeof(SlotDev) * nq, cudaMemcpyHostToDevice, s), "slots");
    LevelCtl c;
    std::memset(&c, 0, sizeof(c));
    for (int q = 0; q < nq; ++q) c.bfs_bits[q >> 6] |= 1ULL << (q & 63);
    for (int i = 0; i < kMaxW; ++i) c.expand[i] = ~0ULL;
    c.forced_dir = -1;
    c.halt_level = -1;
    c.mode = symmetric ? CGP_MODE_HYBRID : CGP_MODE_PUSH;
    c.pull_vertex_threshold = static_cast<unsigned long long>(0.15 * static_cast<double>(V)) + 1;
    c.pull_edge_threshold = static_cast<unsigned long long>(0.20 * static_cast<double>(num_edges)) + 1;
    ck(cudaMemcpyAsync(g.ctl, &c, sizeof(c), cudaMemcpyHostToDevice, s), "control block");
    uint32_t* flag = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(g.ctl) + offsetof(LevelCtl, status));
    if (offset_bytes == 8)
      k_check_csr<int64_t><<<148 * 4, kBlock, 0, s>>>(row_offsets, col_indices, V, num_edges, flag);
    else
      k_check_csr<int32_t><<<148 * 4, kBlock, 0, s>>>(row_offsets, col_indices, V, num_edges, flag);
    uint32_t bad = 0;
    ck(cudaMemcpyAsync(&bad, flag, sizeof(bad), cudaMemcpyDeviceToHost, s), "read csr check");
    ck(cudaStreamSynchronize(s), "csr check");
    if (bad != 0) return set_error(CGP_ERR_INVALID_ARG, "malformed CSR (offsets or column range)");
    DevGraph G;
    std::memset(&G, 0, sizeof(G));
    G.row = row_offsets;
    G.col = col_indices;
    G.prow = row_offsets;
    G.pcol = col_indices;
    G.V = V;
    G.E = num_edges;
    G.heavy_degree = INT64_MAX;  // no heavy table: large lists go to whole warps
    const bool pull = symmetric != 0;
    switch (W) {
      case 1: run_w<1>(g, G, pull, V, nq, g.values, offset_bytes, s); break;
      case 2: run_w<2>(g, G, pull, V, nq, g.values, offset_bytes, s); break;
      default: run_w<4>(g, G, pull, V, nq, g.values, offset_bytes, s); break;
    }
    ck(cudaGetLastError(), "noalloc launch");
    ck(cudaStreamSynchronize(s), "noalloc");
    const uint32_t dstatus = read_status(g, s);
    if (dstatus != 0)
      return set_error(CGP_ERR_DEVICE, "device status " + std::to_string(dstatus));
    return CGP_OK;
  } catch (...) {
    return translate_exception();
  }
}
