// Device code of the multi-query traversal engine (sm_100a).
//
// One traversal group holds up to 64*W queries; every vertex carries W 64-bit
// mask words.  Per level the host-free control block (LevelCtl) decides the
// direction on the device, so a whole chunk of levels can be captured in one
// CUDA graph and replayed without host synchronisation.
//
// Reference correspondence (paths relative to the reference project root):
//   push  : expand_shared_node_{,warp_}kernel, frontier_engine.hxx:678-943,
//           expand_shared_node_{,warp_}hybrid_kernel, hybrid_engine.hxx:132-330
//   pull  : fused_ge_bfs_pull_*, frontier_engine.hxx:1561-1740 (bottom-up BFS)
//   next-frontier marking : mark_next_shared_frontier[_with_signal],
//           frontier_engine.hxx:117-173 (here warp-aggregated)
//   min relaxation : apply_min_reduce, reduce_ops.hxx:40-56 (here a single
//           atomicMin on the ordered uint32 image of the value)
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "device_types.cuh"

namespace cgp {
namespace dev {

// ------------------------------------------------------------------ utils
template <int W>
__device__ __forceinline__ void load_mask(const uint64_t* p, uint64_t (&m)[W]) {
  if constexpr (W % 2 == 0) {
#pragma unroll
    for (int i = 0; i < W; i += 2) {
      ulonglong2 x = *reinterpret_cast<const ulonglong2*>(p + i);
      m[i] = x.x;
      m[i + 1] = x.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) m[i] = p[i];
  }
}

// Asks L2 to fetch the line holding p (no register is written, nothing waits).
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

template <int W>
__device__ __forceinline__ void store_mask(uint64_t* p, const uint64_t (&m)[W]) {
  if constexpr (W % 2 == 0) {
#pragma unroll
    for (int i = 0; i < W; i += 2) {
      *reinterpret_cast<ulonglong2*>(p + i) = make_ulonglong2(m[i], m[i + 1]);
    }
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) p[i] = m[i];
  }
}

template <int W>
__device__ __forceinline__ bool mask_any(const uint64_t (&m)[W]) {
  uint64_t a = 0;
#pragma unroll
  for (int i = 0; i < W; ++i) a |= m[i];
  return a != 0;
}

__device__ __forceinline__ uint64_t atomic_or64(uint64_t* p, uint64_t v) {
  return static_cast<uint64_t>(atomicOr(reinterpret_cast<unsigned long long*>(p),
                                        static_cast<unsigned long long>(v)));
}

// All 32 lanes call.  Lanes with `pred` append `v` to `list` (one atomicAdd
// per warp) and add `deg` to the edge counter.
__device__ __forceinline__ void warp_append(bool pred, int32_t v, uint64_t deg,
                                            int32_t* list,
                                            unsigned long long* count,
                                            unsigned long long* edges, int lane) {
  unsigned m = __ballot_sync(kFull, pred);
  if (m == 0) return;
  unsigned long long d = pred ? deg : 0ULL;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(kFull, d, o);
  int leader = __ffs(m) - 1;
  unsigned long long base = 0;
  if (lane == leader) {
    base = atomicAdd(count, static_cast<unsigned long long>(__popc(m)));
    atomicAdd(edges, d);
  }
  base = __shfl_sync(kFull, base, leader);
  if (pred) list[base + __popc(m & ((1u << lane) - 1u))] = v;
}

// Warp-sums `x` and lane 0 adds it to *dst (all lanes call).
__device__ __forceinline__ void warp_add(unsigned long long x, unsigned long long* dst, int lane) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  if (lane == 0 && x) atomicAdd(dst, x);
}

template <int W>
__device__ __forceinline__ void warp_or_reduce(uint64_t (&m)[W]) {
  // two redux.sync per word (32-bit halves) instead of a 5-step shuffle tree
#pragma unroll
  for (int i = 0; i < W; ++i) {
    const unsigned lo = __reduce_or_sync(kFull, static_cast<unsigned>(m[i]));
    const unsigned hi = __reduce_or_sync(kFull, static_cast<unsigned>(m[i] >> 32));
    m[i] = (static_cast<uint64_t>(hi) << 32) | lo;
  }
}

// ORs each warp's union into ctl->active[par] (lane 0, nonzero words only).
template <int W>
__device__ __forceinline__ void flush_union(uint64_t (&uni)[W], uint64_t* dst,
                                            int lane) {
  warp_or_reduce<W>(uni);
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < W; ++i)
      if (uni[i]) atomic_or64(dst + i, uni[i]);
  }
}

// Position of the j-th (0-based) set bit of a 64-bit word, by halving with
// population counts.
__device__ __forceinline__ int select_bit64(uint64_t x, int j) {
  int pos = 0;
  int c = __popc(static_cast<unsigned>(x));
  if (j >= c) {
    j -= c;
    x >>= 32;
    pos += 32;
  }
  unsigned w = static_cast<unsigned>(x);
  c = __popc(w & 0xffffu);
  if (j >= c) { j -= c; w >>= 16; pos += 16; }
  c = __popc(w & 0xffu);
  if (j >= c) { j -= c; w >>= 8; pos += 8; }
  c = __popc(w & 0xfu);
  if (j >= c) { j -= c; w >>= 4; pos += 4; }
  c = __popc(w & 0x3u);
  if (j >= c) { j -= c; w >>= 2; pos += 2; }
  if (j >= static_cast<int>(w & 1u)) pos += 1;
  return pos;
}

// j-th (0-based) set bit of a W-word mask.
template <int W>
__device__ __forceinline__ int jth_set_bit(const uint64_t* bits, int j) {
#pragma unroll
  for (int i = 0; i < W; ++i) {
    const int c = __popcll(bits[i]);
    if (j < c) return i * 64 + select_bit64(bits[i], j);
    j -= c;
  }
  return -1;
}

// Bit c: 32-slot chunk c of the mask has a bit set.
template <int W>
__device__ __forceinline__ uint32_t chunk_bits(const uint64_t (&m)[W]) {
  uint32_t c = 0;
#pragma unroll
  for (int i = 0; i < W; ++i) {
    c |= (static_cast<uint32_t>(m[i]) != 0u ? 1u : 0u) << (2 * i);
    c |= (static_cast<uint32_t>(m[i] >> 32) != 0u ? 1u : 0u) << (2 * i + 1);
  }
  return c;
}

// Frontier summary of vertex u at `level`: its 32-slot chunks with a frontier
// bit, when the summary was written for this level (a stale word reads as
// "no chunk").  Only ever used to skip mask and row loads: a vertex of the
// current frontier always has its word, so no frontier bit is missed.
__device__ __forceinline__ uint32_t summary_chunks(const uint64_t* fsum, int level, int32_t u) {
  const uint64_t x = fsum[u];
  return (x >> 32) == static_cast<uint64_t>(level + 1) ? static_cast<uint32_t>(x) : 0u;
}

// Pointers of the current level.
struct LevelView {
  int level;
  int par;
  const int32_t* list;
  int32_t* nlist;
  const uint64_t* fcur;
  uint64_t* fnext;
  unsigned long long* ncount;
  unsigned long long* nedges;
  uint64_t* nactive;
};

__device__ __forceinline__ LevelView level_view(const GroupDev& g) {
  LevelView lv;
  lv.level = g.ctl->level;
  lv.par = lv.level & 1;
  lv.list = lv.par ? g.list1 : g.list0;
  lv.nlist = lv.par ? g.list0 : g.list1;
  lv.fcur = lv.par ? g.fbuf1 : g.fbuf0;
  lv.fnext = lv.par ? g.fbuf0 : g.fbuf1;
  lv.ncount = &g.ctl->count[lv.par ^ 1];
  lv.nedges = &g.ctl->edges[lv.par ^ 1];
  lv.nactive = g.ctl->active[lv.par ^ 1];
  return lv;
}

// Frontier vertices that a push level's tile kernels expand themselves: out-
// degree at most the returned limit.  Larger lists go to the heavy queue as
// kHeavyChunk-edge CTA work items: lists above heavy_degree always, and every
// list above 32 edges when the frontier is small (<= kSmallFrontier vertices,
// e.g. the sources' level) or skewed (more than 64 out-edges per vertex on
// average, e.g. the hubs reached by the sources): there a tile of 32 such
// vertices would be one warp's serial work while most warps of the grid have
// nothing to do.  (The heavy queue holds every vertex of out-degree > 32.)
constexpr unsigned long long kSmallFrontier = 4096;

__device__ __forceinline__ int64_t push_light_limit(const GroupDev& g, const DevGraph& G,
                                                    unsigned long long count,
                                                    unsigned long long edges) {
  const bool spread = count <= kSmallFrontier || edges > 64ULL * count;
  return (g.hq_vertex != nullptr && spread && G.heavy_degree > 32) ? 32 : G.heavy_degree;
}

// ------------------------------------------------------- depth recording
// Records depth `depth_abs` (level + 1) for the newly visited bits `nw` of
// vertex n: direct mode writes values[n][q] = depth_abs - base[q]; planes
// mode ORs the bits into the planes of depth_abs's set bits.
template <int W, int DEPTH>
__device__ __forceinline__ void record_depth(const GroupDev& g, int64_t V,
                                            int32_t n, const uint64_t (&nw)[W],
                                            int depth_abs, bool exclusive) {
  if constexpr (DEPTH == kDepthPlanes) {
    const int K = g.ctl->num_planes;
    for (int b = 0; b < K; ++b) {
      if (((depth_abs >> b) & 1) == 0) continue;
      uint64_t* p = g.planes + static_cast<size_t>(b) * static_cast<size_t>(V) * W +
                    static_cast<size_t>(n) * W;
#pragma unroll
      for (int i = 0; i < W; ++i) {
        if (!nw[i]) continue;
        if (exclusive) p[i] |= nw[i];
        else atomic_or64(p + i, nw[i]);
      }
    }
  } else if constexpr (DEPTH == kDepthDirect) {
    uint32_t* row = g.values + static_cast<size_t>(n) * static_cast<size_t>(g.Qg);
#pragma unroll
    for (int i = 0; i < W; ++i) {
      uint64_t b = nw[i];
      while (b) {
        int q = i * 64 + __ffsll(static_cast<long long>(b)) - 1;
        b &= b - 1;
        row[q] = static_cast<uint32_t>(depth_abs - g.slots[q].base);
      }
    }
  }
}

// --------------------------------------------------------------- BFS push
// One edge u->n of a push level for the visited-mask bits f of u.
template <int W, int DEPTH>
__device__ __forceinline__ bool bfs_visit(const GroupDev& g, int64_t V,
                                          const LevelView& lv, int32_t n,
                                          const uint64_t (&f)[W],
                                          uint64_t (&uni)[W],
                                          unsigned long long& pairs) {
  uint64_t* vis = g.visited + static_cast<size_t>(n) * W;
  uint64_t cur[W];
  load_mask<W>(vis, cur);
  uint64_t d[W];
  uint64_t any = 0;
#pragma unroll
  for (int i = 0; i < W; ++i) {
    d[i] = f[i] & ~cur[i];
    any |= d[i];
  }
  if (!any) return false;
  uint64_t nw[W];
  uint64_t anyn = 0;
#pragma unroll
  for (int i = 0; i < W; ++i) {
    nw[i] = 0;
    if (d[i]) {
      uint64_t old = atomic_or64(vis + i, d[i]);
      nw[i] = d[i] & ~old;
      anyn |= nw[i];
    }
  }
  if (!anyn) return false;
  uint64_t* fn = lv.fnext + static_cast<size_t>(n) * W;
#pragma unroll
  for (int i = 0; i < W; ++i) {
    if (nw[i]) {
      atomic_or64(fn + i, nw[i]);
      uni[i] |= nw[i];
      pairs += __popcll(nw[i]);
    }
  }
  record_depth<W, DEPTH>(g, V, n, nw, lv.level + 1, false);
  return atomicMax(g.stamp + n, lv.level + 1) < lv.level + 1;
}

template <typename OT>
__device__ __forceinline__ uint64_t degree_of(const void* row, int32_t v) {
  return static_cast<uint64_t>(row_at<OT>(row, v + 1) - row_at<OT>(row, v));
}

// Appends the n vertices buffered in lanes 0..n-1 to the next frontier list
// with one reservation, adding their out-degrees to the edge counter (all
// lanes call).
template <typename OT>
__device__ __forceinline__ void flush_appends(int32_t v, int n, const DevGraph& G,
                                              const LevelView& lv, int lane) {
  unsigned long long e = lane < n ? degree_of<OT>(G.row, v) : 0ULL;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(kFull, e, o);
  unsigned long long base = 0;
  if (lane == 0) {
    base = atomicAdd(lv.ncount, static_cast<unsigned long long>(n));
    atomicAdd(lv.nedges, e);
  }
  base = __shfl_sync(kFull, base, 0);
  if (lane < n) lv.nlist[base + lane] = v;
}

// Per-warp buffer of vertices to append to the next frontier: lane i holds
// the i-th, and a reservation on the list's shared counters is made once per
// 32 vertices instead of once per step (those two counters are the most
// contended words of a level).  All lanes call add() and flush().
struct WarpAppender {
  int32_t v = 0;  // lane i: pending vertex i
  int n = 0;      // pending count (uniform)

  template <typename OT>
  __device__ __forceinline__ void add(bool pred, int32_t x, const DevGraph& G,
                                      const LevelView& lv, int lane) {
    const unsigned m = __ballot_sync(kFull, pred);
    if (m == 0) return;
    const int c = __popc(m);
    if (n + c > 32) flush<OT>(G, lv, lane);
    const int k = lane - n;  // this lane receives the k-th appended vertex
    const bool take = k >= 0 && k < c;
    const int src = take ? select_bit64(m, k) : lane;
    const int32_t got = __shfl_sync(kFull, x, src);
    if (take) v = got;
    n += c;
  }

  template <typename OT>
  __device__ __forceinline__ void flush(const DevGraph& G, const LevelView& lv, int lane) {
    if (n > 0) flush_appends<OT>(v, n, G, lv, lane);
    n = 0;
  }
};

// Push level, non-heavy frontier vertices: one warp per tile of 32 list
// entries; vertices with degree > 32 are expanded by the whole warp one at a
// time, smaller ones edge-balanced across the warp through a warp scan.
template <int W, typename OT, int DEPTH>
__global__ void __launch_bounds__(kBlock) k_bfs_push(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->dir != kDirPush) return;
  const LevelView lv = level_view(g);
  WarpAppender ap;
  const unsigned long long n = ctl->count[lv.par];
  const int64_t light = push_light_limit(g, G, n, ctl->edges[lv.par]);
  uint64_t sel[W];
#pragma unroll
  for (int i = 0; i < W; ++i) sel[i] = ctl->bfs_bits[i] & ctl->expand[i];
  if (!mask_any<W>(sel)) return;

  __shared__ int64_t s_beg[kWarpsPerBlock][32];
  __shared__ int32_t s_inc[kWarpsPerBlock][32];
  __shared__ uint64_t s_f[kWarpsPerBlock][32][W];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const unsigned long long gw = (static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nw = (static_cast<unsigned long long>(gridDim.x) * blockDim.x) >> 5;
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long pairs = 0;

  for (unsigned long long tile = gw; tile * 32 < n; tile += nw) {
    const unsigned long long idx = tile * 32 + lane;
    const bool valid = idx < n;
    int32_t u = valid ? lv.list[idx] : 0;
    int64_t beg = 0, end = 0;
    uint64_t f[W];
#pragma unroll
    for (int i = 0; i < W; ++i) f[i] = 0;
    if (valid) {
      beg = row_at<OT>(G.row, u);
      end = row_at<OT>(G.row, static_cast<int64_t>(u) + 1);
      load_mask<W>(lv.fcur + static_cast<size_t>(u) * W, f);
#pragma unroll
      for (int i = 0; i < W; ++i) f[i] &= sel[i];
    }
    const int64_t deg = end - beg;
    const bool work = valid && mask_any<W>(f) && deg > 0 && deg <= light;

    unsigned big = __ballot_sync(kFull, work && deg > 32);
    while (big) {
      const int src = __ffs(big) - 1;
      big &= big - 1;
      const int64_t bb = __shfl_sync(kFull, beg, src);
      const int64_t be = __shfl_sync(kFull, end, src);
      uint64_t bf[W];
#pragma unroll
      for (int i = 0; i < W; ++i) bf[i] = __shfl_sync(kFull, f[i], src);
      for (int64_t e0 = bb; e0 < be; e0 += 32) {
        const int64_t e = e0 + lane;
        int32_t nb = 0;
        bool app = false;
        if (e < be) {
          nb = G.col[e];
          app = bfs_visit<W, DEPTH>(g, G.V, lv, nb, bf, uni, pairs);
        }
        ap.add<OT>(app, nb, G, lv, lane);
      }
    }

    int sdeg = (work && deg <= 32) ? static_cast<int>(deg) : 0;
    int inc = sdeg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(kFull, inc, o);
      if (lane >= o) inc += t;
    }
    const int total = __shfl_sync(kFull, inc, 31);
    if (total == 0) continue;
    s_beg[wib][lane] = beg;
    s_inc[wib][lane] = inc;
#pragma unroll
    for (int i = 0; i < W; ++i) s_f[wib][lane][i] = f[i];
    __syncwarp();
    for (int b0 = 0; b0 < total; b0 += 32) {
      const int p = b0 + lane;
      int32_t nb = 0;
      bool app = false;
      if (p < total) {
        int lo = 0, hi = 31;
        while (lo < hi) {
          int mid = (lo + hi) >> 1;
          if (s_inc[wib][mid] > p) hi = mid;
          else lo = mid + 1;
        }
        const int start = lo ? s_inc[wib][lo - 1] : 0;
        const int64_t e = s_beg[wib][lo] + (p - start);
        uint64_t of[W];
#pragma unroll
        for (int i = 0; i < W; ++i) of[i] = s_f[wib][lo][i];
        nb = G.col[e];
        app = bfs_visit<W, DEPTH>(g, G.V, lv, nb, of, uni, pairs);
      }
      ap.add<OT>(app, nb, G, lv, lane);
    }
    __syncwarp();
  }
  ap.flush<OT>(G, lv, lane);
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(pairs, &g.ctl->lc.new_pairs, lane);
}

// Heavy frontier queue.  At the start of a push level the frontier list is
// scanned once and every vertex of degree > heavy_degree is queued with its
// range of kHeavyChunk-edge chunks; one 64-bit atomicAdd hands out both the
// queue slot (high bits) and the first chunk (low bits), so chunk starts grow
// with the slot and a chunk finds its vertex by binary search.  The heavy
// push kernels then visit only the heavy vertices of this frontier instead of
// every heavy vertex of the graph.
constexpr int kQueueShift = 40;

template <typename OT>
__global__ void __launch_bounds__(kBlock) k_heavy_queue(GroupDev g, DevGraph G) {
  LevelCtl* ctl = g.ctl;
  if (ctl->done || (ctl->dir != kDirPush && !ctl->sscatter)) return;
  const LevelView lv = level_view(g);
  const unsigned long long n = ctl->count[lv.par];
  const int64_t light = push_light_limit(g, G, n, ctl->edges[lv.par]);
  for (unsigned long long i = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
       i < n; i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    const int32_t u = lv.list[i];
    const int64_t deg = row_at<OT>(G.row, static_cast<int64_t>(u) + 1) - row_at<OT>(G.row, u);
    if (deg <= light) continue;
    const unsigned long long chunks = static_cast<unsigned long long>((deg + kHeavyChunk - 1) / kHeavyChunk);
    const unsigned long long old = atomicAdd(&ctl->hq_packed, (1ULL << kQueueShift) | chunks);
    const unsigned long long slot = old >> kQueueShift;
    if (slot >= static_cast<unsigned long long>(g.hq_cap)) {  // cannot happen with unique lists
      atomicOr(&ctl->status, kStatusQueueOverflow);
      continue;
    }
    g.hq_vertex[slot] = u;
    g.hq_start[slot] = static_cast<int64_t>(old & ((1ULL << kQueueShift) - 1));
  }
}

// Queue slot of chunk c (the last slot whose first chunk is <= c).
__device__ __forceinline__ int heavy_queue_slot(const GroupDev& g, int nq, int64_t c) {
  int lo = 0, hi = nq - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (g.hq_start[mid] <= c) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Push level, heavy frontier vertices: the static heavy list is cut into
// kHeavyChunk-edge work items spread over all CTAs.
template <int W, typename OT, int DEPTH>
__global__ void __launch_bounds__(kBlock) k_bfs_push_heavy(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->dir != kDirPush) return;
  const unsigned long long hq = ctl->hq_packed;
  const int nq = static_cast<int>(min(static_cast<long long>(hq >> kQueueShift),
                                      static_cast<long long>(g.hq_cap)));
  const int64_t nchunks = static_cast<int64_t>(hq & ((1ULL << kQueueShift) - 1));
  if (nq == 0) return;
  const LevelView lv = level_view(g);
  WarpAppender ap;
  __shared__ int32_t s_h;
  const int lane = threadIdx.x & 31;
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long pairs = 0;
  for (int64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    if (threadIdx.x == 0) s_h = heavy_queue_slot(g, nq, c);
    __syncthreads();
    const int h = s_h;
    __syncthreads();
    const int32_t u = g.hq_vertex[h];
    uint64_t f[W];
    load_mask<W>(lv.fcur + static_cast<size_t>(u) * W, f);
#pragma unroll
    for (int i = 0; i < W; ++i) f[i] &= ctl->bfs_bits[i] & ctl->expand[i];
    if (!mask_any<W>(f)) continue;
    const int64_t beg = row_at<OT>(G.row, u);
    const int64_t end = row_at<OT>(G.row, static_cast<int64_t>(u) + 1);
    const int64_t cb = beg + (c - g.hq_start[h]) * kHeavyChunk;
    const int64_t ce = min(end, cb + kHeavyChunk);
    for (int64_t e0 = cb + (threadIdx.x & ~31); e0 < ce; e0 += blockDim.x) {
      const int64_t e = e0 + lane;
      int32_t nb = 0;
      bool app = false;
      if (e < ce) {
        nb = G.col[e];
        app = bfs_visit<W, DEPTH>(g, G.V, lv, nb, f, uni, pairs);
      }
      ap.add<OT>(app, nb, G, lv, lane);
    }
  }
  ap.flush<OT>(G, lv, lane);
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(pairs, &g.ctl->lc.new_pairs, lane);
}

// Which light-vertex pull form a BFS pull level uses.  The chunked form
// (k_bfs_pull_chunked) keeps 32 in-edges in flight per warp but checks early
// exit once per 32-edge batch; the lane-per-vertex form (k_bfs_pull) stops a
// vertex after the first in-edges that cover its needed bits.  The chunked
// form runs where few vertices stop early: the first pull level after push
// levels (bits are still rare, almost every in-edge is read) and levels after
// a pull level that read at least half of the in-edges.
__device__ __forceinline__ bool bfs_pull_chunked_level(const LevelCtl* ctl, int64_t E) {
  if (ctl->bfs_chunked != 1) return false;
  return ctl->prev_dir != kDirPull || 2 * ctl->prev_pull_edges >= static_cast<unsigned long long>(E);
}

// Zeroes the next-frontier buffer where the previous frontier left bits
// (exactly the vertices of that frontier's list).  Push levels only: a pull
// level rewrites every vertex's next mask.
template <int W>
__global__ void __launch_bounds__(kBlock) k_clear_next(GroupDev g, int64_t E) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done) return;
  // a lane-per-vertex pull level in vertex order rewrites every vertex's next
  // mask; the chunked one and the in-degree-ordered one (which skips vertices
  // without in-edges) write only the vertices they pull
  if (ctl->dir != kDirPush && !bfs_pull_chunked_level(ctl, E) && ctl->bfs_chunked != 2) return;
  const LevelView lv = level_view(g);
  const unsigned long long n = ctl->prev_count;
  const int32_t* plist = lv.nlist;  // list of the previous frontier
  for (unsigned long long i = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
       i < n; i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    uint64_t z[W];
#pragma unroll
    for (int k = 0; k < W; ++k) z[k] = 0;
    store_mask<W>(lv.fnext + static_cast<size_t>(plist[i]) * W, z);
  }
}

// --------------------------------------------------------------- BFS pull
// Finishes one pulled vertex: writes its next mask, visited and depth.
template <int W, int DEPTH>
__device__ __forceinline__ void pull_commit(const GroupDev& g, int64_t V,
                                            const LevelView& lv, int32_t v,
                                            const uint64_t (&vis)[W],
                                            const uint64_t (&nw)[W],
                                            uint64_t (&uni)[W],
                                            unsigned long long& pairs) {
  store_mask<W>(lv.fnext + static_cast<size_t>(v) * W, nw);
  if (!mask_any<W>(nw)) return;
  uint64_t nv[W];
#pragma unroll
  for (int i = 0; i < W; ++i) {
    nv[i] = vis[i] | nw[i];
    uni[i] |= nw[i];
    pairs += __popcll(nw[i]);
  }
  store_mask<W>(g.visited + static_cast<size_t>(v) * W, nv);
  record_depth<W, DEPTH>(g, V, v, nw, lv.level + 1, true);
  // a later SSSP push of the same level must not append v a second time
  g.stamp[v] = lv.level + 1;
}

// A pull level whose frontier holds fewer than 1/16 of the vertices screens
// in-edges by the frontier summary: a source outside the frontier costs an
// 8-byte word that stays in L2 instead of its W-word mask.
__device__ __forceinline__ bool bfs_pull_uses_summary(const GroupDev& g, const LevelCtl* ctl,
                                                      const LevelView& lv, int64_t V) {
  return g.fsum != nullptr && ctl->dir == kDirPull &&
         16ULL * ctl->count[lv.par] < static_cast<unsigned long long>(V);
}

// Pull level (bottom-up): every non-heavy vertex with unvisited active bits
// ORs the current-frontier masks of its in-neighbours until every needed bit
// is found (early exit).  Reads only the current frontier, so depths are
// exactly level-synchronous.  Vertex order by default (a tile is 32
// consecutive vertices); with bfs_chunked == 2 the tiles run over the light
// table's vertices of in-degree 1..32 in decreasing in-degree order, so the
// lanes of a warp walk lists of about the same length (the next masks of the
// vertices left out are zeroed by k_clear_next).
template <int W, typename OT, int DEPTH>
__global__ void __launch_bounds__(kBlock, (W <= 4 ? 3 : 1)) k_bfs_pull(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->dir != kDirPull) return;
  if (G.n_plight_chunks > 0 && bfs_pull_chunked_level(ctl, G.E)) return;
  const LevelView lv = level_view(g);
  uint64_t act[W];
#pragma unroll
  for (int i = 0; i < W; ++i)
    act[i] = ctl->active[lv.par][i] & ctl->bfs_bits[i] & ctl->expand[i];
  const int lane = threadIdx.x & 31;
  const unsigned long long gw = (static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = (static_cast<unsigned long long>(gridDim.x) * blockDim.x) >> 5;
  const unsigned long long V = static_cast<unsigned long long>(G.V);
  const bool use_sum = bfs_pull_uses_summary(g, ctl, lv, G.V);
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long pairs = 0, pverts = 0, pedges = 0;
  const bool sorted = ctl->bfs_chunked == 2;
  // tiles over vertex ids, or over the light table's entries n_pmid .. end
  const unsigned long long n_items =
      sorted ? static_cast<unsigned long long>(G.plight_chunk_start[G.n_plight_chunks] - G.n_pmid) : V;

  for (unsigned long long tile = gw; tile * 32 < n_items; tile += nwarps) {
    const unsigned long long vv = tile * 32 + lane;
    const bool valid = vv < n_items;
    const int32_t v = !valid ? 0 : sorted ? G.plight[G.n_pmid + vv] : static_cast<int32_t>(vv);
    uint64_t need[W], acc[W];
    int64_t beg = 0, end = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      need[i] = 0;
      acc[i] = 0;
    }
    if (valid) {
      beg = row_at<OT>(G.prow, v);
      end = row_at<OT>(G.prow, static_cast<int64_t>(v) + 1);
      uint64_t vis[W];
      load_mask<W>(g.visited + static_cast<size_t>(v) * W, vis);
#pragma unroll
      for (int i = 0; i < W; ++i) need[i] = ~vis[i] & act[i];
    }
    const int64_t deg = end - beg;
    // heavy lists are the heavy kernels'; lists of 33 .. heavy_degree in-edges
    // are k_bfs_pull_mid's when the light table lists them
    const bool heavy = deg > G.heavy_degree || (G.n_pmid > 0 && deg > 32);
    const bool work = valid && !heavy && deg > 0 && mask_any<W>(need);
    pverts += work ? 1 : 0;
    if (work && deg <= 32) {
      const uint32_t nch = chunk_bits<W>(need);
      // four in-edges per step: their column and mask loads are independent
      // and stay in flight together; early exit is checked once per step
      for (int64_t e = beg; e < end; e += 4) {
        int32_t us[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) us[j] = (e + j < end) ? G.pcol[e + j] : -1;
        if (use_sum) {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (us[j] >= 0 && !(summary_chunks(g.fsum, lv.level, us[j]) & nch)) us[j] = -1;
        }
        pedges += static_cast<unsigned long long>(end - e < 4 ? end - e : 4);
        bool full = true;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (us[j] < 0) continue;
          uint64_t fu[W];
          load_mask<W>(lv.fcur + static_cast<size_t>(us[j]) * W, fu);
#pragma unroll
          for (int i = 0; i < W; ++i) acc[i] |= fu[i] & need[i];
        }
#pragma unroll
        for (int i = 0; i < W; ++i) full &= acc[i] == need[i];
        if (full) break;
      }
    }
    unsigned big = __ballot_sync(kFull, work && deg > 32);
    while (big) {
      const int src = __ffs(big) - 1;
      big &= big - 1;
      const int64_t bb = __shfl_sync(kFull, beg, src);
      const int64_t be = __shfl_sync(kFull, end, src);
      uint64_t bn[W], a[W];
#pragma unroll
      for (int i = 0; i < W; ++i) {
        bn[i] = __shfl_sync(kFull, need[i], src);
        a[i] = 0;
      }
      const uint32_t bch = chunk_bits<W>(bn);
      for (int64_t e0 = bb; e0 < be; e0 += 32) {
        const int64_t e = e0 + lane;
        if (e < be) {
          ++pedges;
          const int32_t u = G.pcol[e];
          if (!use_sum || (summary_chunks(g.fsum, lv.level, u) & bch)) {
            uint64_t fu[W];
            load_mask<W>(lv.fcur + static_cast<size_t>(u) * W, fu);
#pragma unroll
            for (int i = 0; i < W; ++i) a[i] |= fu[i] & bn[i];
          }
        }
        warp_or_reduce<W>(a);
        bool full = true;
#pragma unroll
        for (int i = 0; i < W; ++i) full &= a[i] == bn[i];
        if (full) break;
      }
      if (lane == src) {
#pragma unroll
        for (int i = 0; i < W; ++i) acc[i] = a[i];
      }
    }
    bool app = false;
    if (valid && !heavy) {
      uint64_t nwm[W], vis[W];
#pragma unroll
      for (int i = 0; i < W; ++i) nwm[i] = acc[i] & need[i];
      // visited again (this warp's vertex: unchanged since the tile began);
      // not kept in registers across the in-edge loop
      load_mask<W>(g.visited + static_cast<size_t>(v) * W, vis);
      pull_commit<W, DEPTH>(g, G.V, lv, v, vis, nwm, uni, pairs);
      app = mask_any<W>(nwm);
    }
    warp_append(app, v, static_cast<uint64_t>(deg), lv.nlist, lv.ncount, lv.nedges, lane);
  }
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(pairs, &g.ctl->lc.new_pairs, lane);
  warp_add(pverts, &g.ctl->lc.pull_vertices, lane);
  warp_add(pedges, &g.ctl->lc.pull_edges, lane);
}

// Pull level (bottom-up), light vertices in CTA chunks of the pull CSR's light
// chunk table (<= kLightChunkVerts vertices, <= kLightChunkEdges in-edges):
// the CTA's warps split the chunk's in-edges evenly across vertex boundaries,
// each lane loads one in-edge's source frontier mask and ORs its needed bits
// into the vertex's accumulator in shared memory; before a batch a lane skips
// its in-edge once the vertex's accumulator covers its need (early exit per
// 32-edge batch).  After a barrier each vertex is committed once: next-frontier
// words (cleared beforehand by k_clear_next), visited, depth, stamp, append.
// Reads only the current frontier, so depths stay exactly level-synchronous.
template <int W, typename OT, int DEPTH>
__global__ void __launch_bounds__(kBlock) k_bfs_pull_chunked(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->dir != kDirPull || G.n_plight_chunks == 0 ||
      !bfs_pull_chunked_level(ctl, G.E))
    return;
  const LevelView lv = level_view(g);
  __shared__ int32_t s_v[kLightChunkVerts];
  __shared__ int64_t s_beg[kLightChunkVerts];
  __shared__ int32_t s_pre[kLightChunkVerts + 1];
  __shared__ unsigned long long s_need[kLightChunkVerts][W];
  __shared__ unsigned long long s_acc[kLightChunkVerts][W];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  uint64_t act[W];
#pragma unroll
  for (int i = 0; i < W; ++i)
    act[i] = ctl->active[lv.par][i] & ctl->bfs_bits[i] & ctl->expand[i];
  const bool use_sum = bfs_pull_uses_summary(g, ctl, lv, G.V);
  WarpAppender ap;
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long pairs = 0, pverts = 0, pedges = 0;
  for (int c = blockIdx.x; c < G.n_plight_chunks; c += gridDim.x) {
    const int cs = G.plight_chunk_start[c];
    const int nv = G.plight_chunk_start[c + 1] - cs;
    if (wib == 0) {
      int32_t v = 0;
      int64_t b = 0;
      int d = 0;
      if (lane < nv) {
        v = G.plight[cs + lane];
        b = row_at<OT>(G.prow, v);
        uint64_t vis[W];
        load_mask<W>(g.visited + static_cast<size_t>(v) * W, vis);
        bool any = false;
#pragma unroll
        for (int i = 0; i < W; ++i) {
          const uint64_t nd = ~vis[i] & act[i];
          s_need[lane][i] = nd;
          s_acc[lane][i] = 0;
          any |= nd != 0;
        }
        // a vertex that needs nothing contributes no in-edges to the walk
        d = any ? static_cast<int>(row_at<OT>(G.prow, static_cast<int64_t>(v) + 1) - b) : 0;
        pverts += any ? 1 : 0;
      }
      int inc = d;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += t;
      }
      if (lane < nv) {
        s_v[lane] = v;
        s_beg[lane] = b;
        s_pre[lane + 1] = inc;
      }
      if (lane == 0) s_pre[0] = 0;
    }
    __syncthreads();
    const int total = s_pre[nv];
    const int seg = (total + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const int fa = min(total, wib * seg);
    const int fb = min(total, fa + seg);
    for (int f0 = fa; f0 < fb; f0 += 32) {
      const int f = f0 + lane;
      if (f < fb) {
        int lo = 0, hi = nv - 1;  // owner: last k with s_pre[k] <= f
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s_pre[mid] <= f) lo = mid;
          else hi = mid - 1;
        }
        const int k = lo;
        uint64_t nd[W];
        bool open = false;
#pragma unroll
        for (int i = 0; i < W; ++i) {
          nd[i] = s_need[k][i];
          open |= (s_acc[k][i] & nd[i]) != nd[i];
        }
        if (open) {
          ++pedges;
          const int32_t u = G.pcol[s_beg[k] + (f - s_pre[k])];
          if (!use_sum || (summary_chunks(g.fsum, lv.level, u) & chunk_bits<W>(nd))) {
            uint64_t fu[W];
            load_mask<W>(lv.fcur + static_cast<size_t>(u) * W, fu);
#pragma unroll
            for (int i = 0; i < W; ++i) {
              const uint64_t x = fu[i] & nd[i];
              if (x) atomicOr(&s_acc[k][i], static_cast<unsigned long long>(x));
            }
          }
        }
      }
    }
    __syncthreads();
    // commit: warp wib takes vertices wib, wib + 8, ... (lane 0 of the warp)
    for (int k = wib; k < nv; k += kWarpsPerBlock) {
      bool app = false;
      const int32_t v = s_v[k];
      if (lane == 0) {
        uint64_t nw[W], vis[W];
        bool any = false;
#pragma unroll
        for (int i = 0; i < W; ++i) {
          nw[i] = s_acc[k][i] & s_need[k][i];
          any |= nw[i] != 0;
        }
        if (any) {
          load_mask<W>(g.visited + static_cast<size_t>(v) * W, vis);
          uint64_t nv2[W];
#pragma unroll
          for (int i = 0; i < W; ++i) {
            nv2[i] = vis[i] | nw[i];
            uni[i] |= nw[i];
            pairs += __popcll(nw[i]);
          }
          store_mask<W>(g.visited + static_cast<size_t>(v) * W, nv2);
          store_mask<W>(lv.fnext + static_cast<size_t>(v) * W, nw);
          record_depth<W, DEPTH>(g, G.V, v, nw, lv.level + 1, true);
          app = g.stamp[v] < lv.level + 1;
          g.stamp[v] = lv.level + 1;
        }
      }
      ap.add<OT>(app, v, G, lv, lane);
    }
    __syncthreads();
  }
  ap.flush<OT>(G, lv, lane);
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(pairs, &g.ctl->lc.new_pairs, lane);
  warp_add(pverts, &g.ctl->lc.pull_vertices, lane);
  warp_add(pedges, &g.ctl->lc.pull_edges, lane);
}

// Pull level, vertices with 33 .. heavy_degree in-edges (the first n_pmid
// entries of the pull CSR's light table, largest first): a warp per vertex,
// 64 in-edges per step (two column -> mask loads in flight per lane, then a
// warp OR-reduce and the early-exit test), one commit per vertex.  In the
// lane-per-vertex tile kernel these lists were a warp's serial work with one
// 32-edge step in flight; here they have a kernel and a register budget of
// their own.  Every listed vertex's next mask is written (zero when nothing
// is new), as the tile kernel does for its vertices.
template <int W, typename OT, int DEPTH>
__global__ void __launch_bounds__(kBlock, 3) k_bfs_pull_mid(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->dir != kDirPull || G.n_pmid == 0) return;
  if (G.n_plight_chunks > 0 && bfs_pull_chunked_level(ctl, G.E)) return;
  const LevelView lv = level_view(g);
  uint64_t act[W];
#pragma unroll
  for (int i = 0; i < W; ++i)
    act[i] = ctl->active[lv.par][i] & ctl->bfs_bits[i] & ctl->expand[i];
  const bool use_sum = bfs_pull_uses_summary(g, ctl, lv, G.V);
  const int lane = threadIdx.x & 31;
  const long long gw = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  WarpAppender ap;
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long pairs = 0, pverts = 0, pedges = 0;
  for (long long i = gw; i < G.n_pmid; i += nwarps) {
    const int32_t v = G.plight[i];
    uint64_t vis[W], need[W];
    load_mask<W>(g.visited + static_cast<size_t>(v) * W, vis);
    bool any = false;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      need[k] = ~vis[k] & act[k];
      any |= need[k] != 0;
    }
    uint64_t a[W];
#pragma unroll
    for (int k = 0; k < W; ++k) a[k] = 0;
    if (any) {  // uniform
      if (lane == 0) ++pverts;
      const int64_t beg = row_at<OT>(G.prow, v);
      const int64_t end = row_at<OT>(G.prow, static_cast<int64_t>(v) + 1);
      const uint32_t nch = chunk_bits<W>(need);
      for (int64_t e0 = beg; e0 < end; e0 += 64) {
        int32_t u0 = -1, u1 = -1;
        if (e0 + lane < end) u0 = G.pcol[e0 + lane];
        if (e0 + 32 + lane < end) u1 = G.pcol[e0 + 32 + lane];
        pedges += (u0 >= 0 ? 1 : 0) + (u1 >= 0 ? 1 : 0);
        if (use_sum) {
          if (u0 >= 0 && !(summary_chunks(g.fsum, lv.level, u0) & nch)) u0 = -1;
          if (u1 >= 0 && !(summary_chunks(g.fsum, lv.level, u1) & nch)) u1 = -1;
        }
        uint64_t f0[W], f1[W];
#pragma unroll
        for (int k = 0; k < W; ++k) {
          f0[k] = 0;
          f1[k] = 0;
        }
        if (u0 >= 0) load_mask<W>(lv.fcur + static_cast<size_t>(u0) * W, f0);
        if (u1 >= 0) load_mask<W>(lv.fcur + static_cast<size_t>(u1) * W, f1);
#pragma unroll
        for (int k = 0; k < W; ++k) a[k] |= (f0[k] | f1[k]) & need[k];
        warp_or_reduce<W>(a);
        bool full = true;
#pragma unroll
        for (int k = 0; k < W; ++k) full &= a[k] == need[k];
        if (full) break;
      }
    }
    bool app = false;
    if (lane == 0) {
      uint64_t nw[W];
#pragma unroll
      for (int k = 0; k < W; ++k) nw[k] = a[k] & need[k];
      pull_commit<W, DEPTH>(g, G.V, lv, v, vis, nw, uni, pairs);
      app = mask_any<W>(nw);
    }
    ap.add<OT>(app, v, G, lv, lane);
  }
  ap.flush<OT>(G, lv, lane);
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(pairs, &g.ctl->lc.new_pairs, lane);
  warp_add(pverts, &g.ctl->lc.pull_vertices, lane);
  warp_add(pedges, &g.ctl->lc.pull_edges, lane);
}

// Pull level, heavy vertices: chunks of their in-edges spread over CTAs; each
// CTA ORs its chunk into hacc[h] (skipping chunks once hacc covers the need).
template <int W, typename OT>
__global__ void __launch_bounds__(kBlock) k_bfs_pull_heavy(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->dir != kDirPull || G.n_pheavy == 0) return;
  const LevelView lv = level_view(g);
  __shared__ int s_skip;
  __shared__ uint64_t s_red[kWarpsPerBlock][W];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  for (int64_t c = blockIdx.x; c < G.pheavy_chunks; c += gridDim.x) {
    __syncthreads();  // the previous chunk's s_skip is read
    const int h = G.pheavy_ch[c];
    const int32_t v = G.pheavy[h];
    uint64_t vis[W], need[W];
    load_mask<W>(g.visited + static_cast<size_t>(v) * W, vis);
    bool anyneed = false;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      need[i] = ~vis[i] & ctl->active[lv.par][i] & ctl->bfs_bits[i] & ctl->expand[i];
      anyneed |= need[i] != 0;
    }
    if (threadIdx.x == 0) {
      bool covered = true;
      const volatile uint64_t* ha = g.hacc + static_cast<size_t>(h) * W;
#pragma unroll
      for (int i = 0; i < W; ++i) covered &= (ha[i] & need[i]) == need[i];
      s_skip = (!anyneed || covered) ? 1 : 0;
    }
    __syncthreads();
    if (s_skip) continue;
    const int64_t cb = G.pheavy_cb[c];
    const int64_t ce = G.pheavy_ce[c];
    uint64_t a[W];
#pragma unroll
    for (int i = 0; i < W; ++i) a[i] = 0;
    if (threadIdx.x == 0) atomicAdd(&g.ctl->lc.pull_edges, static_cast<unsigned long long>(ce - cb));
    const bool use_sum = bfs_pull_uses_summary(g, ctl, lv, G.V);
    const uint32_t nch = chunk_bits<W>(need);
    for (int64_t e = cb + threadIdx.x; e < ce; e += blockDim.x) {
      const int32_t u = G.pcol[e];
      if (use_sum && !(summary_chunks(g.fsum, lv.level, u) & nch)) continue;
      uint64_t fu[W];
      load_mask<W>(lv.fcur + static_cast<size_t>(u) * W, fu);
#pragma unroll
      for (int i = 0; i < W; ++i) a[i] |= fu[i] & need[i];
    }
    warp_or_reduce<W>(a);
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < W; ++i) s_red[wib][i] = a[i];
    }
    __syncthreads();
    if (threadIdx.x < W) {
      uint64_t r = 0;
      for (int k = 0; k < kWarpsPerBlock; ++k) r |= s_red[k][threadIdx.x];
      if (r) atomic_or64(g.hacc + static_cast<size_t>(h) * W + threadIdx.x, r);
    }
    __syncthreads();
  }
}

// Commits the heavy vertices of a pull level and resets their accumulators.
template <int W, typename OT, int DEPTH>
__global__ void __launch_bounds__(kBlock) k_bfs_pull_heavy_commit(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->dir != kDirPull || G.n_pheavy == 0) return;
  const LevelView lv = level_view(g);
  const int lane = threadIdx.x & 31;
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long pairs = 0, pverts = 0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31);
       base < G.n_pheavy; base += stride) {
    const int64_t h = base + lane;
    bool app = false;
    int32_t v = 0;
    uint64_t deg = 0;
    if (h < G.n_pheavy) {
      v = G.pheavy[h];
      uint64_t vis[W], nwm[W], acc[W];
      load_mask<W>(g.visited + static_cast<size_t>(v) * W, vis);
      load_mask<W>(g.hacc + static_cast<size_t>(h) * W, acc);
#pragma unroll
      for (int i = 0; i < W; ++i) {
        nwm[i] = acc[i] & ~vis[i] & ctl->active[lv.par][i] & ctl->bfs_bits[i] & ctl->expand[i];
        acc[i] = 0;
      }
      store_mask<W>(g.hacc + static_cast<size_t>(h) * W, acc);
      bool anyneed = false;
#pragma unroll
      for (int i = 0; i < W; ++i)
        anyneed |= (~vis[i] & ctl->active[lv.par][i] & ctl->bfs_bits[i] & ctl->expand[i]) != 0;
      pverts += anyneed ? 1 : 0;
      pull_commit<W, DEPTH>(g, G.V, lv, v, vis, nwm, uni, pairs);
      app = mask_any<W>(nwm);
      deg = degree_of<OT>(G.prow, v);
    }
    warp_append(app, v, deg, lv.nlist, lv.ncount, lv.nedges, lane);
  }
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(pairs, &g.ctl->lc.new_pairs, lane);
  warp_add(pverts, &g.ctl->lc.pull_vertices, lane);
}

// -------------------------------------------------------------- SSSP push
template <int WK>
__device__ __forceinline__ uint32_t relax(uint32_t du, const void* w, int64_t e) {
  if constexpr (WK == kWeightF32) {
    float r = __fadd_rn(__uint_as_float(du), static_cast<const float*>(w)[e]);
    return __float_as_uint(r);
  } else {
    uint32_t wt = (WK == kWeightU32) ? static_cast<const uint32_t*>(w)[e] : 1u;
    return du > 0xffffffffu - wt ? 0xffffffffu : du + wt;
  }
}

// One (edge, query) relaxation: values are compared as uint32, which orders
// non-negative floats exactly like their values (+inf = 0x7f800000).
template <int W, int WK>
__device__ __forceinline__ bool sssp_relax(const GroupDev& g, const LevelView& lv,
                                           int32_t u, int32_t n, int q,
                                           const void* w, int64_t e,
                                           uint64_t (&uni)[W],
                                           unsigned long long& improved) {
  const size_t Qg = static_cast<size_t>(g.Qg);
  const uint32_t du = g.values[static_cast<size_t>(u) * Qg + q];
  const uint32_t cand = relax<WK>(du, w, e);
  uint32_t* dst = g.values + static_cast<size_t>(n) * Qg + q;
  if (cand >= *dst) return false;
  const uint32_t old = atomicMin(dst, cand);
  if (cand >= old) return false;
  const uint64_t bit = 1ULL << (q & 63);
  // hub destinations receive many improvements per level: a plain read of
  // the frontier word and of the stamp skips atomics that would change
  // nothing (bits and stamps only grow within a level)
  uint64_t* fw = lv.fnext + static_cast<size_t>(n) * W + (q >> 6);
  if (!(*fw & bit)) atomic_or64(fw, bit);
  uni[q >> 6] |= bit;
  ++improved;
  if (g.stamp[n] >= lv.level + 1) return false;
  return atomicMax(g.stamp + n, lv.level + 1) < lv.level + 1;
}

// Second half of sssp_relax, for callers that loaded the destination value
// themselves (cand < the value they read): the atomicMin and its frontier,
// union and stamp updates.  True when n must be appended.
template <int W>
__device__ __forceinline__ bool sssp_commit(const GroupDev& g, const LevelView& lv, int32_t n,
                                            int q, uint32_t cand, uint64_t (&uni)[W],
                                            unsigned long long& improved) {
  uint32_t* dst = g.values + static_cast<size_t>(n) * static_cast<size_t>(g.Qg) + q;
  const uint32_t old = atomicMin(dst, cand);
  if (cand >= old) return false;
  const uint64_t bit = 1ULL << (q & 63);
  uint64_t* fw = lv.fnext + static_cast<size_t>(n) * W + (q >> 6);
  if (!(*fw & bit)) atomic_or64(fw, bit);
  uni[q >> 6] |= bit;
  ++improved;
  if (g.stamp[n] >= lv.level + 1) return false;
  return atomicMax(g.stamp + n, lv.level + 1) < lv.level + 1;
}

// Pairs handled per lane per step by the sparse scatter loops: their column,
// source and destination loads are independent and issued together.
constexpr int kPairSteps = 4;

// Relaxation with the weight already loaded (raw 32-bit pattern).
template <int WK>
__device__ __forceinline__ uint32_t relax_w(uint32_t du, uint32_t wbits) {
  if constexpr (WK == kWeightF32) {
    return __float_as_uint(__fadd_rn(__uint_as_float(du), __uint_as_float(wbits)));
  } else {
    const uint32_t wt = (WK == kWeightU32) ? wbits : 1u;
    return du > 0xffffffffu - wt ? 0xffffffffu : du + wt;
  }
}

template <int WK>
__device__ __forceinline__ uint32_t weight_bits(const void* w, int64_t e) {
  if constexpr (WK == kWeightNone) {
    return 1u;
  } else {
    return static_cast<const uint32_t*>(w)[e];
  }
}

// Vertices with more active SSSP bits than this take the dense path.
constexpr int kDenseBits = 16;

// Dense SSSP relaxation of edges [eb, ee) of vertex u by one warp (all lanes
// call).  Lane j owns query 32c+j of every 32-bit chunk c of the vertex's
// active mask: u's distances stay in registers, and per edge each active
// chunk costs one coalesced 128-byte load of the neighbour's row, a compare,
// and an atomicMin only where it improves; the improved bits of a chunk are
// combined by a ballot into one atomicOr of the next-frontier word.
template <int W, typename OT, int WK, int U>
__device__ __forceinline__ void sssp_dense_edges(const GroupDev& g, const DevGraph& G,
                                                 const LevelView& lv, int32_t u,
                                                 const uint64_t (&bits)[W], int64_t eb,
                                                 int64_t ee, int lane, uint64_t (&uni)[W],
                                                 unsigned long long& improved,
                                                 WarpAppender& ap) {
  const size_t Qg = static_cast<size_t>(g.Qg);
  uint32_t half[2 * W];
  uint32_t du[2 * W];
  bool act[2 * W];
#pragma unroll
  for (int c = 0; c < 2 * W; ++c) {
    half[c] = static_cast<uint32_t>(bits[c >> 1] >> (32 * (c & 1)));
    act[c] = (half[c] >> lane) & 1u;
    du[c] = act[c] ? g.values[static_cast<size_t>(u) * Qg + 32 * c + lane] : 0xffffffffu;
  }
  for (int64_t e0 = eb; e0 < ee; e0 += 32) {
    const int64_t e = e0 + lane;
    int32_t nl = 0;
    uint32_t wl = 0;
    if (e < ee) {
      nl = G.col[e];
      wl = weight_bits<WK>(G.w, e);
    }
    const int cnt = static_cast<int>(ee - e0 < 32 ? ee - e0 : 32);
    // U edges per step (1 or 2): U x (active chunks) row loads in flight per warp
    for (int i = 0; i < cnt; i += U) {
      const bool two = U == 2 && i + 1 < cnt;
      const int32_t nb0 = __shfl_sync(kFull, nl, i);
      const uint32_t wt0 = __shfl_sync(kFull, wl, i);
      const int32_t nb1 = __shfl_sync(kFull, nl, two ? i + 1 : i);
      const uint32_t wt1 = __shfl_sync(kFull, wl, two ? i + 1 : i);
      uint32_t* row0 = g.values + static_cast<size_t>(nb0) * Qg + lane;
      uint32_t* row1 = g.values + static_cast<size_t>(nb1) * Qg + lane;
      uint32_t cur0[2 * W], cur1[2 * W];
#pragma unroll
      for (int c = 0; c < 2 * W; ++c) {
        cur0[c] = act[c] ? row0[32 * c] : 0u;
        cur1[c] = (act[c] && two) ? row1[32 * c] : 0u;
      }
      bool better = false;
#pragma unroll
      for (int c = 0; c < 2 * W; ++c) {
        better |= act[c] && relax_w<WK>(du[c], wt0) < cur0[c];
        better |= act[c] && two && relax_w<WK>(du[c], wt1) < cur1[c];
      }
      // improvements are rare: atomics and ballots only when some lane of the
      // warp has a better candidate for one of the two edges
      if (!__any_sync(kFull, better)) continue;
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        if (t == 1 && !two) break;
        const int32_t nb = t ? nb1 : nb0;
        const uint32_t wt = t ? wt1 : wt0;
        uint32_t* row = t ? row1 : row0;
        bool any = false;
#pragma unroll
        for (int c = 0; c < 2 * W; ++c) {
          if (half[c] == 0) continue;
          const uint32_t cand = relax_w<WK>(du[c], wt);
          bool imp = false;
          if (act[c] && cand < (t ? cur1[c] : cur0[c])) imp = cand < atomicMin(row + 32 * c, cand);
          const unsigned m = __ballot_sync(kFull, imp);
          if (m) {
            any = true;
            if (lane == 0) {
              const uint64_t bitsw = static_cast<uint64_t>(m) << (32 * (c & 1));
              atomic_or64(lv.fnext + static_cast<size_t>(nb) * W + (c >> 1), bitsw);
              uni[c >> 1] |= bitsw;
              improved += __popc(m);
            }
          }
        }
        bool app = false;
        if (any && lane == 0 && g.stamp[nb] < lv.level + 1)
          app = atomicMax(g.stamp + nb, lv.level + 1) < lv.level + 1;
        ap.add<OT>(app, nb, G, lv, lane);
      }
    }
  }
}

// Dense SSSP vertices of a level, one warp per vertex (the tile kernel
// queued them), so that this loop gets a register budget of its own.
template <int W, typename OT, int WK, int U>
__global__ void __launch_bounds__(kBlock, (U == 1 ? 4 : 3)) k_sssp_dense(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || !ctl->sscatter) return;
  const LevelView lv = level_view(g);
  WarpAppender ap;
  const unsigned long long n = ctl->dense_count;
  const int lane = threadIdx.x & 31;
  const unsigned long long gw = (static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = (static_cast<unsigned long long>(gridDim.x) * blockDim.x) >> 5;
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long improved = 0;
  for (unsigned long long i = gw; i < n; i += nwarps) {
    const int32_t u = g.dense_list[i];
    const int64_t beg = row_at<OT>(G.row, u);
    const int64_t end = row_at<OT>(G.row, static_cast<int64_t>(u) + 1);
    uint64_t b[W];
    load_mask<W>(lv.fcur + static_cast<size_t>(u) * W, b);
#pragma unroll
    for (int k = 0; k < W; ++k) b[k] &= ctl->ssel[k];
    sssp_dense_edges<W, OT, WK, U>(g, G, lv, u, b, beg, end, lane, uni, improved, ap);
  }
  ap.flush<OT>(G, lv, lane);
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(improved, &g.ctl->lc.improved, lane);
}

// SSSP push over the frontier list: the (edge, active query) pairs of a tile
// of 32 vertices are flattened and spread evenly over the warp's lanes, so a
// vertex with k active queries and degree d costs k*d/32 warp steps.
template <int W, typename OT, int WK>
__global__ void __launch_bounds__(kBlock) k_sssp_push(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || !ctl->sscatter) return;
  const LevelView lv = level_view(g);
  WarpAppender ap;
  const unsigned long long n = ctl->count[lv.par];
  const int64_t light = push_light_limit(g, G, n, ctl->edges[lv.par]);
  uint64_t sel[W];
#pragma unroll
  for (int i = 0; i < W; ++i) sel[i] = ctl->ssel[i];
  if (!mask_any<W>(sel)) return;
  __shared__ int64_t s_beg[kWarpsPerBlock][32];
  __shared__ long long s_inc[kWarpsPerBlock][32];
  __shared__ int32_t s_k[kWarpsPerBlock][32];
  __shared__ int32_t s_u[kWarpsPerBlock][32];
  __shared__ uint64_t s_b[kWarpsPerBlock][32][W];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const unsigned long long gw = (static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = (static_cast<unsigned long long>(gridDim.x) * blockDim.x) >> 5;
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long improved = 0, spairs = 0, sactive = 0;
  for (unsigned long long tile = gw; tile * 32 < n; tile += nwarps) {
    const unsigned long long idx = tile * 32 + lane;
    const bool valid = idx < n;
    int32_t u = valid ? lv.list[idx] : 0;
    int64_t beg = 0, end = 0;
    uint64_t b[W];
    int k = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) b[i] = 0;
    if (valid) {
      beg = row_at<OT>(G.row, u);
      end = row_at<OT>(G.row, static_cast<int64_t>(u) + 1);
      load_mask<W>(lv.fcur + static_cast<size_t>(u) * W, b);
#pragma unroll
      for (int i = 0; i < W; ++i) {
        b[i] &= sel[i];
        k += __popcll(b[i]);
      }
    }
    const int64_t deg = end - beg;
    const bool work = valid && k > 0 && deg > 0 && deg <= light;
    spairs += work ? static_cast<unsigned long long>(k) * static_cast<unsigned long long>(deg) : 0ULL;
    sactive += static_cast<unsigned long long>(k);
    // vertices with many active queries go to the dense kernel
    {
      const bool dq = work && k > kDenseBits;
      const unsigned m = __ballot_sync(kFull, dq);
      if (m) {
        unsigned long long base = 0;
        if (lane == __ffs(m) - 1)
          base = atomicAdd(&g.ctl->dense_count, static_cast<unsigned long long>(__popc(m)));
        base = __shfl_sync(kFull, base, __ffs(m) - 1);
        if (dq) g.dense_list[base + __popc(m & ((1u << lane) - 1u))] = u;
      }
    }
    // the rest: (edge, query) pairs flattened over the lanes
    long long wk = (work && k <= kDenseBits) ? static_cast<long long>(k) * deg : 0;
    long long inc = wk;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long t = __shfl_up_sync(kFull, inc, o);
      if (lane >= o) inc += t;
    }
    const long long total = __shfl_sync(kFull, inc, 31);
    if (total == 0) continue;
    s_beg[wib][lane] = beg;
    s_inc[wib][lane] = inc;
    s_k[wib][lane] = k;
    s_u[wib][lane] = u;
#pragma unroll
    for (int i = 0; i < W; ++i) s_b[wib][lane][i] = b[i];
    __syncwarp();
    const size_t Qg = static_cast<size_t>(g.Qg);
    for (long long b0 = 0; b0 < total; b0 += 32 * kPairSteps) {
      int32_t nb[kPairSteps];
      int qq[kPairSteps];
      uint32_t cand[kPairSteps], cur[kPairSteps];
#pragma unroll
      for (int t = 0; t < kPairSteps; ++t) {
        const long long p = b0 + 32 * t + lane;
        nb[t] = 0;
        qq[t] = 0;
        cand[t] = 0xffffffffu;
        if (p < total) {
          int lo = 0, hi = 31;
          while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (s_inc[wib][mid] > p) hi = mid;
            else lo = mid + 1;
          }
          const long long start = lo ? s_inc[wib][lo - 1] : 0;
          const int local = static_cast<int>(p - start);  // < kDenseBits * heavy_degree
          const int ko = s_k[wib][lo];
          const int eoff = local / ko;
          const int j = local - eoff * ko;
          qq[t] = jth_set_bit<W>(s_b[wib][lo], j);
          const int64_t e = s_beg[wib][lo] + eoff;
          nb[t] = G.col[e];
          cand[t] = relax<WK>(g.values[static_cast<size_t>(s_u[wib][lo]) * Qg + qq[t]], G.w, e);
        }
      }
#pragma unroll
      for (int t = 0; t < kPairSteps; ++t)
        cur[t] = cand[t] != 0xffffffffu ? g.values[static_cast<size_t>(nb[t]) * Qg + qq[t]] : 0u;
#pragma unroll
      for (int t = 0; t < kPairSteps; ++t) {
        const bool app = cand[t] < cur[t] && sssp_commit<W>(g, lv, nb[t], qq[t], cand[t], uni, improved);
        ap.add<OT>(app, nb[t], G, lv, lane);
      }
    }
    __syncwarp();
  }
  ap.flush<OT>(G, lv, lane);
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(improved, &g.ctl->lc.improved, lane);
  warp_add(spairs, &g.ctl->lc.sssp_pairs, lane);
  warp_add(sactive, &g.ctl->lc.sssp_active, lane);
}

// SSSP push for heavy frontier vertices: per chunk of kHeavyChunk edges the
// CTA lists the active query ids once and walks (edge, query) pairs.
template <int W, typename OT, int WK>
__global__ void __launch_bounds__(kBlock) k_sssp_push_heavy(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || !ctl->sscatter) return;
  const unsigned long long hq = ctl->hq_packed;
  const int nq = static_cast<int>(min(static_cast<long long>(hq >> kQueueShift),
                                      static_cast<long long>(g.hq_cap)));
  const int64_t nchunks = static_cast<int64_t>(hq & ((1ULL << kQueueShift) - 1));
  if (nq == 0) return;
  const LevelView lv = level_view(g);
  WarpAppender ap;
  __shared__ int32_t s_h;
  __shared__ int32_t s_k;
  __shared__ int16_t s_q[kMaxW * 64];
  __shared__ int32_t s_wpre[W + 1];
  const int lane = threadIdx.x & 31;
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long improved = 0;
  for (int64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    if (threadIdx.x == 0) s_h = heavy_queue_slot(g, nq, c);
    __syncthreads();
    const int h = s_h;
    const int32_t u = g.hq_vertex[h];
    uint64_t b[W];
    load_mask<W>(lv.fcur + static_cast<size_t>(u) * W, b);
#pragma unroll
    for (int i = 0; i < W; ++i) b[i] &= ctl->ssel[i];
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int i = 0; i < W; ++i) {
        s_wpre[i] = acc;
        acc += __popcll(b[i]);
      }
      s_wpre[W] = acc;
      s_k = acc;
    }
    __syncthreads();
    const int k = s_k;
    if (k == 0) {
      __syncthreads();
      continue;
    }
    if (k > kDenseBits) {
      // each warp takes a contiguous slice of the chunk's edges
      const int64_t beg = row_at<OT>(G.row, u);
      const int64_t end = row_at<OT>(G.row, static_cast<int64_t>(u) + 1);
      const int64_t cb = beg + (c - g.hq_start[h]) * kHeavyChunk;
      const int64_t ce = min(end, cb + kHeavyChunk);
      if (threadIdx.x == 0) {
        atomicAdd(&g.ctl->lc.sssp_pairs, static_cast<unsigned long long>(ce - cb) * k);
        if (c == g.hq_start[h]) atomicAdd(&g.ctl->lc.sssp_active, static_cast<unsigned long long>(k));
      }
      const int nw = blockDim.x >> 5;
      const int64_t seg = (ce - cb + nw - 1) / nw;
      const int64_t wb = cb + (threadIdx.x >> 5) * seg;
      const int64_t we = min(ce, wb + seg);
      sssp_dense_edges<W, OT, WK, 1>(g, G, lv, u, b, wb, we, lane, uni, improved, ap);
      __syncthreads();
      continue;
    }
    for (int t = threadIdx.x; t < W * 64; t += blockDim.x) {
      const int i = t >> 6, bit = t & 63;
      if ((b[i] >> bit) & 1ULL)
        s_q[s_wpre[i] + __popcll(b[i] & ((1ULL << bit) - 1ULL))] = static_cast<int16_t>(t);
    }
    __syncthreads();
    const int64_t beg = row_at<OT>(G.row, u);
    const int64_t end = row_at<OT>(G.row, static_cast<int64_t>(u) + 1);
    const int64_t cb = beg + (c - g.hq_start[h]) * kHeavyChunk;
    const int64_t ce = min(end, cb + kHeavyChunk);
    const long long pairs = static_cast<long long>(ce - cb) * k;
    if (threadIdx.x == 0) {
      atomicAdd(&g.ctl->lc.sssp_pairs, static_cast<unsigned long long>(pairs));
      if (c == g.hq_start[h]) atomicAdd(&g.ctl->lc.sssp_active, static_cast<unsigned long long>(k));
    }
    const size_t Qg = static_cast<size_t>(g.Qg);
    for (long long p0 = threadIdx.x & ~31; p0 < pairs; p0 += kPairSteps * blockDim.x) {
      int32_t nb[kPairSteps];
      int qq[kPairSteps];
      uint32_t cand[kPairSteps], cur[kPairSteps];
#pragma unroll
      for (int t = 0; t < kPairSteps; ++t) {
        const long long p = p0 + t * blockDim.x + lane;
        nb[t] = 0;
        qq[t] = 0;
        cand[t] = 0xffffffffu;
        if (p < pairs) {
          const int eoff = static_cast<int>(p) / k;  // pairs <= kHeavyChunk * kDenseBits
          qq[t] = s_q[static_cast<int>(p) - eoff * k];
          const int64_t e = cb + eoff;
          nb[t] = G.col[e];
          cand[t] = relax<WK>(g.values[static_cast<size_t>(u) * Qg + qq[t]], G.w, e);
        }
      }
#pragma unroll
      for (int t = 0; t < kPairSteps; ++t)
        cur[t] = cand[t] != 0xffffffffu ? g.values[static_cast<size_t>(nb[t]) * Qg + qq[t]] : 0u;
#pragma unroll
      for (int t = 0; t < kPairSteps; ++t) {
        const bool app = cand[t] < cur[t] && sssp_commit<W>(g, lv, nb[t], qq[t], cand[t], uni, improved);
        ap.add<OT>(app, nb[t], G, lv, lane);
      }
    }
    __syncthreads();
  }
  ap.flush<OT>(G, lv, lane);
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(improved, &g.ctl->lc.improved, lane);
}


// ------------------------------------------------------------ SSSP gather
// Dense SSSP levels (most vertices in the frontier for many queries) run as a
// gather instead of a scatter: the warp that owns vertex v takes the minimum
// of dist[u][q] + w(u, v) over v's in-edges for all its SSSP slots at once,
// then writes the improved entries of v's row with plain stores.  No
// distance atomics, no per-(edge, query) frontier atomics: the improved bits
// of a 32-slot chunk come from one ballot.  Lane j owns slot 32c + j of
// chunk c; the sources' rows are read for every SSSP slot of the chunk (an
// entry that is not in the frontier relaxes to a value that cannot improve
// v, or to one that another relaxation would produce anyway), so per edge the
// warp issues 2W coalesced 128-byte loads and no data-dependent branches.
// Several in-edges are in flight per warp (GatherSteps) to cover latency.

// Relaxation of a stored value `du` over an edge with raw weight bits.  The
// unreached markers (0xffffffff; +inf for f32) never improve anything.
template <int WK>
__device__ __forceinline__ uint32_t gather_relax(uint32_t du, uint32_t wbits) {
  if constexpr (WK == kWeightF32) {
    return du >= 0x7f800000u
               ? 0xffffffffu
               : __float_as_uint(__fadd_rn(__uint_as_float(du), __uint_as_float(wbits)));
  } else {
    const uint32_t wt = (WK == kWeightU32) ? wbits : 1u;
    return min(du, ~wt) + wt;  // saturates at 0xffffffff
  }
}

// In-edges gathered together per warp step: 2W x steps row loads per lane.
template <int W>
struct GatherSteps {
  static constexpr int value = W >= 16 ? 1 : (W >= 8 ? 2 : (W >= 4 ? 4 : 8));
};

// Bit c of the result: this lane's slot of chunk c is an SSSP slot that
// gathers at this level.
template <int W>
__device__ __forceinline__ uint32_t lane_sssp_chunks(const LevelCtl* ctl, int lane) {
  uint32_t sel = 0;
#pragma unroll
  for (int c = 0; c < 2 * W; ++c)
    sel |= static_cast<uint32_t>((ctl->gsel[c >> 1] >> (32 * (c & 1) + lane)) & 1ULL) << c;
  return sel;
}

// min-accumulates relaxations over in-edges [eb, ee) of the pull CSR into
// best[c] (lane's slot of chunk c).  Edges whose source has no SSSP frontier
// bit are skipped by a ballot.  All lanes call.
template <int W, int WK>
__device__ __forceinline__ void gather_edges(const GroupDev& g, const DevGraph& G,
                                             const LevelView& lv, const uint64_t* sb,
                                             uint32_t lsel, int64_t eb, int64_t ee, int lane,
                                             uint32_t (&best)[2 * W],
                                             unsigned long long& pairs,
                                             unsigned& scanned) {
  constexpr int C = 2 * W;
  constexpr int S = GatherSteps<W>::value;
  const size_t Qg = static_cast<size_t>(g.Qg);
  for (int64_t e0 = eb; e0 < ee; e0 += 32) {
    const int64_t e = e0 + lane;
    int32_t u = 0;
    uint32_t wb = 0;
    int k = 0;
    if (e < ee) {
      u = G.pcol[e];
      wb = weight_bits<WK>(G.pw, e);
      uint64_t m[W];
      load_mask<W>(lv.fcur + static_cast<size_t>(u) * W, m);
#pragma unroll
      for (int i = 0; i < W; ++i) k += __popcll(m[i] & sb[i]);
      ++scanned;
    }
    pairs += static_cast<unsigned long long>(k);
    unsigned live = __ballot_sync(kFull, k > 0);
    while (live) {
      int32_t us[S];
      uint32_t ws[S];
      bool ok[S];
#pragma unroll
      for (int t = 0; t < S; ++t) {
        ok[t] = live != 0;
        const int j = (__ffs(live) - 1) & 31;
        live &= live - 1;
        us[t] = __shfl_sync(kFull, u, j);
        ws[t] = __shfl_sync(kFull, wb, j);
      }
      uint32_t cur[S][C];
#pragma unroll
      for (int t = 0; t < S; ++t) {
        const uint32_t* row = g.values + static_cast<size_t>(us[t]) * Qg + lane;
#pragma unroll
        for (int c = 0; c < C; ++c)
          cur[t][c] = (ok[t] && ((lsel >> c) & 1u)) ? __ldcg(row + 32 * c) : 0xffffffffu;
      }
#pragma unroll
      for (int t = 0; t < S; ++t) {
#pragma unroll
        for (int c = 0; c < C; ++c) best[c] = min(best[c], gather_relax<WK>(cur[t][c], ws[t]));
      }
    }
  }
}

// Gather level, vertices of in-degree <= heavy_degree: one warp per vertex.
template <int W, typename OT, int WK>
__global__ void __launch_bounds__(kBlock, (W <= 4 ? 3 : 2)) k_sssp_pull(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->sdir != kDirPull) return;
  const LevelView lv = level_view(g);
  constexpr int C = 2 * W;
  const int lane = threadIdx.x & 31;
  const uint64_t* sb = ctl->gsel;
  const uint32_t lsel = lane_sssp_chunks<W>(ctl, lane);
  const unsigned long long gw = (static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = (static_cast<unsigned long long>(gridDim.x) * blockDim.x) >> 5;
  const size_t Qg = static_cast<size_t>(g.Qg);
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long improved = 0, pairs = 0;
  unsigned scanned = 0, verts = 0;
  for (unsigned long long vv = gw; vv < static_cast<unsigned long long>(G.V); vv += nwarps) {
    const int32_t v = static_cast<int32_t>(vv);
    const int64_t beg = row_at<OT>(G.prow, v);
    const int64_t end = row_at<OT>(G.prow, static_cast<int64_t>(v) + 1);
    if (end == beg || end - beg > G.heavy_degree) continue;
    if (lane == 0) ++verts;  // one count per vertex, not per lane
    uint32_t* row = g.values + static_cast<size_t>(v) * Qg + lane;
    uint32_t best[C];
#pragma unroll
    for (int c = 0; c < C; ++c) best[c] = ((lsel >> c) & 1u) ? row[32 * c] : 0u;
    gather_edges<W, WK>(g, G, lv, sb, lsel, beg, end, lane, best, pairs, scanned);
    uint64_t nw[W];
#pragma unroll
    for (int i = 0; i < W; ++i) nw[i] = 0;
    // the warp owns v's row this level: the entries read above are unchanged
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const bool imp = ((lsel >> c) & 1u) && best[c] < row[32 * c];
      if (imp) row[32 * c] = best[c];
      nw[c >> 1] |= static_cast<uint64_t>(__ballot_sync(kFull, imp)) << (32 * (c & 1));
    }
    bool app = false;
    if (lane == 0 && mask_any<W>(nw)) {
#pragma unroll
      for (int i = 0; i < W; ++i) {
        if (!nw[i]) continue;
        atomic_or64(lv.fnext + static_cast<size_t>(v) * W + i, nw[i]);
        uni[i] |= nw[i];
        improved += __popcll(nw[i]);
      }
      app = atomicMax(g.stamp + v, lv.level + 1) < lv.level + 1;
    }
    warp_append(app, v, app ? degree_of<OT>(G.row, v) : 0, lv.nlist, lv.ncount, lv.nedges, lane);
  }
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(improved, &g.ctl->lc.improved, lane);
  warp_add(pairs, &g.ctl->lc.sssp_pairs, lane);
  warp_add(scanned, &g.ctl->lc.spull_edges, lane);
  warp_add(verts, &g.ctl->lc.spull_vertices, lane);
}

// Gather level, heavy vertices (in-degree > heavy_degree): a CTA takes a
// chunk of kHeavyChunk in-edges, its warps min-reduce slices into shared
// memory, and the chunk's result is committed with one atomicMin per slot.
template <int W, typename OT, int WK>
__global__ void __launch_bounds__(kBlock) k_sssp_pull_heavy(GroupDev g, DevGraph G) {
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->sdir != kDirPull || G.n_pheavy == 0) return;
  const LevelView lv = level_view(g);
  constexpr int C = 2 * W;
  __shared__ uint32_t s_best[C * 32];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const uint64_t* sb = ctl->gsel;
  const uint32_t lsel = lane_sssp_chunks<W>(ctl, lane);
  const size_t Qg = static_cast<size_t>(g.Qg);
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long improved = 0, pairs = 0;
  unsigned scanned = 0;
  // every heavy vertex is gathered once per launch (all its chunks)
  if (blockIdx.x == 0 && threadIdx.x == 0)
    atomicAdd(&g.ctl->lc.spull_vertices, static_cast<unsigned long long>(G.n_pheavy));
  for (int64_t ch = blockIdx.x; ch < G.pheavy_chunks; ch += gridDim.x) {
    // the chunk's vertex and edge range: independent loads, no search
    const int32_t v = G.pheavy[G.pheavy_ch[ch]];
    const int64_t cb = G.pheavy_cb[ch];
    const int64_t ce = G.pheavy_ce[ch];
    for (int i = threadIdx.x; i < C * 32; i += blockDim.x) s_best[i] = 0xffffffffu;
    __syncthreads();
    const int64_t seg = (ce - cb + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const int64_t wb = cb + wib * seg;
    const int64_t we = min(ce, wb + seg);
    uint32_t best[C];
#pragma unroll
    for (int c = 0; c < C; ++c) best[c] = 0xffffffffu;
    gather_edges<W, WK>(g, G, lv, sb, lsel, wb, we, lane, best, pairs, scanned);
#pragma unroll
    for (int c = 0; c < C; ++c)
      if (best[c] != 0xffffffffu) atomicMin(&s_best[32 * c + lane], best[c]);
    __syncthreads();
    // commit: warp wib takes chunks wib, wib + 8, ...
    bool any = false;
    for (int c = wib; c < C; c += kWarpsPerBlock) {
      const int q = 32 * c + lane;
      bool imp = false;
      if ((lsel >> c) & 1u) {
        const uint32_t b = s_best[q];
        uint32_t* p = g.values + static_cast<size_t>(v) * Qg + q;
        if (b < *p) imp = b < atomicMin(p, b);
      }
      const unsigned m = __ballot_sync(kFull, imp);
      if (m) {
        any = true;
        if (lane == 0) {
          const uint64_t bits = static_cast<uint64_t>(m) << (32 * (c & 1));
          atomic_or64(lv.fnext + static_cast<size_t>(v) * W + (c >> 1), bits);
          uni[c >> 1] |= bits;
          improved += __popc(m);
        }
      }
    }
    bool app = false;
    if (any && lane == 0) app = atomicMax(g.stamp + v, lv.level + 1) < lv.level + 1;
    warp_append(app, v, app ? degree_of<OT>(G.row, v) : 0, lv.nlist, lv.ncount, lv.nedges, lane);
    __syncthreads();
  }
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(improved, &g.ctl->lc.improved, lane);
  warp_add(pairs, &g.ctl->lc.sssp_pairs, lane);
  warp_add(scanned, &g.ctl->lc.spull_edges, lane);
}


// ------------------------------------------------- SSSP gather, vectorised
// The same gather with vector loads, for groups whose rows are 16-byte
// aligned and hold a multiple of the vector width (the usual case): lane l
// owns the kElem consecutive slots (32r + l)*kElem .. +kElem of each part r,
// so a row costs kParts vector loads per lane instead of 2W scalar ones.
// The live in-edges of a 32-edge batch are compacted into shared memory by
// a ballot prefix, and full groups of kSteps edges are gathered without any
// per-load predicate.
template <int W>
struct GatherVec {
  static constexpr int kElem = W == 1 ? 2 : 4;      // slots per vector load
  static constexpr int kParts = 2 * W / kElem;      // vector loads per lane per row
  static constexpr int kSlots = kParts * kElem;     // slots per lane
  static constexpr int kSteps = W <= 2 ? 8 : (W == 4 ? 4 : (W == 8 ? 2 : 1));
  static constexpr int kLanesPerHalf = 32 / kElem;  // lanes covering one 32-bit mask half
};

template <int E>
__device__ __forceinline__ void load_vec_cg(const uint32_t* p, uint32_t* x) {
  if constexpr (E == 4) {
    const uint4 v = __ldcg(reinterpret_cast<const uint4*>(p));
    x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
  } else {
    const uint2 v = __ldcg(reinterpret_cast<const uint2*>(p));
    x[0] = v.x; x[1] = v.y;
  }
}

template <int E>
__device__ __forceinline__ void load_vec(const uint32_t* p, uint32_t* x) {
  if constexpr (E == 4) {
    const uint4 v = *reinterpret_cast<const uint4*>(p);
    x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
  } else {
    const uint2 v = *reinterpret_cast<const uint2*>(p);
    x[0] = v.x; x[1] = v.y;
  }
}

template <int E>
__device__ __forceinline__ void store_vec(uint32_t* p, const uint32_t* x) {
  if constexpr (E == 4) *reinterpret_cast<uint4*>(p) = make_uint4(x[0], x[1], x[2], x[3]);
  else *reinterpret_cast<uint2*>(p) = make_uint2(x[0], x[1]);
}

// best[j] = min(best[j], relax(du[j], w)) for the lane's slots.
template <int WK, int N>
__device__ __forceinline__ void relax_min_row(uint32_t (&best)[N], const uint32_t* du,
                                              uint32_t wbits) {
  if constexpr (WK == kWeightF32) {
#pragma unroll
    for (int j = 0; j < N; ++j) best[j] = min(best[j], gather_relax<WK>(du[j], wbits));
  } else {
    const uint32_t wt = (WK == kWeightU32) ? wbits : 1u;
    const uint32_t lim = ~wt;
#pragma unroll
    for (int j = 0; j < N; ++j) best[j] = min(best[j], min(du[j], lim) + wt);
  }
}

// Lane masks for the vectorised gather: bit r of *parts: the lane's vector of
// part r lies inside the row (slot < Qg) and holds a slot that gathers at this
// level (otherwise the lane neither loads nor commits it: a 32-slot chunk
// without gathering slots is never read); bit j of *slots: slot j of the lane
// gathers.
template <int W>
__device__ __forceinline__ void gather_vec_masks(const uint64_t* gsel, int Qg, int lane,
                                                 uint32_t* parts, uint32_t* slots) {
  using GV = GatherVec<W>;
  uint32_t pm = 0, sm = 0;
#pragma unroll
  for (int r = 0; r < GV::kParts; ++r) {
    const int base = (32 * r + lane) * GV::kElem;
#pragma unroll
    for (int k = 0; k < GV::kElem; ++k) {
      const int q = base + k;
      if (q < Qg && ((gsel[q >> 6] >> (q & 63)) & 1ULL)) sm |= 1u << (r * GV::kElem + k);
    }
    if (base < Qg && ((sm >> (r * GV::kElem)) & ((1u << GV::kElem) - 1u))) pm |= 1u << r;
  }
  *parts = pm;
  *slots = sm;
}

// ORs the lanes' per-slot bits into 64-bit frontier words: `bits` holds the
// lane's kSlots bits (slot r*kElem + k at bit r*kElem + k).  For each part,
// the lane whose slots start a word receives it in words[r] (0 elsewhere).
template <int W>
__device__ __forceinline__ void gather_vec_words(uint32_t bits, int lane,
                                                 uint64_t (&words)[GatherVec<W>::kParts]) {
  using GV = GatherVec<W>;
  constexpr int E = GV::kElem;
  constexpr int L = GV::kLanesPerHalf;
#pragma unroll
  for (int r = 0; r < GV::kParts; ++r) {
    uint32_t h = ((bits >> (r * E)) & ((1u << E) - 1u)) << (E * (lane % L));
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) h |= __shfl_xor_sync(kFull, h, o);
    const uint32_t hi = __shfl_down_sync(kFull, h, L);
    words[r] = (lane % (2 * L) == 0) ? (static_cast<uint64_t>(hi) << 32) | h : 0ULL;
  }
}

// 32-slot chunks that hold a gathering SSSP slot at this level.
template <int W>
__device__ __forceinline__ uint32_t gather_chunks(const uint64_t* gsel) {
  uint64_t gs[W];
#pragma unroll
  for (int i = 0; i < W; ++i) gs[i] = gsel[i];
  return chunk_bits<W>(gs);
}

template <int W>
__device__ __forceinline__ uint32_t gather_chunks(const LevelCtl* ctl) {
  return gather_chunks<W>(ctl->gsel);
}

// Whether the gather screens in-edges by their source's frontier chunks (-1)
// or reads every in-edge's source row whole (the number of gathering slots).
// With the frontier summary: a whole-row gather reads E x (gathering chunks)
// row chunks, a screened one only the live ones, which the summary kernel
// counted (live_chunks); screening pays when fewer than 4/5 of them are live,
// and costs an 8-byte L2 word per in-edge.  Without it (no summary buffer):
// screen when the frontier's out-edges are less than half of all edges or its
// entries are sparse (the previous level improved fewer than 1/32 of the
// frontier's vertices x SSSP slots), reading the sources' W-word masks.
template <int W>
__device__ __forceinline__ int gather_screen_qs(const GroupDev& g, const LevelCtl* ctl,
                                                const LevelView& lv, int64_t E) {
  int qs = 0;
#pragma unroll
  for (int i = 0; i < W; ++i) qs += __popcll(ctl->gsel[i]);
  if (g.fsum != nullptr) {
    const unsigned long long whole =
        static_cast<unsigned long long>(E) * static_cast<unsigned long long>(__popc(gather_chunks<W>(ctl)));
    return 5 * ctl->lc.live_chunks < 4 * whole ? -1 : qs;
  }
  if (2 * ctl->edges[lv.par] < static_cast<unsigned long long>(E)) return -1;
  if (32 * ctl->prev_improved < ctl->count[lv.par] * static_cast<unsigned long long>(qs)) return -1;
  return qs;
}

// Writes the frontier summary of the current frontier's vertices on SSSP
// gather levels and sparse BFS pull levels (other levels return at once), and
// on gather levels counts the live row chunks a screened gather would read
// (out-degree x gathering chunks with a frontier bit).  Words of vertices
// outside the frontier keep an older level's stamp and read as empty.
template <int W, typename OT>
__global__ void __launch_bounds__(kBlock) k_frontier_summary(GroupDev g, DevGraph G) {
  LevelCtl* ctl = g.ctl;
  if (ctl->done) return;
  const LevelView lv = level_view(g);
  const bool sssp = ctl->sdir == kDirPull;
  if (!sssp && !bfs_pull_uses_summary(g, ctl, lv, G.V)) return;
  const unsigned long long n = ctl->count[lv.par];
  const uint64_t stamp = static_cast<uint64_t>(lv.level + 1) << 32;
  const uint32_t gch = gather_chunks<W>(ctl);
  const int lane = threadIdx.x & 31;
  unsigned long long live = 0;
  const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  for (unsigned long long i0 = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31);
       i0 < n; i0 += stride) {
    const unsigned long long i = i0 + lane;
    if (i < n) {
      const int32_t v = lv.list[i];
      uint64_t m[W];
      load_mask<W>(lv.fcur + static_cast<size_t>(v) * W, m);
      const uint32_t cm = chunk_bits<W>(m);
      g.fsum[v] = stamp | cm;
      if (sssp) live += __popc(cm & gch) * degree_of<OT>(G.row, v);
    }
  }
  if (sssp) warp_add(live, &ctl->lc.live_chunks, lane);
}

// Whether the lane reads part r of a source row whose 32-slot chunk bits are
// `cm`.
template <int W>
__device__ __forceinline__ bool chunk_live(uint32_t cm, int r, int lane) {
  constexpr int E = GatherVec<W>::kElem;
  return (cm >> (((32 * r + lane) * E) >> 5)) & 1u;
}

// Gathers in-edges [eb, ee) into best[] (vector layout).  `stage` is this
// warp's 32-entry shared staging array.  All lanes call.
template <int W, int WK, bool kChunks = true>
__device__ __forceinline__ void gather_edges_vec(const GroupDev& g, const DevGraph& G,
                                                 const LevelView& lv, const uint64_t* sb,
                                                 uint32_t pmask, int64_t eb, int64_t ee,
                                                 int lane, int4* stage,
                                                 uint32_t (&best)[GatherVec<W>::kSlots],
                                                 unsigned long long& pairs,
                                                 unsigned& scanned, int screen_qs,
                                                 uint32_t gch) {
  using GV = GatherVec<W>;
  constexpr int E = GV::kElem;
  constexpr int P = GV::kParts;
  constexpr int S = GV::kSteps;
  const size_t Qg = static_cast<size_t>(g.Qg);
  const uint32_t* lanebase = g.values + lane * E;
  for (int64_t e0 = eb; e0 < ee; e0 += 32) {
    const int64_t e = e0 + lane;
    int k = 0;
    int32_t u = 0;
    uint32_t wb = 0;
    uint32_t cm = 0xffffffffu;  // 32-slot chunks of the source row to read
    if (e < ee) {
      u = G.pcol[e];
      wb = weight_bits<WK>(G.pw, e);
      if (screen_qs < 0 && g.fsum != nullptr) {
        // sparse frontier: skip in-edges whose source has no gathering
        // frontier chunk, and the source row's chunks without one, by the
        // frontier summary (pairs are counted per 32-slot chunk)
        cm = summary_chunks(g.fsum, lv.level, u) & gch;
        k = __popc(cm) << 5;
      } else if (screen_qs < 0) {
        // the same from the source's W-word mask
        uint64_t m[W];
        load_mask<W>(lv.fcur + static_cast<size_t>(u) * W, m);
        // the next batch's source masks move to L2 while this batch's rows load
        if (e + 32 < ee) prefetch_l2(lv.fcur + static_cast<size_t>(G.pcol[e + 32]) * W);
#pragma unroll
        for (int i = 0; i < W; ++i) {
          m[i] &= sb[i];
          k += __popcll(m[i]);
        }
        if constexpr (kChunks) cm = chunk_bits<W>(m);
      } else {
        k = screen_qs;  // dense frontier: every in-edge is gathered (no mask load)
      }
      ++scanned;
    }
    pairs += static_cast<unsigned long long>(k);
    const unsigned lm = __ballot_sync(kFull, k > 0);
    if (k > 0)
      stage[__popc(lm & ((1u << lane) - 1u))] =
          make_int4(u, static_cast<int>(wb), 0, kChunks ? static_cast<int>(cm) : -1);
    __syncwarp();
    const int n = __popc(lm);
    int i = 0;
    for (; i + S <= n; i += S) {
      int4 ed[S];
#pragma unroll
      for (int t = 0; t < S; ++t) ed[t] = stage[i + t];
      uint32_t cur[S][GV::kSlots];
#pragma unroll
      for (int t = 0; t < S; ++t) {
        const uint32_t* row = lanebase + static_cast<size_t>(ed[t].x) * Qg;
#pragma unroll
        for (int r = 0; r < P; ++r) {
          if (((pmask >> r) & 1u) && (!kChunks || chunk_live<W>(static_cast<uint32_t>(ed[t].w), r, lane))) {
            load_vec_cg<E>(row + 32 * E * r, &cur[t][r * E]);
          } else {
#pragma unroll
            for (int q = 0; q < E; ++q) cur[t][r * E + q] = 0xffffffffu;
          }
        }
      }
#pragma unroll
      for (int t = 0; t < S; ++t) relax_min_row<WK>(best, cur[t], static_cast<uint32_t>(ed[t].y));
    }
    if (i < n) {
      // the remaining 1..S-1 edges in one step (uniform predicates), so that
      // a short list costs one round trip instead of one per edge
      int4 ed[S];
#pragma unroll
      for (int t = 0; t < S; ++t) ed[t] = stage[i + t < n ? i + t : i];
      uint32_t cur[S][GV::kSlots];
#pragma unroll
      for (int t = 0; t < S; ++t) {
        const uint32_t* row = lanebase + static_cast<size_t>(ed[t].x) * Qg;
#pragma unroll
        for (int r = 0; r < P; ++r) {
          if (i + t < n && ((pmask >> r) & 1u) && (!kChunks || chunk_live<W>(static_cast<uint32_t>(ed[t].w), r, lane))) {
            load_vec_cg<E>(row + 32 * E * r, &cur[t][r * E]);
          } else {
#pragma unroll
            for (int q = 0; q < E; ++q) cur[t][r * E + q] = 0xffffffffu;
          }
        }
      }
#pragma unroll
      for (int t = 0; t < S; ++t) relax_min_row<WK>(best, cur[t], static_cast<uint32_t>(ed[t].y));
    }
    __syncwarp();
  }
}


// Gather level (vectorised), vertices of in-degree <= heavy_degree.
template <int W, typename OT, int WK>
__global__ void __launch_bounds__(kBlock, (W == 4 ? 4 : (W <= 8 ? 3 : 2))) k_sssp_pull_vec(GroupDev g, DevGraph G) {
  using GV = GatherVec<W>;
  constexpr int E = GV::kElem;
  constexpr int P = GV::kParts;
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->sdir != kDirPull) return;
  __shared__ int4 s_stage[kWarpsPerBlock][32];
  const LevelView lv = level_view(g);
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const uint64_t* sb = ctl->gsel;
  uint32_t pmask, smask;
  gather_vec_masks<W>(ctl->gsel, g.Qg, lane, &pmask, &smask);
  const unsigned long long gw = (static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = (static_cast<unsigned long long>(gridDim.x) * blockDim.x) >> 5;
  const size_t Qg = static_cast<size_t>(g.Qg);
  uint32_t uacc = 0;
  unsigned long long improved = 0, pairs = 0;
  unsigned scanned = 0, verts = 0;
  int32_t pend_v = 0;  // lane i: i-th vertex waiting to be appended
  int pend_n = 0;      // uniform
  const int screen_qs = gather_screen_qs<W>(g, ctl, lv, G.E);
  const uint32_t gch = gather_chunks<W>(ctl);
  const unsigned long long V = static_cast<unsigned long long>(G.V);
  // the next vertex's offsets are loaded while the current one is gathered
  int64_t nbeg = 0, nend = 0;
  if (gw < V) {
    nbeg = row_at<OT>(G.prow, static_cast<int64_t>(gw));
    nend = row_at<OT>(G.prow, static_cast<int64_t>(gw) + 1);
  }
  for (unsigned long long vv = gw; vv < V; vv += nwarps) {
    const int32_t v = static_cast<int32_t>(vv);
    const int64_t beg = nbeg, end = nend;
    if (vv + nwarps < V) {
      nbeg = row_at<OT>(G.prow, static_cast<int64_t>(vv + nwarps));
      nend = row_at<OT>(G.prow, static_cast<int64_t>(vv + nwarps) + 1);
    }
    if (end == beg || end - beg > G.heavy_degree) continue;
    if (lane == 0) ++verts;  // one count per vertex, not per lane
    uint32_t* row = g.values + static_cast<size_t>(v) * Qg + lane * E;
    uint32_t best[GV::kSlots];
#pragma unroll
    for (int r = 0; r < P; ++r) {
      if ((pmask >> r) & 1u) {
        load_vec<E>(row + 32 * E * r, &best[r * E]);
      } else {
#pragma unroll
        for (int q = 0; q < E; ++q) best[r * E + q] = 0u;
      }
    }
    gather_edges_vec<W, WK>(g, G, lv, sb, pmask, beg, end, lane, s_stage[wib], best, pairs,
                            scanned, screen_qs, gch);
    // commit (the warp owns v's row this level: the row read above is current)
    uint32_t imp = 0;
#pragma unroll
    for (int r = 0; r < P; ++r) {
      if (!((pmask >> r) & 1u)) continue;
      uint32_t o[E], nv[E];
      load_vec<E>(row + 32 * E * r, o);
      uint32_t b = 0;
#pragma unroll
      for (int q = 0; q < E; ++q) {
        const int j = r * E + q;
        const bool up = ((smask >> j) & 1u) && best[j] < o[q];
        nv[q] = up ? best[j] : o[q];
        b |= static_cast<uint32_t>(up) << q;
      }
      if (b) store_vec<E>(row + 32 * E * r, nv);
      imp |= b << (r * E);
    }
    if (!__any_sync(kFull, imp != 0)) continue;
    improved += __popc(imp);
    uacc |= imp;
    uint64_t words[P];
    gather_vec_words<W>(imp, lane, words);
    // v is this warp's alone during the kernel (earlier kernels of the level
    // are complete, heavy vertices are not in this kernel): its frontier
    // words and stamp need no atomics
#pragma unroll
    for (int r = 0; r < P; ++r) {
      if (words[r]) {
        const int wi = ((32 * r + lane) * E) >> 6;
        lv.fnext[static_cast<size_t>(v) * W + wi] |= words[r];
      }
    }
    if (g.stamp[v] < lv.level + 1) {  // uniform: every lane reads the same word
      __syncwarp();
      if (lane == 0) g.stamp[v] = lv.level + 1;
      // appends are buffered in the lanes and reserved 32 at a time
      if (lane == pend_n) pend_v = v;
      if (++pend_n == 32) {
        flush_appends<OT>(pend_v, pend_n, G, lv, lane);
        pend_n = 0;
      }
    }
  }
  if (pend_n > 0) flush_appends<OT>(pend_v, pend_n, G, lv, lane);
  {
    uint64_t words[P];
    gather_vec_words<W>(uacc, lane, words);
#pragma unroll
    for (int r = 0; r < P; ++r)
      if (words[r]) atomic_or64(lv.nactive + (((32 * r + lane) * E) >> 6), words[r]);
  }
  warp_add(improved, &g.ctl->lc.improved, lane);
  warp_add(pairs, &g.ctl->lc.sssp_pairs, lane);
  warp_add(scanned, &g.ctl->lc.spull_edges, lane);
  warp_add(verts, &g.ctl->lc.spull_vertices, lane);
}

// Owner of in-edge f0 + lane in a chunk whose vertex k starts at prefix
// position pre_k (lane k passes its own pre_k, INT_MAX beyond the chunk;
// every chunk vertex has an in-edge, so the starts are distinct): the last k
// with pre_k <= f0 + lane.  One ballot and one OR-reduction per 32 in-edges
// instead of a binary search per lane.  All lanes call.
__device__ __forceinline__ int chunk_edge_owner(int my_pre, int f0, int lane) {
  const int k0 = __popc(__ballot_sync(kFull, my_pre <= f0)) - 1;
  // bit (pre_k - f0) for the vertices that start inside (f0, f0 + 32)
  const unsigned d = static_cast<unsigned>(my_pre - f0 - 1);
  const unsigned starts = __reduce_or_sync(kFull, d < 31u ? 2u << d : 0u);
  const unsigned upto = lane == 31 ? 0xffffffffu : (2u << lane) - 1u;
  return k0 + __popc(starts & upto);
}

// Gather level (vectorised), light vertices in CTA chunks.  A chunk is a
// run of up to kLightChunkVerts light vertices with at most kLightChunkEdges
// in-edges in total (static table of the pull CSR).  The CTA's warps split
// the chunk's in-edges evenly, across vertex boundaries, so every warp keeps
// several source rows in flight all the time instead of stalling on each
// small vertex's chain of dependent loads; a warp min-reduces its run of one
// vertex into that vertex's row in shared memory, and after a barrier each
// vertex is committed once (compare, store, frontier words, append: no
// atomics, the chunk owns its vertices).  W <= 4 (a row of 64W slots fits
// 32 times in 32 KB of shared memory).  Wider groups (WF = 8 or 16 words)
// are gathered in slices of W words: blockIdx.y is the slice, each CTA owns
// its vertices' slice of the row, and the frontier append is claimed with an
// atomic on the stamp (the slices of a vertex commit in different CTAs).
template <int W, typename OT, int WK, int WF = W>
__global__ void __launch_bounds__(kBlock, 3) k_sssp_pull_chunked(GroupDev g, DevGraph G) {
  static_assert(W <= 4, "chunked gather holds 32 rows of at most 256 slots");
  static_assert(WF % W == 0, "a group is a whole number of slices");
  using GV = GatherVec<W>;
  constexpr int E = GV::kElem;
  constexpr int P = GV::kParts;
  constexpr int S = GV::kSteps < 4 ? GV::kSteps : 4;
  constexpr int R = 64 * W;
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->sdir != kDirPull || G.n_plight_chunks == 0) return;
  const LevelView lv = level_view(g);
  __shared__ __align__(16) uint32_t s_best[kLightChunkVerts * R];
  __shared__ int4 s_stage[kWarpsPerBlock][32];
  __shared__ int32_t s_v[kLightChunkVerts];
  __shared__ int64_t s_beg[kLightChunkVerts];
  __shared__ int32_t s_pre[kLightChunkVerts + 1];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int sl = WF > W ? static_cast<int>(blockIdx.y) : 0;  // slice of W words
  const int s0 = sl * 64 * W;                                  // its first slot
  const uint64_t* sb = ctl->gsel + sl * W;
  uint32_t pmask, smask;
  gather_vec_masks<W>(sb, g.Qg - s0, lane, &pmask, &smask);
  const uint32_t gch = gather_chunks<W>(sb);
  if (gch == 0) return;  // no gathering slot in this slice (uniform over the CTA)
  // screen or read whole rows: one decision for the whole group
  int screen_qs = gather_screen_qs<WF>(g, ctl, lv, G.E);
  if (screen_qs >= 0) {
    screen_qs = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) screen_qs += __popcll(sb[i]);
  }
  const size_t Qg = static_cast<size_t>(g.Qg);
  const uint32_t* lanebase = g.values + s0 + lane * E;
  WarpAppender ap;
  uint32_t uacc = 0;
  unsigned long long improved = 0, pairs = 0;
  unsigned scanned = 0, verts = 0;
  for (int c = blockIdx.x; c < G.n_plight_chunks; c += gridDim.x) {
    const int cs = G.plight_chunk_start[c];
    const int nv = G.plight_chunk_start[c + 1] - cs;
    if (wib == 0) {
      // vertex, first in-edge and in-edge prefix come from the table: three
      // independent loads (no chain through the offsets)
      if (lane < nv) {
        s_v[lane] = G.plight[cs + lane];
        s_beg[lane] = G.plight_beg[cs + lane];
        s_pre[lane + 1] = G.plight_pre[cs + lane];
      }
      if (lane == 0) s_pre[0] = 0;
    }
    for (int i = threadIdx.x; i < nv * R; i += blockDim.x) s_best[i] = 0xffffffffu;
    __syncthreads();
    // the rows the commit reads: the 2W lines of 128 bytes of each vertex's
    // slice move to L2 while the chunk gathers
    {
      const int k = static_cast<int>(threadIdx.x >> 3), ln = static_cast<int>(threadIdx.x & 7);
      if (k < nv && ln < 2 * W && s0 + ln * 32 < g.Qg)
        prefetch_l2(g.values + static_cast<size_t>(s_v[k]) * Qg + s0 + ln * 32);
    }
    const int total = s_pre[nv];
    const int seg = (total + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const int fa = min(total, wib * seg);
    const int fb = min(total, fa + seg);
    uint32_t best[GV::kSlots];
#pragma unroll
    for (int j = 0; j < GV::kSlots; ++j) best[j] = 0xffffffffu;
    int cur_k = -1;
    // adds this warp's run of vertex cur_k into its shared row
    auto flush_row = [&]() {
      uint32_t* row = s_best + cur_k * R;
#pragma unroll
      for (int j = 0; j < GV::kSlots; ++j) {
        if (best[j] != 0xffffffffu) atomicMin(row + (32 * (j / E) + lane) * E + (j % E), best[j]);
        best[j] = 0xffffffffu;
      }
    };
    int4* stage = s_stage[wib];
    for (int f0 = fa; f0 < fb; f0 += 32) {
      const int f = f0 + lane;
      int cnt = 0;
      int32_t u = 0;
      uint32_t wb = 0;
      uint32_t cm = 0xffffffffu;  // 32-slot chunks of the source row to read
      const int k = chunk_edge_owner(lane < nv ? s_pre[lane] : 0x7fffffff, f0, lane);
      if (f < fb) {
        const int64_t e = s_beg[k] + (f - s_pre[k]);
        u = G.pcol[e];
        wb = weight_bits<WK>(G.pw, e);
        if (screen_qs < 0 && g.fsum != nullptr) {
          cm = (summary_chunks(g.fsum, lv.level, u) >> (2 * W * sl)) & gch;
          cnt = __popc(cm) << 5;
        } else if (screen_qs < 0) {
          uint64_t m[W];
          load_mask<W>(lv.fcur + static_cast<size_t>(u) * WF + sl * W, m);
          // the next batch's source masks move to L2 while this batch's rows load
          const int fn = f + 32;
          if (fn < fb) {
            int a = k, b = nv - 1;  // owner of fn: last k' >= k with s_pre[k'] <= fn
            while (a < b) {
              const int mid = (a + b + 1) >> 1;
              if (s_pre[mid] <= fn) a = mid;
              else b = mid - 1;
            }
            prefetch_l2(lv.fcur + static_cast<size_t>(G.pcol[s_beg[a] + (fn - s_pre[a])]) * WF + sl * W);
          }
#pragma unroll
          for (int i = 0; i < W; ++i) {
            m[i] &= sb[i];
            cnt += __popcll(m[i]);
          }
          cm = chunk_bits<W>(m);
        } else {
          cnt = screen_qs;
        }
        if (sl == 0) ++scanned;  // in-edges counted once per group
        if (cnt > 0 && fb - fa <= 32) {
          // a warp whose whole share is one batch (chunks of low in-degree
          // vertices, where the gather waits on latency): the source row's
          // live 128-byte chunks move to L2 now, so that the staged row loads
          // below wait on L2 rather than on DRAM (on longer shares the extra
          // requests slowed the bandwidth-bound dense levels)
          const uint32_t* rb = g.values + static_cast<size_t>(u) * Qg + s0;
          uint32_t lines = cm & gch;
          while (lines) {
            prefetch_l2(rb + 32 * (__ffs(lines) - 1));
            lines &= lines - 1;
          }
        }
      }
      pairs += static_cast<unsigned long long>(cnt);
      const unsigned lm = __ballot_sync(kFull, cnt > 0);
      if (cnt > 0)
        stage[__popc(lm & ((1u << lane) - 1u))] = make_int4(u, static_cast<int>(wb), k, static_cast<int>(cm));
      __syncwarp();
      const int n = __popc(lm);
      for (int i = 0; i < n; i += S) {
        int4 ed[S];
#pragma unroll
        for (int t = 0; t < S; ++t) ed[t] = stage[i + t < n ? i + t : i];
        uint32_t cur[S][GV::kSlots];
#pragma unroll
        for (int t = 0; t < S; ++t) {
          const uint32_t* row = lanebase + static_cast<size_t>(ed[t].x) * Qg;
#pragma unroll
          for (int r = 0; r < P; ++r) {
            if (i + t < n && ((pmask >> r) & 1u) && chunk_live<W>(static_cast<uint32_t>(ed[t].w), r, lane)) {
              load_vec_cg<E>(row + 32 * E * r, &cur[t][r * E]);
            } else {
#pragma unroll
              for (int q = 0; q < E; ++q) cur[t][r * E + q] = 0xffffffffu;
            }
          }
        }
#pragma unroll
        for (int t = 0; t < S; ++t) {
          if (i + t >= n) break;  // uniform
          if (ed[t].z != cur_k) {  // uniform: a new vertex starts
            if (cur_k >= 0) flush_row();
            cur_k = ed[t].z;
          }
          relax_min_row<WK>(best, cur[t], static_cast<uint32_t>(ed[t].y));
        }
      }
      __syncwarp();
    }
    if (cur_k >= 0) flush_row();
    __syncthreads();
    // commit: warp wib takes vertices wib, wib + 8, ...
    for (int k = wib; k < nv; k += kWarpsPerBlock) {
      const int32_t v = s_v[k];
      uint32_t* row = g.values + static_cast<size_t>(v) * Qg + s0 + lane * E;
      const uint32_t* srow = s_best + k * R + lane * E;
      uint32_t imp = 0;
#pragma unroll
      for (int r = 0; r < P; ++r) {
        if (!((pmask >> r) & 1u)) continue;
        uint32_t o[E], b[E], nvv[E];
        load_vec<E>(row + 32 * E * r, o);
        if constexpr (E == 4) {
          const uint4 x = *reinterpret_cast<const uint4*>(srow + 32 * E * r);
          b[0] = x.x; b[1] = x.y; b[2] = x.z; b[3] = x.w;
        } else {
          const uint2 x = *reinterpret_cast<const uint2*>(srow + 32 * E * r);
          b[0] = x.x; b[1] = x.y;
        }
        uint32_t bits = 0;
#pragma unroll
        for (int q = 0; q < E; ++q) {
          const bool up = ((smask >> (r * E + q)) & 1u) && b[q] < o[q];
          nvv[q] = up ? b[q] : o[q];
          bits |= static_cast<uint32_t>(up) << q;
        }
        if (bits) store_vec<E>(row + 32 * E * r, nvv);
        imp |= bits << (r * E);
      }
      if (lane == 0 && sl == 0) ++verts;
      if (!__any_sync(kFull, imp != 0)) continue;
      improved += __popc(imp);
      uacc |= imp;
      uint64_t words[P];
      gather_vec_words<W>(imp, lane, words);
#pragma unroll
      for (int r = 0; r < P; ++r) {
        if (words[r]) {
          const int wi = ((32 * r + lane) * E) >> 6;
          lv.fnext[static_cast<size_t>(v) * WF + sl * W + wi] |= words[r];
        }
      }
      bool fresh;
      if constexpr (WF > W) {
        int old = 0;
        if (lane == 0) old = atomicMax(g.stamp + v, lv.level + 1);
        fresh = __shfl_sync(kFull, old, 0) < lv.level + 1;
      } else {
        fresh = g.stamp[v] < lv.level + 1;  // uniform
        __syncwarp();
        if (fresh && lane == 0) g.stamp[v] = lv.level + 1;
      }
      ap.add<OT>(fresh && lane == 0, v, G, lv, lane);
    }
    __syncthreads();
  }
  ap.flush<OT>(G, lv, lane);
  {
    uint64_t words[P];
    gather_vec_words<W>(uacc, lane, words);
#pragma unroll
    for (int r = 0; r < P; ++r)
      if (words[r]) atomic_or64(lv.nactive + sl * W + (((32 * r + lane) * E) >> 6), words[r]);
  }
  warp_add(improved, &g.ctl->lc.improved, lane);
  warp_add(pairs, &g.ctl->lc.sssp_pairs, lane);
  warp_add(scanned, &g.ctl->lc.spull_edges, lane);
  warp_add(verts, &g.ctl->lc.spull_vertices, lane);
}

// Gather level (vectorised), heavy vertices: CTA per 2048-edge chunk, warps
// min-reduce their slices into shared memory, one atomicMin per slot.
// kMode 0: every gather level, whole source rows; 1: only levels that read
// whole rows (dense entries); 2: only screened levels (sparse entries), with
// the source rows' 32-slot chunks without frontier bits skipped.  Modes 1 and 2
// are launched together (groups of <= 256 slots) so that each level runs the
// variant whose register budget suits it.
template <int W, typename OT, int WK, int kMode>
__global__ void __launch_bounds__(kBlock) k_sssp_pull_heavy_vec(GroupDev g, DevGraph G) {
  using GV = GatherVec<W>;
  constexpr int E = GV::kElem;
  constexpr int C = 2 * W;
  const LevelCtl* ctl = g.ctl;
  if (ctl->done || ctl->sdir != kDirPull || G.n_pheavy == 0) return;
  const LevelView lv = level_view(g);
  __shared__ uint32_t s_best[C * 32];
  __shared__ int4 s_stage[kWarpsPerBlock][32];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const uint64_t* sb = ctl->gsel;
  uint32_t pmask, smask;
  gather_vec_masks<W>(ctl->gsel, g.Qg, lane, &pmask, &smask);
  const uint32_t lsel = lane_sssp_chunks<W>(ctl, lane);
  const int screen_qs = gather_screen_qs<W>(g, ctl, lv, G.E);
  const uint32_t gch = gather_chunks<W>(ctl);
  if ((kMode == 1 && screen_qs < 0) || (kMode == 2 && screen_qs >= 0)) return;
  const size_t Qg = static_cast<size_t>(g.Qg);
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  unsigned long long improved = 0, pairs = 0;
  unsigned scanned = 0;
  // every heavy vertex is gathered once per launch (all its chunks)
  if (blockIdx.x == 0 && threadIdx.x == 0)
    atomicAdd(&g.ctl->lc.spull_vertices, static_cast<unsigned long long>(G.n_pheavy));
  for (int64_t ch = blockIdx.x; ch < G.pheavy_chunks; ch += gridDim.x) {
    // the chunk's vertex and edge range: independent loads, no search
    const int32_t v = G.pheavy[G.pheavy_ch[ch]];
    const int64_t cb = G.pheavy_cb[ch];
    const int64_t ce = G.pheavy_ce[ch];
    for (int i = threadIdx.x; i < C * 32; i += blockDim.x) s_best[i] = 0xffffffffu;
    __syncthreads();
    const int64_t seg = (ce - cb + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const int64_t wb = cb + wib * seg;
    const int64_t we = min(ce, wb + seg);
    uint32_t best[GV::kSlots];
#pragma unroll
    for (int j = 0; j < GV::kSlots; ++j) best[j] = 0xffffffffu;
    gather_edges_vec<W, WK, kMode == 2>(g, G, lv, sb, pmask, wb, we, lane, s_stage[wib], best,
                                        pairs, scanned, screen_qs, gch);
#pragma unroll
    for (int j = 0; j < GV::kSlots; ++j) {
      const int q = (32 * (j / E) + lane) * E + (j % E);
      if (((smask >> j) & 1u) && best[j] != 0xffffffffu) atomicMin(&s_best[q], best[j]);
    }
    __syncthreads();
    // commit: warp wib takes 32-slot chunks wib, wib + 8, ... (lane j <-> slot 32c + j)
    bool any = false;
    for (int c = wib; c < C; c += kWarpsPerBlock) {
      const int q = 32 * c + lane;
      bool imp = false;
      if ((lsel >> c) & 1u) {
        const uint32_t b = s_best[q];
        uint32_t* p = g.values + static_cast<size_t>(v) * Qg + q;
        if (b < *p) imp = b < atomicMin(p, b);
      }
      const unsigned m = __ballot_sync(kFull, imp);
      if (m) {
        any = true;
        if (lane == 0) {
          const uint64_t bits = static_cast<uint64_t>(m) << (32 * (c & 1));
          atomic_or64(lv.fnext + static_cast<size_t>(v) * W + (c >> 1), bits);
          uni[c >> 1] |= bits;
          improved += __popc(m);
        }
      }
    }
    bool app = false;
    if (any && lane == 0) app = atomicMax(g.stamp + v, lv.level + 1) < lv.level + 1;
    // one append per improved vertex-chunk: rare, a plain warp append
    warp_append(app, v, app ? degree_of<OT>(G.row, v) : 0, lv.nlist, lv.ncount, lv.nedges, lane);
    __syncthreads();
  }
  flush_union<W>(uni, lv.nactive, lane);
  warp_add(improved, &g.ctl->lc.improved, lane);
  warp_add(pairs, &g.ctl->lc.sssp_pairs, lane);
  warp_add(scanned, &g.ctl->lc.spull_edges, lane);
}

// --------------------------------------------------------- level control
__device__ __forceinline__ int32_t decide_dir(const LevelCtl* ctl, unsigned long long count,
                                              unsigned long long edges, bool has_bfs) {
  if (!has_bfs) return kDirPush;
  if (ctl->forced_dir >= 0) return ctl->forced_dir;
  if (ctl->mode == 0) return kDirPush;   // CGP_MODE_PUSH
  if (ctl->mode == 1) return kDirPull;   // CGP_MODE_PULL
  return (edges >= ctl->pull_edge_threshold || count >= ctl->pull_vertex_threshold)
             ? kDirPull : kDirPush;
}

// SSSP direction of the next level: gather once the frontier's edges reach
// the threshold (dense levels), scatter otherwise.
template <int W>
__device__ __forceinline__ bool any_bits(const uint64_t* m) {
  uint64_t a = 0;
  for (int i = 0; i < W; ++i) a |= m[i];
  return a != 0;
}

// Group-wide SSSP direction of a level whose frontier has `count` vertices
// and `edges` out-edges.  Hybrid: gather when the edges reach the edge
// threshold and the estimated (edge, slot) pairs a scatter would relax — the
// previous level's improvements x the frontier's mean out-degree — reach
// sssp_pull_pair_unit per SSSP 32-slot chunk: a scatter costs per pair, a
// gather per (in-edge, gathering chunk), so a wide group whose frontier
// carries one or two bits per vertex (a grid's first and last levels) keeps
// scattering although its frontier touches half the edges.
template <int W>
__device__ __forceinline__ int32_t decide_sdir(const LevelCtl* ctl, unsigned long long count,
                                               unsigned long long edges) {
  if (!any_bits<W>(ctl->sssp_bits) || !ctl->sssp_gather) return kDirPush;
  if (ctl->forced_dir >= 0) return ctl->forced_dir;
  if (ctl->mode == 0) return kDirPush;
  if (ctl->mode == 1) return kDirPull;
  if (edges < ctl->sssp_pull_edge_threshold) return kDirPush;
  if (ctl->sssp_pull_pair_unit > 0) {
    int chunks = 0;
    for (int i = 0; i < W; ++i)
      chunks += (static_cast<uint32_t>(ctl->sssp_bits[i]) != 0u) + ((ctl->sssp_bits[i] >> 32) != 0ULL);
    const double pairs = static_cast<double>(ctl->prev_improved) * static_cast<double>(edges) /
                         static_cast<double>(count > 0 ? count : 1ULL);
    if (pairs < static_cast<double>(ctl->sssp_pull_pair_unit) * chunks) return kDirPush;
  }
  return kDirPull;
}

// Splits the SSSP slots of the next level into gathering (gsel) and
// scattering (ssel) ones.  Group-wide by default (every slot takes
// `group_dir`); with chunk_dir in hybrid mode each 32-slot chunk gathers when
// the out-edges of the next frontier's vertices that carry one of its bits
// (cedges, summed by k_chunk_census) reach the gather threshold and the
// chunk's (edge, slot) pairs (cpairs) reach sssp_pull_pair_unit, so a few
// queries in their dense phase do not make every other slot gather too, and a
// chunk whose last improvements are few scatters them.  Consumes (zeroes)
// cedges and cpairs.
template <int W>
__device__ __forceinline__ void split_sssp_slots(LevelCtl* ctl, int32_t group_dir) {
  const bool per_chunk = ctl->chunk_dir && ctl->mode == 2 && ctl->forced_dir < 0 &&
                         ctl->sssp_gather;
  bool g_any = false, s_any = false;
  for (int i = 0; i < W; ++i) {
    uint64_t gm = 0;
    if (per_chunk) {
      for (int h = 0; h < 2; ++h) {
        const uint64_t half = 0xffffffffULL << (32 * h);
        // as the group rule: enough frontier edges, and enough (edge, slot)
        // pairs that a scatter would cost more than the chunk's gather
        if (ctl->cedges[2 * i + h] >= ctl->sssp_pull_edge_threshold &&
            (ctl->sssp_pull_pair_unit == 0 || ctl->cpairs[2 * i + h] >= ctl->sssp_pull_pair_unit))
          gm |= half;
      }
    } else if (group_dir == kDirPull) {
      gm = ~0ULL;
    }
    ctl->gsel[i] = ctl->sssp_bits[i] & gm;
    ctl->ssel[i] = ctl->sssp_bits[i] & ~gm;
    g_any |= ctl->gsel[i] != 0;
    s_any |= ctl->ssel[i] != 0;
    for (int h = 0; h < 2; ++h) {
      ctl->sssp_chunk_levels += static_cast<uint32_t>(ctl->sssp_bits[i] >> (32 * h)) != 0u;
      ctl->gather_chunk_levels += static_cast<uint32_t>(ctl->gsel[i] >> (32 * h)) != 0u;
    }
  }
  for (int c = 0; c < 2 * kMaxW; ++c) ctl->cedges[c] = ctl->cpairs[c] = 0;
  ctl->sdir = g_any ? kDirPull : kDirPush;
  ctl->sscatter = s_any ? 1 : 0;
}

// Expand mask for `level`: k-hop slots stop once their depth reaches k.
template <int W>
__device__ void compute_expand(LevelCtl* ctl, const SlotDev* slots, int Qg, int level) {
  for (int i = 0; i < W; ++i) ctl->expand[i] = ~0ULL;
  for (int q = 0; q < Qg; ++q) {
    const SlotDev s = slots[q];
    if (s.kind == 3 && level - s.base >= s.k) ctl->expand[q >> 6] &= ~(1ULL << (q & 63));
  }
}

// End of a level (one thread): profile, convergence, and the set-up of the
// next level (counter reset, direction, expand mask).
template <int W>
__device__ void level_end(GroupDev& g) {
  LevelCtl* ctl = g.ctl;
  if (ctl->done) return;
  const int l = ctl->level;
  const int par = l & 1;
  const unsigned long long nextc = ctl->count[par ^ 1];
  if (g.prof != nullptr && l < ctl->profile_cap) {
    LevelProfile p;
    p.level = l;
    p.dir = ctl->dir;
    p.frontier = ctl->count[par];
    p.edges = ctl->edges[par];
    p.next = nextc;
    p.active0 = ctl->active[par ^ 1][0];
    p.new_pairs = ctl->lc.new_pairs;
    p.pull_vertices = ctl->lc.pull_vertices;
    p.pull_edges = ctl->lc.pull_edges;
    p.sssp_pairs = ctl->lc.sssp_pairs;
    p.sssp_active = ctl->lc.sssp_active;
    p.improved = ctl->lc.improved;
    p.spull_vertices = ctl->lc.spull_vertices;
    p.spull_edges = ctl->lc.spull_edges;
    p.sdir = ctl->sdir;
    p.reserved = 0;
    g.prof[l] = p;
  }
  ctl->total.new_pairs += ctl->lc.new_pairs;
  ctl->total.pull_vertices += ctl->lc.pull_vertices;
  ctl->total.pull_edges += ctl->lc.pull_edges;
  ctl->total.sssp_pairs += ctl->lc.sssp_pairs;
  ctl->total.sssp_active += ctl->lc.sssp_active;
  ctl->total.improved += ctl->lc.improved;
  ctl->prev_improved = ctl->lc.improved;
  ctl->prev_pull_edges = ctl->lc.pull_edges;
  ctl->prev_dir = ctl->dir;
  ctl->total.spull_vertices += ctl->lc.spull_vertices;
  ctl->total.spull_edges += ctl->lc.spull_edges;
  ctl->lc = LevelCounters{};
  ctl->dense_count = 0;
  ctl->hq_packed = 0;
  ctl->total_frontier += ctl->count[par];
  ctl->total_edges += ctl->edges[par];
  if (ctl->dir == kDirPush) ctl->push_levels++;
  else ctl->pull_levels++;
  ctl->level = l + 1;
  // Set up level l+1 even when it is empty, so that a serving loop can add
  // sources to it and resume.
  ctl->prev_count = ctl->count[par];
  ctl->count[par] = 0;
  ctl->edges[par] = 0;
  for (int i = 0; i < W; ++i) ctl->active[par][i] = 0;
  compute_expand<W>(ctl, g.slots, g.Qg, l + 1);
  ctl->dir = decide_dir(ctl, nextc, ctl->edges[par ^ 1], any_bits<W>(ctl->bfs_bits));
  split_sssp_slots<W>(ctl, decide_sdir<W>(ctl, nextc, ctl->edges[par ^ 1]));
  if (nextc == 0 || (ctl->max_iterations > 0 && l + 1 >= ctl->max_iterations)) {
    ctl->done = 1;
    return;
  }
  // Pauses (done = 2): depth planes hold depths < 2^num_planes and level l+1
  // writes depth l+2; or the caller asked to stop at halt_level.  The host
  // resumes by clearing `done`.
  if (ctl->num_planes > 0 && ((l + 2) >> ctl->num_planes) != 0) {
    ctl->status |= kStatusPlanesExhausted;
    ctl->done = 2;
  }
  if (ctl->halt_level >= 0 && l + 1 >= ctl->halt_level) ctl->done = 2;
}

template <int W>
__global__ void k_level_end(GroupDev g) {
  if (threadIdx.x == 0) level_end<W>(g);
}

// Per 32-slot chunk, the out-edges of the next frontier's vertices that carry
// an SSSP bit of the chunk (input of the per-chunk direction decision).  Runs
// after the level's kernels, before its level end: each lane takes a vertex
// of the next frontier list, the warp sums its chunks, lane 0 adds them.
template <int W, typename OT>
__global__ void __launch_bounds__(kBlock) k_chunk_census(GroupDev g, DevGraph G) {
  LevelCtl* ctl = g.ctl;
  if (ctl->done || !ctl->chunk_dir) return;
  const LevelView lv = level_view(g);
  const unsigned long long n = *lv.ncount;
  const int lane = threadIdx.x & 31;
  unsigned long long acc[2 * W], pacc[2 * W];
#pragma unroll
  for (int c = 0; c < 2 * W; ++c) acc[c] = pacc[c] = 0;
  const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  for (unsigned long long i0 = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31);
       i0 < n; i0 += stride) {
    const unsigned long long i = i0 + lane;
    if (i < n) {
      const int32_t v = lv.nlist[i];
      const unsigned long long d = degree_of<OT>(G.row, v);
      uint64_t m[W];
      load_mask<W>(lv.fnext + static_cast<size_t>(v) * W, m);
#pragma unroll
      for (int w = 0; w < W; ++w) {
        const uint64_t x = m[w] & ctl->sssp_bits[w];
        const int lo = __popc(static_cast<uint32_t>(x)), hi = __popc(static_cast<uint32_t>(x >> 32));
        if (lo) acc[2 * w] += d;
        if (hi) acc[2 * w + 1] += d;
        pacc[2 * w] += d * static_cast<unsigned long long>(lo);
        pacc[2 * w + 1] += d * static_cast<unsigned long long>(hi);
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 2 * W; ++c) {
    unsigned long long x = acc[c], y = pacc[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_xor_sync(kFull, x, o);
      y += __shfl_xor_sync(kFull, y, o);
    }
    if (lane == 0 && x) {
      atomicAdd(&ctl->cedges[c], x);
      atomicAdd(&ctl->cpairs[c], y);
    }
  }
}

// Level end inside a device-looped CUDA graph (a WHILE conditional node whose
// body is one level): sets the loop condition from the done flag, so the
// whole traversal runs without the host.  A traversal that is still running
// at `level_cap` levels (more than any converging BFS/SSSP needs) stops with
// kStatusLevelCap instead of looping on.
template <int W>
__global__ void k_level_end_loop(GroupDev g, cudaGraphConditionalHandle loop, int32_t level_cap) {
  if (threadIdx.x != 0) return;
  level_end<W>(g);
  LevelCtl* ctl = g.ctl;
  if (ctl->done == 0 && ctl->level >= level_cap) {
    ctl->status |= kStatusLevelCap;
    ctl->done = 3;
  }
  cudaGraphSetConditional(loop, ctl->done == 0 ? 1u : 0u);
}

// Seeds the sources of every slot (one block).  Level 0 starts afterwards.
template <int W, typename OT>
__global__ void k_seed(GroupDev g, DevGraph G) {
  LevelCtl* ctl = g.ctl;
  const int lane = threadIdx.x & 31;
  uint64_t uni[W];
#pragma unroll
  for (int i = 0; i < W; ++i) uni[i] = 0;
  for (int base = threadIdx.x & ~31; base < g.Qg; base += blockDim.x) {
    const int q = base + lane;
    bool app = false;
    int32_t src = 0;
    uint64_t deg = 0;
    if (q < g.Qg) {
      const SlotDev s = g.slots[q];
      if (s.kind != 2 && s.source >= 0) {  // WCC slots are not traversal slots
        src = s.source;
        const uint64_t bit = 1ULL << (q & 63);
        if (s.kind != 1) atomic_or64(g.visited + static_cast<size_t>(src) * W + (q >> 6), bit);
        atomic_or64(g.fbuf0 + static_cast<size_t>(src) * W + (q >> 6), bit);
        if (g.values != nullptr) g.values[static_cast<size_t>(src) * g.Qg + q] = 0u;
        uni[q >> 6] |= bit;
        app = atomicMax(g.stamp + src, 0) < 0;
        deg = degree_of<OT>(G.row, src);
      }
    }
    warp_append(app, src, deg, g.list0, &ctl->count[0], &ctl->edges[0], lane);
  }
  flush_union<W>(uni, ctl->active[0], lane);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    compute_expand<W>(ctl, g.slots, g.Qg, 0);
    ctl->dir = decide_dir(ctl, ctl->count[0], ctl->edges[0], any_bits<W>(ctl->bfs_bits));
    // the sources' level: every slot starts with the group's direction
    split_sssp_slots<W>(ctl, decide_sdir<W>(ctl, ctl->count[0], ctl->edges[0]));
    if (ctl->count[0] == 0) ctl->done = 1;
  }
}

// --------------------------------------------------------------- output
// Fills the working values with each slot's "unreached" marker, or with
// `uniform` everywhere when it is nonzero (the serving layout, where a slot
// changes kind between requests).  Warp per vertex row, lanes over slots.
static __global__ void k_fill_values(uint32_t* values, const SlotDev* slots, int Qg,
                                     int64_t V, uint32_t f32_inf_for_sssp, uint32_t uniform) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t v = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; v < V;
       v += warps) {
    uint32_t* row = values + static_cast<size_t>(v) * Qg;
    for (int q = lane; q < Qg; q += 32) {
      uint32_t x = uniform;
      if (!uniform) {
        const int kind = slots[q].kind;
        x = kind == 1 ? f32_inf_for_sssp : (kind == 2 ? 0u : 0x7fffffffu);
      }
      row[q] = x;
    }
  }
}

// Depth planes -> int32 depths (INT32_MAX where the visited bit is clear).
// Vertex-major output: warp per vertex, lanes over queries (coalesced row
// writes).  Query-major output: blockIdx.y walks queries, threads walk
// vertices (coalesced column writes).
template <int W>
__device__ __forceinline__ uint32_t plane_depth(const uint64_t* visited, const uint64_t* planes,
                                                int K, int64_t V, int64_t v, int q) {
  const size_t word = static_cast<size_t>(v) * W + (q >> 6);
  const uint64_t bit = 1ULL << (q & 63);
  if (!(visited[word] & bit)) return 0x7fffffffu;
  uint32_t d = 0;
  for (int b = 0; b < K; ++b)
    if (planes[static_cast<size_t>(b) * V * W + word] & bit) d |= 1u << b;
  return d;
}

template <int W>
__global__ void k_materialize_planes(const uint64_t* visited, const uint64_t* planes,
                                     int K, int64_t V, int Qg, OutMap om, int query_major) {
  if (query_major) {
    for (int q = blockIdx.y; q < Qg; q += gridDim.y) {
      uint32_t* col = om.out + static_cast<int64_t>(om.qmap[q]) * om.sq;
      for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
           v += static_cast<int64_t>(gridDim.x) * blockDim.x)
        col[v * om.sv] = plane_depth<W>(visited, planes, K, V, v, q);
    }
    return;
  }
  if (blockIdx.y != 0) return;
  // vertex-major: each lane owns 8 consecutive queries of a 256-query block,
  // loads their visited word and the K plane words once, and writes the 8
  // depths (two 16-byte stores when the columns are contiguous and aligned).
  const int lane = threadIdx.x & 31;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  const bool vec = om.qmap_contiguous && (om.sv % 4 == 0) && om.sq == 1 && (om.qmap[0] % 4 == 0);
  for (int64_t v = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; v < V;
       v += warps) {
    uint32_t* row = om.out + v * om.sv;
    for (int q0 = 8 * lane; q0 < Qg; q0 += 256) {
      const size_t word = static_cast<size_t>(v) * W + (q0 >> 6);
      const int sh = q0 & 63;
      const uint32_t vis = static_cast<uint32_t>(visited[word] >> sh) & 0xffu;
      uint32_t d[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) d[j] = 0;
      // the first 8 planes are loaded together, then folded in
      uint64_t pw[8];
#pragma unroll
      for (int b = 0; b < 8; ++b)
        pw[b] = b < K ? planes[static_cast<size_t>(b) * V * W + word] : 0ULL;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const uint32_t pl = static_cast<uint32_t>(pw[b] >> sh) & 0xffu;
#pragma unroll
        for (int j = 0; j < 8; ++j) d[j] |= ((pl >> j) & 1u) << b;
      }
      for (int b = 8; b < K; ++b) {
        const uint32_t pl =
            static_cast<uint32_t>(planes[static_cast<size_t>(b) * V * W + word] >> sh) & 0xffu;
#pragma unroll
        for (int j = 0; j < 8; ++j) d[j] |= ((pl >> j) & 1u) << b;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (!((vis >> j) & 1u)) d[j] = 0x7fffffffu;
      if (vec && q0 + 8 <= Qg) {
        uint4* dst = reinterpret_cast<uint4*>(row + om.qmap[q0]);
        dst[0] = make_uint4(d[0], d[1], d[2], d[3]);
        dst[1] = make_uint4(d[4], d[5], d[6], d[7]);
      } else {
        for (int j = 0; j < 8 && q0 + j < Qg; ++j)
          row[static_cast<int64_t>(om.qmap[q0 + j]) * om.sq] = d[j];
      }
    }
  }
}

// Working values -> output mapping (skips WCC slots); same mappings.
static __global__ void k_copy_values(const uint32_t* values, const SlotDev* slots, int64_t V,
                                     int Qg, OutMap om, int query_major) {
  if (query_major) {
    for (int q = blockIdx.y; q < Qg; q += gridDim.y) {
      if (slots[q].kind == 2) continue;
      uint32_t* col = om.out + static_cast<int64_t>(om.qmap[q]) * om.sq;
      for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
           v += static_cast<int64_t>(gridDim.x) * blockDim.x)
        col[v * om.sv] = values[static_cast<size_t>(v) * Qg + q];
    }
    return;
  }
  if (blockIdx.y != 0) return;
  const int lane = threadIdx.x & 31;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t v = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; v < V;
       v += warps) {
    const uint32_t* src = values + static_cast<size_t>(v) * Qg;
    uint32_t* row = om.out + v * om.sv;
    for (int q = lane; q < Qg; q += 32)
      if (slots[q].kind != 2) row[static_cast<int64_t>(om.qmap[q]) * om.sq] = src[q];
  }
}

}  // namespace dev
}  // namespace cgp
