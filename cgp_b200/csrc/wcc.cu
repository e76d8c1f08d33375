// Weakly connected components by min-label hooking (union-find).
//
// The reference runs WCC as label propagation inside the frontier loop
// (init_wcc_all_vertices_kernel, hybrid_engine.hxx:95-123, min-reduce push),
// which needs O(diameter) levels.  Its fixpoint is the minimum vertex id of
// each component (cpu_wcc, puercgp/examples/mtx_loader.hxx:328-356).  Here the
// same labels come from one union-find pass: roots are always linked under
// the smaller root, so every root is its component's minimum id, followed by
// a pointer-jumping pass that writes label[v] = root(v).
#include "engine.h"

namespace cgp {
namespace {

using namespace dev;

__global__ void k_uf_init(int32_t* parent, int64_t V) {
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
       v += static_cast<int64_t>(gridDim.x) * blockDim.x)
    parent[v] = static_cast<int32_t>(v);
}

// Root of x; shortens the path on the way (parent[x] < x for non-roots, so
// racing shortcuts only ever point further up the same tree).
__device__ __forceinline__ int32_t uf_find(int32_t* parent, int32_t x) {
  volatile int32_t* p = parent;
  int32_t cur = p[x];
  if (cur == x) return x;
  int32_t prev = x;
  for (;;) {
    const int32_t next = p[cur];
    if (next == cur) break;
    p[prev] = next;
    prev = cur;
    cur = next;
  }
  return cur;
}

// Joins the sets of a and b, linking the larger root under the smaller.
__device__ __forceinline__ void uf_union(int32_t* parent, int32_t a, int32_t b) {
  int32_t ra = uf_find(parent, a);
  int32_t rb = uf_find(parent, b);
  while (ra != rb) {
    if (ra < rb) {
      const int32_t t = ra;
      ra = rb;
      rb = t;
    }
    // ra > rb: try to hang ra below rb
    const int32_t old = atomicCAS(parent + ra, ra, rb);
    if (old == ra) return;
    ra = uf_find(parent, old);
    rb = uf_find(parent, rb);
  }
}

// Every CSR entry u->v joins u and v.  On a symmetric CSR each undirected
// edge is visited once (v < u).  Warp per tile of 32 vertices; vertices with
// more than 32 entries are walked by the whole warp.
template <typename OT>
__global__ void __launch_bounds__(kBlock) k_uf_hook(const void* row, const int32_t* col,
                                                    int32_t* parent, int64_t V, int symmetric) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t tile = gw; tile * 32 < V; tile += nw) {
    const int64_t u = tile * 32 + lane;
    int64_t beg = 0, end = 0;
    if (u < V) {
      beg = row_at<OT>(row, u);
      end = row_at<OT>(row, u + 1);
    }
    if (end - beg <= 32) {
      for (int64_t e = beg; e < end; ++e) {
        const int32_t v = col[e];
        if (!symmetric || v < u) uf_union(parent, static_cast<int32_t>(u), v);
      }
    }
    unsigned big = __ballot_sync(kFull, end - beg > 32);
    while (big) {
      const int src = __ffs(big) - 1;
      big &= big - 1;
      const int64_t bu = __shfl_sync(kFull, u, src);
      const int64_t bb = __shfl_sync(kFull, beg, src);
      const int64_t be = __shfl_sync(kFull, end, src);
      for (int64_t e = bb + lane; e < be; e += 32) {
        const int32_t v = col[e];
        if (!symmetric || v < bu) uf_union(parent, static_cast<int32_t>(bu), v);
      }
    }
  }
}

// Root of x without shortening the path.  The label pass writes roots into
// the parent array itself, so it must not also store shortcuts: a late
// shortcut store to parent[y] could replace y's finished label (its root)
// with an intermediate ancestor.
__device__ __forceinline__ int32_t uf_root(const int32_t* parent, int32_t x) {
  const volatile int32_t* p = parent;
  int32_t cur = x;
  for (;;) {
    const int32_t next = p[cur];
    if (next == cur) return cur;
    cur = next;
  }
}

// labels[v] = root(v), in place over the parent array: each entry is written
// once, by its own thread, with an ancestor of v, so concurrent readers still
// follow valid parent chains.
__global__ void k_uf_labels(int32_t* parent, int64_t V) {
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
       v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t r = uf_root(parent, static_cast<int32_t>(v));
    reinterpret_cast<volatile int32_t*>(parent)[v] = r;
  }
}

__global__ void k_broadcast(const uint32_t* labels, int64_t V, OutMap om, int colidx) {
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
       v += static_cast<int64_t>(gridDim.x) * blockDim.x)
    om.out[v * om.sv + static_cast<int64_t>(colidx) * om.sq] = labels[v];
}

}  // namespace

void wcc_labels(GraphImpl* g, uint32_t* labels, cudaStream_t s) {
  // parent array lives in `labels` itself (int32 view); the final pass
  // rewrites every entry with its root.
  int32_t* parent = reinterpret_cast<int32_t*>(labels);
  const int blocks = g->num_sms * 8;
  k_uf_init<<<blocks, kBlock, 0, s>>>(parent, g->V);
  if (g->offset_bytes == 8)
    k_uf_hook<int64_t><<<blocks, kBlock, 0, s>>>(g->row.p, g->col.as<int32_t>(), parent, g->V,
                                                g->symmetric ? 1 : 0);
  else
    k_uf_hook<int32_t><<<blocks, kBlock, 0, s>>>(g->row.p, g->col.as<int32_t>(), parent, g->V,
                                                g->symmetric ? 1 : 0);
  k_uf_labels<<<blocks, kBlock, 0, s>>>(parent, g->V);
  ck(cudaGetLastError(), "wcc");
}

void broadcast_labels(const uint32_t* labels, int64_t V, OutMap om, int col, cudaStream_t s) {
  k_broadcast<<<256, kBlock, 0, s>>>(labels, V, om, col);
  ck(cudaGetLastError(), "wcc broadcast");
}

}  // namespace cgp
