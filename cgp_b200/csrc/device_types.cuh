// Device-side data structures of the traversal engine, shared by every
// translation unit (no kernels here).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace cgp {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBlock = 256;
constexpr int kWarpsPerBlock = kBlock / 32;
constexpr int kHeavyChunk = 2048;  // edges of a heavy vertex per CTA work item
constexpr int kMaxW = 16;
constexpr int kMaxPlanes = 24;
constexpr int kLightChunkVerts = 32;    // light vertices per chunked-gather CTA item
constexpr int kLightChunkEdges = 2048;  // and their in-edges

enum : int32_t { kDirPush = 0, kDirPull = 1 };
enum : int32_t { kDepthNone = 0, kDepthDirect = 1, kDepthPlanes = 2 };
enum : int32_t { kWeightNone = 0, kWeightU32 = 1, kWeightF32 = 2 };

// status bits reported back to the host
enum : uint32_t {
  kStatusPlanesExhausted = 1u,  // depth planes too few for the level reached
  kStatusLevelCap = 2u,         // a device-looped traversal reached its level cap
  kStatusQueueOverflow = 4u,    // the heavy frontier queue was full (entry dropped)
};

struct LevelProfile {
  int32_t level;
  int32_t dir;
  unsigned long long frontier;      // U_l: unique frontier vertices
  unsigned long long edges;         // D_l: their out-degree sum
  unsigned long long next;          // U_{l+1}
  unsigned long long active0;       // next-frontier slot bits, first word
  unsigned long long new_pairs;     // N_l: (query, vertex) pairs newly reached (BFS bits)
  unsigned long long pull_vertices; // P_l: vertices scanned by a pull level
  unsigned long long pull_edges;    // S_l: in-edges read before early exit
  unsigned long long sssp_pairs;    // A_l: (edge, active query) relaxations attempted
  unsigned long long sssp_active;   // sum over frontier vertices of active SSSP bits
  unsigned long long improved;      // SSSP (query, vertex) improvements
  unsigned long long spull_vertices; // vertices an SSSP gather level scanned
  unsigned long long spull_edges;    // in-edges an SSSP gather level scanned
  int32_t sdir;                     // SSSP direction of the level (push / gather)
  int32_t reserved;
};

// Per-level work counters (reset by the level-end kernel).
struct LevelCounters {
  unsigned long long new_pairs;
  unsigned long long pull_vertices;
  unsigned long long pull_edges;
  unsigned long long sssp_pairs;
  unsigned long long sssp_active;
  unsigned long long improved;
  unsigned long long spull_vertices;
  unsigned long long spull_edges;
  unsigned long long live_chunks;  // sum over frontier vertices of out-degree x gathering
                                   // chunks with a frontier bit (row chunks a screened
                                   // gather reads)
};

// Control block of one traversal group (device memory).
struct LevelCtl {
  unsigned long long count[2];  // unique frontier sizes by level parity
  unsigned long long edges[2];  // sum of out-degrees of those frontiers
  unsigned long long prev_count;
  unsigned long long total_frontier;
  unsigned long long total_edges;
  uint64_t active[2][kMaxW];    // OR of the frontier masks by parity
  uint64_t expand[kMaxW];       // bits allowed to expand at the current level
  uint64_t bfs_bits[kMaxW];     // slots with visited-mask semantics (BFS, k-hop)
  uint64_t sssp_bits[kMaxW];    // slots with min-reduce semantics (SSSP)
  uint64_t gsel[kMaxW];         // SSSP slots that gather (pull) at the current level
  uint64_t ssel[kMaxW];         // SSSP slots that scatter (push) at the current level
  unsigned long long cpairs[2 * kMaxW];  // per 32-slot chunk: (out-edge, SSSP bit) pairs of
                                         // the next frontier (what a scatter would relax)
  unsigned long long cedges[2 * kMaxW];  // per 32-slot chunk: out-edges of the next
                                         // frontier's vertices with an SSSP bit in it
  unsigned long long sssp_chunk_levels;    // sum over levels of chunks with SSSP slots
  unsigned long long gather_chunk_levels;  // ... and of those that gathered
  int32_t sscatter;             // ssel has a bit: the scatter kernels have work
  int32_t chunk_dir;            // SSSP direction decided per 32-slot chunk
  int32_t level;
  int32_t dir;                  // BFS direction of the current level
  int32_t sdir;                 // SSSP direction: push (scatter) or pull (gather)
  int32_t sssp_gather;          // gather kernels are launched (pull CSR + weights exist)
  int32_t done;
  uint32_t status;
  int32_t forced_dir;           // -1: decide; else direction of the next level
  int32_t halt_level;           // stop (without converging) once level reaches it; <0 none
  int32_t push_levels;
  int32_t pull_levels;
  int32_t max_iterations;       // 0: unbounded
  int32_t mode;                 // CGP_MODE_*
  int32_t num_planes;
  int32_t profile_cap;
  unsigned long long pull_vertex_threshold;
  unsigned long long pull_edge_threshold;
  unsigned long long sssp_pull_edge_threshold;  // gather when frontier edges reach it
  unsigned long long sssp_pull_pair_unit;  // ... and est. pairs reach it x SSSP chunks (0: off)
  unsigned long long dense_count;  // SSSP vertices queued for the dense kernel this level
  unsigned long long hq_packed;    // heavy frontier queue: count << 40 | chunks, this level
  unsigned long long prev_improved; // SSSP entries improved by the previous level
  unsigned long long prev_pull_edges; // in-edges the previous BFS pull level read
  int32_t prev_dir;                 // BFS direction of the previous level
  int32_t bfs_chunked;              // the BFS pull may run in CTA chunks (chunk table built)
  LevelCounters lc;                // counters of the current level
  LevelCounters total;             // sums over all levels
};

// Per-slot metadata.
struct SlotDev {
  int32_t kind;    // CGP_KIND_*
  int32_t source;
  int32_t k;       // hop bound (k-hop)
  int32_t base;    // level at which the slot was admitted
};

struct DevGraph {
  const void* row;       // int32 or int64 offsets (template OT)
  const int32_t* col;
  const void* w;
  const void* prow;      // CSR used by pull (the transpose for directed graphs)
  const int32_t* pcol;
  const void* pw;        // weights aligned with pcol: pw[e] = weight of pcol[e] -> v
  int64_t V;
  int64_t E;
  const int32_t* heavy;             // vertices with out-degree > heavy_degree
  const int64_t* heavy_chunk_start; // [n_heavy + 1] prefix of chunk counts
  int32_t n_heavy;
  int64_t heavy_chunks;
  const int32_t* pheavy;            // same for the pull CSR
  const int64_t* pheavy_chunk_start;
  const int32_t* pheavy_ch;         // per 2048-edge chunk: table index of its vertex
  const int64_t* pheavy_cb;         // per chunk: first in-edge
  const int64_t* pheavy_ce;         // per chunk: one past its last in-edge
  int32_t n_pheavy;
  int64_t pheavy_chunks;
  int64_t heavy_degree;
  const int32_t* plight;             // light vertices of the pull CSR (chunked gathers)
  const int32_t* plight_chunk_start; // [n_plight_chunks + 1]
  const int64_t* plight_beg;         // first pull-CSR in-edge of plight[i]
  const int32_t* plight_pre;         // in-edges of plight[i]'s chunk up to and including it
  int32_t n_plight_chunks;
  int32_t n_pmid;                    // plight[0 .. n_pmid) have in-degree > 32 (BFS pull mid kernel)
};

struct GroupDev {
  uint64_t* visited;   // [V*W]
  uint64_t* fbuf0;     // [V*W] frontier masks, level parity 0
  uint64_t* fbuf1;
  int32_t* list0;      // unique frontier vertex lists
  int32_t* list1;
  int32_t* stamp;      // last level (+1) a vertex was appended in push
  uint64_t* planes;    // [K][V*W] depth bit planes
  uint32_t* values;    // [V*Qg] vertex-major values (SSSP, direct depths)
  uint64_t* hacc;      // [n_pheavy*W] pull accumulators of heavy vertices
  uint64_t* fsum;      // [V] frontier summary: (level + 1) << 32 | 32-slot chunks with a
                       // frontier bit, written for the frontier's vertices on levels that
                       // screen sources by it (nullptr: not kept)
  int32_t* dense_list; // [V] SSSP frontier vertices with many active bits
  int32_t* hq_vertex;  // [n_heavy] heavy vertices of the current frontier
  int64_t* hq_start;   // [n_heavy] their first chunk in the level's chunk space
  int64_t hq_cap;      // entries of hq_vertex / hq_start
  LevelCtl* ctl;
  LevelProfile* prof;
  const SlotDev* slots;
  int32_t Qg;
};

// Output mapping: group slot q is global query qmap[q]; element (v, gq)
// lives at out[v*sv + gq*sq].
struct OutMap {
  uint32_t* out;
  int64_t sv;
  int64_t sq;
  const int32_t* qmap;
  int32_t qmap_contiguous;  // qmap[q] == qmap[0] + q for every q
};

template <typename OT>
__device__ __forceinline__ int64_t row_at(const void* row, int64_t v) {
  return static_cast<int64_t>(static_cast<const OT*>(row)[v]);
}

}  // namespace dev
}  // namespace cgp
