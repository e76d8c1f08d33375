/*
 * CPU oracle for the concurrent multi-query traversal path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * single-query CPU traversals (puercgp/examples/mtx_loader.hxx:269-356), used
 * by the tests, by smoke() and by the CPU-baseline leg of bench.py as the
 * checker.  Nothing in the shipped library links or calls it.
 *
 * Graphs are CSR with int64 row offsets and int32 column indices.  All
 * per-query outputs are dense arrays of length V.
 */
#ifndef CGP_ORACLE_H
#define CGP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_BFS_INF INT32_MAX
#define ORACLE_U32_INF UINT32_MAX

/* FIFO BFS from `source`; depth[v] = hop count, INT32_MAX if unreached.
 * `max_depth` < 0 means unbounded; otherwise vertices deeper than max_depth
 * stay unreached (k-hop BFS).  Returns the number of CSR entries scanned. */
int64_t oracle_bfs(int64_t V, const int64_t* row, const int32_t* col,
                   int32_t source, int32_t max_depth, int32_t* depth);

/* Binary-heap Dijkstra with float left-fold path sums (distance + w in fp32,
 * round to nearest); +inf if unreached. */
int64_t oracle_sssp_f32(int64_t V, const int64_t* row, const int32_t* col,
                        const float* w, int32_t source, float* dist);

/* Dijkstra with exact uint32 path sums; UINT32_MAX if unreached. */
int64_t oracle_sssp_u32(int64_t V, const int64_t* row, const int32_t* col,
                        const uint32_t* w, int32_t source, uint32_t* dist);

/* In-place min-label propagation to a fixpoint along out-edges, the exact
 * restatement of cpu_wcc (label[v] = min(label[v], label[u]) for v->u).
 * On a symmetric CSR the result is the minimum vertex id of v's component.
 * Returns the number of sweeps. */
int32_t oracle_wcc_label_propagation(int64_t V, const int64_t* row,
                                     const int32_t* col, int32_t max_sweeps,
                                     uint32_t* label);

/* Weakly connected components treating every CSR entry as an undirected
 * edge: label[v] = minimum vertex id of v's weak component (union-find). */
void oracle_wcc_components(int64_t V, const int64_t* row, const int32_t* col,
                           uint32_t* label);

/* Multi-threaded batch runner: runs `nq` independent queries of one kind over
 * `threads` host threads and writes query-major out[q*V + v].
 *   kind 0 = BFS (int32), 1 = SSSP u32 (uint32), 2 = SSSP f32 (float),
 *   3 = k-hop BFS (int32, k from khop[q]).
 * weights may be NULL for BFS.  edges_out[q] (may be NULL) receives
 * sum of out-degrees of the vertices reached by query q. */
void oracle_batch(int32_t kind, int64_t V, const int64_t* row,
                  const int32_t* col, const void* weights,
                  const int32_t* sources, const int32_t* khop, int32_t nq,
                  int32_t threads, void* out, int64_t* edges_out);

#ifdef __cplusplus
}
#endif

#endif
