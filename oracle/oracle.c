/*
 * CPU oracle: plain-C restatement of the reference's CPU traversals.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load this; the shipped library never does.
 *
 * Each function cites the reference routine it restates (paths relative to
 * the reference project root).
 */
#include "oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- BFS ---- */
/* Restates puercgp_examples::cpu_bfs (puercgp/examples/mtx_loader.hxx:269-290):
 * FIFO queue, the first discovery writes depth[parent] + 1.  max_depth >= 0
 * stops expansion at that depth (the k-hop query kind, which the reference
 * does not have; k < 0 is the reference behaviour). */
int64_t oracle_bfs(int64_t V, const int64_t* row, const int32_t* col,
                   int32_t source, int32_t max_depth, int32_t* depth) {
  int32_t* queue = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V > 0 ? V : 1));
  int64_t head = 0, tail = 0, scanned = 0;
  for (int64_t v = 0; v < V; ++v) depth[v] = ORACLE_BFS_INF;
  depth[source] = 0;
  queue[tail++] = source;
  while (head < tail) {
    int32_t v = queue[head++];
    if (max_depth >= 0 && depth[v] >= max_depth) continue;
    for (int64_t e = row[v]; e < row[v + 1]; ++e) {
      int32_t nb = col[e];
      ++scanned;
      if (depth[nb] == ORACLE_BFS_INF) {
        depth[nb] = depth[v] + 1;
        queue[tail++] = nb;
      }
    }
  }
  free(queue);
  return scanned;
}

/* ------------------------------------------------------------- heaps ---- */
typedef struct {
  double key; /* float or uint32 distance, exactly representable */
  int32_t v;
} heap_item;

typedef struct {
  heap_item* a;
  int64_t n, cap;
} heap_t;

/* Ordering of std::greater<std::pair<float,int>>: (key, vertex) lexicographic. */
static int item_less(heap_item x, heap_item y) {
  return x.key < y.key || (x.key == y.key && x.v < y.v);
}

static void heap_push(heap_t* h, heap_item it) {
  if (h->n == h->cap) {
    h->cap = h->cap ? h->cap * 2 : 1024;
    h->a = (heap_item*)realloc(h->a, sizeof(heap_item) * (size_t)h->cap);
  }
  int64_t i = h->n++;
  while (i > 0) {
    int64_t p = (i - 1) / 2;
    if (!item_less(it, h->a[p])) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i] = it;
}

static heap_item heap_pop(heap_t* h) {
  heap_item top = h->a[0];
  heap_item last = h->a[--h->n];
  int64_t i = 0;
  for (;;) {
    int64_t l = 2 * i + 1;
    if (l >= h->n) break;
    int64_t c = (l + 1 < h->n && item_less(h->a[l + 1], h->a[l])) ? l + 1 : l;
    if (!item_less(h->a[c], last)) break;
    h->a[i] = h->a[c];
    i = c;
  }
  if (h->n > 0) h->a[i] = last;
  return top;
}

/* --------------------------------------------------------------- SSSP ---- */
/* Restates puercgp_examples::cpu_sssp (puercgp/examples/mtx_loader.hxx:292-319):
 * lazy-deletion binary heap, candidate = distance + w evaluated in fp32,
 * relax when candidate < dist[nb], skip stale heap entries. */
int64_t oracle_sssp_f32(int64_t V, const int64_t* row, const int32_t* col,
                        const float* w, int32_t source, float* dist) {
  const float inf = __builtin_inff();
  heap_t h = {0, 0, 0};
  int64_t scanned = 0;
  for (int64_t v = 0; v < V; ++v) dist[v] = inf;
  dist[source] = 0.0f;
  heap_item s = {0.0, source};
  heap_push(&h, s);
  while (h.n > 0) {
    heap_item it = heap_pop(&h);
    float d = (float)it.key;
    if (d != dist[it.v]) continue;
    for (int64_t e = row[it.v]; e < row[it.v + 1]; ++e) {
      int32_t nb = col[e];
      volatile float cand = d + (w ? w[e] : 1.0f); /* fp32 rounding, no contraction */
      ++scanned;
      if (cand < dist[nb]) {
        dist[nb] = cand;
        heap_item ni = {(double)cand, nb};
        heap_push(&h, ni);
      }
    }
  }
  free(h.a);
  return scanned;
}

/* Same algorithm with exact unsigned integer sums (uint32 weights).  With
 * weights below 2^24 and path sums below 2^24 it equals oracle_sssp_f32 on the
 * same weights converted to float. */
int64_t oracle_sssp_u32(int64_t V, const int64_t* row, const int32_t* col,
                        const uint32_t* w, int32_t source, uint32_t* dist) {
  heap_t h = {0, 0, 0};
  int64_t scanned = 0;
  for (int64_t v = 0; v < V; ++v) dist[v] = ORACLE_U32_INF;
  dist[source] = 0;
  heap_item s = {0.0, source};
  heap_push(&h, s);
  while (h.n > 0) {
    heap_item it = heap_pop(&h);
    uint32_t d = (uint32_t)it.key;
    if (d != dist[it.v]) continue;
    for (int64_t e = row[it.v]; e < row[it.v + 1]; ++e) {
      int32_t nb = col[e];
      uint64_t cand = (uint64_t)d + (w ? w[e] : 1u);
      ++scanned;
      if (cand > ORACLE_U32_INF) cand = ORACLE_U32_INF;
      if ((uint32_t)cand < dist[nb]) {
        dist[nb] = (uint32_t)cand;
        heap_item ni = {(double)cand, nb};
        heap_push(&h, ni);
      }
    }
  }
  free(h.a);
  return scanned;
}

/* ---------------------------------------------------------------- WCC ---- */
/* Restates puercgp_examples::cpu_wcc (puercgp/examples/mtx_loader.hxx:328-356):
 * label[v] = v; sweep v = 0..V-1 taking the minimum label over v's CSR
 * neighbours, updating in place, until a sweep changes nothing. */
int32_t oracle_wcc_label_propagation(int64_t V, const int64_t* row,
                                     const int32_t* col, int32_t max_sweeps,
                                     uint32_t* label) {
  int32_t sweeps = 0;
  for (int64_t v = 0; v < V; ++v) label[v] = (uint32_t)v;
  for (int32_t it = 0; it < max_sweeps; ++it) {
    int changed = 0;
    ++sweeps;
    for (int64_t v = 0; v < V; ++v) {
      uint32_t cur = label[v], best = cur;
      for (int64_t e = row[v]; e < row[v + 1]; ++e) {
        uint32_t nb = label[col[e]];
        if (nb < best) best = nb;
      }
      if (best < cur) {
        label[v] = best;
        changed = 1;
      }
    }
    if (!changed) break;
  }
  return sweeps;
}

static uint32_t uf_find(uint32_t* parent, uint32_t x) {
  while (parent[x] != x) {
    parent[x] = parent[parent[x]];
    x = parent[x];
  }
  return x;
}

/* Union-find with the larger root linked under the smaller one, so every
 * root is the minimum id of its set.  On a symmetric CSR this is the fixpoint
 * of oracle_wcc_label_propagation; on a directed CSR it is the weakly
 * connected component minimum (every entry u->v joins u and v). */
void oracle_wcc_components(int64_t V, const int64_t* row, const int32_t* col,
                           uint32_t* label) {
  for (int64_t v = 0; v < V; ++v) label[v] = (uint32_t)v;
  for (int64_t u = 0; u < V; ++u) {
    for (int64_t e = row[u]; e < row[u + 1]; ++e) {
      uint32_t a = uf_find(label, (uint32_t)u);
      uint32_t b = uf_find(label, (uint32_t)col[e]);
      if (a == b) continue;
      if (a < b) label[b] = a;
      else label[a] = b;
    }
  }
  for (int64_t v = 0; v < V; ++v) label[v] = uf_find(label, (uint32_t)v);
}

/* -------------------------------------------------------------- batch ---- */
typedef struct {
  int32_t kind;
  int64_t V;
  const int64_t* row;
  const int32_t* col;
  const void* weights;
  const int32_t* sources;
  const int32_t* khop;
  int32_t nq;
  void* out;
  int64_t* edges_out;
  int32_t next; /* guarded by lock */
  pthread_mutex_t lock;
} batch_job;

static void* batch_worker(void* arg) {
  batch_job* j = (batch_job*)arg;
  for (;;) {
    pthread_mutex_lock(&j->lock);
    int32_t q = j->next++;
    pthread_mutex_unlock(&j->lock);
    if (q >= j->nq) break;
    size_t off = (size_t)q * (size_t)j->V;
    int64_t reached_edges = 0;
    if (j->kind == 0 || j->kind == 3) {
      int32_t* d = (int32_t*)j->out + off;
      oracle_bfs(j->V, j->row, j->col, j->sources[q],
                 j->kind == 3 ? j->khop[q] : -1, d);
      for (int64_t v = 0; v < j->V; ++v)
        if (d[v] != ORACLE_BFS_INF) reached_edges += j->row[v + 1] - j->row[v];
    } else if (j->kind == 1) {
      uint32_t* d = (uint32_t*)j->out + off;
      oracle_sssp_u32(j->V, j->row, j->col, (const uint32_t*)j->weights,
                      j->sources[q], d);
      for (int64_t v = 0; v < j->V; ++v)
        if (d[v] != ORACLE_U32_INF) reached_edges += j->row[v + 1] - j->row[v];
    } else {
      float* d = (float*)j->out + off;
      oracle_sssp_f32(j->V, j->row, j->col, (const float*)j->weights,
                      j->sources[q], d);
      for (int64_t v = 0; v < j->V; ++v)
        if (d[v] != __builtin_inff()) reached_edges += j->row[v + 1] - j->row[v];
    }
    if (j->edges_out) j->edges_out[q] = reached_edges;
  }
  return NULL;
}

void oracle_batch(int32_t kind, int64_t V, const int64_t* row,
                  const int32_t* col, const void* weights,
                  const int32_t* sources, const int32_t* khop, int32_t nq,
                  int32_t threads, void* out, int64_t* edges_out) {
  batch_job j;
  j.kind = kind;
  j.V = V;
  j.row = row;
  j.col = col;
  j.weights = weights;
  j.sources = sources;
  j.khop = khop;
  j.nq = nq;
  j.out = out;
  j.edges_out = edges_out;
  j.next = 0;
  pthread_mutex_init(&j.lock, NULL);
  if (threads < 1) threads = 1;
  if (threads > nq) threads = nq > 0 ? nq : 1;
  pthread_t* tids = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
  for (int32_t t = 0; t < threads; ++t) pthread_create(&tids[t], NULL, batch_worker, &j);
  for (int32_t t = 0; t < threads; ++t) pthread_join(tids[t], NULL);
  free(tids);
  pthread_mutex_destroy(&j.lock);
}
