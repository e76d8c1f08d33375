// Continuous-batching server over one or more traversal groups of bitmask
// slots.
//
// Replaces replenish_frontier_engine / run_replenish_pipeline
// (puercgp/include/puercgp/engine/replenish_engine.hxx:42-573).  The
// reference takes all N queries up front and, after every level, detects
// converged slots from the active-slot union, snapshots them into a row-major
// buffer, clears them and injects the next pending query.  Here requests
// arrive at any time through cgp_server_submit; a host thread admits them
// into free slots at level boundaries while the others keep running, retires
// converged slots (snapshot + reset in one pass over V), and records per
// request submit / admit / finish times.  Differences that fix reference
// hazards: every slot has its own base level, so a BFS admitted at level L
// writes depth = level + 1 - L (the reference writes the global level,
// hybrid_engine.hxx:175); WCC requests are answered from one union-find pass
// instead of occupying a slot; slot state uses one "unreached" word
// (0xffffffff) for every kind, mapped to the kind's marker on retire.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>
#include <unordered_map>

#include "engine.h"
#include "kernels.cuh"

namespace cgp {
namespace {

using namespace dev;

constexpr uint32_t kServeInf = 0xffffffffu;
constexpr int kRetireBatch = 32;

struct AdmitReq {
  int32_t slot;
  int32_t kind;
  int32_t source;
  int32_t k;
};

struct RetireReq {
  int32_t slot;
  int32_t kind;
  int32_t has_out;
  int32_t reserved;
  uint32_t* dst;  // the request's device output, or NULL: staging row i
};

// Seeds newly admitted slots into the frontier of the current level (one
// block, between levels).
template <int W, typename OT>
__global__ void k_admit(GroupDev g, DevGraph G, const AdmitReq* reqs, int n) {
  LevelCtl* ctl = g.ctl;
  const int L = ctl->level;
  const int par = L & 1;
  uint64_t* fcur = par ? g.fbuf1 : g.fbuf0;
  int32_t* list = par ? g.list1 : g.list0;
  SlotDev* slots = const_cast<SlotDev*>(g.slots);
  const int lane = threadIdx.x & 31;
  for (int base = threadIdx.x & ~31; base < n; base += blockDim.x) {
    const int i = base + lane;
    bool app = false;
    int32_t src = 0;
    uint64_t deg = 0;
    if (i < n) {
      const AdmitReq r = reqs[i];
      const int s = r.slot;
      const int w = s >> 6;
      const uint64_t bit = 1ULL << (s & 63);
      SlotDev sd;
      sd.kind = r.kind;
      sd.source = r.source;
      sd.k = r.k;
      sd.base = L;
      slots[s] = sd;
      const bool bfs_like = r.kind == 0 || r.kind == 3;
      // a new SSSP slot scatters from its source until the level ends decide
      // its chunk's direction again
      atomicAnd(reinterpret_cast<unsigned long long*>(&ctl->gsel[w]), ~bit);
      if (bfs_like) {
        atomic_or64(&ctl->bfs_bits[w], bit);
        atomicAnd(reinterpret_cast<unsigned long long*>(&ctl->sssp_bits[w]), ~bit);
        atomicAnd(reinterpret_cast<unsigned long long*>(&ctl->ssel[w]), ~bit);
        atomic_or64(g.visited + static_cast<size_t>(r.source) * W + w, bit);
      } else {
        atomic_or64(&ctl->sssp_bits[w], bit);
        atomic_or64(&ctl->ssel[w], bit);
        atomicAnd(reinterpret_cast<unsigned long long*>(&ctl->bfs_bits[w]), ~bit);
      }
      if (r.kind == 3 && r.k <= 0)
        atomicAnd(reinterpret_cast<unsigned long long*>(&ctl->expand[w]), ~bit);
      else
        atomic_or64(&ctl->expand[w], bit);
      g.values[static_cast<size_t>(r.source) * g.Qg + s] = 0u;
      atomic_or64(fcur + static_cast<size_t>(r.source) * W + w, bit);
      atomic_or64(&ctl->active[par][w], bit);
      src = r.source;
      app = atomicMax(g.stamp + src, L) < L;
      deg = degree_of<OT>(G.row, src);
    }
    warp_append(app, src, deg, list, &ctl->count[par], &ctl->edges[par], lane);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0 && ctl->count[par] > 0) {
    ctl->done = 0;
    ctl->dir = decide_dir(ctl, ctl->count[par], ctl->edges[par], any_bits<W>(ctl->bfs_bits));
    if (ctl->chunk_dir) {
      ctl->sdir = any_bits<W>(ctl->gsel) ? kDirPull : kDirPush;
      ctl->sscatter = any_bits<W>(ctl->ssel) ? 1 : 0;
    } else {
      split_sssp_slots<W>(ctl, decide_sdir<W>(ctl, ctl->count[par], ctl->edges[par]));
    }
  }
}

// Retires slots: snapshot each slot column (mapped to its kind's unreached
// marker) into the request's device output, or staging row i for a host
// output, reset the column, and clear the slots' visited bits (and frontier
// bits when a running request was cancelled).  A CTA takes 64 vertices: its
// warps read the retiring slots of one vertex row together (lane i <-> slot
// i, all within the row's 1 KB), stage them in shared memory, and then write
// every slot's output row contiguously.
constexpr int kRetireTile = 64;

template <int W>
__global__ void __launch_bounds__(kBlock) k_retire(GroupDev g, int64_t V, const RetireReq* reqs,
                                                   int n, uint32_t* staging, const uint64_t* clear,
                                                   int clear_frontier, uint32_t f32) {
  __shared__ uint32_t tile[kRetireBatch][kRetireTile + 1];
  __shared__ RetireReq rq[kRetireBatch];
  if (threadIdx.x < n) rq[threadIdx.x] = reqs[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  bool any_out = false;
  for (int i = 0; i < n; ++i) any_out |= rq[i].has_out != 0;
  for (int64_t v0 = static_cast<int64_t>(blockIdx.x) * kRetireTile; v0 < V;
       v0 += static_cast<int64_t>(gridDim.x) * kRetireTile) {
    // each warp reads its 8 rows' slots first (8 independent loads per lane)
    constexpr int kPer = kRetireTile / kWarpsPerBlock;
    uint32_t xs[kPer];
    RetireReq r{};
    if (lane < n) r = rq[lane];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int64_t v = v0 + wib + k * kWarpsPerBlock;
      xs[k] = (lane < n && v < V) ? g.values[static_cast<size_t>(v) * g.Qg + r.slot] : kServeInf;
    }
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int j = wib + k * kWarpsPerBlock;
      const int64_t v = v0 + j;
      if (v >= V) break;
      if (lane < n) {
        g.values[static_cast<size_t>(v) * g.Qg + r.slot] = kServeInf;
        uint32_t x = xs[k];
        if (x == kServeInf) {
          if (r.kind == 0 || r.kind == 3) x = 0x7fffffffu;
          else if (f32) x = 0x7f800000u;
        }
        tile[lane][j] = x;
      }
      if (lane < W && clear[lane]) {
        const size_t wi = static_cast<size_t>(v) * W + lane;
        g.visited[wi] &= ~clear[lane];
        if (clear_frontier) {
          g.fbuf0[wi] &= ~clear[lane];
          g.fbuf1[wi] &= ~clear[lane];
        }
      }
    }
    __syncthreads();
    if (any_out) {
      for (int t = threadIdx.x; t < n * kRetireTile; t += blockDim.x) {
        const int i = t / kRetireTile, j = t % kRetireTile;
        if (rq[i].has_out && v0 + j < V) {
          uint32_t* row = rq[i].dst ? rq[i].dst : staging + static_cast<size_t>(i) * V;
          row[v0 + j] = tile[i][j];
        }
      }
    }
    __syncthreads();
  }
}

template <int W, typename OT>
void launch_admit(const GroupDev& g, const DevGraph& G, const AdmitReq* r, int n, cudaStream_t s) {
  k_admit<W, OT><<<1, kBlock, 0, s>>>(g, G, r, n);
}

template <int W>
void launch_retire(const GroupDev& g, int64_t V, const RetireReq* r, int n, uint32_t* st,
                   const uint64_t* clear, int cf, uint32_t f32, int blocks, cudaStream_t s) {
  k_retire<W><<<blocks, kBlock, 0, s>>>(g, V, r, n, st, clear, cf, f32);
}

struct Request {
  cgp_query q{};
  void* out = nullptr;
  bool out_dev = false;
  int state = 0;  // 0 queued, 1 running, 2 done, 3 cancelled, 4 failed
  int slot = -1;
  int admit_level = -1;
  int completion_level = -1;
  double t_submit = 0, t_admit = 0, t_finish = 0;
  bool cancel = false;
};

}  // namespace
}  // namespace cgp

using namespace cgp;
using namespace cgp::dev;

// One traversal group of the server: its own workspace (masks, values,
// control block), stream and admission buffers.  Slots of group g are the
// global slots [base, base + S).
struct ServeGroup {
  std::unique_ptr<Workspace> ws;
  GroupSpec spec;
  cudaStream_t stream = nullptr;
  int S = 0;
  int W = 1;
  int base = 0;
  int active = 0;        // occupied slots
  bool cohort = false;   // group-cohort policy: a cohort runs here (no admissions)
  int32_t level = 0;     // device level at the last read
  int64_t levels_done = 0;
  int64_t sssp_chunk_levels = 0, gather_chunk_levels = 0;
  DevBuf admit_dev, retire_dev, clear_dev;
  AdmitReq* h_admit = nullptr;
  RetireReq* h_retire = nullptr;
  uint64_t* h_clear = nullptr;
  int32_t* h_level = nullptr;
  int nadmit = 0;        // admissions of the current pass
  bool ran = false;      // levels were enqueued in the current pass
};

struct cgp_server {
  GraphImpl* g = nullptr;
  cgp_options o{};
  int S = 0;             // total slots over all groups
  std::vector<ServeGroup> groups;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv;       // work arrived / stop
  std::condition_variable done_cv;  // a request finished
  std::deque<uint64_t> pending;
  std::unordered_map<uint64_t, Request> reqs;
  std::vector<int64_t> slot_ticket;  // by global slot
  int active = 0;
  bool stop = false;
  uint64_t next_ticket = 1;
  int64_t completed = 0;
  int64_t levels = 0;
  double busy_ms = 0;
  double admit_ms = 0;
  double retire_ms = 0;
  int64_t retire_passes = 0;
  int64_t sssp_chunk_levels = 0;
  int64_t gather_chunk_levels = 0;
  int64_t state_bytes = 0;
  bool wcc_ready = false;
  std::string fatal;
  DevBuf staging;        // retire snapshots (groups retire one after another)
  std::unique_ptr<Workspace> wcc_ws;  // WCC labels
  std::unique_ptr<KernelTimer> kt;  // per-class kernel times (profile_kernels)
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  void loop();
  int pick_slot(int* group, int32_t kind);
  void finish_wcc(std::vector<uint64_t>& tickets);
  void retire(ServeGroup& gr, std::vector<int>& local_slots, bool forced);
  void release_pinned();
};

namespace {

using AdmitFn = void (*)(const GroupDev&, const DevGraph&, const AdmitReq*, int, cudaStream_t);
using RetireFn = void (*)(const GroupDev&, int64_t, const RetireReq*, int, uint32_t*,
                          const uint64_t*, int, uint32_t, int, cudaStream_t);

template <int W>
AdmitFn admit_for(int ob) {
  return ob == 8 ? launch_admit<W, int64_t> : launch_admit<W, int32_t>;
}

AdmitFn pick_admit(int W, int ob) {
  switch (W) {
    case 1: return admit_for<1>(ob);
    case 2: return admit_for<2>(ob);
    case 4: return admit_for<4>(ob);
    case 8: return admit_for<8>(ob);
    default: return admit_for<16>(ob);
  }
}

RetireFn pick_retire(int W) {
  switch (W) {
    case 1: return launch_retire<1>;
    case 2: return launch_retire<2>;
    case 4: return launch_retire<4>;
    case 8: return launch_retire<8>;
    default: return launch_retire<16>;
  }
}

GroupDev server_dev(const ServeGroup& gr) {
  GroupDev g{};
  Workspace* ws = gr.ws.get();
  g.visited = ws->visited.as<uint64_t>();
  g.fbuf0 = ws->fbuf0.as<uint64_t>();
  g.fbuf1 = ws->fbuf1.as<uint64_t>();
  g.list0 = ws->list0.as<int32_t>();
  g.list1 = ws->list1.as<int32_t>();
  g.stamp = ws->stamp.as<int32_t>();
  g.planes = nullptr;
  g.values = ws->values.as<uint32_t>();
  g.hacc = ws->hacc.as<uint64_t>();
  g.fsum = ws->fsum.as<uint64_t>();
  g.dense_list = ws->dense.as<int32_t>();
  g.hq_vertex = nullptr;
  g.hq_start = nullptr;
  g.ctl = ws->ctl.as<LevelCtl>();
  g.prof = nullptr;
  g.slots = ws->slots.as<SlotDev>();
  g.Qg = gr.S;
  return g;
}

}  // namespace

void cgp_server::release_pinned() {
  for (ServeGroup& gr : groups) {
    if (gr.stream) cudaStreamSynchronize(gr.stream);
    if (gr.h_admit) cudaFreeHost(gr.h_admit);
    if (gr.h_retire) cudaFreeHost(gr.h_retire);
    if (gr.h_clear) cudaFreeHost(gr.h_clear);
    if (gr.h_level) cudaFreeHost(gr.h_level);
    gr.h_admit = nullptr;
    gr.h_retire = nullptr;
    gr.h_clear = nullptr;
    gr.h_level = nullptr;
  }
}

void cgp_server::finish_wcc(std::vector<uint64_t>& tickets) {
  if (tickets.empty()) return;
  cudaStream_t s = wcc_ws->stream;
  if (!wcc_ready) {
    wcc_ws->wcc.ensure(static_cast<size_t>(g->V) * 4);
    wcc_labels(g, wcc_ws->wcc.as<uint32_t>(), s);
    wcc_ready = true;
  }
  std::vector<std::pair<void*, bool>> outs;
  {
    std::lock_guard<std::mutex> lk(mu);
    for (uint64_t t : tickets) outs.emplace_back(reqs[t].out, reqs[t].out_dev);
  }
  for (auto& o : outs)
    if (o.first)
      ck(cudaMemcpyAsync(o.first, wcc_ws->wcc.p, static_cast<size_t>(g->V) * 4,
                         o.second ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s),
         "wcc result");
  ck(cudaStreamSynchronize(s), "wcc");
  std::lock_guard<std::mutex> lk(mu);
  const double t = now_ms();
  for (uint64_t tk : tickets) {
    Request& r = reqs[tk];
    r.state = 2;
    r.t_admit = r.t_admit > 0 ? r.t_admit : t;
    r.t_finish = t;
    r.completion_level = 0;
    ++completed;
  }
  done_cv.notify_all();
}

// Retires local slots of group gr: snapshots their columns into the staging
// rows, resets them, copies the results out, in passes of kRetireBatch.
void cgp_server::retire(ServeGroup& gr, std::vector<int>& to_retire, bool forced) {
  const double t_start = now_ms();
  const int64_t V = g->V;
  const uint32_t f32 = g->weight_kind == CGP_WEIGHT_F32 ? 1u : 0u;
  RetireFn rf = pick_retire(gr.W);
  for (size_t b = 0; b < to_retire.size(); b += kRetireBatch) {
    const int n = static_cast<int>(std::min<size_t>(kRetireBatch, to_retire.size() - b));
    std::memset(gr.h_clear, 0, kMaxWords * 8);
    std::vector<uint64_t> tickets(n);
    std::vector<std::pair<void*, bool>> outs(n);
    {
      std::lock_guard<std::mutex> lk(mu);
      for (int i = 0; i < n; ++i) {
        const int s = to_retire[b + i];
        tickets[i] = static_cast<uint64_t>(slot_ticket[gr.base + s]);
        Request& r = reqs[tickets[i]];
        outs[i] = {r.out, r.out_dev};
        gr.h_retire[i].slot = s;
        gr.h_retire[i].kind = r.q.kind;
        gr.h_retire[i].has_out = (r.out != nullptr && !r.cancel) ? 1 : 0;
        // device outputs are written by the retire kernel itself
        gr.h_retire[i].dst = r.out_dev ? static_cast<uint32_t*>(r.out) : nullptr;
        gr.h_clear[s >> 6] |= 1ULL << (s & 63);
      }
    }
    ck(cudaMemcpyAsync(gr.retire_dev.p, gr.h_retire, n * sizeof(RetireReq), cudaMemcpyHostToDevice,
                       gr.stream), "upload retire");
    ck(cudaMemcpyAsync(gr.clear_dev.p, gr.h_clear, kMaxWords * 8, cudaMemcpyHostToDevice, gr.stream),
       "upload clear");
    rf(server_dev(gr), V, gr.retire_dev.as<RetireReq>(), n, staging.as<uint32_t>(),
       gr.clear_dev.as<uint64_t>(), forced ? 1 : 0, f32, g->num_sms * 4, gr.stream);
    ck(cudaGetLastError(), "retire");
    for (int i = 0; i < n; ++i) {
      if (gr.h_retire[i].has_out && !outs[i].second)
        ck(cudaMemcpyAsync(outs[i].first, staging.as<uint32_t>() + static_cast<size_t>(i) * V,
                           static_cast<size_t>(V) * 4, cudaMemcpyDeviceToHost, gr.stream),
           "result copy");
    }
    ck(cudaStreamSynchronize(gr.stream), "retire");
    std::lock_guard<std::mutex> lk(mu);
    const double t = now_ms();
    for (int i = 0; i < n; ++i) {
      Request& r = reqs[tickets[i]];
      r.state = r.cancel ? 3 : 2;
      r.t_finish = t;
      r.completion_level = gr.level - r.admit_level;
      slot_ticket[gr.base + gr.h_retire[i].slot] = -1;
      --gr.active;
      --active;
      ++completed;
    }
    ++retire_passes;
    done_cv.notify_all();
  }
  retire_ms += now_ms() - t_start;
}

// A free global slot for the next admission (mu held), or -1; *group gets
// its group.  Slots are taken in 32-slot cohorts, so that requests that
// arrive together share a chunk and pass through their sparse and dense
// phases together (what the per-chunk SSSP direction needs): first a chunk
// already taken by this admission pass, then an empty chunk, then the chunk
// whose occupants were admitted last.  Policies (cgp_options.serve_admission):
//  * 0, free slots: any free slot, in that order of preference.
//  * 1, chunk cohorts: a chunk with occupants from earlier passes takes no one.
//  * 2, group cohorts: a group takes requests only while it is empty or
//    filling in this pass, so each group runs one cohort at a time and every
//    gather level of the group serves all of its SSSP requests; with two or
//    more groups, arrivals open a cohort in an idle group while the others
//    run, and the groups' levels overlap on the device.  Inside the group,
//    SSSP requests fill the slots from the bottom and BFS-like ones from the
//    top, so a gather reads only the chunks that hold SSSP slots.
// (Separating SSSP from BFS-like requests into chunks of their own under the
// free-slot policy was measured too: lower capacity on R-MAT 24, 329 against
// 380 q/s at 500 q/s
// offered, since a saturated server refills single freed slots and an
// all-SSSP chunk then gathers at most levels.)
int cgp_server::pick_slot(int* group, int32_t kind) {
  const int pol = o.serve_admission;
  if (pol == 2) {
    // group cohorts: the group this pass fills, else an empty one; inside it
    // SSSP requests take the lowest free slots and BFS-like ones the highest,
    // so the cohort's SSSP slots share as few 32-slot chunks as possible and
    // its gather levels read only those chunks of each source row
    int gsel = -1;
    for (int gi = 0; gi < static_cast<int>(groups.size()); ++gi) {
      const ServeGroup& gr = groups[gi];
      if (gr.nadmit > 0 && gr.nadmit < gr.S) {
        gsel = gi;
        break;
      }
      if (gsel < 0 && !gr.cohort && gr.active == 0) gsel = gi;
    }
    *group = gsel;
    if (gsel < 0) return -1;
    const ServeGroup& gr = groups[gsel];
    const bool low = kind == CGP_KIND_SSSP;
    for (int k = 0; k < gr.S; ++k) {
      const int i = low ? k : gr.S - 1 - k;
      if (slot_ticket[gr.base + i] < 0) return gr.base + i;
    }
    *group = -1;
    return -1;
  }
  int best = -1, best_g = -1;
  long long best_key = -1;
  for (int gi = 0; gi < static_cast<int>(groups.size()); ++gi) {
    ServeGroup& gr = groups[gi];
    if (pol == 2 && gr.cohort && gr.nadmit == 0) continue;  // a cohort runs here
    for (int c0 = 0; c0 < gr.S; c0 += 32) {
      const int c1 = std::min(gr.S, c0 + 32);
      int free_slot = -1, occupied = 0, newest = -1;
      bool this_pass = false;
      for (int i = c0; i < c1; ++i) {
        const int64_t t = slot_ticket[gr.base + i];
        if (t < 0) {
          if (free_slot < 0) free_slot = i;
          continue;
        }
        ++occupied;
        const int al = reqs[static_cast<uint64_t>(t)].admit_level;
        if (al < 0) this_pass = true;  // level set once the admission kernel ran
        newest = std::max(newest, al);
      }
      if (free_slot < 0) continue;
      if (pol == 1 && occupied > 0 && !this_pass) continue;
      long long key = this_pass ? (3LL << 40) : occupied == 0 ? (2LL << 40) : newest;
      if (pol == 2 && gr.nadmit > 0) key += 4LL << 40;  // one cohort per pass stays together
      if (key > best_key) {
        best_key = key;
        best = gr.base + free_slot;
        best_g = gi;
      }
    }
  }
  *group = best_g;
  return best;
}

void cgp_server::loop() {
  try {
    ck(cudaSetDevice(g->device), "cudaSetDevice");
    const int per = o.levels_per_sync > 0 ? o.levels_per_sync : 2;
    for (;;) {
      std::vector<uint64_t> wcc_tickets;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait_for(lk, std::chrono::milliseconds(50),
                    [&] { return stop || !pending.empty() || active > 0; });
        if (stop) break;
        for (ServeGroup& gr : groups) gr.nadmit = 0;
        const double t = now_ms();
        while (!pending.empty()) {
          const uint64_t tk = pending.front();
          Request& r = reqs[tk];
          if (r.cancel) {
            pending.pop_front();
            r.state = 3;
            r.t_finish = t;
            done_cv.notify_all();
            continue;
          }
          if (r.q.kind == CGP_KIND_WCC) {
            pending.pop_front();
            r.state = 1;
            r.t_admit = t;
            wcc_tickets.push_back(tk);
            continue;
          }
          int gi = -1;
          const int s = pick_slot(&gi, r.q.kind);
          if (s < 0) break;
          ServeGroup& gr = groups[gi];
          pending.pop_front();
          slot_ticket[s] = static_cast<int64_t>(tk);
          ++gr.active;
          ++active;
          r.state = 1;
          r.slot = s;
          r.t_admit = t;
          AdmitReq& a = gr.h_admit[gr.nadmit++];
          a.slot = s - gr.base;
          a.kind = r.q.kind;
          a.source = r.q.source;
          a.k = r.q.k;
        }
      }
      finish_wcc(wcc_tickets);
      const double ta = now_ms();
      bool admitted = false;
      for (ServeGroup& gr : groups) {
        if (gr.nadmit == 0) continue;
        admitted = true;
        ck(cudaMemcpyAsync(gr.h_level, reinterpret_cast<char*>(gr.ws->ctl.p) + offsetof(LevelCtl, level),
                           sizeof(int32_t), cudaMemcpyDeviceToHost, gr.stream), "read level");
        ck(cudaMemcpyAsync(gr.admit_dev.p, gr.h_admit, gr.nadmit * sizeof(AdmitReq),
                           cudaMemcpyHostToDevice, gr.stream), "upload admits");
        pick_admit(gr.W, g->offset_bytes)(server_dev(gr), g->dev_graph(heavy_threshold(o)),
                                          gr.admit_dev.as<AdmitReq>(), gr.nadmit, gr.stream);
        ck(cudaGetLastError(), "admit");
      }
      if (admitted) {
        for (ServeGroup& gr : groups)
          if (gr.nadmit > 0) ck(cudaStreamSynchronize(gr.stream), "admit");
        std::lock_guard<std::mutex> lk(mu);
        for (ServeGroup& gr : groups) {
          if (gr.nadmit == 0) continue;
          for (int i = 0; i < gr.nadmit; ++i)
            reqs[static_cast<uint64_t>(slot_ticket[gr.base + gr.h_admit[i].slot])].admit_level =
                *gr.h_level;
          gr.cohort = true;
        }
        admit_ms += now_ms() - ta;
      }
      const double tb = now_ms();
      // levels: every group with requests runs `per` levels; without kernel
      // timing the groups' level chunks are enqueued on their own streams
      // first and waited for afterwards, so they overlap on the device
      bool any = false;
      for (ServeGroup& gr : groups) {
        gr.ran = false;
        int act;
        {
          std::lock_guard<std::mutex> lk(mu);
          act = gr.active;
        }
        if (act == 0) {
          gr.cohort = false;
          continue;
        }
        gr.ran = true;
        any = true;
        if (kt) {
          GroupRun r;
          group_enact(g, gr.ws.get(), gr.spec, o, gr.stream, &r, per, kt.get());
          kt->flush();
        } else {
          group_enqueue_levels(g, gr.ws.get(), gr.spec, o, gr.stream, per);
        }
        ck(cudaMemcpyAsync(gr.ws->hctl, gr.ws->ctl.p, sizeof(LevelCtl), cudaMemcpyDeviceToHost,
                           gr.stream), "read ctl");
      }
      if (!any) continue;
      for (ServeGroup& gr : groups)
        if (gr.ran) ck(cudaStreamSynchronize(gr.stream), "levels");
      busy_ms += now_ms() - tb;
      for (ServeGroup& gr : groups) {
        if (!gr.ran) continue;
        const LevelCtl& c = gr.ws->hctl[0];
        if (c.status & kStatusQueueOverflow)
          throw ApiError{CGP_ERR_DEVICE, "heavy frontier queue overflow"};
        gr.level = c.level;
        gr.levels_done = c.level;
        gr.sssp_chunk_levels = static_cast<int64_t>(c.sssp_chunk_levels);
        gr.gather_chunk_levels = static_cast<int64_t>(c.gather_chunk_levels);
        // converged: occupied, admitted before the current level, no frontier bit
        std::vector<int> conv, forced;
        {
          std::lock_guard<std::mutex> lk(mu);
          const uint64_t* act_bits = c.active[c.level & 1];
          for (int s = 0; s < gr.S; ++s) {
            const int64_t t = slot_ticket[gr.base + s];
            if (t < 0) continue;
            Request& q = reqs[static_cast<uint64_t>(t)];
            const bool live = c.done != 1 && ((act_bits[s >> 6] >> (s & 63)) & 1ULL);
            if (q.cancel) forced.push_back(s);
            else if (q.admit_level < c.level && !live) conv.push_back(s);
          }
          levels = 0;
          sssp_chunk_levels = 0;
          gather_chunk_levels = 0;
          for (const ServeGroup& x : groups) {
            levels += x.levels_done;
            sssp_chunk_levels += x.sssp_chunk_levels;
            gather_chunk_levels += x.gather_chunk_levels;
          }
        }
        if (!conv.empty()) retire(gr, conv, false);
        if (!forced.empty()) retire(gr, forced, true);
        std::lock_guard<std::mutex> lk(mu);
        if (gr.active == 0) gr.cohort = false;
      }
    }
  } catch (...) {
    cgp_status st = translate_exception();
    char buf[512];
    cgp_last_error(buf, sizeof(buf));
    std::lock_guard<std::mutex> lk(mu);
    fatal = std::string(cgp_status_name(st)) + ": " + buf;
    for (auto& kv : reqs)
      if (kv.second.state < 2) {
        kv.second.state = 4;
        kv.second.t_finish = now_ms();
      }
    done_cv.notify_all();
  }
}

extern "C" {

cgp_status cgp_server_create(cgp_graph* graph, int32_t slots, const cgp_options* opts,
                             int64_t max_state_bytes, cgp_server** out) {
  clear_error();
  if (out == nullptr) return set_error(CGP_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (graph == nullptr) return set_error(CGP_ERR_INVALID_ARG, "graph is NULL");
  if (slots <= 0 || slots > kMaxWords * 64)
    return set_error(CGP_ERR_INVALID_ARG, "slots must be in [1, 1024]");
  if (opts && (opts->serve_admission < 0 || opts->serve_admission > 2))
    return set_error(CGP_ERR_INVALID_ARG, "serve_admission must be 0, 1 or 2");
  if (opts && (opts->serve_groups < 0 || opts->serve_groups > 8))
    return set_error(CGP_ERR_INVALID_ARG, "serve_groups must be in [0, 8]");
  auto* sv = new (std::nothrow) cgp_server();
  if (!sv) return set_error(CGP_ERR_OOM, "host allocation failed");
  try {
    GraphImpl* g = &graph->impl;
    ck(cudaSetDevice(g->device), "cudaSetDevice");
    sv->g = g;
    if (opts) sv->o = *opts;
    else cgp_options_init(&sv->o);
    sv->o.profile_iterations = 0;
    sv->o.max_iterations = 0;
    // groups: one unless asked (on R-MAT 24 serving, one 256-slot group of
    // cohorts sustained 500 q/s at p99 0.66 s; two groups of 128 or 256 slots
    // gave 0.96 / 1.09 s: two cohorts at a time share every level's per-edge
    // cost); never more groups than slots
    int G = sv->o.serve_groups > 0 ? sv->o.serve_groups : 1;
    G = std::max(1, std::min(G, static_cast<int>(slots)));
    // admission by device memory: slot width x |V| for the values, plus the
    // per-vertex masks of each group, plus the retire staging rows
    size_t free_b = 0, total_b = 0;
    ck(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const int64_t budget = max_state_bytes > 0 ? max_state_bytes
                                               : static_cast<int64_t>(0.8 * static_cast<double>(free_b));
    auto need_for = [&](int total) {
      int64_t b = static_cast<int64_t>(kRetireBatch) * g->V * 4;
      for (int i = 0; i < G; ++i) {
        const int Sg = total / G + (i < total % G ? 1 : 0);
        if (Sg > 0) b += group_state_bytes(g, choose_words(Sg, sv->o.mask_words), Sg, kDepthDirect);
      }
      return b;
    };
    int S = std::max(slots, G);
    while (S > G && need_for(S) > budget) --S;
    if (S < G) S = G;
    const int64_t need = need_for(S);
    if (need > budget) throw ApiError{CGP_ERR_OOM, "not enough device memory for one slot"};
    sv->S = S;
    sv->state_bytes = need;
    sv->slot_ticket.assign(S, -1);
    sv->groups.resize(G);
    int base = 0;
    for (int i = 0; i < G; ++i) {
      ServeGroup& gr = sv->groups[i];
      gr.S = S / G + (i < S % G ? 1 : 0);
      gr.base = base;
      base += gr.S;
      gr.W = choose_words(gr.S, sv->o.mask_words);
      gr.ws = std::make_unique<Workspace>(g->device);
      gr.stream = gr.ws->stream;
      gr.spec.W = gr.W;
      gr.spec.Qg = gr.S;
      gr.spec.slots.assign(gr.S, SlotDev{-1, -1, 0, 0});
      gr.spec.depth_mode = kDepthDirect;
      gr.spec.has_bfs = true;
      gr.spec.has_sssp = true;
      gr.spec.uniform_inf = kServeInf;
      gr.spec.serving = true;
      group_prepare(g, gr.ws.get(), gr.spec, sv->o, gr.stream);
      gr.admit_dev.ensure(kMaxWords * 64 * sizeof(AdmitReq));
      gr.retire_dev.ensure(kRetireBatch * sizeof(RetireReq));
      gr.clear_dev.ensure(kMaxWords * 8);
      ck(cudaHostAlloc(reinterpret_cast<void**>(&gr.h_admit), kMaxWords * 64 * sizeof(AdmitReq),
                       cudaHostAllocDefault), "pinned");
      ck(cudaHostAlloc(reinterpret_cast<void**>(&gr.h_retire), kRetireBatch * sizeof(RetireReq),
                       cudaHostAllocDefault), "pinned");
      ck(cudaHostAlloc(reinterpret_cast<void**>(&gr.h_clear), kMaxWords * 8, cudaHostAllocDefault),
         "pinned");
      ck(cudaHostAlloc(reinterpret_cast<void**>(&gr.h_level), sizeof(int32_t), cudaHostAllocDefault),
         "pinned");
    }
    sv->staging.ensure(static_cast<size_t>(kRetireBatch) * g->V * 4);
    sv->wcc_ws = std::make_unique<Workspace>(g->device);
    for (ServeGroup& gr : sv->groups) ck(cudaStreamSynchronize(gr.stream), "server init");
    if (sv->o.profile_kernels) sv->kt = std::make_unique<KernelTimer>();
    sv->th = std::thread([sv] { sv->loop(); });
    *out = sv;
    return CGP_OK;
  } catch (...) {
    cgp_status st = translate_exception();
    sv->release_pinned();
    delete sv;
    return st;
  }
}

cgp_status cgp_server_destroy(cgp_server* sv) {
  clear_error();
  if (sv == nullptr) return CGP_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv.notify_all();
  if (sv->th.joinable()) sv->th.join();
  sv->release_pinned();
  delete sv;
  return CGP_OK;
}

cgp_status cgp_server_submit(cgp_server* sv, const cgp_query* q, void* out, int32_t out_on_device,
                             uint64_t* ticket) {
  clear_error();
  if (sv == nullptr || q == nullptr || ticket == nullptr)
    return set_error(CGP_ERR_INVALID_ARG, "NULL argument");
  if (q->kind < CGP_KIND_BFS || q->kind > CGP_KIND_KHOP)
    return set_error(CGP_ERR_INVALID_ARG, "unknown query kind");
  if (q->kind != CGP_KIND_WCC && (q->source < 0 || q->source >= sv->g->V))
    return set_error(CGP_ERR_INVALID_ARG, "query source out of range");
  if (q->kind == CGP_KIND_KHOP && q->k < 0)
    return set_error(CGP_ERR_INVALID_ARG, "k-hop bound must be non-negative");
  std::lock_guard<std::mutex> lk(sv->mu);
  if (!sv->fatal.empty()) return set_error(CGP_ERR_CUDA, "server failed: " + sv->fatal);
  const uint64_t t = sv->next_ticket++;
  Request r;
  r.q = *q;
  r.out = out;
  r.out_dev = out_on_device != 0;
  r.t_submit = sv->now_ms();
  sv->reqs.emplace(t, r);
  sv->pending.push_back(t);
  *ticket = t;
  sv->cv.notify_all();
  return CGP_OK;
}

static void fill_info(const Request& r, cgp_request_info* info) {
  if (!info) return;
  info->state = r.state;
  info->slot = r.slot;
  info->admit_level = r.admit_level;
  info->completion_level = r.completion_level;
  info->submit_time_ms = r.t_submit;
  info->admit_time_ms = r.t_admit;
  info->finish_time_ms = r.t_finish;
}

cgp_status cgp_server_poll(cgp_server* sv, uint64_t ticket, cgp_request_info* info) {
  clear_error();
  if (sv == nullptr) return set_error(CGP_ERR_INVALID_ARG, "server is NULL");
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return set_error(CGP_ERR_NOT_FOUND, "unknown ticket");
  fill_info(it->second, info);
  return CGP_OK;
}

cgp_status cgp_server_wait(cgp_server* sv, uint64_t ticket, int32_t timeout_ms,
                           cgp_request_info* info) {
  clear_error();
  if (sv == nullptr) return set_error(CGP_ERR_INVALID_ARG, "server is NULL");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return set_error(CGP_ERR_NOT_FOUND, "unknown ticket");
  const auto pred = [&] { return sv->reqs[ticket].state >= 2; };
  if (timeout_ms < 0) sv->done_cv.wait(lk, pred);
  else if (!sv->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred))
    return set_error(CGP_ERR_TIMEOUT, "request not finished");
  const Request& r = sv->reqs[ticket];
  fill_info(r, info);
  if (r.state == 3) return set_error(CGP_ERR_CANCELLED, "request cancelled");
  if (r.state == 4) return set_error(CGP_ERR_CUDA, "server failed: " + sv->fatal);
  return CGP_OK;
}

cgp_status cgp_server_cancel(cgp_server* sv, uint64_t ticket) {
  clear_error();
  if (sv == nullptr) return set_error(CGP_ERR_INVALID_ARG, "server is NULL");
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return set_error(CGP_ERR_NOT_FOUND, "unknown ticket");
  if (it->second.state < 2) it->second.cancel = true;
  sv->cv.notify_all();
  return CGP_OK;
}

cgp_status cgp_server_drain(cgp_server* sv, int32_t timeout_ms) {
  clear_error();
  if (sv == nullptr) return set_error(CGP_ERR_INVALID_ARG, "server is NULL");
  std::unique_lock<std::mutex> lk(sv->mu);
  const auto pred = [&] {
    if (!sv->fatal.empty()) return true;
    for (auto& kv : sv->reqs)
      if (kv.second.state < 2) return false;
    return true;
  };
  if (timeout_ms < 0) sv->done_cv.wait(lk, pred);
  else if (!sv->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred))
    return set_error(CGP_ERR_TIMEOUT, "requests still running");
  if (!sv->fatal.empty()) return set_error(CGP_ERR_CUDA, "server failed: " + sv->fatal);
  return CGP_OK;
}

cgp_status cgp_server_get_stats(cgp_server* sv, cgp_server_stats* st) {
  clear_error();
  if (sv == nullptr || st == nullptr) return set_error(CGP_ERR_INVALID_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  st->slots = sv->S;
  st->active_slots = sv->active;
  st->queued = static_cast<int64_t>(sv->pending.size());
  st->completed = sv->completed;
  st->levels = sv->levels;
  st->busy_ms = sv->busy_ms;
  st->state_bytes = sv->state_bytes;
  st->admit_ms = sv->admit_ms;
  st->retire_ms = sv->retire_ms;
  st->retire_passes = sv->retire_passes;
  st->sssp_chunk_levels = sv->sssp_chunk_levels;
  st->gather_chunk_levels = sv->gather_chunk_levels;
  for (int c = 0; c < 12; ++c) st->kernel_ms[c] = sv->kt && c < kNumClasses ? sv->kt->ms[c] : 0.0;
  return CGP_OK;
}

}  // extern "C"
