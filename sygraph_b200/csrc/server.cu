// Query serving with continuous batching (no counterpart in the reference,
// whose algorithms run one call at a time on one queue): several graphs stay
// resident, BFS / SSSP queries arrive from any host thread, and a dispatcher
// thread keeps `slots` CUDA streams busy.
//
//   admission   a query starts when a slot is free and the workspace it needs
//               (per slot and graph: a batched-BFS, BFS or SSSP instance)
//               exists or fits in the memory budget after evicting idle
//               workspaces, least recently used first; otherwise it waits.
//   batching    when a slot frees, every pending BFS query of the oldest
//               query's graph (up to max_batch) runs as one bit-parallel
//               batched launch; fewer than min_batch run as single traversals.
//               SSSP queries run singly (near-far when sssp_delta > 0).
//   overlap     each launch is a persistent kernel capped to ctas_per_slot
//               CTAs, so launches of different slots are resident together.
//   results     copied on the slot's stream into the caller's host buffer
//               (pinned memory keeps the copy asynchronous); the latency of a
//               query is submit to completion on the host clock.
// Results equal the single-query entry points bit for bit: the batched BFS
// computes exactly the per-source depths and SSSP's fixed point does not
// depend on the schedule.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now().time_since_epoch()).count();
}

struct Query {
  uint64_t ticket = 0;
  uint32_t graph = 0, source = 0;
  int kind = SG_QUERY_BFS;
  void* host_out = nullptr;
  sg_query_result res{};
  bool done = false;
};

enum WsKind { kWsBfs = 0, kWsBatch = 1, kWsSssp = 2 };

struct Workspace {
  void* handle = nullptr;  // sg_bfs / sg_msbfs / sg_sssp
  uint64_t bytes = 0;
  uint64_t last_use = 0;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  bool busy = false;
  uint32_t graph = 0;
  int ws_kind = 0;
  std::vector<uint64_t> batch;  // tickets
  // workspaces of this slot, by (graph, kind)
  std::unordered_map<uint64_t, Workspace> ws;
};

uint64_t ws_key(uint32_t graph, int kind) { return ((uint64_t)graph << 2) | (uint64_t)kind; }

}  // namespace

struct sg_server_s {
  sg_server_config cfg{};
  int device = 0;
  std::vector<sg_graph> graphs;
  std::vector<Slot> slots;
  std::deque<uint64_t> pending;         // tickets in arrival order
  std::vector<Query> queries;           // by ticket
  uint64_t ws_bytes = 0, peak_ws_bytes = 0;
  sg_server_stats stats{};
  std::mutex mu;
  std::condition_variable cv_submit;    // wakes the dispatcher
  std::condition_variable cv_done;      // wakes waiters
  std::thread worker;
  std::atomic<bool> stop{false};
  uint64_t use_clock = 0;
};

namespace {

uint32_t bits_of(uint64_t x) {
  uint32_t b = 1;
  while (b < 32 && (x >> b)) b++;
  return b;
}

// Device bytes a workspace of this kind holds (allocation sizes of the
// instances, rounded up; used for admission, so it errs high).
uint64_t ws_estimate(const sg_graph g, int kind, uint32_t max_batch) {
  const uint64_t n = g->n, m = g->m, w0 = (n + 31) / 32;
  const uint64_t fixed = 512 * 1024;  // counters, barrier, level log
  switch (kind) {
    case kWsBfs:  // depths and first in-neighbours, bitmaps, heavy lists
      return fixed + 8 * n + 4 * 6 * w0 + 16 * (m / 256 + 1);
    case kWsBatch:
      return fixed + 8 * n * (4 + bits_of(n ? n - 1 : 0)) + 4 * n * max_batch + 4 * 8 * w0 + 16 * (m / 256 + 1);
    default:
      return fixed + 8 * n + 16 * n + 4 * 8 * w0;
  }
}

void ws_destroy(int kind, Workspace& w) {
  if (!w.handle) return;
  if (kind == kWsBfs) sg_bfs_destroy((sg_bfs)w.handle);
  if (kind == kWsBatch) sg_msbfs_destroy((sg_msbfs)w.handle);
  if (kind == kWsSssp) sg_sssp_destroy((sg_sssp)w.handle);
  w.handle = nullptr;
}

uint32_t slot_ctas(const sg_server_s* s) {
  if (s->cfg.ctas_per_slot) return s->cfg.ctas_per_slot;
  const uint32_t total = 2u * (uint32_t)sgb::device_props().sm_count;
  return std::max<uint32_t>(1, total / std::max<uint32_t>(1, s->cfg.slots));
}

// Frees idle workspaces (not the one slot `keep_slot` is about to use, not
// those of running launches), least recently used first, until `need` more
// bytes fit.  Returns whether they fit.
bool make_room(sg_server_s* s, uint64_t need, uint32_t keep_slot, uint64_t keep_key) {
  if (s->ws_bytes + need <= s->cfg.memory_budget) return true;
  for (;;) {
    // idle slots first (destroying an instance waits for its stream), then LRU
    Slot* best_slot = nullptr;
    uint64_t best_key = 0, best_rank = ~0ull;
    for (uint32_t i = 0; i < s->slots.size(); i++) {
      Slot& sl = s->slots[i];
      for (auto& kv : sl.ws) {
        if (i == keep_slot && kv.first == keep_key) continue;
        if (sl.busy && kv.first == ws_key(sl.graph, sl.ws_kind)) continue;
        const uint64_t rank = (sl.busy ? (1ull << 62) : 0ull) + kv.second.last_use;
        if (rank < best_rank) {
          best_rank = rank;
          best_slot = &sl;
          best_key = kv.first;
        }
      }
    }
    if (!best_slot) return false;
    Workspace& w = best_slot->ws[best_key];
    ws_destroy((int)(best_key & 3), w);
    s->ws_bytes -= w.bytes;
    best_slot->ws.erase(best_key);
    s->stats.evictions++;
    if (s->ws_bytes + need <= s->cfg.memory_budget) return true;
  }
}

// The workspace of (slot, graph, kind), created on demand.  SG_ERR_NOMEM
// when it cannot fit now; `never` tells whether it can never fit.
sg_status get_workspace(sg_server_s* s, uint32_t slot, uint32_t graph, int kind, Workspace** out, bool* never) {
  *never = false;
  Slot& sl = s->slots[slot];
  const uint64_t key = ws_key(graph, kind);
  auto it = sl.ws.find(key);
  if (it != sl.ws.end()) {
    it->second.last_use = ++s->use_clock;
    *out = &it->second;
    return SG_OK;
  }
  sg_graph g = s->graphs[graph];
  const uint64_t est = ws_estimate(g, kind, s->cfg.max_batch);
  if (est > s->cfg.memory_budget) {
    *never = true;
    return SG_ERR_NOMEM;
  }
  if (!make_room(s, est, slot, key)) return SG_ERR_NOMEM;
  Workspace w;
  sg_status st = SG_OK;
  const uint32_t ctas = slot_ctas(s);
  if (kind == kWsBfs) {
    sg_bfs b = nullptr;
    st = sg_bfs_create(g, &b);
    if (st == SG_OK) st = sg_bfs_set_launch(b, sl.stream, ctas);
    w.handle = b;
  } else if (kind == kWsBatch) {
    sg_msbfs h = nullptr;
    st = sg_msbfs_create(g, s->cfg.max_batch, &h);
    if (st == SG_OK) st = sg_msbfs_set_launch(h, sl.stream, ctas);
    w.handle = h;
  } else {
    sg_sssp p = nullptr;
    st = sg_sssp_create(g, &p);
    if (st == SG_OK) st = sg_sssp_set_launch(p, sl.stream, ctas);
    if (st == SG_OK) st = sg_sssp_set_delta(p, s->cfg.sssp_delta);
    w.handle = p;
  }
  if (st != SG_OK) {
    ws_destroy(kind, w);
    return st;
  }
  w.bytes = est;
  w.last_use = ++s->use_clock;
  s->ws_bytes += est;
  s->peak_ws_bytes = std::max(s->peak_ws_bytes, s->ws_bytes);
  auto ins = sl.ws.emplace(key, w);
  *out = &ins.first->second;
  return SG_OK;
}

constexpr float kBatchAlpha = 4.0f, kBatchBeta = 24.0f;  // batched BFS direction switch (bench.py MS_ALPHA)
constexpr float kAlpha = 15.0f, kBeta = 24.0f;           // single BFS: the reference heuristic

sg_status launch(sg_server_s* s, uint32_t si, const std::vector<uint64_t>& tickets, uint32_t graph, int kind,
                 Workspace* w) {
  Slot& sl = s->slots[si];
  sg_graph g = s->graphs[graph];
  const uint64_t t = now_ns();
  for (uint64_t tk : tickets) {
    s->queries[tk].res.start_ns = t;
    s->queries[tk].res.batch_size = (uint32_t)tickets.size();
  }
  const uint64_t bytes = 4ull * g->n;
  if (kind == kWsBatch) {
    std::vector<uint32_t> src;
    for (uint64_t tk : tickets) src.push_back(s->queries[tk].source);
    sg_msbfs h = (sg_msbfs)w->handle;
    SG_TRY(sg_msbfs_run_async(h, src.data(), (uint32_t)src.size(), SG_BFS_HYBRID, kBatchAlpha, kBatchBeta));
    const uint32_t* d = nullptr;
    SG_TRY(sg_msbfs_depths_device(h, &d));
    for (size_t i = 0; i < tickets.size(); i++) {
      void* out = s->queries[tickets[i]].host_out;
      if (out) SG_CUDA(cudaMemcpyAsync(out, d + i * (size_t)g->n, bytes, cudaMemcpyDeviceToHost, sl.stream));
    }
    s->stats.batched_queries += tickets.size();
  } else if (kind == kWsBfs) {
    sg_bfs b = (sg_bfs)w->handle;
    SG_TRY(sg_bfs_init(b, s->queries[tickets[0]].source));
    SG_TRY(sg_bfs_run_async(b, SG_BFS_HYBRID, kAlpha, kBeta));
    const uint32_t* d = nullptr;
    SG_TRY(sg_bfs_distances_device(b, &d));
    void* out = s->queries[tickets[0]].host_out;
    if (out) SG_CUDA(cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, sl.stream));
  } else {
    sg_sssp p = (sg_sssp)w->handle;
    SG_TRY(sg_sssp_init(p, s->queries[tickets[0]].source));
    SG_TRY(sg_sssp_run_async(p));
    const void* d = nullptr;
    SG_TRY(sg_sssp_distances_device(p, &d));
    void* out = s->queries[tickets[0]].host_out;
    if (out) SG_CUDA(cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, sl.stream));
  }
  SG_CUDA(cudaEventRecord(sl.ev, sl.stream));
  sl.busy = true;
  sl.batch = tickets;
  sl.graph = graph;
  sl.ws_kind = kind;
  s->stats.launches++;
  return SG_OK;
}

void finish(sg_server_s* s, const std::vector<uint64_t>& tickets, sg_status st) {
  const uint64_t t = now_ns();
  for (uint64_t tk : tickets) {
    Query& q = s->queries[tk];
    q.res.status = st;
    q.res.end_ns = t;
    q.done = true;
    if (st == SG_OK)
      s->stats.completed++;
    else
      s->stats.failed++;
  }
}

// Picks the next launch from the head of the queue.  Returns false when the
// head must wait (no free slot, or its workspace does not fit yet).
bool admit_one(sg_server_s* s) {
  if (s->pending.empty()) return false;
  const Query& q0 = s->queries[s->pending.front()];
  std::vector<uint64_t> tickets;
  int kind = kWsSssp;
  if (q0.kind == SG_QUERY_BFS) {
    for (uint64_t tk : s->pending) {
      const Query& q = s->queries[tk];
      if (q.kind == SG_QUERY_BFS && q.graph == q0.graph) tickets.push_back(tk);
      if (tickets.size() == s->cfg.max_batch) break;
    }
    kind = tickets.size() >= s->cfg.min_batch ? kWsBatch : kWsBfs;
    if (kind == kWsBfs) tickets.resize(1);
    if (kind == kWsBatch && ws_estimate(s->graphs[q0.graph], kWsBatch, s->cfg.max_batch) > s->cfg.memory_budget) {
      kind = kWsBfs;  // a batch workspace can never fit: single traversals
      tickets.resize(1);
    }
  } else {
    tickets.push_back(s->pending.front());
  }
  // a free slot, preferring one that holds the workspace already
  int si = -1;
  const uint64_t key = ws_key(q0.graph, kind);
  for (uint32_t i = 0; i < s->slots.size(); i++) {
    if (s->slots[i].busy) continue;
    if (si < 0) si = (int)i;
    if (s->slots[i].ws.count(key)) {
      si = (int)i;
      break;
    }
  }
  if (si < 0) return false;
  Workspace* w = nullptr;
  bool never = false;
  sg_status st = get_workspace(s, (uint32_t)si, q0.graph, kind, &w, &never);
  if (st == SG_ERR_NOMEM && !never) {
    s->stats.deferred_admissions++;
    return false;
  }
  // the chosen tickets leave the queue
  std::deque<uint64_t> rest;
  size_t j = 0;
  for (uint64_t tk : s->pending) {
    if (j < tickets.size() && tk == tickets[j])
      j++;
    else
      rest.push_back(tk);
  }
  s->pending.swap(rest);
  if (st == SG_OK) st = launch(s, (uint32_t)si, tickets, q0.graph, kind, w);
  if (st != SG_OK) {
    cudaStreamSynchronize(s->slots[si].stream);
    s->slots[si].busy = false;
    finish(s, tickets, st);
    s->cv_done.notify_all();
  }
  return true;
}

void dispatcher(sg_server_s* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop.load()) {
    bool completed = false;
    for (Slot& sl : s->slots) {
      if (!sl.busy) continue;
      const cudaError_t e = cudaEventQuery(sl.ev);
      if (e == cudaErrorNotReady) continue;
      sl.busy = false;
      sg_status st = e == cudaSuccess ? SG_OK : SG_ERR_CUDA;
      if (e != cudaSuccess) cudaGetLastError();
      if (st == SG_OK) {  // a launch whose grid barrier timed out did not finish its work
        auto it = sl.ws.find(ws_key(sl.graph, sl.ws_kind));
        if (it != sl.ws.end()) {
          if (sl.ws_kind == kWsBfs) st = sgb::bfs_launch_status((sg_bfs)it->second.handle);
          if (sl.ws_kind == kWsBatch) st = sgb::msbfs_launch_status((sg_msbfs)it->second.handle);
          if (sl.ws_kind == kWsSssp) st = sgb::sssp_launch_status((sg_sssp)it->second.handle);
        }
      }
      finish(s, sl.batch, st);
      sl.batch.clear();
      completed = true;
    }
    if (completed) s->cv_done.notify_all();
    while (admit_one(s)) {
    }
    bool any_busy = false;
    for (const Slot& sl : s->slots) any_busy |= sl.busy;
    if (any_busy) {
      // poll completions at a few-microsecond grain without holding the lock
      lk.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(2));
      lk.lock();
    } else {
      s->cv_submit.wait_for(lk, std::chrono::milliseconds(2));
    }
  }
}

}  // namespace

extern "C" {

sg_status sg_server_create(const sg_server_config* cfg, sg_server* out) {
  sgb::clear_error();
  SG_REQUIRE(out, SG_ERR_INVALID, "NULL argument");
  *out = nullptr;
  sg_server_config c{};
  if (cfg) c = *cfg;
  if (!c.slots) c.slots = 4;
  if (!c.max_batch) c.max_batch = 64;
  if (!c.min_batch) c.min_batch = 16;
  SG_REQUIRE(c.slots <= 64, SG_ERR_INVALID, "at most 64 slots");
  SG_REQUIRE(c.max_batch <= 64, SG_ERR_INVALID, "a batch holds at most 64 queries");
  SG_REQUIRE(c.sssp_delta >= 0.0, SG_ERR_INVALID, "sssp_delta must be non-negative");
  if (!c.memory_budget) {
    size_t f = 0, t = 0;
    SG_CUDA(cudaMemGetInfo(&f, &t));
    c.memory_budget = f / 2;
  }
  sg_server s = new sg_server_s();
  s->cfg = c;
  cudaGetDevice(&s->device);
  s->slots.resize(c.slots);
  for (Slot& sl : s->slots) {
    if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      for (Slot& x : s->slots) {
        if (x.ev) cudaEventDestroy(x.ev);
        if (x.stream) cudaStreamDestroy(x.stream);
      }
      delete s;
      return sgb::fail(SG_ERR_CUDA, "server: stream or event creation failed");
    }
  }
  s->worker = std::thread(dispatcher, s);
  *out = s;
  return SG_OK;
}

sg_status sg_server_destroy(sg_server s) {
  if (!s) return SG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_submit.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (Slot& sl : s->slots) {
    cudaStreamSynchronize(sl.stream);
    for (auto& kv : sl.ws) ws_destroy((int)(kv.first & 3), kv.second);
    cudaEventDestroy(sl.ev);
    cudaStreamDestroy(sl.stream);
  }
  delete s;
  return SG_OK;
}

sg_status sg_server_add_graph(sg_server s, sg_graph g, uint32_t* graph_id) {
  sgb::clear_error();
  SG_REQUIRE(s && g && graph_id, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaStreamSynchronize(g->stream));  // the upload is complete before any slot reads it
  std::lock_guard<std::mutex> lk(s->mu);
  *graph_id = (uint32_t)s->graphs.size();
  s->graphs.push_back(g);
  return SG_OK;
}

sg_status sg_server_prepare(sg_server s, uint32_t graph_id) {
  sgb::clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  SG_REQUIRE(graph_id < s->graphs.size(), SG_ERR_INVALID, "unknown graph id");
  const sg_graph g = s->graphs[graph_id];
  bool short_of_memory = false;
  for (uint32_t si = 0; si < s->slots.size(); si++)
    for (int kind : {kWsBfs, kWsBatch, kWsSssp}) {
      if (kind == kWsSssp && g->value_type == SG_WEIGHT_NONE) continue;
      if (s->slots[si].ws.count(ws_key(graph_id, kind))) continue;
      if (s->ws_bytes + ws_estimate(g, kind, s->cfg.max_batch) > s->cfg.memory_budget) {
        short_of_memory = true;  // (no eviction for a prepared workspace)
        continue;
      }
      Workspace* w = nullptr;
      bool never = false;
      SG_TRY(get_workspace(s, si, graph_id, kind, &w, &never));
    }
  if (short_of_memory) return sgb::fail(SG_ERR_NOMEM, "server: some workspaces do not fit in the memory budget");
  return SG_OK;
}

sg_status sg_server_submit(sg_server s, uint32_t graph_id, int kind, uint32_t source, void* host_out,
                           uint64_t* ticket) {
  sgb::clear_error();
  SG_REQUIRE(s && ticket, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(kind == SG_QUERY_BFS || kind == SG_QUERY_SSSP, SG_ERR_INVALID, "unknown query kind");
  std::lock_guard<std::mutex> lk(s->mu);
  SG_REQUIRE(graph_id < s->graphs.size(), SG_ERR_INVALID, "unknown graph id");
  const sg_graph g = s->graphs[graph_id];
  SG_REQUIRE(source < g->n, SG_ERR_INVALID, "source out of range");
  SG_REQUIRE(kind == SG_QUERY_BFS || g->value_type != SG_WEIGHT_NONE, SG_ERR_INVALID,
             "SSSP needs a weighted graph");
  Query q;
  q.ticket = s->queries.size();
  q.graph = graph_id;
  q.kind = kind;
  q.source = source;
  q.host_out = host_out;
  q.res.status = SG_ERR_NOT_INITIALIZED;
  q.res.graph = graph_id;
  q.res.kind = kind;
  q.res.source = source;
  q.res.submit_ns = now_ns();
  s->queries.push_back(q);
  s->pending.push_back(q.ticket);
  s->stats.submitted++;
  *ticket = q.ticket;
  s->cv_submit.notify_one();
  return SG_OK;
}

sg_status sg_server_wait(sg_server s, uint64_t ticket, double timeout_s, sg_query_result* result) {
  SG_REQUIRE(s, SG_ERR_INVALID, "NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  SG_REQUIRE(ticket < s->queries.size(), SG_ERR_INVALID, "unknown ticket");
  const auto until = Clock::now() + std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9);
  while (!s->queries[ticket].done)
    if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout && !s->queries[ticket].done)
      return sgb::fail(SG_ERR_TIMEOUT, "server: the query has not completed");
  if (result) *result = s->queries[ticket].res;
  return SG_OK;
}

sg_status sg_server_drain(sg_server s, double timeout_s) {
  SG_REQUIRE(s, SG_ERR_INVALID, "NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  const auto until = Clock::now() + std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9);
  while (s->stats.completed + s->stats.failed < s->stats.submitted)
    if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout &&
        s->stats.completed + s->stats.failed < s->stats.submitted)
      return sgb::fail(SG_ERR_TIMEOUT, "server: queries still running");
  return SG_OK;
}

sg_status sg_server_get_stats(sg_server s, sg_server_stats* stats) {
  SG_REQUIRE(s && stats, SG_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *stats = s->stats;
  stats->workspace_bytes = s->ws_bytes;
  stats->peak_workspace_bytes = s->peak_ws_bytes;
  stats->memory_budget = s->cfg.memory_budget;
  return SG_OK;
}

}  // extern "C"
