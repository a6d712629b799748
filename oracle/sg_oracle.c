/*
 * sg_oracle.c -- CPU restatement of SYgraph's frontier algorithms.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * sygraph_b200: only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference leg of bench.py load it.  Nothing in the product links it.
 *
 * Every function restates the algorithm of one reference file (paths are
 * relative to the SYgraph project root).  The reference itself is SYCL and
 * cannot be compiled without a SYCL compiler, so parity is pinned by running
 * these functions on the reference's own known-answer fixtures
 * (tests/include/test_utils.hpp, include/sygraph/io/matrices.hpp) and checking
 * the answers its tests assert (tests/algorithms/*.cpp, tests/operators/*.cpp).
 *
 * Conventions shared with the reference:
 *   - vertex ids, row offsets and column indices are uint32;
 *   - an unreached BFS depth / SSSP distance is n+1 (bfs.hpp:67, sssp.hpp:43),
 *     cast to the distance type;
 *   - BFS direction: 0 = push, 1 = pull, 2 = hybrid (bfs.hpp:29).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <omp.h>

#define OR_PUSH 0
#define OR_PULL 1
#define OR_HYBRID 2

static inline int or_threads(int nthreads) { return nthreads > 0 ? nthreads : omp_get_max_threads(); }

/* ------------------------------------------------------------------------- */
/* BFS                                                                        */
/* ------------------------------------------------------------------------- */

/* Level-synchronous BFS exactly as the example validator walks it
 * (examples/bfs/bfs.cpp:16-56): depth[source] = 0, unreached = n+1. */
void or_bfs_levels(uint32_t n, const uint32_t* ro, const uint32_t* col, uint32_t src, uint32_t* depth) {
  const uint32_t inf = n + 1;
  for (uint32_t i = 0; i < n; i++) depth[i] = inf;
  uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint64_t head = 0, tail = 0;
  depth[src] = 0;
  q[tail++] = src;
  while (head < tail) {
    uint32_t v = q[head++];
    for (uint32_t e = ro[v]; e < ro[v + 1]; e++) {
      uint32_t u = col[e];
      if (depth[u] == inf) {
        depth[u] = depth[v] + 1;
        q[tail++] = u;
      }
    }
  }
  free(q);
}

/* Frontier BFS restating BFS::run (include/sygraph/algorithms/bfs.hpp:153-238)
 * with the push functor (:185-191), the pull functor (:201-207) over the
 * inverse graph (operators/advance/common.hpp:49-75, pull candidates are the
 * vertices NOT in the input frontier; the in-neighbour must be IN it; the
 * candidate stops at its first successful edge, workgroup_mapped.hpp:151-175)
 * and the hybrid heuristic (bfs.hpp:284-350):
 *   push -> pull  when (float)(uint32)sum_deg(out) > (float)(uint32)sum_deg(unvisited) / alpha
 *   pull -> push  when (float)|out| < (float)n / beta
 * Returns the number of iterations (BFSRunDetails::iterations); steps[i] is 0
 * for a push step and 1 for a pull step (push_steps / pull_steps). OpenMP. */
int64_t or_bfs_frontier(uint32_t n, const uint32_t* ro, const uint32_t* col, const uint32_t* iro, const uint32_t* icol,
                        uint32_t src, int direction, float alpha, float beta, uint32_t* depth, uint8_t* steps,
                        uint64_t steps_cap, int nthreads) {
  const int nt = or_threads(nthreads);
  const uint32_t inf = n + 1;
  uint8_t* in_flag = (uint8_t*)calloc(n ? n : 1, 1);
  uint8_t* out_flag = (uint8_t*)calloc(n ? n : 1, 1);
  uint32_t* in_list = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t* out_list = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint64_t in_size = 0;

#pragma omp parallel for num_threads(nt) schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) depth[i] = inf;
  depth[src] = 0;
  in_flag[src] = 1;
  in_list[0] = src;
  in_size = 1;

  int push = direction != OR_PULL;
  int64_t iter = 0;
  while (in_size > 0) {
    if ((uint64_t)iter < steps_cap) steps[iter] = push ? 0 : 1;
    const uint32_t next_depth = (uint32_t)iter + 1;
    if (push) {
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
      for (int64_t i = 0; i < (int64_t)in_size; i++) {
        uint32_t v = in_list[i];
        for (uint32_t e = ro[v]; e < ro[v + 1]; e++) {
          uint32_t u = col[e];
          /* functor: if (distances[dst] == size + 1) { distances[dst] = iter + 1; return true; } */
          if (__atomic_load_n(&depth[u], __ATOMIC_RELAXED) == inf) {
            __atomic_store_n(&depth[u], next_depth, __ATOMIC_RELAXED);
            __atomic_store_n(&out_flag[u], 1, __ATOMIC_RELAXED);
          }
        }
      }
    } else {
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
      for (int64_t vv = 0; vv < (int64_t)n; vv++) {
        uint32_t v = (uint32_t)vv;
        if (in_flag[v]) continue; /* check(): pull candidates are outside the input frontier */
        if (depth[v] != inf) continue; /* the functor returns false for every edge of a visited candidate */
        for (uint32_t e = iro[v]; e < iro[v + 1]; e++) {
          uint32_t u = icol[e];
          if (!in_flag[u]) continue; /* isValidNeighbor(): in-neighbour must be in the frontier */
          if (depth[u] == (uint32_t)iter) {
            depth[v] = next_depth;
            out_flag[v] = 1;
            break; /* short-circuit after the first successful edge */
          }
        }
      }
    }
    /* compact out_flag into out_list (order does not matter) */
    uint64_t out_size = 0;
    for (uint32_t v = 0; v < n; v++)
      if (out_flag[v]) out_list[out_size++] = v;

    if (direction == OR_HYBRID) {
      if (push) {
        uint64_t fd = 0, ud = 0;
#pragma omp parallel for num_threads(nt) reduction(+ : fd) schedule(static)
        for (int64_t i = 0; i < (int64_t)out_size; i++) fd += ro[out_list[i] + 1] - ro[out_list[i]];
#pragma omp parallel for num_threads(nt) reduction(+ : ud) schedule(static)
        for (int64_t v = 0; v < (int64_t)n; v++)
          if (depth[v] == inf) ud += ro[v + 1] - ro[v];
        uint32_t fd32 = (uint32_t)fd, ud32 = (uint32_t)ud;
        if ((float)fd32 > (float)ud32 / alpha) push = 0;
      } else {
        if ((float)out_size < (float)n / beta) push = 1;
      }
    }
    /* swap(in, out); out.clear() */
    for (uint64_t i = 0; i < in_size; i++) in_flag[in_list[i]] = 0;
    uint8_t* tf = in_flag; in_flag = out_flag; out_flag = tf;
    uint32_t* tl = in_list; in_list = out_list; out_list = tl;
    in_size = out_size;
    iter++;
  }
  free(in_flag); free(out_flag); free(in_list); free(out_list);
  return iter;
}

/* ------------------------------------------------------------------------- */
/* SSSP                                                                       */
/* ------------------------------------------------------------------------- */

/* Binary min-heap of (key, vertex) used by the Dijkstra validator. */
typedef struct { double key; uint32_t v; } or_heap_item;
typedef struct { or_heap_item* a; uint64_t n, cap; } or_heap;

static void or_heap_push(or_heap* h, double key, uint32_t v) {
  if (h->n == h->cap) { h->cap = h->cap ? 2 * h->cap : 1024; h->a = (or_heap_item*)realloc(h->a, h->cap * sizeof(or_heap_item)); }
  uint64_t i = h->n++;
  while (i > 0) {
    uint64_t p = (i - 1) / 2;
    if (h->a[p].key <= key) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i].key = key; h->a[i].v = v;
}

static or_heap_item or_heap_pop(or_heap* h) {
  or_heap_item top = h->a[0];
  or_heap_item last = h->a[--h->n];
  uint64_t i = 0;
  for (;;) {
    uint64_t c = 2 * i + 1;
    if (c >= h->n) break;
    if (c + 1 < h->n && h->a[c + 1].key < h->a[c].key) c++;
    if (last.key <= h->a[c].key) break;
    h->a[i] = h->a[c];
    i = c;
  }
  if (h->n) h->a[i] = last;
  return top;
}

/* Dijkstra with fp32 distances, as the example validator computes them
 * (examples/sssp/sssp.cpp:23-66): new_dist = curr_dist + w in fp32, distances
 * start at (float)(n+1).  The fixed point is the same as the frontier
 * Bellman-Ford of algorithms/sssp.hpp:178-196 because fl(d + w) is monotone in d. */
void or_sssp_dijkstra_f32(uint32_t n, const uint32_t* ro, const uint32_t* col, const float* w, uint32_t src, float* dist) {
  const float inf = (float)(n + 1);
  for (uint32_t i = 0; i < n; i++) dist[i] = inf;
  dist[src] = 0.0f;
  or_heap h = {0};
  or_heap_push(&h, 0.0, src);
  while (h.n) {
    or_heap_item it = or_heap_pop(&h);
    float d = (float)it.key;
    if (d > dist[it.v]) continue; /* stale entry: relaxing from it cannot lower anything */
    for (uint32_t e = ro[it.v]; e < ro[it.v + 1]; e++) {
      float nd = d + w[e];
      uint32_t u = col[e];
      if (nd < dist[u]) { dist[u] = nd; or_heap_push(&h, (double)nd, u); }
    }
  }
  free(h.a);
}

/* Same with uint32 weights / distances (the grid workload's weight type). */
void or_sssp_dijkstra_u32(uint32_t n, const uint32_t* ro, const uint32_t* col, const uint32_t* w, uint32_t src, uint32_t* dist) {
  const uint32_t inf = n + 1;
  for (uint32_t i = 0; i < n; i++) dist[i] = inf;
  dist[src] = 0;
  or_heap h = {0};
  or_heap_push(&h, 0.0, src);
  while (h.n) {
    or_heap_item it = or_heap_pop(&h);
    uint32_t d = (uint32_t)it.key;
    if (d > dist[it.v]) continue;
    for (uint32_t e = ro[it.v]; e < ro[it.v + 1]; e++) {
      uint32_t nd = d + w[e];
      uint32_t u = col[e];
      if (nd < dist[u]) { dist[u] = nd; or_heap_push(&h, (double)nd, u); }
    }
  }
  free(h.a);
}

static inline float or_atomic_min_f32(float* p, float v) {
  /* non-negative floats order like their uint32 bit patterns */
  uint32_t* pu = (uint32_t*)p;
  uint32_t nv; memcpy(&nv, &v, 4);
  uint32_t old = __atomic_load_n(pu, __ATOMIC_RELAXED);
  while (nv < old && !__atomic_compare_exchange_n(pu, &old, nv, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
  float of; memcpy(&of, &old, 4);
  return of;
}

/* Frontier Bellman-Ford restating SSSP::run (algorithms/sssp.hpp:152-210):
 * each frontier vertex relaxes its out-edges with fetch_min (:180-189) and a
 * destination whose distance dropped joins the next frontier; the filter step
 * (:192-196) only de-duplicates, which the flag array does here.
 * Returns the number of iterations.  OpenMP (the timed CPU baseline). */
int64_t or_sssp_frontier_f32(uint32_t n, const uint32_t* ro, const uint32_t* col, const float* w, uint32_t src, float* dist,
                             int nthreads) {
  const int nt = or_threads(nthreads);
  const float inf = (float)(n + 1);
  uint8_t* out_flag = (uint8_t*)calloc(n ? n : 1, 1);
  uint32_t* in_list = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t* out_list = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) dist[i] = inf;
  dist[src] = 0.0f;
  in_list[0] = src;
  uint64_t in_size = 1;
  int64_t iter = 0;
  while (in_size) {
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)in_size; i++) {
      uint32_t v = in_list[i];
      float dv;
      {
        uint32_t b = __atomic_load_n((uint32_t*)&dist[v], __ATOMIC_RELAXED);
        memcpy(&dv, &b, 4);
      }
      for (uint32_t e = ro[v]; e < ro[v + 1]; e++) {
        uint32_t u = col[e];
        float nd = dv + w[e];
        float old = or_atomic_min_f32(&dist[u], nd);
        if (nd < old) __atomic_store_n(&out_flag[u], 1, __ATOMIC_RELAXED);
      }
    }
    uint64_t out_size = 0;
    for (uint32_t v = 0; v < n; v++)
      if (out_flag[v]) { out_list[out_size++] = v; out_flag[v] = 0; }
    uint32_t* t = in_list; in_list = out_list; out_list = t;
    in_size = out_size;
    iter++;
  }
  free(out_flag); free(in_list); free(out_list);
  return iter;
}

/* ------------------------------------------------------------------------- */
/* Connected components: maximum-label propagation                           */
/* ------------------------------------------------------------------------- */

/* Restates CC::run (algorithms/cc.hpp:103-169): labels[i] = i, one pass over
 * every edge, then frontier passes; along an edge src->dst the larger label
 * wins ("if dst_label < src_label store src_label", :137-142, :151-156).  The
 * reference's load/compare/store is not atomic and can lose an update; the
 * intended fixed point -- label(v) = max id over the vertices that reach v,
 * the maximum id of v's component when the graph is symmetric -- is what this
 * worklist computes deterministically. */
void or_cc_maxlabel(uint32_t n, const uint32_t* ro, const uint32_t* col, uint32_t* labels) {
  for (uint32_t i = 0; i < n; i++) labels[i] = i;
  uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint8_t* inq = (uint8_t*)calloc(n ? n : 1, 1);
  uint64_t head = 0, count = 0; /* ring buffer of capacity n */
  for (uint32_t v = 0; v < n; v++) { q[count++] = v; inq[v] = 1; }
  while (count) {
    uint32_t v = q[head];
    head = (head + 1) % n;
    count--;
    inq[v] = 0;
    uint32_t lv = labels[v];
    for (uint32_t e = ro[v]; e < ro[v + 1]; e++) {
      uint32_t u = col[e];
      if (labels[u] < lv) {
        labels[u] = lv;
        if (!inq[u]) { inq[u] = 1; q[(head + count) % n] = u; count++; }
      }
    }
  }
  free(q); free(inq);
}

/* ------------------------------------------------------------------------- */
/* Betweenness centrality (Brandes), FP64                                    */
/* ------------------------------------------------------------------------- */

/* Restates BC::run (algorithms/bc.hpp:118-200) in FP64 for each source s of
 * srcs[0..k): forward levels with sigma[dst] += sigma[src] along edges whose
 * dst label is label[src]+1 (:140-165); backward in reverse level order,
 * delta[src] += sigma[src]/sigma[dst]*(1+delta[dst]) for src != s (:167-194).
 * bc[v] accumulates delta_s(v) over the sources (no 1/2 factor, no
 * normalisation).  Sources run in parallel, one per thread. */
void or_bc(uint32_t n, const uint32_t* ro, const uint32_t* col, const uint32_t* srcs, uint32_t k, double* bc, int nthreads) {
  const int nt = or_threads(nthreads);
  memset(bc, 0, sizeof(double) * n);
#pragma omp parallel num_threads(nt)
  {
    double* local_bc = (double*)calloc(n ? n : 1, sizeof(double));
    uint32_t* label = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    double* sigma = (double*)malloc(sizeof(double) * (n ? n : 1));
    double* delta = (double*)malloc(sizeof(double) * (n ? n : 1));
    uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
#pragma omp for schedule(dynamic, 1)
    for (int64_t si = 0; si < (int64_t)k; si++) {
      uint32_t s = srcs[si];
      for (uint32_t i = 0; i < n; i++) { label[i] = UINT32_MAX; sigma[i] = 0.0; delta[i] = 0.0; }
      label[s] = 0; sigma[s] = 1.0;
      uint64_t head = 0, tail = 0;
      order[tail++] = s;
      while (head < tail) {
        uint32_t v = order[head++];
        for (uint32_t e = ro[v]; e < ro[v + 1]; e++) {
          uint32_t u = col[e];
          if (label[u] == UINT32_MAX) { label[u] = label[v] + 1; order[tail++] = u; }
          if (label[u] == label[v] + 1) sigma[u] += sigma[v];
        }
      }
      /* BFS order is non-decreasing in level: walk it backwards */
      for (int64_t i = (int64_t)tail - 1; i >= 0; i--) {
        uint32_t v = order[i];
        if (v == s) continue;
        double acc = 0.0;
        for (uint32_t e = ro[v]; e < ro[v + 1]; e++) {
          uint32_t u = col[e];
          if (label[u] != UINT32_MAX && label[v] + 1 == label[u]) acc += sigma[v] / sigma[u] * (1.0 + delta[u]);
        }
        delta[v] = acc;
        local_bc[v] += acc;
      }
    }
#pragma omp critical
    for (uint32_t i = 0; i < n; i++) bc[i] += local_bc[i];
    free(local_bc); free(label); free(sigma); free(delta); free(order);
  }
}

/* ------------------------------------------------------------------------- */
/* Triangle counting                                                          */
/* ------------------------------------------------------------------------- */

/* Per-vertex counts with the reference's convention (algorithms/tc.hpp:80-107
 * without its over-count, see below): for every edge (u,v) with u < v,
 * triangles[u] += |N(u) n N(v)| by a two-pointer merge of the sorted lists.
 * The reference adds the running count inside the merge loop (tc.hpp:104),
 * which over-counts whenever a match is not the merge's last step; this
 * restatement adds it once.  Returns sum(triangles)/3 (tc.hpp:120-138) in
 * uint64.  Cost is sum over edges of deg(u)+deg(v): small graphs only. */
uint64_t or_tc_edge_merge(uint32_t n, const uint32_t* ro, const uint32_t* col, uint64_t* per_vertex, int nthreads) {
  const int nt = or_threads(nthreads);
  uint64_t total = 0;
#pragma omp parallel for num_threads(nt) reduction(+ : total) schedule(dynamic, 16)
  for (int64_t uu = 0; uu < (int64_t)n; uu++) {
    uint32_t u = (uint32_t)uu;
    uint64_t tu = 0;
    for (uint32_t e = ro[u]; e < ro[u + 1]; e++) {
      uint32_t v = col[e];
      if (u >= v) continue;
      uint32_t a = ro[u], ae = ro[u + 1], b = ro[v], be = ro[v + 1];
      while (a < ae && b < be) {
        if (col[a] == col[b]) { tu++; a++; b++; }
        else if (col[a] < col[b]) a++;
        else b++;
      }
    }
    if (per_vertex) per_vertex[u] = tu;
    total += tu;
  }
  return total / 3;
}

/* Exact triangle count of a symmetric graph on the degree-ordered DAG: each
 * edge is kept once, from the endpoint with the smaller (degree, id) key, and
 * each triangle is found once as N+(u) n N+(v) for a DAG edge u->v.  Marker
 * array per thread.  When per_vertex is non-NULL it receives the reference's
 * per-vertex convention: a triangle a<b<c adds 2 to a and 1 to b. */
uint64_t or_tc_dag(uint32_t n, const uint32_t* ro, const uint32_t* col, uint64_t* per_vertex, int nthreads) {
  const int nt = or_threads(nthreads);
  /* build the DAG */
  uint32_t* dro = (uint32_t*)malloc(sizeof(uint32_t) * ((uint64_t)n + 1));
  dro[0] = 0;
  for (uint32_t u = 0; u < n; u++) {
    uint32_t du = ro[u + 1] - ro[u], c = 0;
    for (uint32_t e = ro[u]; e < ro[u + 1]; e++) {
      uint32_t v = col[e], dv = ro[v + 1] - ro[v];
      if (du < dv || (du == dv && u < v)) c++;
    }
    dro[u + 1] = dro[u] + c;
  }
  uint32_t* dcol = (uint32_t*)malloc(sizeof(uint32_t) * (dro[n] ? dro[n] : 1));
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256)
  for (int64_t uu = 0; uu < (int64_t)n; uu++) {
    uint32_t u = (uint32_t)uu, du = ro[u + 1] - ro[u], p = dro[u];
    for (uint32_t e = ro[u]; e < ro[u + 1]; e++) {
      uint32_t v = col[e], dv = ro[v + 1] - ro[v];
      if (du < dv || (du == dv && u < v)) dcol[p++] = v;
    }
  }
  if (per_vertex) memset(per_vertex, 0, sizeof(uint64_t) * n);
  uint64_t total = 0;
#pragma omp parallel num_threads(nt) reduction(+ : total)
  {
    uint8_t* mark = (uint8_t*)calloc(n ? n : 1, 1);
#pragma omp for schedule(dynamic, 64)
    for (int64_t uu = 0; uu < (int64_t)n; uu++) {
      uint32_t u = (uint32_t)uu;
      for (uint32_t e = dro[u]; e < dro[u + 1]; e++) mark[dcol[e]] = 1;
      for (uint32_t e = dro[u]; e < dro[u + 1]; e++) {
        uint32_t v = dcol[e];
        for (uint32_t f = dro[v]; f < dro[v + 1]; f++) {
          uint32_t w = dcol[f];
          if (mark[w]) {
            total++;
            if (per_vertex) {
              uint32_t a = u, b = v, c = w, t;
              if (a > b) { t = a; a = b; b = t; }
              if (b > c) { t = b; b = c; c = t; }
              if (a > b) { t = a; a = b; b = t; }
              __atomic_fetch_add(&per_vertex[a], 2, __ATOMIC_RELAXED);
              __atomic_fetch_add(&per_vertex[b], 1, __ATOMIC_RELAXED);
            }
          }
        }
      }
      for (uint32_t e = dro[u]; e < dro[u + 1]; e++) mark[dcol[e]] = 0;
    }
    free(mark);
  }
  free(dro); free(dcol);
  return total;
}

/* ------------------------------------------------------------------------- */
/* Multi-source BFS (checker for the batched bit-parallel kernels)           */
/* ------------------------------------------------------------------------- */

/* Independent level-synchronous BFS per source (examples/bfs/bfs.cpp:16-56),
 * one source per thread; depth is k x n, row-major by source. */
void or_bfs_multi(uint32_t n, const uint32_t* ro, const uint32_t* col, const uint32_t* srcs, uint32_t k, uint32_t* depth,
                  int nthreads) {
  const int nt = or_threads(nthreads);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1)
  for (int64_t i = 0; i < (int64_t)k; i++) or_bfs_levels(n, ro, col, srcs[i], depth + (uint64_t)i * n);
}

/* Sum of degrees over reached vertices: the reference's visited-edge count
 * behind its MTEPS figure (algorithms/bfs.hpp:88-99, utils/profiler.hpp:65-67). */
uint64_t or_visited_edges(uint32_t n, const uint32_t* ro, const uint32_t* depth, uint32_t unreached) {
  uint64_t s = 0;
  for (uint32_t v = 0; v < n; v++)
    if (depth[v] != unreached) s += ro[v + 1] - ro[v];
  return s;
}

/* ------------------------------------------------------------------------- */
/* Benchmark inputs without the product library                              */
/* ------------------------------------------------------------------------- */

/* The seeded RMAT graph of the benchmarks, restated so the CPU baseline arm
 * builds its input without loading the product library: the same draws, so
 * the same CSR bit for bit (tested against sg_rmat_generate).  Every random
 * number is the splitmix64 finaliser (Steele, Lea, Flood 2014) of a counter:
 *   hash2(seed, i) = mix64(mix64(seed) ^ i).
 * Pair i draws its quadrant at level l (most significant bit first) from the
 * high 32 bits of mix64(hash2(seed, i) + l) at even l and the low 32 bits of
 * the same word at the odd l after it, as a fraction of 2^32 against the
 * cumulative probabilities a, a+b, a+b+c: quadrant 0 keeps both bits, 1 sets
 * the column bit, 2 the row bit, 3 both.  Ids are relabelled by a
 * Fisher-Yates shuffle (i from n-1 down to 1 swaps perm[i] with
 * perm[hash2(perm_seed, i) % (i+1)]; perm_seed 0 = identity).  Self-loops are
 * dropped, both directions kept, duplicates removed, rows sorted.  The weight
 * of the unordered pair {lo, hi} is h = hash2(weight_seed, lo << 32 | hi):
 * float32 ((h >> 40) + 1) * 2^-24 on (0, 1], or uint32 (h >> 58) + 1 on
 * [1, 64]. */
static inline uint64_t or_mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
static inline uint64_t or_hash2(uint64_t seed, uint64_t i) { return or_mix64(or_mix64(seed) ^ i); }

static uint32_t or_pair_weight_bits(uint64_t seed, uint32_t u, uint32_t v, int value_type) {
  const uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
  const uint64_t h = or_hash2(seed, ((uint64_t)lo << 32) | hi);
  if (value_type == 1) {
    float w = (float)((h >> 40) + 1) * (1.0f / 16777216.0f);
    uint32_t bits;
    memcpy(&bits, &w, 4);
    return bits;
  }
  return (uint32_t)(h >> 58) + 1u;
}

/* LSD radix sort of n keys on their low key_bits bits, 11-bit digits, each
 * thread counting and scattering its own contiguous range (stable). */
static int or_radix_sort(uint64_t* keys, size_t n, int key_bits) {
  if (n < 2) return 0;
  uint64_t* tmp = (uint64_t*)malloc(sizeof(uint64_t) * n);
  if (!tmp) return -1;
  const int digit = 11, nb = 1 << 11;
  const int nt = omp_get_max_threads();
  size_t* hist = (size_t*)malloc(sizeof(size_t) * (size_t)nt * nb);
  if (!hist) {
    free(tmp);
    return -1;
  }
  uint64_t *src = keys, *dst = tmp;
  int passes = 0;
  for (int shift = 0; shift < key_bits; shift += digit, passes++) {
    memset(hist, 0, sizeof(size_t) * (size_t)nt * nb);
#pragma omp parallel num_threads(nt)
    {
      const int t = omp_get_thread_num();
      const size_t lo = n * t / nt, hi = n * (t + 1) / nt;
      size_t* h = hist + (size_t)t * nb;
      for (size_t i = lo; i < hi; i++) h[(src[i] >> shift) & (nb - 1)]++;
#pragma omp barrier
#pragma omp single
      {
        size_t sum = 0;
        for (int b = 0; b < nb; b++)
          for (int tt = 0; tt < nt; tt++) {
            const size_t c = hist[(size_t)tt * nb + b];
            hist[(size_t)tt * nb + b] = sum;
            sum += c;
          }
      }
      for (size_t i = lo; i < hi; i++) dst[h[(src[i] >> shift) & (nb - 1)]++] = src[i];
    }
    uint64_t* sw = src;
    src = dst;
    dst = sw;
  }
  if (passes & 1) memcpy(keys, src, sizeof(uint64_t) * n);
  free(tmp);
  free(hist);
  return 0;
}

/* Returns m, or -1 on failure; *ro (n+1), *col (m) and *val (m, or NULL for
 * value_type 0) are malloc'd and released with or_free. */
int64_t or_rmat_generate(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                         uint64_t weight_seed, uint64_t perm_seed, int value_type, uint32_t** ro_out,
                         uint32_t** col_out, uint32_t** val_out) {
  if (scale < 1 || scale > 30) return -1;
  const uint32_t n = 1u << scale;
  const uint64_t pairs = (uint64_t)edge_factor * n;
  const double ab = a + b, abc = a + b + c;
  uint32_t* perm = (uint32_t*)malloc(sizeof(uint32_t) * n);
  uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * 2 * (pairs ? pairs : 1));
  if (!perm || !keys) {
    free(perm);
    free(keys);
    return -1;
  }
  for (uint32_t i = 0; i < n; i++) perm[i] = i;
  if (perm_seed)
    for (uint32_t i = n - 1; i > 0; i--) {
      const uint32_t j = (uint32_t)(or_hash2(perm_seed, i) % ((uint64_t)i + 1));
      const uint32_t t = perm[i];
      perm[i] = perm[j];
      perm[j] = t;
    }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)pairs; i++) {
    const uint64_t st = or_hash2(seed, (uint64_t)i);
    uint32_t u = 0, v = 0;
    uint64_t r = 0;
    for (uint32_t l = 0; l < scale; l++) {
      if ((l & 1) == 0) r = or_mix64(st + l);
      const double x = (double)((l & 1) ? (r & 0xffffffffu) : (r >> 32)) * (1.0 / 4294967296.0);
      const uint32_t bit = 1u << (scale - 1 - l);
      if (x < a) {
      } else if (x < ab) {
        v |= bit;
      } else if (x < abc) {
        u |= bit;
      } else {
        u |= bit;
        v |= bit;
      }
    }
    u = perm[u];
    v = perm[v];
    if (u == v) {
      keys[2 * i] = keys[2 * i + 1] = ~0ull;
    } else {
      keys[2 * i] = ((uint64_t)u << scale) | v;
      keys[2 * i + 1] = ((uint64_t)v << scale) | u;
    }
  }
  free(perm);
  size_t k = 0;
  for (size_t i = 0; i < 2 * pairs; i++)
    if (keys[i] != ~0ull) keys[k++] = keys[i];
  if (or_radix_sort(keys, k, 2 * (int)scale) != 0) {
    free(keys);
    return -1;
  }
  size_t m = 0;
  for (size_t i = 0; i < k; i++)
    if (m == 0 || keys[i] != keys[m - 1]) keys[m++] = keys[i];
  uint32_t* ro = (uint32_t*)calloc((size_t)n + 1, sizeof(uint32_t));
  uint32_t* col = (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1));
  uint32_t* val = value_type ? (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1)) : NULL;
  if (!ro || !col || (value_type && !val)) {
    free(keys);
    free(ro);
    free(col);
    free(val);
    return -1;
  }
  const uint64_t low = (1ull << scale) - 1;
  for (size_t i = 0; i < m; i++) ro[(keys[i] >> scale) + 1]++;
  for (uint32_t v = 0; v < n; v++) ro[v + 1] += ro[v];
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)m; i++) {
    const uint32_t s = (uint32_t)(keys[i] >> scale), d = (uint32_t)(keys[i] & low);
    col[i] = d;
    if (val) val[i] = or_pair_weight_bits(weight_seed, s, d, value_type);
  }
  free(keys);
  *ro_out = ro;
  *col_out = col;
  *val_out = val;
  return (int64_t)m;
}

/* k distinct vertices with degree > 0: candidate i is hash2(seed, i) % n,
 * skipped when taken or isolated (the benchmarks' source draw).  Returns 0,
 * or -1 when fewer than k vertices have edges. */
int or_sample_sources(uint32_t n, const uint32_t* ro, uint32_t k, uint64_t seed, uint32_t* out) {
  uint64_t nonzero = 0;
  for (uint32_t v = 0; v < n; v++) nonzero += ro[v + 1] > ro[v];
  if (nonzero < k) return -1;
  uint8_t* taken = (uint8_t*)calloc(n ? n : 1, 1);
  if (!taken) return -1;
  uint32_t got = 0;
  for (uint64_t i = 0; got < k; i++) {
    const uint32_t v = (uint32_t)(or_hash2(seed, i) % n);
    if (taken[v] || ro[v + 1] == ro[v]) continue;
    taken[v] = 1;
    out[got++] = v;
  }
  free(taken);
  return 0;
}

void or_free(void* p) { free(p); }
