/*
 * sygraph_b200.h -- C ABI of libsygraph_b200.so, the B200 (sm_100a) frontier
 * hot path of SYgraph.
 *
 * SYgraph is a header-only C++20/SYCL library with no FFI: its boundary is
 * the template API under include/sygraph/ called in-process on one
 * sycl::queue.  Each entry point below names the reference interface it
 * replaces (file:line, relative to the SYgraph project root).  The C++20
 * header layer in include/sygraph/ (same names as the reference) is built on
 * these calls; templated advances with user lambdas instantiate the kernels
 * of include/sygraph/detail/advance_kernels.cuh directly.
 *
 * Conventions
 *   - Every call returns an sg_status; SG_OK is 0.  No C++ exception crosses
 *     this boundary.  sg_last_error() gives the message of the last failure
 *     on the calling thread.  Where the reference throws std::runtime_error
 *     (unsupported combinations, uninitialised instances) these calls return
 *     SG_ERR_INVALID / SG_ERR_UNSUPPORTED / SG_ERR_NOT_INITIALIZED.
 *   - Vertex ids, row offsets and column indices are uint32 (the reference's
 *     index_t; every example and test instantiates uint32, e.g.
 *     tests/include/test_utils.hpp:63).  Edge weights are float32 or uint32.
 *   - `stream` is a cudaStream_t passed as void*; NULL means the legacy
 *     default stream.  Objects remember the stream they were created with,
 *     as GraphCSR holds its queue (graph/impls/graph_csr.hpp:434).
 *   - Pointers named host_* are host memory; dev_* are device memory.
 *   - Device-side persistent loops use bounded waits: a wait that runs out
 *     returns SG_ERR_TIMEOUT instead of hanging.
 */
#ifndef SYGRAPH_B200_H
#define SYGRAPH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status -- */
typedef int sg_status;
#define SG_OK 0
#define SG_ERR_INVALID 1         /* bad argument: std::runtime_error in the reference */
#define SG_ERR_CUDA 2            /* a CUDA runtime call failed */
#define SG_ERR_NOMEM 3           /* device or host allocation failed / over budget */
#define SG_ERR_TIMEOUT 4         /* a bounded device-side wait ran out */
#define SG_ERR_UNSUPPORTED 5     /* "Load balancer not implemented" (operators/advance/advance.hpp:63,138) */
#define SG_ERR_NOT_INITIALIZED 6 /* "BFS instance not initialized" (algorithms/bfs.hpp:155) */

/* Message of the last failed call on this thread ("" when none). */
const char* sg_last_error(void);
/* Static name of a status code. */
const char* sg_status_string(sg_status s);
/* Library version string. */
const char* sg_version(void);

/* ---------------------------------------------------------------- enums -- */
/* operators/config.hpp:10-37 */
#define SG_DIR_PUSH 0
#define SG_DIR_PULL 1     /* pull with short-circuit after the first successful edge */
#define SG_DIR_PULL_ALL 2 /* pull without short-circuit */

#define SG_LB_WORKITEM_MAPPED 0  /* one thread per candidate vertex */
#define SG_LB_SUBGROUP_MAPPED 1  /* one warp per candidate vertex */
#define SG_LB_WORKGROUP_MAPPED 2 /* CTA-wide degree scan, edge-parallel (the reference default) */
#define SG_LB_BUCKETING 3        /* lane / warp / CTA buckets by degree */

/* frontier/frontier_settings.hpp:13-27 */
#define SG_VIEW_GRAPH 0
#define SG_VIEW_VERTEX 1
#define SG_VIEW_EDGE 2
#define SG_VIEW_NONE 3

/* operators/config.hpp:31-32 */
#define SG_SIZE_FETCH_FROM_MEMORY (-1)
#define SG_SIZE_INFER_FROM_DEVICE 0

/* algorithms/bfs.hpp:29 */
#define SG_BFS_PUSH 0
#define SG_BFS_PULL 1
#define SG_BFS_HYBRID 2
/* Not in the reference: the learned selector (sg_bfs_set_selector) picks each
 * level's strategy, with the hybrid heuristic as its fallback. */
#define SG_BFS_LEARNED 3

/* Per-level strategies of the fused BFS engine (direction x mapping). */
#define SG_STRATEGY_PUSH_WARP 0
#define SG_STRATEGY_PUSH_CTA 1
#define SG_STRATEGY_PULL_WARP 2
#define SG_STRATEGY_PULL_CTA 3
#define SG_STRATEGY_PULL_ALL_WARP 4
#define SG_STRATEGY_PULL_ALL_CTA 5

#define SG_WEIGHT_NONE 0
#define SG_WEIGHT_F32 1
#define SG_WEIGHT_U32 2

/* graph/properties.hpp:29-32 and the binary CSR flags (io/read_csr.hpp:22-25) */
#define SG_GRAPH_DIRECTED 1u
#define SG_GRAPH_WEIGHTED 2u

/* ------------------------------------------------------ device helpers -- */
sg_status sg_device_count(int* count);
sg_status sg_set_device(int device);
sg_status sg_device_info(int* sm_count, uint64_t* free_bytes, uint64_t* total_bytes);
/* Plain device memory helpers for callers without a CUDA toolchain. */
sg_status sg_malloc_device(uint64_t bytes, void** dev_ptr);
sg_status sg_free_device(void* dev_ptr);
sg_status sg_malloc_host_pinned(uint64_t bytes, void** host_ptr);
sg_status sg_free_host_pinned(void* host_ptr);
/* kind: 0 host->device, 1 device->host, 2 device->device, 3 default (unified addressing) */
sg_status sg_memcpy(void* dst, const void* src, uint64_t bytes, int kind, void* stream);
/* As sg_memcpy, enqueued on `stream` only (no synchronisation for any kind):
 * for pipelines that overlap a result's copy with the next launch; the
 * caller synchronises the stream before reading a device->host copy. */
sg_status sg_memcpy_async(void* dst, const void* src, uint64_t bytes, int kind, void* stream);
sg_status sg_memset(void* dev_ptr, int value, uint64_t bytes, void* stream);
/* A non-blocking stream (does not synchronise with the legacy default stream). */
/* Diagnostic of the bounded grid barrier every fused engine uses (not in the
 * reference): launches `blocks` (1-64) cooperative blocks, all of which but
 * `skip_block` (none when it is >= blocks) wait at one grid barrier polling
 * at most `spin_limit` (1 - 2^20) times.  *timed_out = blocks whose wait ran
 * out, *error_flag = the barrier's error word the engines report as
 * SG_ERR_TIMEOUT.  A block that never arrives makes every other block give up
 * and return; no wait is unbounded. */
sg_status sg_debug_barrier_check(uint32_t blocks, uint32_t skip_block, uint64_t spin_limit, uint32_t* timed_out,
                                 uint32_t* error_flag);
sg_status sg_stream_create(void** stream);
sg_status sg_stream_destroy(void* stream);
sg_status sg_stream_synchronize(void* stream);
/* Device timing for callers without a CUDA toolchain: an event recorded on
 * `stream` (NULL: the legacy default stream), and the milliseconds between
 * two recorded events (waits for `end`). */
sg_status sg_event_record(void* stream, void** event);
sg_status sg_event_elapsed_ms(void* start, void* end, float* ms);
sg_status sg_event_destroy(void* event);
sg_status sg_device_synchronize(void);
/* Number of kernels this library has launched in this process (all entry
 * points, all devices); used to report launch counts. */
uint64_t sg_kernel_launch_count(void);

/* ---------------------------------------------------------------- graph -- */
typedef struct sg_graph_s* sg_graph;

/* Device view of one CSR direction; pointers are device memory owned by the graph. */
typedef struct {
  uint32_t n;
  uint64_t m;
  const uint32_t* row_offsets;
  const uint32_t* column_indices;
  const void* values; /* float32 or uint32 per value_type; NULL when unweighted */
  int value_type;
} sg_graph_view;

/* graph::build::fromCSR<Space>(q, csr, Properties) (graph/build.hpp:31-41),
 * GraphCSR::initializeGraphStorage (graph/impls/graph_csr.hpp:394-426).
 * Copies the host CSR to the device.  host_values may be NULL (every weight
 * is then 1, as fromMM does for pattern matrices).  When flags has
 * SG_GRAPH_DIRECTED the inverse (incoming-edge) CSR is built as well
 * (formats/csr.hpp:179-209); otherwise the inverse view aliases the forward
 * one (graph_csr.hpp:424). */
sg_status sg_graph_create_csr(const uint32_t* host_row_offsets, const uint32_t* host_column_indices,
                              const void* host_values, int value_type, uint32_t n, uint64_t m, uint32_t flags,
                              void* stream, sg_graph* out);
/* Edge list -> device graph, built on the device (the step before the path;
 * the reference builds on the host: io/read_csr.hpp:260-300 fromCOO,
 * formats/csr.hpp:179-209 invert, graph_csr.hpp:394-426 upload).  The same
 * CSR as sg_csr_from_edges followed by sg_graph_create_csr: symmetrize adds
 * (v,u) for every edge (u,v) with u != v and makes the graph undirected,
 * dedupe keeps the first of repeated pairs in edge order, drop_self_loops
 * drops (v,v); rows sorted by column; values NULL or value_type
 * SG_WEIGHT_NONE means every weight 1.  Without symmetrize the graph is
 * directed and its inverse CSR is built too.  src / dst / values are device
 * pointers when device_pointers, else host arrays (copied first).  Edge
 * entries (2 * count when symmetrised) must be below 2^32; an endpoint >= n
 * is SG_ERR_INVALID. */
sg_status sg_graph_create_coo(const uint32_t* src, const uint32_t* dst, const void* values, int value_type,
                              uint32_t n, uint64_t count, int symmetrize, int dedupe, int drop_self_loops,
                              int device_pointers, void* stream, sg_graph* out);
sg_status sg_graph_destroy(sg_graph g);
sg_status sg_graph_info(sg_graph g, uint32_t* n, uint64_t* m, uint32_t* flags, int* value_type);
/* GraphCSR::getDeviceGraph / getInverseDeviceGraph (graph_csr.hpp:300-320). */
sg_status sg_graph_device_view(sg_graph g, int inverse, sg_graph_view* view);
sg_status sg_graph_set_stream(sg_graph g, void* stream);
/* Host copy of row offsets / columns (GraphCSR::getRowOffsets etc.). */
sg_status sg_graph_copy_csr(sg_graph g, int inverse, uint32_t* host_row_offsets, uint32_t* host_column_indices,
                            void* host_values);
/* GraphCSRDevice::getDegree (graph_csr.hpp:64), host query. */
sg_status sg_graph_degree(sg_graph g, uint32_t v, uint32_t* degree);
sg_status sg_graph_memory_bytes(sg_graph g, uint64_t* bytes);
/* The rows of the forward CSR sorted by weight (equal weights keep their
 * column order), the adjacency delta-stepping SSSP reads; built on the
 * device on first use and kept with the graph.  *symmetric = 1 when every
 * row is strictly increasing in column and every edge's reverse carries the
 * same weight (the pull phases of delta-stepping need it).  Output arrays are
 * host arrays of m entries (either may be NULL).  No counterpart in the
 * reference, which has no delta-stepping. */
sg_status sg_graph_weight_sorted(sg_graph g, uint32_t* host_column_indices, void* host_values, int* symmetric);

/* ------------------------------------------------------------- frontier -- */
typedef struct sg_frontier_s* sg_frontier;

/* Device view of a two-level bitmap frontier (MLBDevice, frontier/impls/mlb_frontier.hpp:58-153). */
typedef struct {
  uint32_t num_elems;
  uint32_t words0; /* ceil(num_elems/32) */
  uint32_t words1; /* ceil(words0/32) */
  uint32_t* level0;
  uint32_t* level1;
  int32_t* offsets;       /* compacted active-word indices */
  uint32_t* offsets_size; /* device scalar */
} sg_frontier_view;

/* FrontierMLB(q, num_elems) (mlb_frontier.hpp:162-179) / makeFrontier (frontier/frontier.hpp:68-80). */
sg_status sg_frontier_create(uint32_t num_elems, void* stream, sg_frontier* out);
sg_status sg_frontier_destroy(sg_frontier f);
sg_status sg_frontier_device_view(sg_frontier f, sg_frontier_view* view);
sg_status sg_frontier_num_elems(sg_frontier f, uint32_t* num_elems);
/* FrontierMLB::clear (mlb:367-380) */
sg_status sg_frontier_clear(sg_frontier f);
/* FrontierMLB::insert / remove / check (mlb:248-285) */
sg_status sg_frontier_insert(sg_frontier f, uint32_t idx);
sg_status sg_frontier_remove(sg_frontier f, uint32_t idx);
sg_status sg_frontier_check(sg_frontier f, uint32_t idx, int* present);
/* Bulk insert of a host list (many FrontierMLB::insert calls in one launch). */
sg_status sg_frontier_insert_list(sg_frontier f, const uint32_t* host_ids, uint64_t count);
/* FrontierMLB::empty (mlb:216-246) and size (mlb:287-311). */
sg_status sg_frontier_empty(sg_frontier f, int* empty);
sg_status sg_frontier_size(sg_frontier f, uint64_t* size);
/* FrontierMLB::merge / intersect (mlb:313-337): level-0 OR / AND.  Both
 * levels are kept consistent here (the reference leaves level 1 stale). */
sg_status sg_frontier_merge(sg_frontier f, sg_frontier other);
sg_status sg_frontier_intersect(sg_frontier f, sg_frontier other);
/* frontier::swap (frontier/frontier.hpp:94-101, mlb:444) */
sg_status sg_frontier_swap(sg_frontier a, sg_frontier b);
/* FrontierMLB::computeActiveFrontier(invert) (mlb:388-442): writes the
 * indices of non-empty level-0 words (invert=0) or of non-full words
 * (invert=1) into the offsets list, warp-ballot compaction.  When
 * host_active_words is non-NULL the count is copied back (a blocking read,
 * as buildAdvanceLaunchConfig does at operators/advance/common.hpp:112-119). */
sg_status sg_frontier_compact(sg_frontier f, int invert, uint32_t* host_active_words);
/* FrontierMLB::saveState / loadState (mlb:339-365): both levels to/from host. */
sg_status sg_frontier_save(sg_frontier f, uint32_t* host_level0, uint32_t* host_level1);
sg_status sg_frontier_load(sg_frontier f, const uint32_t* host_level0, const uint32_t* host_level1);
/* Flags of every element (1 byte each), for tests and tools. */
sg_status sg_frontier_to_flags(sg_frontier f, uint8_t* host_flags);

/* ------------------------------------------------------------- operators -- */
/* Built-in device functors for sg_advance.  The templated C++ API accepts any
 * device lambda; through the C ABI a functor is one of these, with its state
 * in sg_op_args (device pointers p[] and scalars u[] / f[]). */
#define SG_OP_BFS_PUSH 0     /* bfs.hpp:185-191: p0=uint32 depth, u0=sentinel(n+1), u1=iter */
#define SG_OP_BFS_PULL 1     /* bfs.hpp:201-207: same args; src = candidate, dst = in-frontier neighbour */
#define SG_OP_SSSP_RELAX 2   /* sssp.hpp:180-189: p0=distances (f32 or u32 per the graph's value_type) */
#define SG_OP_CC_MAX 3       /* cc.hpp:137-142 with an atomic max: p0=uint32 labels */
#define SG_OP_BC_FORWARD 4   /* bc.hpp:144-153: p0=uint32 labels, p1=float sigma, u0=invalid label */
#define SG_OP_BC_BACKWARD 5  /* bc.hpp:174-186: p0=labels, p1=sigma, p2=delta, p3=bc, u0=source */
#define SG_OP_COUNT_VISITS 6 /* tests/operators/advance_pull.cpp:29-32: p0=uint32 visits; atomicAdd(visits[src],1); true */
#define SG_OP_NONZERO_DEGREE 7 /* tests/operators/advance_graph.cpp:19: degree(src) != 0 */
#define SG_OP_BFS_VISIT_FLAG 8 /* tests/operators/advance.cpp:29-36: p0=uint8 visited, p1=uint64 distances */
#define SG_OP_TRUE 9           /* always true (pure frontier expansion) */

typedef struct {
  void* p[4];
  uint32_t u[4];
  float f[4];
} sg_op_args;

/* advance::frontier<Direction, Lb, InView, OutView>(G, in, out, f, expected_size)
 * (operators/advance/advance.hpp:116-218) and advance::vertices<Lb, OutView>(G, out, f)
 * (advance.hpp:46-87).
 *   in_view  : SG_VIEW_VERTEX (needs `in`) or SG_VIEW_GRAPH (every vertex, `in` ignored)
 *   out_view : SG_VIEW_VERTEX (needs `out`) or SG_VIEW_NONE
 *   expected_size : SG_SIZE_FETCH_FROM_MEMORY, SG_SIZE_INFER_FROM_DEVICE or a
 *     positive hint.  The active-word count is always read on the device, so
 *     none of them costs a host round trip.
 * Pull directions walk the inverse graph (common.hpp:147). */
sg_status sg_advance(sg_graph g, sg_frontier in, sg_frontier out, int direction, int load_balancer, int in_view,
                     int out_view, int op, const sg_op_args* args, int expected_size);

#define SG_PRED_EVEN 0        /* tests/operators/filter_compute.cpp:15: v % 2 == 0 */
#define SG_PRED_LESS_THAN 1   /* filter_compute.cpp:19: v < u0 */
#define SG_PRED_ITER_MARK 2   /* sssp.hpp:546-550: p0=int32 visited, u0=iter; false if visited[v]==iter else mark, true */
#define SG_PRED_FLAG 3        /* p0=uint8 flags: flags[v] != 0 */

/* filter::external(G, in, out, pred) (operators/filter/filter.hpp:41-69):
 * out.clear(), then out gets every v in `in` with pred(v). */
sg_status sg_filter_external(sg_graph g, sg_frontier in, sg_frontier out, int pred, const sg_op_args* args);
/* filter::inplace(G, f, pred): removes every v in f with pred(v). */
sg_status sg_filter_inplace(sg_graph g, sg_frontier f, int pred, const sg_op_args* args);

#define SG_FN_MARK 0         /* filter_compute.cpp:26: p0=uint32 seen; seen[v] = 1 */
#define SG_FN_SET_U8 1       /* advance_pull.cpp:36: p0=uint8 flags; flags[v] = 1 */
#define SG_RED_VERTEX_ID 0   /* filter_compute.cpp:35-36: acc += v */
#define SG_RED_DEGREE 1      /* bfs.hpp:290-291: acc += degree(v) */
#define SG_RED_COUNT 2       /* acc += 1 */

/* compute::execute<vertex>(G, f, fn) (operators/for/for.hpp:48-60). */
sg_status sg_compute_execute(sg_graph g, sg_frontier f, int fn, const sg_op_args* args);
/* compute::reduce<vertex, plus<R>>(G, f, acc, fn) (for.hpp:62-92); the sum is
 * returned in *host_result (64-bit). */
sg_status sg_compute_reduce(sg_graph g, sg_frontier f, int fn, const sg_op_args* args, uint64_t* host_result);
/* intersection::execute(G, in1, in2, out, f) (operators/intersection/intersection.hpp:44-55):
 * out = in1 AND in2. */
sg_status sg_intersection_execute(sg_graph g, sg_frontier in1, sg_frontier in2, sg_frontier out);
/* GraphCSRDevice::getIntersectionCount (graph_csr.hpp:109-135) for a batch of
 * vertex pairs: counts[i] = |N(a[i]) n N(b[i])| over sorted adjacency. */
sg_status sg_segmented_intersection(sg_graph g, const uint32_t* dev_a, const uint32_t* dev_b, uint64_t pairs,
                                    uint32_t* dev_counts);

/* ------------------------------------------------------------ algorithms -- */
#define SG_MAX_LOGGED_LEVELS 4096

/* BFSRunDetails (algorithms/bfs.hpp:31-35).  step_is_pull[i] records the
 * direction of step i for the first SG_MAX_LOGGED_LEVELS steps. */
typedef struct {
  uint64_t iterations;
  uint64_t push_steps;
  uint64_t pull_steps;
  uint64_t visited_vertices;
  uint64_t visited_edges; /* sum of degrees of reached vertices (bfs.hpp:88-99) */
  uint8_t step_is_pull[SG_MAX_LOGGED_LEVELS];
} sg_bfs_details;

/* Per-level record kept by the fused traversal engines (one per step). */
typedef struct {
  uint32_t level;
  uint32_t strategy;      /* direction * 2 + load balancer (0 warp-mapped, 1 CTA-mapped) */
  uint32_t frontier_size; /* |F| processed in this step */
  uint32_t next_size;     /* |F'| produced */
  uint64_t frontier_degree;   /* sum of degrees over F */
  uint64_t next_degree;       /* sum of degrees over F' */
  uint64_t unexplored_degree; /* sum of degrees over unvisited vertices after the step */
  uint64_t t_start_ns;        /* device global timer at the step's start */
  uint64_t t_end_ns;
} sg_level_record;

typedef struct sg_bfs_s* sg_bfs;

/* BFS(G) + init(source) + run(direction, alpha, beta) + getDistances()
 * (algorithms/bfs.hpp:129-278), as one fused device-side traversal: frontier
 * compaction, advance, size / degree bookkeeping, the direction heuristic and
 * termination run inside one persistent kernel with no host round trip per
 * level.  Depths are uint32 with n+1 for unreached (bfs.hpp:67). */
sg_status sg_bfs_create(sg_graph g, sg_bfs* out);
sg_status sg_bfs_destroy(sg_bfs b);
sg_status sg_bfs_init(sg_bfs b, uint32_t source);
sg_status sg_bfs_reset(sg_bfs b);
sg_status sg_bfs_run(sg_bfs b, int direction, float alpha, float beta, sg_bfs_details* details);
/* Same as sg_bfs_run but enqueues only: no host synchronisation and no
 * details; for timing loops and graph capture. */
sg_status sg_bfs_run_async(sg_bfs b, int direction, float alpha, float beta);
sg_status sg_bfs_get_distances(sg_bfs b, uint32_t* host_depth);
sg_status sg_bfs_distances_device(sg_bfs b, const uint32_t** dev_depth);
sg_status sg_bfs_level_records(sg_bfs b, sg_level_record* host_records, uint32_t cap, uint32_t* count);
/* One-shot form: host depth out (n entries). */
sg_status sg_run_bfs(sg_graph g, uint32_t source, int direction, float alpha, float beta, uint32_t* host_depth,
                 sg_bfs_details* details);

/* BFS that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc when they need a traversal: code
 * on a latency-critical path (cudaMalloc may synchronise the device and take
 * milliseconds), or a plug-in whose host application owns all device memory
 * and passes in only input and output buffers.  The caller passes the device
 * CSR (forward, and the inverse CSR of a directed graph; NULL inverse means
 * the graph is undirected) and a device array of n depths (n+1 = unreached,
 * same values as sg_bfs_run).  m must equal row_offsets[n] of the forward
 * and of the inverse CSR (read back and checked: SG_ERR_INVALID otherwise).
 * All working memory is one static device array of about 11 MB inside this
 * library, held by every GPU that loads it until the process exits; graphs
 * above 2^22 vertices or 2^27 edges are rejected with SG_ERR_INVALID.  The
 * first call on a device looks up that array's address (once per device);
 * make that first call before any stream capture.  Every call shares the
 * array: calls whose work overlaps on the GPU (other streams, other threads)
 * race and must be serialised by the caller.  The call is synchronous: it
 * waits on `stream` for the edge-count check and again for the traversal to
 * finish; *host_iterations (optional) gets the number of BFS levels. */
sg_status sg_bfs_noalloc(const uint32_t* dev_row_offsets, const uint32_t* dev_column_indices,
                         const uint32_t* dev_inv_row_offsets, const uint32_t* dev_inv_column_indices, uint32_t n,
                         uint64_t m, uint32_t source, int direction, float alpha, float beta, uint32_t* dev_depth,
                         uint64_t* host_iterations, void* stream);

/* Batched multi-source BFS: up to 64 BFS::run traversals of one graph
 * (algorithms/bfs.hpp:153-238) in one persistent kernel, bit-parallel (one
 * 64-bit frontier / seen word per vertex).  Per source the depths equal the
 * single-source ones.  Depths are a source-major k x n uint32 array
 * (n+1 = unreached). */
typedef struct sg_msbfs_s* sg_msbfs;
typedef struct {
  uint64_t iterations;
  uint64_t push_steps;
  uint64_t pull_steps;
  uint64_t reached_edges; /* sum over sources of the degrees of reached vertices */
} sg_msbfs_details;
sg_status sg_msbfs_create(sg_graph g, uint32_t max_sources, sg_msbfs* out);
sg_status sg_msbfs_destroy(sg_msbfs h);
sg_status sg_msbfs_run(sg_msbfs h, const uint32_t* host_sources, uint32_t k, int direction, float alpha, float beta,
                       sg_msbfs_details* details);
sg_status sg_msbfs_run_async(sg_msbfs h, const uint32_t* host_sources, uint32_t k, int direction, float alpha,
                             float beta);
sg_status sg_msbfs_get_depths(sg_msbfs h, uint32_t* host_depth);
/* As sg_sssp_set_launch. */
sg_status sg_msbfs_set_launch(sg_msbfs h, void* stream, uint32_t max_ctas);
sg_status sg_msbfs_depths_device(sg_msbfs h, const uint32_t** dev_depth);
/* Per-level log of the last batch (strategy 0 push / 2 pull, sizes and
 * degrees of the frontier union, device timestamps), as sg_bfs_level_records. */
sg_status sg_msbfs_level_records(sg_msbfs h, sg_level_record* host_records, uint32_t cap, uint32_t* count);

/* Learned strategy selector (no counterpart in the reference, whose
 * direction choice is the degree-threshold heuristic of bfs.hpp:325-350): a
 * 12 -> 32 -> 32 -> 6 FP32 MLP predicting the log-time of a traversal level
 * under each strategy (push / pull / pull_all x warp- / CTA-mapped).  The
 * parameter block is sg_mlp_param_count() floats: w1[32][12], b1[32],
 * w2[32][32], b2[32], w3[6][32], b3[6], then input mean[12], 1/std[12] and the
 * trusted range lo[12], hi[12].  Training runs on the device with this
 * library's own forward / backward / Adam kernels. */
typedef struct sg_mlp_s* sg_mlp;
uint32_t sg_mlp_param_count(void);
sg_status sg_mlp_create(const float* host_params /* NULL: seeded initialisation */, sg_mlp* out);
sg_status sg_mlp_destroy(sg_mlp h);
sg_status sg_mlp_get_params(sg_mlp h, float* host_params);
sg_status sg_mlp_set_params(sg_mlp h, const float* host_params);
/* dev_y[n][6] = MLP(dev_x[n][12]) */
sg_status sg_mlp_forward(sg_mlp h, const float* dev_x, uint32_t n, float* dev_y);
/* Gradient of the masked mean squared error 0.5*mask*(y-t)^2 over n samples
 * (trainable parameters; the normalisation entries get 0). */
sg_status sg_mlp_gradient(sg_mlp h, const float* dev_x, const float* dev_t, const float* dev_mask, uint32_t n,
                          float* host_grad, float* host_loss);
/* `steps` full-batch Adam steps on that loss. */
sg_status sg_mlp_train(sg_mlp h, const float* dev_x, const float* dev_t, const float* dev_mask, uint32_t n,
                       uint32_t steps, float lr, float weight_decay, float* host_final_loss);

/* Scheduling controls of the batched BFS (no counterpart in the reference,
 * whose batch of traversals does not exist; none changes any depth):
 *   sg_msbfs_set_schedule  forces the direction of level i (0 push, 2 pull,
 *                          -1 the mode decides) for i < len; len 0 clears it
 *   sg_msbfs_set_selector  the MLP of SG_BFS_LEARNED (NULL detaches it): it
 *                          is asked, between push/warp and pull/warp, where
 *                          the hybrid heuristic would switch direction on a
 *                          frontier of min_frontier..max_frontier * n vertices,
 *                          and overrules the heuristic when it predicts the
 *                          heuristic's choice `margin` slower in log-time
 *   sg_msbfs_log_features  records the twelve selector features of each
 *                          level decision (frontier = the union over the
 *                          sources, visited = vertices every source reached);
 *                          sg_msbfs_level_features reads them. */
sg_status sg_msbfs_set_schedule(sg_msbfs h, const int* host_directions, uint32_t len);
sg_status sg_msbfs_set_selector(sg_msbfs h, sg_mlp mlp, float margin, float min_frontier, float max_frontier);
sg_status sg_msbfs_log_features(sg_msbfs h, int enable);
sg_status sg_msbfs_level_features(sg_msbfs h, float* host_features, uint32_t cap_levels, uint32_t* count);

/* Scheduling controls of the fused BFS engine (no counterpart in the
 * reference; none changes any depth):
 *   sg_bfs_set_schedule  forces the strategy of level i (SG_STRATEGY_*, or -1
 *                        to let the mode decide) for i < len; len 0 clears it
 *   sg_bfs_set_selector  the MLP used by SG_BFS_LEARNED and the strategies it
 *                        may choose (bit mask over SG_STRATEGY_*)
 *   sg_bfs_set_selector_margin  the predicted log-time gain the MLP needs to
 *                        overrule the hybrid heuristic's choice (default 0.05)
 *   sg_bfs_log_features  records the twelve selector features of each level
 *                        decision; sg_bfs_level_features reads them (12 floats
 *                        per level, level 0 first). */
/* As sg_sssp_set_launch. */
sg_status sg_bfs_set_launch(sg_bfs b, void* stream, uint32_t max_ctas);
sg_status sg_bfs_set_schedule(sg_bfs b, const int* host_strategies, uint32_t len);
sg_status sg_bfs_set_selector(sg_bfs b, sg_mlp mlp, uint32_t allowed);
/* Probe order of short-circuit pull levels: bit L of reverse_levels (L < 64)
 * makes level L probe each vertex's in-neighbours from the back of its sorted
 * list (the parents of late-level vertices tend to have high ids).  Any
 * parent gives the same depth; only the work changes. */
sg_status sg_bfs_set_pull_order(sg_bfs b, uint64_t reverse_levels);
/* Form of the short-circuit pull: 0 (the default) ranks the unvisited
 * vertices of 32 of a warp's bitmap words across its lanes, four candidates
 * per lane in flight; 2 or 4 take that many words per warp step, one lane per
 * vertex of a word.  Every form gives the same depths. */
sg_status sg_bfs_set_pull_words(sg_bfs b, uint32_t words);
sg_status sg_bfs_set_selector_margin(sg_bfs b, float margin);
/* Learned mode: a frontier smaller than fraction * n keeps the heuristic's
 * choice without an inference (when that choice is allowed).  Default 1e-3;
 * 0 asks the MLP on every level. */
sg_status sg_bfs_set_selector_min_frontier(sg_bfs b, float fraction);
/* Learned mode: a frontier larger than fraction * n keeps the heuristic's
 * choice without an inference (when that choice is allowed).  Default 1
 * (no limit); the model file stores the range chosen in training. */
sg_status sg_bfs_set_selector_max_frontier(sg_bfs b, float fraction);
/* Learned mode: the MLP is consulted only on graphs whose mean-degree feature
 * log2(1 + m/n) / 8 lies in [lo, hi]; on other graphs the launch carries no
 * MLP (no parameter staging, no inference) and the heuristic decides every
 * level.  The model file stores the range of the training graphs on which
 * the model overruled the heuristic.  Default: every graph. */
sg_status sg_bfs_set_selector_graph_range(sg_bfs b, float lo, float hi);
sg_status sg_bfs_log_features(sg_bfs b, int enable);
sg_status sg_bfs_level_features(sg_bfs b, float* host_features, uint32_t cap_levels, uint32_t* count);

/* SSSP(G) + init + run + getDistance (algorithms/sssp.hpp:109-217): frontier
 * Bellman-Ford with atomicMin, fused.  Distances have the graph's weight type
 * (float32 or uint32); unreached = (weight_t)(n+1) (sssp.hpp:43). */
typedef struct sg_sssp_s* sg_sssp;
sg_status sg_sssp_create(sg_graph g, sg_sssp* out);
sg_status sg_sssp_destroy(sg_sssp s);
sg_status sg_sssp_init(sg_sssp s, uint32_t source);
sg_status sg_sssp_run(sg_sssp s, uint64_t* iterations);
/* Near-far bucketing (not in the reference): relaxations to a distance
 * below a threshold stay in the frontier, the others wait until the frontier
 * empties and the threshold moves up by delta.  Distances are unchanged (the
 * same fixed point); the iteration count and the work are not.  0 (the
 * default) is the reference's frontier Bellman-Ford. */
sg_status sg_sssp_set_delta(sg_sssp s, double delta);
/* With near-far bucketing: once a refill leaves fewer than fraction * n
 * vertices waiting beyond the threshold, the next refill takes all of them
 * and the rest runs as plain frontier Bellman-Ford (every edge).  The sparse
 * end of the distance range then takes a few iterations instead of one bucket
 * per delta.  Default 1/4; 0 keeps bucketing to the end. */
sg_status sg_sssp_set_tail(sg_sssp s, double fraction);
/* With near-far bucketing, on graphs whose weighted rows are symmetric
 * (every edge's reverse present with the same weight; checked once per
 * graph): a bucket whose heavy edges number more than m / ratio relaxes them
 * by pull, each vertex beyond the bucket scanning its weight-sorted row up
 * to the first weight that can no longer improve it.  Default 8; 0 always
 * pushes. */
sg_status sg_sssp_set_heavy_pull(sg_sssp s, uint32_t ratio);
/* Same graphs: an iteration of a bucket whose frontier holds more than
 * n / ratio vertices relaxes the light edges by pull (each vertex scans the
 * light prefix of its weight-sorted row, frontier neighbours only, up to the
 * first weight that can no longer improve it).  Default 0 (always push). */
sg_status sg_sssp_set_light_pull(sg_sssp s, uint32_t ratio);
/* Pull iterations (not in the reference): an iteration whose frontier
 * out-degree times `ratio` exceeds the edge count runs as one pull sweep
 * (every vertex takes the minimum over its in-neighbours in the frontier, no
 * atomics) instead of a push.  Distances are unchanged; 0 (the default) is
 * push only, as the reference. */
sg_status sg_sssp_set_pull(sg_sssp s, uint32_t ratio);
/* Per-step log of the last run (frontier size and out-degree, vertices
 * improved, device timestamps), as sg_bfs_level_records.  strategy: 0 push
 * iteration, 2 pull sweep; with near-far bucketing also 4, the heavy-edge
 * phase of a bucket (frontier_size = the bucket's vertices), and 5, a refill
 * pass (frontier_size = vertices moved to the frontier, next_size = vertices
 * left beyond the threshold).  In the push iterations of near-far bucketing
 * without light pulls, next_size counts frontier marks, an upper bound on the
 * vertices of the next frontier (zero exactly when it is empty). */
sg_status sg_sssp_level_records(sg_sssp s, sg_level_record* host_records, uint32_t cap, uint32_t* count);
/* Stream of this instance's launches and copies (NULL: the graph's stream)
 * and a cap on its persistent grid in CTAs of 512 threads (0: two per SM on
 * every SM), so that several instances
 * can share the GPU.  Waits for work queued on the previous stream.  The
 * stream must stay valid until the instance is destroyed or given another. */
sg_status sg_sssp_set_launch(sg_sssp s, void* stream, uint32_t max_ctas);
sg_status sg_sssp_run_async(sg_sssp s);
sg_status sg_sssp_get_distances(sg_sssp s, void* host_dist);
sg_status sg_sssp_distances_device(sg_sssp s, const void** dev_dist);

/* Learned heavy phases of delta-stepping SSSP (no counterpart in the
 * reference, which has no buckets; none changes any distance):
 *   sg_sssp_set_selector  the MLP (NULL detaches it) that chooses, at a
 *                         bucket's heavy phase, between pushing the bucket's
 *                         heavy edges and pulling them into the vertices
 *                         beyond the bucket (its outputs 0 and 2), where the
 *                         graph allows pull (symmetric weighted rows) and the
 *                         bucket's heavy edges number min_heavy..max_heavy * m
 *                         (the model file stores the range chosen in
 *                         training); the sg_sssp_set_heavy_pull rule stands
 *                         unless the model predicts it `margin` slower in
 *                         log-time
 *   sg_sssp_log_features  records the twelve features of each heavy phase
 *                         (bucket vertices and heavy edges, heavy edges not
 *                         yet relaxed, vertices settled, previous bucket,
 *                         previous direction); sg_sssp_level_features reads
 *                         them, one row per heavy phase. */
sg_status sg_sssp_set_selector(sg_sssp s, sg_mlp mlp, float margin, float min_heavy, float max_heavy);
sg_status sg_sssp_log_features(sg_sssp s, int enable);
sg_status sg_sssp_level_features(sg_sssp s, float* host_features, uint32_t cap, uint32_t* count);
sg_status sg_run_sssp(sg_graph g, uint32_t source, void* host_dist, uint64_t* iterations);

/* CC(G) + init + run (algorithms/cc.hpp:82-169): labels[v] = max id over the
 * vertices reaching v.  The instance owns the label array and the engine's
 * workspace (cc.hpp:54), so that runs allocate nothing; runs are enqueued on
 * the graph's stream.  Methods: the reference's maximum-label propagation
 * with atomicMax (SG_CC_PROPAGATION, every directed graph), or, on an
 * undirected graph (whose rows hold every edge both ways), lock-free
 * union-find in the Afforest order (one sampled neighbour per vertex, then
 * the other edges of the vertices outside the largest component) followed by
 * the largest id of each component (SG_CC_UNION_FIND): the same labels.
 * SG_CC_AUTO picks union-find for undirected graphs. */
#define SG_CC_AUTO 0
#define SG_CC_PROPAGATION 1
#define SG_CC_UNION_FIND 2
typedef struct sg_cc_s* sg_cc_handle;
sg_status sg_cc_create(sg_graph g, sg_cc_handle* out);
sg_status sg_cc_destroy(sg_cc_handle c);
sg_status sg_cc_set_method(sg_cc_handle c, int method);
sg_status sg_cc_run_async(sg_cc_handle c);
/* iterations = propagation levels, the first one over every vertex (1 for
 * union-find: one pass over the edges) */
sg_status sg_cc_run(sg_cc_handle c, uint64_t* iterations);
sg_status sg_cc_get_labels(sg_cc_handle c, uint32_t* host_labels);
sg_status sg_cc_labels_device(sg_cc_handle c, const uint32_t** dev_labels);
/* One-shot: create, run, copy the labels (when non-NULL), destroy. */
sg_status sg_cc(sg_graph g, uint32_t* host_labels, uint64_t* iterations);

/* BC(G) + init(source) + run (algorithms/bc.hpp:86-200) for each of k
 * sources; host_bc[v] = sum over sources of the Brandes dependency
 * delta_s(v), v != s, float32. */
sg_status sg_bc(sg_graph g, const uint32_t* host_sources, uint32_t k, float* host_bc);

/* Batched BC (no counterpart in the reference, which runs one source per
 * BC::run): up to 64 sources per launch as bit-parallel frontiers, the same
 * sum as sg_bc over those sources (float32; every sum in a fixed order, so
 * repeated runs give identical bits).  The per-level frontier history sizes
 * the device memory: history_levels = 0 picks it from the graph size, and a
 * deeper traversal enlarges it and runs again (SG_ERR_NOMEM when it cannot). */
typedef struct sg_bc_batch_s* sg_bc_batch;
typedef struct {
  uint64_t iterations;      /* forward levels */
  uint64_t reached_edges;   /* sum over (source, reached vertex) of its out-degree */
  uint64_t history_levels;  /* history capacity used */
  uint64_t history_retries; /* runs repeated after enlarging the history */
} sg_bc_batch_details;
sg_status sg_bc_batch_create(sg_graph g, uint32_t history_levels, sg_bc_batch* out);
sg_status sg_bc_batch_destroy(sg_bc_batch h);
/* accumulate != 0 adds this batch into the device bc array instead of
 * overwriting it. */
sg_status sg_bc_batch_run_async(sg_bc_batch h, const uint32_t* host_sources, uint32_t k, int accumulate);
sg_status sg_bc_batch_run(sg_bc_batch h, const uint32_t* host_sources, uint32_t k, int accumulate,
                          sg_bc_batch_details* details);
/* As sg_sssp_set_launch. */
sg_status sg_bc_batch_set_launch(sg_bc_batch h, void* stream, uint32_t max_ctas);
sg_status sg_bc_batch_get(sg_bc_batch h, float* host_bc);
sg_status sg_bc_batch_bc_device(sg_bc_batch h, const float** dev_bc);
/* Log of the last batch: forward levels first (strategy 0: marked sparse
 * level, 2: pull over every vertex not done), then backward levels (7). */
sg_status sg_bc_batch_level_records(sg_bc_batch h, sg_level_record* host_records, uint32_t cap, uint32_t* count);
/* One-shot: any number of sources, in batches of 64. */
sg_status sg_bc_batched(sg_graph g, const uint32_t* host_sources, uint32_t k, float* host_bc);

/* TC(G) + init + run + getNumTriangles (algorithms/tc.hpp:58-138), exact,
 * uint64: every run orients the edges into the degree-ordered DAG and
 * intersects N+(u) with N+(v) for every DAG edge through shared-memory hash
 * sets, streaming the shorter row.  Rows need not be sorted; the graph must
 * have no parallel edges (self-loops are ignored).
 * getNumTriangles(v), the per-vertex count, is for every edge (u,v) with
 * u < v, |N(u) n N(v)| added to u.  The instance owns the DAG, its reverse
 * lists and the work lists (about 8m + 28n bytes), so that runs allocate
 * nothing; runs are enqueued on the graph's stream. */
typedef struct sg_tc_s* sg_tc_handle;
sg_status sg_tc_create(sg_graph g, sg_tc_handle* out);
sg_status sg_tc_destroy(sg_tc_handle t);
/* per_vertex != 0 also accumulates the per-vertex counts (8n more bytes) */
sg_status sg_tc_run_async(sg_tc_handle t, int per_vertex);
sg_status sg_tc_run(sg_tc_handle t, int per_vertex, uint64_t* total);
sg_status sg_tc_get_total(sg_tc_handle t, uint64_t* total);
/* shorter != 0 (the default): every DAG edge streams the shorter of its two
 * rows against the other's set (reverse lists built each run); 0: always the
 * head's row against the tail's set (no reverse lists).  Same counts. */
sg_status sg_tc_set_shorter_rows(sg_tc_handle t, int shorter);
sg_status sg_tc_get_per_vertex(sg_tc_handle t, uint64_t* host_per_vertex);
/* One-shot; host_per_vertex may be NULL. */
sg_status sg_tc(sg_graph g, uint64_t* total, uint64_t* host_per_vertex);

/* -------------------------------------------------------------- serving -- */
/* Query serving with continuous batching (no counterpart in the reference,
 * which runs one algorithm call at a time).  Graphs stay resident; queries are
 * submitted from any host thread and a dispatcher thread runs them on `slots`
 * CUDA streams, each launch capped to ctas_per_slot CTAs so that launches of
 * different slots overlap on the GPU.  A query is admitted when a slot is free
 * and its workspace (per slot and graph) fits in memory_budget, after idle
 * workspaces are evicted least recently used first; otherwise it waits.  When
 * a slot frees, the pending BFS queries of the oldest query's graph (up to
 * max_batch, at least min_batch) run as one batched launch; SSSP queries run
 * singly, near-far with sssp_delta when it is > 0.  Each result equals the
 * single-query entry point's, bit for bit.  host_out receives n depths
 * (uint32) or distances (the graph's weight type); pinned memory keeps the
 * copy asynchronous, NULL skips it. */
typedef struct sg_server_s* sg_server;
typedef struct {
  uint32_t slots;          /* concurrent launches (0: 4) */
  uint32_t max_batch;      /* BFS queries per batched launch, <= 64 (0: 64) */
  uint32_t min_batch;      /* fewer pending BFS queries of a graph run singly (0: 16) */
  uint32_t ctas_per_slot;  /* persistent grid per launch (0: 2 * SMs / slots) */
  uint64_t memory_budget;  /* workspace bytes (0: half the free device memory) */
  double sssp_delta;       /* near-far step of SSSP queries (0: the reference schedule) */
} sg_server_config;
#define SG_QUERY_BFS 0
#define SG_QUERY_SSSP 1
typedef struct {
  sg_status status;
  uint32_t graph, source, batch_size;
  int kind;
  uint64_t submit_ns, start_ns, end_ns; /* host steady clock */
} sg_query_result;
typedef struct {
  uint64_t submitted, completed, failed, launches, batched_queries;
  uint64_t evictions, deferred_admissions;
  uint64_t workspace_bytes, peak_workspace_bytes, memory_budget;
} sg_server_stats;
sg_status sg_server_create(const sg_server_config* cfg, sg_server* out);
sg_status sg_server_destroy(sg_server s);
sg_status sg_server_add_graph(sg_server s, sg_graph g, uint32_t* graph_id);
/* Creates now, on every slot, each workspace the graph's queries can use (the
 * single and batched BFS and, on a weighted graph, the SSSP instance) that
 * is not there yet and fits in the memory budget without evicting another
 * workspace; SG_ERR_NOMEM when some did not fit.  A workspace is otherwise
 * created by the first query that needs it, and its creation (allocations,
 * host passes over the in-edge offsets for the pull chunk lists) then holds
 * up every query queued behind it. */
sg_status sg_server_prepare(sg_server s, uint32_t graph_id);
sg_status sg_server_submit(sg_server s, uint32_t graph_id, int kind, uint32_t source, void* host_out,
                           uint64_t* ticket);
/* Blocks until the query completes (SG_ERR_TIMEOUT after timeout_s; <= 0 waits without limit). */
sg_status sg_server_wait(sg_server s, uint64_t ticket, double timeout_s, sg_query_result* result);
sg_status sg_server_drain(sg_server s, double timeout_s);
sg_status sg_server_get_stats(sg_server s, sg_server_stats* stats);

/* ------------------------------------------------------- host graph I/O -- */
/* Host CSR owned by the library (malloc'd); free with sg_host_csr_free. */
typedef struct {
  uint32_t n;
  uint64_t m;
  uint32_t* row_offsets;    /* n+1 */
  uint32_t* column_indices; /* m */
  void* values;             /* m entries of value_type, or NULL */
  int value_type;
  uint32_t flags; /* SG_GRAPH_DIRECTED / SG_GRAPH_WEIGHTED */
} sg_host_csr;

typedef struct {
  uint32_t scale;      /* n = 2^scale */
  uint32_t edge_factor; /* generated pairs = edge_factor * n */
  double a, b, c;       /* quadrant probabilities; d = 1-a-b-c */
  uint64_t seed;        /* edge seed */
  uint64_t weight_seed; /* weight seed (weights keyed by the unordered pair) */
  uint64_t perm_seed;   /* 0: no relabelling; else seeded random vertex permutation */
  int value_type;       /* SG_WEIGHT_NONE / F32 ((0,1]) / U32 ([1,64]) */
} sg_rmat_params;

/* Seeded RMAT generator: recursive quadrant choice, then symmetrise, drop
 * self-loops, de-duplicate and sort each adjacency list.  OpenMP host code. */
sg_status sg_rmat_generate(const sg_rmat_params* params, sg_host_csr* out);
/* side x side 4-neighbour grid plus long_range_frac * (grid pairs) uniform
 * random pairs, symmetrised, sorted; weights as in sg_rmat_params. */
sg_status sg_grid_generate(uint32_t side, double long_range_frac, uint64_t seed, uint64_t weight_seed, int value_type,
                           sg_host_csr* out);
/* io::csr::fromCOO (io/read_csr.hpp:260-300) generalised: builds a CSR from
 * an edge list; symmetrize adds (v,u), dedupe drops repeated pairs (keeping
 * the first value), self-loops are dropped when drop_self_loops. */
sg_status sg_csr_from_edges(uint32_t n, const uint32_t* src, const uint32_t* dst, const void* values, int value_type,
                            uint64_t count, int symmetrize, int dedupe, int drop_self_loops, sg_host_csr* out);
/* formats::CSR::invert (formats/csr.hpp:179-209). */
sg_status sg_csr_invert(const sg_host_csr* in, sg_host_csr* out);
/* io::csr::toBinary / fromBinary (io/read_csr.hpp:316-411): the "SYGRCSR"
 * binary layout, including the legacy headerless one on read.  The file stores
 * n+1 row offsets, m column indices and m values (4 bytes each). */
sg_status sg_csr_write_binary(const sg_host_csr* csr, const char* path);
sg_status sg_csr_read_binary(const char* path, int value_type, sg_host_csr* out);
/* io::csr::fromMM (io/read_csr.hpp:88-192): coordinate Matrix Market,
 * general or symmetric, pattern or real/integer. */
sg_status sg_csr_read_mm(const char* path, int value_type, sg_host_csr* out);
void sg_host_csr_free(sg_host_csr* csr);
/* Uniform random sample of k vertices with degree > 0 (seeded, sorted by draw order). */
sg_status sg_sample_sources(const sg_host_csr* csr, uint32_t k, uint64_t seed, uint32_t* out_sources);

#ifdef __cplusplus
}
#endif

#endif /* SYGRAPH_B200_H */
