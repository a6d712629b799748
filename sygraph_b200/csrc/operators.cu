// C ABI of the operator layer: sg_advance (operators/advance/advance.hpp:46-218),
// filter (operators/filter/filter.hpp:41-69), compute (operators/for/for.hpp:48-92),
// intersection (operators/intersection/intersection.hpp:44-55) and the
// segmented intersection of sorted adjacency lists
// (GraphCSRDevice::getIntersectionCount, graph/impls/graph_csr.hpp:109-135).
#include "ops_functors.cuh"

namespace sgb {

sygraph::detail::MLBDev mlb_dev(const sg_frontier_s* f);
sg_status frontier_compact(sg_frontier f, int invert, cudaStream_t stream);
sg_status frontier_clear(sg_frontier f, cudaStream_t stream);
sg_status frontier_rebuild_level1(sg_frontier f, cudaStream_t stream);
sg_status frontier_and(sg_frontier out, sg_frontier a, sg_frontier b, cudaStream_t stream);

namespace {

using namespace sygraph::detail;

template <int Dir, typename W, typename F>
sg_status go(int lb, const GraphDev<W>& g, const AdvanceArgs& a, const F& f, unsigned grid, cudaStream_t s) {
  cudaError_t e = launch_advance<Dir, W, F>(lb, g, a, f, grid, s);
  if (e != cudaSuccess) return cuda_fail(e, "advance launch", __FILE__, __LINE__);
  count_launch();
  return SG_OK;
}

template <typename W, typename F>
sg_status go_dir(int dir, int lb, const GraphDev<W>& g, const AdvanceArgs& a, const F& f, unsigned grid,
                 cudaStream_t s) {
  switch (dir) {
    case SG_DIR_PUSH: return go<kPush>(lb, g, a, f, grid, s);
    case SG_DIR_PULL: return go<kPull>(lb, g, a, f, grid, s);
    case SG_DIR_PULL_ALL: return go<kPullAll>(lb, g, a, f, grid, s);
  }
  return fail(SG_ERR_INVALID, "unknown direction");
}

// Functors that ignore the weight run on the uint32 view of the value array.
sg_status dispatch(int op, const sg_op_args& x, int dir, int lb, const sg_graph_view& v, const AdvanceArgs& a,
                   unsigned grid, cudaStream_t s) {
  GraphDev<uint32_t> gu{v.n, v.m, v.row_offsets, v.column_indices, (const uint32_t*)v.values};
  switch (op) {
    case SG_OP_BFS_PUSH: return go_dir(dir, lb, gu, a, ops::BfsPush{(uint32_t*)x.p[0], x.u[0], x.u[1]}, grid, s);
    case SG_OP_BFS_PULL: return go_dir(dir, lb, gu, a, ops::BfsPull{(uint32_t*)x.p[0], x.u[0], x.u[1]}, grid, s);
    case SG_OP_SSSP_RELAX:
      if (v.value_type == SG_WEIGHT_F32) {
        GraphDev<float> gf{v.n, v.m, v.row_offsets, v.column_indices, (const float*)v.values};
        return go_dir(dir, lb, gf, a, ops::SsspRelax<float>{(float*)x.p[0]}, grid, s);
      }
      return go_dir(dir, lb, gu, a, ops::SsspRelax<uint32_t>{(uint32_t*)x.p[0]}, grid, s);
    case SG_OP_CC_MAX: return go_dir(dir, lb, gu, a, ops::CcMax{(uint32_t*)x.p[0]}, grid, s);
    case SG_OP_BC_FORWARD:
      return go_dir(dir, lb, gu, a, ops::BcForward{(uint32_t*)x.p[0], (float*)x.p[1], x.u[0]}, grid, s);
    case SG_OP_BC_BACKWARD:
      return go_dir(dir, lb, gu, a,
                    ops::BcBackward{(const uint32_t*)x.p[0], (const float*)x.p[1], (float*)x.p[2], (float*)x.p[3],
                                    x.u[0]},
                    grid, s);
    case SG_OP_COUNT_VISITS: return go_dir(dir, lb, gu, a, ops::CountVisits{(uint32_t*)x.p[0]}, grid, s);
    case SG_OP_NONZERO_DEGREE: return go_dir(dir, lb, gu, a, ops::NonzeroDegree{v.row_offsets}, grid, s);
    case SG_OP_BFS_VISIT_FLAG:
      return go_dir(dir, lb, gu, a, ops::BfsVisitFlag{(uint8_t*)x.p[0], (unsigned long long*)x.p[1]}, grid, s);
    case SG_OP_TRUE: return go_dir(dir, lb, gu, a, ops::AlwaysTrue{}, grid, s);
  }
  return fail(SG_ERR_INVALID, "unknown operator");
}

unsigned advance_grid(int expected_size) {
  const unsigned full = (unsigned)device_props().sm_count * 8u;
  if (expected_size > 0) {
    const unsigned want = (unsigned)(((uint64_t)expected_size + 255) / 256);
    return want < 1 ? 1 : (want < full ? want : full);
  }
  return full;
}

template <typename P>
sg_status launch_filter_ext(sg_frontier in, sg_frontier out, uint32_t n, const P& p, cudaStream_t s) {
  filter_external_kernel<<<grid_for((uint64_t)in->words0 * 32, 256), 256, 0, s>>>(mlb_dev(in), mlb_dev(out), n, p);
  SG_CHECK_LAUNCH();
  return SG_OK;
}

template <typename P>
sg_status launch_filter_inp(sg_frontier f, uint32_t n, const P& p, cudaStream_t s) {
  filter_inplace_kernel<<<grid_for((uint64_t)f->words0 * 32, 256), 256, 0, s>>>(mlb_dev(f), n, p);
  SG_CHECK_LAUNCH();
  return SG_OK;
}

// Thread per pair: walk the shorter sorted list and binary-search each id in
// the longer one (the reference walks both with two pointers).
__global__ void __launch_bounds__(256) segmented_intersection_kernel(const uint32_t* __restrict__ ro,
                                                                     const uint32_t* __restrict__ col,
                                                                     const uint32_t* a, const uint32_t* b,
                                                                     uint64_t pairs, uint32_t* counts) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < pairs; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t x = a[i], y = b[i];
    uint32_t xb = ro[x], xe = ro[x + 1], yb = ro[y], ye = ro[y + 1];
    if (xe - xb > ye - yb) {
      uint32_t t = xb; xb = yb; yb = t;
      t = xe; xe = ye; ye = t;
    }
    uint32_t c = 0, lo = yb;
    for (uint32_t e = xb; e < xe && lo < ye; e++) {
      const uint32_t key = col[e];
      uint32_t l = lo, h = ye;
      while (l < h) {
        const uint32_t mid = (l + h) >> 1;
        if (col[mid] < key)
          l = mid + 1;
        else
          h = mid;
      }
      if (l < ye && col[l] == key) {
        c++;
        l++;
      }
      lo = l;
    }
    counts[i] = c;
  }
}

}  // namespace
}  // namespace sgb

using namespace sgb;

extern "C" {

sg_status sg_advance(sg_graph g, sg_frontier in, sg_frontier out, int direction, int load_balancer, int in_view,
                     int out_view, int op, const sg_op_args* args, int expected_size) {
  clear_error();
  SG_REQUIRE(g, SG_ERR_INVALID, "graph is NULL");
  SG_REQUIRE(load_balancer >= SG_LB_WORKITEM_MAPPED && load_balancer <= SG_LB_BUCKETING, SG_ERR_UNSUPPORTED,
             "Load balancer not implemented");
  SG_REQUIRE(direction >= SG_DIR_PUSH && direction <= SG_DIR_PULL_ALL, SG_ERR_INVALID, "unknown direction");
  SG_REQUIRE(in_view == SG_VIEW_VERTEX || in_view == SG_VIEW_GRAPH, SG_ERR_INVALID,
             "Invalid frontier view for the advance input");
  SG_REQUIRE(out_view == SG_VIEW_VERTEX || out_view == SG_VIEW_NONE, SG_ERR_INVALID,
             "Invalid frontier view for the advance output");
  SG_REQUIRE(in_view != SG_VIEW_VERTEX || in, SG_ERR_INVALID, "input frontier is NULL");
  SG_REQUIRE(out_view != SG_VIEW_VERTEX || out, SG_ERR_INVALID, "output frontier is NULL");
  SG_REQUIRE(in_view != SG_VIEW_GRAPH || direction == SG_DIR_PUSH, SG_ERR_INVALID,
             "a graph-view advance is a push over every vertex");
  SG_REQUIRE(expected_size >= SG_SIZE_FETCH_FROM_MEMORY, SG_ERR_INVALID, "Invalid expected_size value");
  if (in) SG_REQUIRE(in->num_elems == g->n, SG_ERR_INVALID, "input frontier size differs from the vertex count");
  if (out) SG_REQUIRE(out->num_elems == g->n, SG_ERR_INVALID, "output frontier size differs from the vertex count");
  sg_op_args x{};
  if (args) x = *args;
  cudaStream_t s = g->stream;
  AdvanceArgs a{};
  a.in_view = in_view;
  a.out_view = out_view;
  a.limit = g->n;
  if (in_view == SG_VIEW_VERTEX) {
    a.in = mlb_dev(in);
    SG_TRY(frontier_compact(in, direction != SG_DIR_PUSH, s));
  }
  if (out_view == SG_VIEW_VERTEX) a.out = mlb_dev(out);
  const sg_graph_view v = g->view(direction != SG_DIR_PUSH);
  return dispatch(op, x, direction, load_balancer, v, a, advance_grid(expected_size), s);
}

sg_status sg_filter_external(sg_graph g, sg_frontier in, sg_frontier out, int pred, const sg_op_args* args) {
  clear_error();
  SG_REQUIRE(g && in && out, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(in != out, SG_ERR_INVALID, "filter::external needs distinct frontiers");
  sg_op_args x{};
  if (args) x = *args;
  cudaStream_t s = g->stream;
  SG_TRY(frontier_compact(in, 0, s));
  SG_TRY(frontier_clear(out, s));
  switch (pred) {
    case SG_PRED_EVEN: return launch_filter_ext(in, out, g->n, ops::PredEven{}, s);
    case SG_PRED_LESS_THAN: return launch_filter_ext(in, out, g->n, ops::PredLess{x.u[0]}, s);
    case SG_PRED_ITER_MARK: return launch_filter_ext(in, out, g->n, ops::PredIterMark{(int32_t*)x.p[0], (int32_t)x.u[0]}, s);
    case SG_PRED_FLAG: return launch_filter_ext(in, out, g->n, ops::PredFlag{(const uint8_t*)x.p[0]}, s);
  }
  return fail(SG_ERR_INVALID, "unknown predicate");
}

sg_status sg_filter_inplace(sg_graph g, sg_frontier f, int pred, const sg_op_args* args) {
  clear_error();
  SG_REQUIRE(g && f, SG_ERR_INVALID, "NULL argument");
  sg_op_args x{};
  if (args) x = *args;
  cudaStream_t s = g->stream;
  SG_TRY(frontier_compact(f, 0, s));
  switch (pred) {
    case SG_PRED_EVEN: return launch_filter_inp(f, g->n, ops::PredEven{}, s);
    case SG_PRED_LESS_THAN: return launch_filter_inp(f, g->n, ops::PredLess{x.u[0]}, s);
    case SG_PRED_ITER_MARK: return launch_filter_inp(f, g->n, ops::PredIterMark{(int32_t*)x.p[0], (int32_t)x.u[0]}, s);
    case SG_PRED_FLAG: return launch_filter_inp(f, g->n, ops::PredFlag{(const uint8_t*)x.p[0]}, s);
  }
  return fail(SG_ERR_INVALID, "unknown predicate");
}

sg_status sg_compute_execute(sg_graph g, sg_frontier f, int fn, const sg_op_args* args) {
  clear_error();
  SG_REQUIRE(g && f, SG_ERR_INVALID, "NULL argument");
  sg_op_args x{};
  if (args) x = *args;
  cudaStream_t s = g->stream;
  SG_TRY(frontier_compact(f, 0, s));
  const unsigned grid = grid_for((uint64_t)f->words0 * 32, 256);
  switch (fn) {
    case SG_FN_MARK:
      compute_execute_kernel<<<grid, 256, 0, s>>>(mlb_dev(f), g->n, ops::FnMark{(uint32_t*)x.p[0]});
      break;
    case SG_FN_SET_U8:
      compute_execute_kernel<<<grid, 256, 0, s>>>(mlb_dev(f), g->n, ops::FnSetU8{(uint8_t*)x.p[0]});
      break;
    default: return fail(SG_ERR_INVALID, "unknown compute function");
  }
  SG_CHECK_LAUNCH();
  return SG_OK;
}

sg_status sg_compute_reduce(sg_graph g, sg_frontier f, int fn, const sg_op_args* args, uint64_t* host_result) {
  clear_error();
  SG_REQUIRE(g && f && host_result, SG_ERR_INVALID, "NULL argument");
  (void)args;
  cudaStream_t s = g->stream;
  SG_TRY(frontier_compact(f, 0, s));
  SG_CUDA(cudaMemsetAsync(f->scratch, 0, sizeof(uint64_t), s));
  const unsigned grid = grid_for((uint64_t)f->words0 * 32, 256);
  unsigned long long* acc = (unsigned long long*)f->scratch;
  switch (fn) {
    case SG_RED_VERTEX_ID: compute_reduce_kernel<<<grid, 256, 0, s>>>(mlb_dev(f), g->n, ops::RedVertexId{}, acc); break;
    case SG_RED_DEGREE:
      compute_reduce_kernel<<<grid, 256, 0, s>>>(mlb_dev(f), g->n, ops::RedDegree{g->fwd.ro}, acc);
      break;
    case SG_RED_COUNT: compute_reduce_kernel<<<grid, 256, 0, s>>>(mlb_dev(f), g->n, ops::RedCount{}, acc); break;
    default: return fail(SG_ERR_INVALID, "unknown reduction");
  }
  SG_CHECK_LAUNCH();
  SG_CUDA(cudaMemcpyAsync(host_result, acc, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  SG_CUDA(cudaStreamSynchronize(s));
  return SG_OK;
}

sg_status sg_intersection_execute(sg_graph g, sg_frontier in1, sg_frontier in2, sg_frontier out) {
  clear_error();
  SG_REQUIRE(g && in1 && in2 && out, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(in1->num_elems == out->num_elems && in2->num_elems == out->num_elems, SG_ERR_INVALID,
             "frontier sizes differ");
  // out.clear(); out.merge(in1); out.intersect(in2) (bitmap_intersect_impl.hpp:21-30) as one pass
  return frontier_and(out, in1, in2, g->stream);
}

sg_status sg_segmented_intersection(sg_graph g, const uint32_t* dev_a, const uint32_t* dev_b, uint64_t pairs,
                                    uint32_t* dev_counts) {
  clear_error();
  SG_REQUIRE(g, SG_ERR_INVALID, "graph is NULL");
  if (pairs == 0) return SG_OK;
  SG_REQUIRE(dev_a && dev_b && dev_counts, SG_ERR_INVALID, "NULL argument");
  segmented_intersection_kernel<<<grid_for(pairs, 256), 256, 0, g->stream>>>(g->fwd.ro, g->fwd.col, dev_a, dev_b,
                                                                            pairs, dev_counts);
  SG_CHECK_LAUNCH();
  return SG_OK;
}

}  // extern "C"
