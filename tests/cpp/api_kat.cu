// The reference's tests (tests/operators/*.cpp, tests/frontier/mlb_frontier.cpp,
// tests/algorithms/*.cpp) written against the C++ header API of
// sygraph_b200: same calls, device lambdas via SYGRAPH_LAMBDA, sygraph::Queue
// in place of sycl::queue.  Fixture matrices arrive on argv
// (name=rows separated by ';') from tests/test_cpp_api.py.
#include <array>
#include <cstring>
#include <limits>

#include "test_utils.hpp"

using namespace sygraph;
using frontier_view_t = frontier::frontier_view;
using frontier_impl_t = frontier::frontier_type;
using load_balance_t = operators::load_balancer;

// tests/operators/advance.cpp
template <load_balance_t LB, typename GraphT>
void run_bfs(GraphT& G) {
  auto& q = G.getQueue();
  auto in_frontier = frontier::makeFrontier<frontier_view_t::vertex, frontier_impl_t::bitmap>(q, G);
  auto out_frontier = frontier::makeFrontier<frontier_view_t::vertex, frontier_impl_t::bitmap>(q, G);
  bool* visited = memory::detail::memoryAlloc<bool, memory::space::shared>(G.getVertexCount(), q);
  size_t* distances = memory::detail::memoryAlloc<size_t, memory::space::shared>(G.getVertexCount(), q);
  for (size_t i = 0; i < G.getVertexCount(); ++i) {
    visited[i] = false;
    distances[i] = 0;
  }
  in_frontier.insert(0);
  visited[0] = true;
  while (!in_frontier.empty()) {
    operators::advance::frontier<LB, frontier_view_t::vertex, frontier_view_t::vertex>(
        G, in_frontier, out_frontier, SYGRAPH_LAMBDA(auto u, auto v, auto, auto)->bool {
          if (!visited[v]) {
            visited[v] = true;
            distances[v] = distances[u] + 1;
            return true;
          }
          return false;
        }).waitAndThrow();
    frontier::swap(in_frontier, out_frontier);
    out_frontier.clear();
  }
  const std::array<size_t, 6> expected{0, 1, 1, 2, 2, 3};
  for (size_t i = 0; i < G.getVertexCount(); ++i) {
    EXPECT(visited[i]);
    EXPECT(distances[i] == expected[i]);
  }
  memory::detail::releaseUSM(visited, q);
  memory::detail::releaseUSM(distances, q);
}

// tests/operators/advance_graph.cpp
template <load_balance_t LB, typename GraphT>
void run_graph_advance(GraphT& G) {
  auto& q = G.getQueue();
  auto out_frontier = frontier::makeFrontier<frontier_view_t::vertex, frontier_impl_t::mlb>(q, G);
  auto device_graph = G.getDeviceGraph();
  operators::advance::vertices<LB, frontier_view_t::vertex>(
      G, out_frontier, SYGRAPH_LAMBDA(auto u, auto, auto, auto)->bool { return device_graph.getDegree(u) != 0; })
      .waitAndThrow();
  const std::array<bool, 6> expected{true, true, true, true, true, false};
  for (size_t i = 0; i < G.getVertexCount(); ++i) EXPECT(out_frontier.check(i) == expected[i]);
}

// tests/operators/advance_pull.cpp
template <load_balance_t LB, typename GraphT>
uint32_t run_pull_case(GraphT& G, bool* active) {
  auto& q = G.getQueue();
  auto in_frontier = frontier::makeFrontier<frontier_view_t::vertex, frontier_impl_t::mlb>(q, G);
  auto out_frontier = frontier::makeFrontier<frontier_view_t::vertex, frontier_impl_t::mlb>(q, G);
  auto visits = memory::detail::memoryAlloc<uint32_t, memory::space::shared>(G.getVertexCount(), q);
  for (size_t i = 0; i < G.getVertexCount(); ++i) {
    visits[i] = 0;
    active[i] = false;
  }
  in_frontier.insert(0);
  in_frontier.insert(1);
  operators::advance::frontier<operators::direction::pull, LB, frontier_view_t::vertex, frontier_view_t::vertex>(
      G, in_frontier, out_frontier,
      SYGRAPH_LAMBDA(auto src, auto, auto, auto)->bool {
        sync::atomicFetchAdd(visits + src, 1U);
        return true;
      },
      frontier::size::infer_from_device)
      .waitAndThrow();
  operators::compute::execute<frontier_view_t::vertex>(G, out_frontier, SYGRAPH_LAMBDA(auto v) { active[v] = true; })
      .waitAndThrow();
  const uint32_t two = visits[2];
  memory::detail::releaseUSM(visits, q);
  return two;
}

// sync::min / cas / load / store / atomicFetchAdd (sync/atomics.hpp:24-100):
// every candidate is applied by 64 threads at once, so the minima are
// contended; the expected values follow operator< (no store unless the
// candidate is strictly less).
template <typename T>
__global__ void sync_min_kernel(T* targets, T* cand, const int* target_of, int k, int copies) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < k * copies) sync::min(targets + target_of[i / copies], cand + i / copies);
}

__global__ void sync_cas_kernel(uint32_t* word, uint32_t* won, uint32_t* seen) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t expected = 0;
  if (sync::cas(word, expected, t + 1)) {
    sync::atomicFetchAdd(won, 1u);
    seen[t] = t + 1;
  } else {
    seen[t] = expected;  // the winner's value
  }
}

__global__ void sync_add_kernel(float* acc, double* dacc, uint64_t* cnt) {
  sync::atomicFetchAdd(acc, 1.0f);
  sync::atomicFetchAdd(dacc, 0.5);
  sync::atomicFetchAdd(cnt, (uint64_t)1);
}

__global__ void sync_load_store_kernel(uint64_t* p, uint64_t* out) {
  if (threadIdx.x == 0) sync::store(p, sync::load(p) * 3 + 1);
  __syncthreads();
  if (threadIdx.x == 1) *out = sync::load(p);
}

template <typename T>
bool same_bits(T a, T b) {
  return std::memcmp(&a, &b, sizeof(T)) == 0;
}

template <typename T>
void run_sync_min(Queue& q) {
  const T inf = std::numeric_limits<T>::infinity(), nan = std::numeric_limits<T>::quiet_NaN();
  // (target start, candidates) -> expected final value
  struct Case {
    T start;
    std::vector<T> cand;
    T want;
  };
  const std::vector<Case> cases{
      {T(5), {T(-1), T(-2.5), T(3), T(-2.4), T(0.5)}, T(-2.5)},  // mixed sign
      {T(-1), {T(-2), T(-0.5), T(4)}, T(-2)},                     // negative start
      {T(0), {T(-0.0)}, T(0)},                                     // -0 is not below +0
      {T(-0.0), {T(0)}, T(-0.0)},                                  // +0 is not below -0
      {T(1), {T(-0.0)}, T(-0.0)},
      {T(-3), {nan}, T(-3)},                                       // NaN is never less
      {inf, {-inf, T(7)}, -inf},
      {T(2), {T(3), T(4)}, T(2)},
  };
  const int copies = 64;
  std::vector<T> cand_h;
  std::vector<int> of_h;
  for (size_t c = 0; c < cases.size(); ++c)
    for (T x : cases[c].cand) {
      cand_h.push_back(x);
      of_h.push_back((int)c);
    }
  const int k = (int)cand_h.size();
  T* targets = memory::detail::memoryAlloc<T, memory::space::shared>(cases.size(), q);
  T* cand = memory::detail::memoryAlloc<T, memory::space::shared>(k, q);
  int* of = memory::detail::memoryAlloc<int, memory::space::shared>(k, q);
  for (size_t c = 0; c < cases.size(); ++c) targets[c] = cases[c].start;
  for (int i = 0; i < k; ++i) {
    cand[i] = cand_h[i];
    of[i] = of_h[i];
  }
  sync_min_kernel<T><<<(k * copies + 255) / 256, 256>>>(targets, cand, of, k, copies);
  EXPECT(cudaDeviceSynchronize() == cudaSuccess);
  for (size_t c = 0; c < cases.size(); ++c) EXPECT(same_bits(targets[c], cases[c].want));
  memory::detail::releaseUSM(targets, q);
  memory::detail::releaseUSM(cand, q);
  memory::detail::releaseUSM(of, q);
}

void run_sync_misc(Queue& q) {
  // integers: hardware minimum, signed and unsigned
  int* si = memory::detail::memoryAlloc<int, memory::space::shared>(1, q);
  int* sc = memory::detail::memoryAlloc<int, memory::space::shared>(3, q);
  int* of = memory::detail::memoryAlloc<int, memory::space::shared>(3, q);
  si[0] = 5;
  sc[0] = -7;
  sc[1] = 3;
  sc[2] = 10;
  of[0] = of[1] = of[2] = 0;
  sync_min_kernel<int><<<1, 192>>>(si, sc, of, 3, 64);
  EXPECT(cudaDeviceSynchronize() == cudaSuccess);
  EXPECT(si[0] == -7);
  // compare-exchange: exactly one of 1024 threads wins, the others see its value
  uint32_t* word = memory::detail::memoryAlloc<uint32_t, memory::space::shared>(2, q);
  uint32_t* seen = memory::detail::memoryAlloc<uint32_t, memory::space::shared>(1024, q);
  word[0] = word[1] = 0;
  sync_cas_kernel<<<4, 256>>>(word, word + 1, seen);
  EXPECT(cudaDeviceSynchronize() == cudaSuccess);
  EXPECT(word[1] == 1 && word[0] != 0);
  for (int t = 0; t < 1024; ++t) EXPECT(seen[t] == word[0]);
  // fetch_add on float, double and 64-bit integers
  float* acc = memory::detail::memoryAlloc<float, memory::space::shared>(1, q);
  double* dacc = memory::detail::memoryAlloc<double, memory::space::shared>(1, q);
  uint64_t* cnt = memory::detail::memoryAlloc<uint64_t, memory::space::shared>(3, q);
  acc[0] = 0.0f;
  dacc[0] = 0.0;
  cnt[0] = 0;
  sync_add_kernel<<<8, 256>>>(acc, dacc, cnt);
  EXPECT(cudaDeviceSynchronize() == cudaSuccess);
  EXPECT(acc[0] == 2048.0f && dacc[0] == 1024.0 && cnt[0] == 2048);
  cnt[1] = 4;
  sync_load_store_kernel<<<1, 32>>>(cnt + 1, cnt + 2);
  EXPECT(cudaDeviceSynchronize() == cudaSuccess);
  EXPECT(cnt[1] == 13 && cnt[2] == 13);
  for (void* p : {(void*)si, (void*)sc, (void*)of, (void*)word, (void*)seen, (void*)acc, (void*)dacc, (void*)cnt})
    memory::detail::releaseUSM(p, q);
}

int main(int argc, char** argv) {
  auto q = tests::makeQueue();
  const std::string symmetric_6nodes = tests::matrixArg(argc, argv, "symmetric_6nodes");
  const std::string two_cc = tests::matrixArg(argc, argv, "two_cc");
  const std::string star_5 = tests::matrixArg(argc, argv, "star_5");
  const std::string line_5 = tests::matrixArg(argc, argv, "line_5");
  const std::string triangle_3 = tests::matrixArg(argc, argv, "triangle_3");
  const std::string weighted_directed_5 = tests::matrixArg(argc, argv, "weighted_directed_5");

  {  // advance.cpp
    auto G = tests::buildGraphFromMatrix(q, symmetric_6nodes);
    run_bfs<load_balance_t::workgroup_mapped>(G);
    run_bfs<load_balance_t::bucketing>(G);
    run_bfs<load_balance_t::subgroup_mapped>(G);
    run_bfs<load_balance_t::workitem_mapped>(G);
    std::puts("advance ok");
  }
  {  // advance_graph.cpp
    auto G = tests::buildGraphFromMatrix(q, two_cc);
    run_graph_advance<load_balance_t::workgroup_mapped>(G);
    run_graph_advance<load_balance_t::bucketing>(G);
    std::puts("advance_graph ok");
  }
  {  // advance_pull.cpp
    auto G = tests::buildGraphFromMatrix(q, symmetric_6nodes);
    bool* wg = memory::detail::memoryAlloc<bool, memory::space::shared>(G.getVertexCount(), q);
    bool* bk = memory::detail::memoryAlloc<bool, memory::space::shared>(G.getVertexCount(), q);
    const auto wv = run_pull_case<load_balance_t::workgroup_mapped>(G, wg);
    const auto bv = run_pull_case<load_balance_t::bucketing>(G, bk);
    for (size_t i = 0; i < G.getVertexCount(); ++i) EXPECT(wg[i] == bk[i]);
    EXPECT(wg[2]);
    EXPECT(wv >= 1);
    EXPECT(bv == 1);
    memory::detail::releaseUSM(wg, q);
    memory::detail::releaseUSM(bk, q);
    std::puts("advance_pull ok");
  }
  {  // filter_compute.cpp
    auto graph = tests::buildGraphFromMatrix(q, star_5);
    auto input = frontier::makeFrontier<frontier_view_t::vertex, frontier_impl_t::mlb>(q, graph);
    auto output = frontier::makeFrontier<frontier_view_t::vertex, frontier_impl_t::mlb>(q, graph);
    for (uint32_t v : {0u, 1u, 2u, 3u, 4u}) input.insert(v);
    operators::filter::external(graph, input, output, SYGRAPH_LAMBDA(auto vertex) { return vertex % 2 == 0; })
        .waitAndThrow();
    tests::expectEqual(tests::activeElements(output), std::vector<uint32_t>{0, 2, 4});
    operators::filter::inplace(graph, input, SYGRAPH_LAMBDA(auto vertex) { return vertex < 2; }).waitAndThrow();
    tests::expectEqual(tests::activeElements(input), std::vector<uint32_t>{2, 3, 4});
    auto seen = memory::detail::memoryAlloc<uint32_t, memory::space::shared>(graph.getVertexCount(), q);
    for (size_t i = 0; i < graph.getVertexCount(); ++i) seen[i] = 0;
    operators::compute::execute<frontier_view_t::vertex>(graph, output, SYGRAPH_LAMBDA(auto vertex) { seen[vertex] = 1; })
        .waitAndThrow();
    std::vector<uint32_t> actual(seen, seen + graph.getVertexCount());
    tests::expectEqual(actual, std::vector<uint32_t>{1, 0, 1, 0, 1});
    uint32_t sum = 0;
    operators::compute::reduce<frontier_view_t::vertex, operators::compute::plus<uint32_t>>(
        graph, output, sum, SYGRAPH_LAMBDA(auto vertex, auto& acc) { acc += static_cast<uint32_t>(vertex); })
        .waitAndThrow();
    EXPECT(sum == 6);
    // a second reduction reuses the graph's accumulator and adds again
    operators::compute::reduce<frontier_view_t::vertex, operators::compute::plus<uint32_t>>(
        graph, output, sum, SYGRAPH_LAMBDA(auto vertex, auto& acc) { acc += static_cast<uint32_t>(vertex); })
        .waitAndThrow();
    EXPECT(sum == 12);
    memory::detail::releaseUSM(seen, q);
    std::puts("filter_compute ok");
  }
  {  // intersection.cpp
    auto graph = tests::buildGraphFromMatrix(q, line_5);
    auto lhs = frontier::makeFrontier<frontier_view_t::vertex, frontier_impl_t::bitmap>(q, graph);
    auto rhs = frontier::makeFrontier<frontier_view_t::vertex, frontier_impl_t::bitmap>(q, graph);
    auto out = frontier::makeFrontier<frontier_view_t::vertex, frontier_impl_t::bitmap>(q, graph);
    for (uint32_t v : {0u, 1u, 3u}) lhs.insert(v);
    for (uint32_t v : {1u, 2u, 3u}) rhs.insert(v);
    operators::intersection::execute(graph, lhs, rhs, out, [](auto) {}).waitAndThrow();
    tests::expectEqual(tests::activeElements(out), std::vector<uint32_t>{1, 3});
    std::puts("intersection ok");
  }
  {  // frontier/mlb_frontier.cpp
    auto graph = tests::buildGraphFromMatrix(q, star_5);
    auto f = frontier::makeFrontier<frontier_view_t::vertex, frontier_impl_t::mlb>(q, graph);
    f.insert(1);
    f.insert(3);
    f.insert(4);
    tests::expectEqual(tests::activeElements(f), std::vector<uint32_t>{1, 3, 4});
    auto saved = f.saveState();
    f.remove(3);
    tests::expectEqual(tests::activeElements(f), std::vector<uint32_t>{1, 4});
    f.clear();
    EXPECT(f.empty());
    f.loadState(saved);
    tests::expectEqual(tests::activeElements(f), std::vector<uint32_t>{1, 3, 4});
    std::puts("mlb_frontier ok");
  }
  {  // algorithms/bfs.cpp
    auto graph = tests::buildGraphFromMatrix(q, line_5);
    uint32_t source = 0;
    algorithms::BFS bfs_push(graph);
    bfs_push.init(source);
    auto pd = bfs_push.run(algorithms::bfs_direction::push);
    tests::expectEqual(bfs_push.getDistances(), std::vector<uint32_t>{0, 1, 2, 3, 4});
    EXPECT(!pd.push_steps.empty() && pd.pull_steps.empty());
    algorithms::BFS bfs_pull(graph);
    bfs_pull.init(source);
    auto ld = bfs_pull.run(algorithms::bfs_direction::pull);
    tests::expectEqual(bfs_pull.getDistances(), std::vector<uint32_t>{0, 1, 2, 3, 4});
    EXPECT(ld.push_steps.empty() && !ld.pull_steps.empty());
    algorithms::BFS bfs_hybrid(graph);
    bfs_hybrid.init(source);
    auto hd = bfs_hybrid.run(algorithms::bfs_direction::hybrid, 1.0f, 1.0f);
    tests::expectEqual(bfs_hybrid.getDistances(), std::vector<uint32_t>{0, 1, 2, 3, 4});
    EXPECT(hd.iterations == 5);
    std::puts("bfs ok");
  }
  {  // algorithms/sssp.cpp
    graph::Properties properties;
    properties.directed = true;
    properties.weighted = true;
    auto graph = tests::buildGraphFromMatrix(q, weighted_directed_5, properties);
    algorithms::SSSP sssp(graph);
    uint32_t source = 0;
    sssp.init(source);
    sssp.run();
    std::vector<uint32_t> d(graph.getVertexCount());
    for (size_t i = 0; i < d.size(); ++i) d[i] = sssp.getDistance(i);
    tests::expectEqual(d, std::vector<uint32_t>{0, 1, 3, 4, 5});
    std::puts("sssp ok");
  }
  {  // algorithms/cc.cpp (no assertion in the reference; the fixed point is checked here)
    auto graph = tests::buildGraphFromMatrix(q, two_cc);
    algorithms::CC cc(graph);
    uint32_t source = 0;
    cc.init(source);
    cc.run();
    tests::expectEqual(cc.getLabels(), std::vector<uint32_t>{4, 4, 4, 4, 4, 5});
    std::puts("cc ok");
  }
  {  // algorithms/tc.cpp
    auto graph = tests::buildGraphFromMatrix(q, triangle_3);
    algorithms::TC tc(graph);
    tc.init();
    tc.run();
    EXPECT(tc.getNumTriangles() == 1);
    std::puts("tc ok");
  }
  {  // algorithms/bc.cpp (no assertion in the reference; Brandes on a path is checked here)
    auto graph = tests::buildGraphFromMatrix(q, line_5);
    algorithms::BC bc(graph);
    bc.init(0u);
    bc.run();
    const std::vector<float> want{0, 3, 2, 1, 0};
    for (size_t i = 0; i < want.size(); ++i) EXPECT(std::abs(bc.getBC()[i] - want[i]) <= 1e-4f * (1 + want[i]));
    std::puts("bc ok");
  }
  {  // sync/atomics.hpp
    run_sync_min<float>(q);
    run_sync_min<double>(q);
    run_sync_misc(q);
    std::puts("sync ok");
  }
  std::puts("ALL OK");
  return 0;
}
