// operators::load_balancer / direction and frontier::size, as in the
// reference (operators/config.hpp:10-37).  subgroup_mapped and
// workitem_mapped are implemented here (the reference throws / does not
// compile for them).
#pragma once

namespace sygraph {
namespace operators {

enum class load_balancer {
  workitem_mapped,
  subgroup_mapped,
  workgroup_mapped,
  bucketing,
};

enum class direction {
  push,
  pull,      // pull with short-circuit: stops after the first valid source edge per vertex
  pull_all,  // pull without short-circuit: processes all source edges per vertex
};

template <direction D>
constexpr bool is_pull() {
  return D == direction::pull || D == direction::pull_all;
}

template <direction D>
constexpr bool is_short_circuit() {
  return D == direction::pull;
}

}  // namespace operators

namespace frontier {

enum class frontier_view { graph, vertex, edge, none };
enum class frontier_type { bitmap, mlb, none };

namespace size {
using frontier_size_t = int;
constexpr frontier_size_t fetch_from_memory = -1;
constexpr frontier_size_t infer_from_device = 0;
}  // namespace size

}  // namespace frontier
}  // namespace sygraph
