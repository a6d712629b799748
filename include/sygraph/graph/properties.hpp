// graph::Properties (graph/properties.hpp:29-32).
#pragma once

namespace sygraph {
namespace graph {

struct Properties {
  bool directed{false};
  bool weighted{false};
};

}  // namespace graph
}  // namespace sygraph
