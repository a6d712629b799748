// SYgraph's C++ API on B200 (sm_100a): include this instead of the
// reference's <sygraph/sygraph.hpp>, compile with nvcc
// (-gencode arch=compute_100a,code=sm_100a --extended-lambda) and link
// libsygraph_b200.so.  Differences a user meets when switching:
//   - sycl::queue becomes sygraph::Queue (a CUDA stream);
//   - device lambdas are written SYGRAPH_LAMBDA(...) (i.e. [=] __device__);
//   - compute::reduce takes sygraph::operators::compute::plus<R>.
#pragma once

#include "sygraph_b200.h"
#include "sygraph/utils/runtime.hpp"
#include "sygraph/operators/config.hpp"
#include "sygraph/formats/csr.hpp"
#include "sygraph/graph/properties.hpp"
#include "sygraph/graph/graph.hpp"
#include "sygraph/io/read_csr.hpp"
#include "sygraph/frontier/frontier.hpp"
#include "sygraph/operators/operators.hpp"
#include "sygraph/algorithms/algorithms.hpp"
#include "sygraph/sync/atomics.hpp"
