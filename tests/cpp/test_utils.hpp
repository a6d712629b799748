// Helpers of the C++ API tests, mirroring the reference's
// tests/include/test_utils.hpp: fixture matrices are read from
// tests/golden/kat.json by the pytest driver and passed on argv.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include <sygraph/sygraph.hpp>

#define EXPECT(cond)                                                              \
  do {                                                                            \
    if (!(cond)) {                                                                \
      std::fprintf(stderr, "%s:%d: expectation failed: %s\n", __FILE__, __LINE__, #cond); \
      std::exit(1);                                                               \
    }                                                                             \
  } while (0)

namespace sygraph::tests {

inline Queue makeQueue() { return Queue(); }

template <typename ValueT = uint32_t>
auto buildGraphFromMatrix(Queue& q, const std::string& matrix, graph::Properties properties = {}) {
  std::istringstream iss{matrix};
  auto csr = io::csr::fromMatrix<ValueT, uint32_t, uint32_t>(iss);
  return graph::build::fromCSR<memory::space::shared>(q, csr, properties);
}

template <typename FrontierT>
std::vector<uint32_t> activeElements(const FrontierT& f) {
  std::vector<uint32_t> out;
  for (size_t i = 0; i < f.getNumElems(); ++i)
    if (f.check(i)) out.push_back((uint32_t)i);
  return out;
}

template <typename T>
void expectEqual(const std::vector<T>& a, const std::vector<T>& b) {
  EXPECT(a.size() == b.size());
  for (size_t i = 0; i < a.size(); ++i) EXPECT(a[i] == b[i]);
}

// argv: pairs "name=matrix-text" where rows are separated by ';'
inline std::string matrixArg(int argc, char** argv, const std::string& name) {
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a.rfind(name + "=", 0) == 0) {
      std::string m = a.substr(name.size() + 1);
      for (auto& c : m)
        if (c == ';') c = '\n';
      return m;
    }
  }
  std::fprintf(stderr, "missing matrix %s\n", name.c_str());
  std::exit(2);
}

}  // namespace sygraph::tests
