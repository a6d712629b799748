// Algorithm classes with the reference's interface (algorithms/bfs.hpp,
// sssp.hpp, cc.hpp, bc.hpp, tc.hpp), each run as one fused device traversal
// of libsygraph_b200.so.
#pragma once

#include <cstdint>
#include <memory>
#include <set>
#include <stdexcept>
#include <vector>

#include "sygraph/graph/graph.hpp"
#include "sygraph/utils/runtime.hpp"

namespace sygraph {
namespace algorithms {

enum class bfs_direction { push, pull, hybrid };

// BFSRunDetails (bfs.hpp:31-35)
struct BFSRunDetails {
  size_t iterations = 0;
  std::set<size_t> push_steps;
  std::set<size_t> pull_steps;
};

template <typename GraphType>
class BFS {
  using vertex_t = typename GraphType::vertex_t;
  using edge_t = typename GraphType::edge_t;

 public:
  BFS(GraphType& g) : _g(g) {}

  void init(const vertex_t& source) {
    if (!_h) {
      sg_bfs b = nullptr;
      sygraph::detail::throw_if(sg_bfs_create(_g.handle(), &b));
      _h = std::shared_ptr<sg_bfs_s>(b, [](sg_bfs x) { sg_bfs_destroy(x); });
    }
    sygraph::detail::throw_if(sg_bfs_init(_h.get(), source));
  }
  void reset() { _h.reset(); }

  BFSRunDetails run(bfs_direction direction = bfs_direction::push, float alpha = 1.0f, float beta = 1.0f) {
    if (!_h) throw std::runtime_error("BFS instance not initialized");
    sg_bfs_details d{};
    sygraph::detail::throw_if(sg_bfs_run(_h.get(), (int)direction, alpha, beta, &d));
    BFSRunDetails out;
    out.iterations = d.iterations;
    for (size_t i = 0; i < d.iterations && i < SG_MAX_LOGGED_LEVELS; i++)
      (d.step_is_pull[i] ? out.pull_steps : out.push_steps).insert(i);
    return out;
  }

  edge_t getDistance(size_t vertex) const { return getDistances()[vertex]; }
  std::vector<edge_t> getDistances() const {
    if (!_h) throw std::runtime_error("BFS instance not initialized");
    std::vector<edge_t> d(_g.getVertexCount());
    sygraph::detail::throw_if(sg_bfs_get_distances(_h.get(), reinterpret_cast<uint32_t*>(d.data())));
    return d;
  }
  // parents are allocated but never written by the reference (bfs.hpp:66-70)
  std::vector<vertex_t> getParents() const { return std::vector<vertex_t>(_g.getVertexCount(), (vertex_t)-1); }

 private:
  GraphType& _g;
  std::shared_ptr<sg_bfs_s> _h;
};

template <typename GraphType>
class SSSP {
  using vertex_t = typename GraphType::vertex_t;
  using weight_t = typename GraphType::weight_t;

 public:
  SSSP(GraphType& g) : _g(g) {}
  void init(const vertex_t& source) {
    if (!_h) {
      sg_sssp s = nullptr;
      sygraph::detail::throw_if(sg_sssp_create(_g.handle(), &s));
      _h = std::shared_ptr<sg_sssp_s>(s, [](sg_sssp x) { sg_sssp_destroy(x); });
    }
    sygraph::detail::throw_if(sg_sssp_init(_h.get(), source));
    _dist.clear();
  }
  void reset() { _h.reset(); }
  template <bool EnableProfiling = false>
  void run() {
    if (!_h) throw std::runtime_error("SSSP instance not initialized");
    uint64_t it = 0;
    sygraph::detail::throw_if(sg_sssp_run(_h.get(), &it));
    _dist.resize(_g.getVertexCount());
    sygraph::detail::throw_if(sg_sssp_get_distances(_h.get(), _dist.data()));
  }
  weight_t getDistance(size_t vertex) const { return _dist.at(vertex); }
  const std::vector<weight_t>& getDistances() const { return _dist; }

 private:
  GraphType& _g;
  std::shared_ptr<sg_sssp_s> _h;
  std::vector<weight_t> _dist;
};

template <typename GraphType>
class CC {
  using vertex_t = typename GraphType::vertex_t;

 public:
  CC(GraphType& g) : _g(g) {}
  void init(const vertex_t& source) {
    _source = source;
    if (!_h) {
      sg_cc_handle c = nullptr;
      sygraph::detail::throw_if(sg_cc_create(_g.handle(), &c));
      _h = std::shared_ptr<sg_cc_s>(c, [](sg_cc_handle x) { sg_cc_destroy(x); });
    }
  }
  void reset() {
    _labels.clear();
    _h.reset();
  }
  template <bool EnableProfiling = false>
  void run() {
    if (!_h) init(_source);
    uint64_t it = 0;
    sygraph::detail::throw_if(sg_cc_run(_h.get(), &it));
    _labels.resize(_g.getVertexCount());
    sygraph::detail::throw_if(sg_cc_get_labels(_h.get(), reinterpret_cast<uint32_t*>(_labels.data())));
  }
  const std::vector<vertex_t>& getLabels() const { return _labels; }

 private:
  GraphType& _g;
  vertex_t _source = 0;
  std::shared_ptr<sg_cc_s> _h;
  std::vector<vertex_t> _labels;
};

template <typename GraphType>
class BC {
  using vertex_t = typename GraphType::vertex_t;

 public:
  BC(GraphType& g) : _g(g) {}
  void init(const vertex_t source) { _sources.assign(1, source); }
  void init(const std::vector<vertex_t>& sources) { _sources = sources; }
  void reset() { _bc.clear(); }
  void run() {
    _bc.resize(_g.getVertexCount());
    sygraph::detail::throw_if(sg_bc(_g.handle(), reinterpret_cast<const uint32_t*>(_sources.data()),
                                    (uint32_t)_sources.size(), _bc.data()));
  }
  const std::vector<float>& getBC() const { return _bc; }

 private:
  GraphType& _g;
  std::vector<vertex_t> _sources;
  std::vector<float> _bc;
};

template <typename GraphType>
class TC {
  using vertex_t = typename GraphType::vertex_t;

 public:
  TC(GraphType& g) : _g(g) {}
  void init() {
    _ran = false;
    if (!_h) {
      sg_tc_handle t = nullptr;
      sygraph::detail::throw_if(sg_tc_create(_g.handle(), &t));
      _h = std::shared_ptr<sg_tc_s>(t, [](sg_tc_handle x) { sg_tc_destroy(x); });
    }
  }
  void reset() {
    _ran = false;
    _h.reset();
  }
  template <bool EnableProfiling = false>
  void run() {
    if (!_h) init();
    sygraph::detail::throw_if(sg_tc_run(_h.get(), /*per_vertex=*/1, &_total));
    _per.resize(_g.getVertexCount());
    sygraph::detail::throw_if(sg_tc_get_per_vertex(_h.get(), _per.data()));
    _ran = true;
  }
  size_t getNumTriangles() const {
    if (!_ran) throw std::runtime_error("TC instance not initialized");
    return _total;
  }
  size_t getNumTriangles(vertex_t v) const {
    if (!_ran) throw std::runtime_error("TC instance not initialized");
    return _per.at(v);
  }

 private:
  GraphType& _g;
  std::shared_ptr<sg_tc_s> _h;
  bool _ran = false;
  uint64_t _total = 0;
  std::vector<uint64_t> _per;
};

}  // namespace algorithms
}  // namespace sygraph
