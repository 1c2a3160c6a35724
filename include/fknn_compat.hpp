// fknn_compat.hpp -- the reference's own C++ entry points, with their
// signatures, over the C ABI of fknn.h.  Include this instead of the
// reference's header and link libfknn.so:
//
//   Bruteforce(nodes, queries, gt)                          utils.h:80
//   bruteforce(dim, k, closest, npoints, codes, alpha, nq, q) bruteforce.h:244
//   bruteforce_subgraph(..., distances, ...)                bruteforce.h:267
//   HybridGraph::Build / sorted_ids / BatchSearch(...)      hybrid_graph.h:37-62
//
// Failures throw std::runtime_error with the library's message (the
// reference throws or exits in the same places).
#ifndef FKNN_COMPAT_HPP_
#define FKNN_COMPAT_HPP_

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "fknn.h"

namespace fknn_compat {

inline void check(int rc) {
  if (rc != FKNN_OK) throw std::runtime_error(std::string("fknn: ") + fknn_last_error());
}

// utils.h:80: exact filtered top-100 of every query, rows [label, ts, 100 dims],
// queries [type, v, l, r, 100 dims]; gt[i] ascending by (distance, id).
inline void Bruteforce(const std::vector<std::vector<float>> &nodes, const std::vector<std::vector<float>> &queries,
                       std::vector<std::vector<uint32_t>> &gt) {
  const uint32_t n = (uint32_t)nodes.size(), nq = (uint32_t)queries.size();
  std::vector<float> rows((size_t)n * 102), qrows((size_t)nq * 104);
  for (uint32_t i = 0; i < n; ++i) {
    if (nodes[i].size() != 102) throw std::runtime_error("Bruteforce: a node row must hold 102 floats");
    std::memcpy(rows.data() + (size_t)i * 102, nodes[i].data(), 102 * sizeof(float));
  }
  for (uint32_t i = 0; i < nq; ++i) {
    if (queries[i].size() != 104) throw std::runtime_error("Bruteforce: a query row must hold 104 floats");
    std::memcpy(qrows.data() + (size_t)i * 104, queries[i].data(), 104 * sizeof(float));
  }
  std::vector<uint32_t> flat((size_t)nq * 100);
  check(fknn_bruteforce_rows(rows.data(), n, qrows.data(), nq, flat.data()));
  gt.assign(nq, std::vector<uint32_t>(100));
  for (uint32_t i = 0; i < nq; ++i) std::memcpy(gt[i].data(), flat.data() + (size_t)i * 100, 100 * sizeof(uint32_t));
}

// bruteforce.h:244 (one query per call, as hybrid_graph.cpp:211 calls it;
// nqueries > 1 batches queries that share the slab).
inline void bruteforce(size_t dim, size_t k, int *closest_points, size_t npoints, char *codes_in, float alpha,
                       size_t nqueries, int8_t *queries_in) {
  check(fknn_sq8_bruteforce(dim, k, closest_points, npoints, codes_in, alpha, nqueries ? nqueries : 1,
                            queries_in));
}

// bruteforce.h:267
inline void bruteforce_subgraph(size_t dim, size_t k, int *closest_points, float *distances, size_t npoints,
                                char *codes_in, float alpha, size_t nqueries, int8_t *queries_in) {
  check(fknn_sq8_bruteforce_subgraph(dim, k, closest_points, distances, npoints, codes_in, alpha,
                                     nqueries ? nqueries : 1, queries_in));
}

// The search form BatchSearch uses; any struct with mode / kprime members
// can stand in for the reference's SearchParams.
struct SearchParams {
  int mode = FKNN_MODE_BF16_RERANK;
  uint32_t kprime = 0;  // 0: the library default
};

// hybrid_graph.h:37-62's batch interface.  Build keeps one resident index
// over the base in original order (with the BF16 copies); BatchSearch takes
// the queries in sorted_ids order, as the reference's does, and writes
// ids[sorted_ids[i] * 100 ..] for query i.  The three re-ordered bases the
// reference passes are not needed: the index holds its own row orders.
struct HybridGraph {
  std::vector<uint32_t> sorted_ids;
  fknn_index *index = nullptr;

  HybridGraph() = default;
  HybridGraph(const HybridGraph &) = delete;
  HybridGraph &operator=(const HybridGraph &) = delete;
  ~HybridGraph() {
    if (index) fknn_index_destroy(index);
  }

  template <class BuildParams = int>
  void Build(const float *vecs, const float *labels, const float *timestamps, int nb, const BuildParams & = {}) {
    if (index) fknn_index_destroy(index);
    index = nullptr;
    fknn_index_opts o{};
    o.build_bf16 = 1;
    check(fknn_index_create(vecs, labels, timestamps, (uint64_t)nb, 100, &o, &index));
  }

  template <class Params = SearchParams>
  void BatchSearch(const float * /*base*/, const float * /*base_by_time*/, const float * /*base_by_full_time*/,
                   const float *vecs, const float *metas, int nq, uint32_t *ids, const Params &params = {}) {
    if (!index) throw std::runtime_error("BatchSearch: Build was not called");
    if ((size_t)nq > sorted_ids.size()) throw std::runtime_error("BatchSearch: sorted_ids shorter than nq");
    fknn_search_opts so{};
    so.mode = mode_of(params, 0);
    so.kprime = kprime_of(params, 0);
    std::vector<uint32_t> tmp((size_t)nq * 100);
    check(fknn_search_ex(index, vecs, metas, (uint32_t)nq, 100, &so, tmp.data(), nullptr, nullptr, nullptr));
    for (int i = 0; i < nq; ++i)
      std::memcpy(ids + (size_t)sorted_ids[i] * 100, tmp.data() + (size_t)i * 100, 100 * sizeof(uint32_t));
  }

 private:
  // the params' mode / kprime members when it has them, else the defaults
  template <class P>
  static auto mode_of(const P &p, int) -> decltype(p.mode, int()) {
    return p.mode;
  }
  template <class P>
  static int mode_of(const P &, long) {
    return FKNN_MODE_BF16_RERANK;
  }
  template <class P>
  static auto kprime_of(const P &p, int) -> decltype(p.kprime, uint32_t()) {
    return p.kprime;
  }
  template <class P>
  static uint32_t kprime_of(const P &, long) {
    return 0;
  }
};

// hybrid_graph.h:37-109 with the reference's own routing
// (hybrid_graph.cpp:147-503) run by fknn_router: the caller fills the
// members the reference's caller fills (baseline.cpp:66-78, after
// ReadSortedBaseTimestamp / ReadSortedQuery) plus the Graph::save bytes of
// each category and time-bucket graph, calls Prepare once with the base in
// original order, then BatchSearch with the reference's arguments.
struct RoutedHybridGraph {
  std::vector<uint32_t> sorted_ids;                    // query order (ReadSortedQuery)
  std::vector<uint32_t> sorted_base_ids;               // category order -> id
  std::vector<uint32_t> sorted_base_ids_by_full_time;  // timestamp order -> id
  std::vector<std::pair<int32_t, std::pair<uint32_t, uint32_t>>> category_map, timestamp_map;  // key -> (start, n)
  std::vector<std::pair<int32_t, std::string>> category_graphs, timestamp_graphs;  // key -> Graph::save bytes
  uint32_t maxc_size = 0, minc_size = 0;
  fknn_router_params params{};
  fknn_router *router = nullptr;

  RoutedHybridGraph() { fknn_router_default_params(&params); }
  RoutedHybridGraph(const RoutedHybridGraph &) = delete;
  RoutedHybridGraph &operator=(const RoutedHybridGraph &) = delete;
  ~RoutedHybridGraph() {
    if (router) fknn_router_destroy(router);
  }

  void Prepare(const float *vecs, const float *labels, const float *timestamps, uint64_t nb, int device = 0) {
    if (router) fknn_router_destroy(router);
    router = nullptr;
    std::vector<fknn_router_subgraph> cats, bks;
    auto add = [](const std::vector<std::pair<int32_t, std::pair<uint32_t, uint32_t>>> &map,
                  const std::vector<std::pair<int32_t, std::string>> &graphs, std::vector<fknn_router_subgraph> &out) {
      for (const auto &kv : map)
        for (const auto &g : graphs)
          if (g.first == kv.first) {
            fknn_router_subgraph sg{};
            sg.key = kv.first;
            sg.start = kv.second.first;
            sg.count = kv.second.second;
            sg.graph_bytes = g.second.data();
            sg.nbytes = g.second.size();
            out.push_back(sg);
          }
    };
    add(category_map, category_graphs, cats);
    add(timestamp_map, timestamp_graphs, bks);
    fknn_router_desc d{};
    d.vecs = vecs;
    d.labels = labels;
    d.ts = timestamps;
    d.n = nb;
    d.sorted_base_ids = sorted_base_ids.data();
    d.sorted_base_ids_by_full_time = sorted_base_ids_by_full_time.data();
    d.categories = cats.data();
    d.ncategories = (uint32_t)cats.size();
    d.buckets = bks.data();
    d.nbuckets = (uint32_t)bks.size();
    d.maxc_size = maxc_size;
    d.minc_size = minc_size;
    d.device = device;
    check(fknn_router_create(&d, &router));
  }

  // vecs / metas in sorted_ids order, as the reference's BatchSearch gets them
  template <class Params = int>
  void BatchSearch(const float * /*base*/, const float * /*base_by_time*/, const float * /*base_by_full_time*/,
                   const float *vecs, const float *metas, int nq, uint32_t *ids, const Params & = {}) {
    if (!router) throw std::runtime_error("BatchSearch: Prepare was not called");
    if ((size_t)nq > sorted_ids.size()) throw std::runtime_error("BatchSearch: sorted_ids shorter than nq");
    std::vector<uint32_t> tmp((size_t)nq * 100);
    check(fknn_router_search(router, vecs, metas, (uint32_t)nq, &params, tmp.data(), nullptr));
    for (int i = 0; i < nq; ++i)
      std::memcpy(ids + (size_t)sorted_ids[i] * 100, tmp.data() + (size_t)i * 100, 100 * sizeof(uint32_t));
  }
};

}  // namespace fknn_compat

#endif  // FKNN_COMPAT_HPP_
