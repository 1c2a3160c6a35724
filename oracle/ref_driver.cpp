// Test infrastructure only: a thin extern "C" driver around the reference's
// own CPU code, compiled from the reference sources where they lie (the
// recipe is oracle/Makefile; outputs go to oracle/_ref/).  Nothing on the
// product path links this file.  It is used to pin the C restatement
// (oracle/fknn_oracle.c) and, in bench.py's reference arm, as the timed CPU
// baseline.
//
// Two shared objects are made from this one file:
//   * REF_EXACT : utils.h Bruteforce (utils.h:80-158) with normal_l2
//                 (distance.h:62-72).  Scalar code, built for baseline x86-64
//                 plus AVX2/FMA exactly as the reference's CMakeLists.txt:14
//                 asks, so it runs on any AVX2 host.
//   * REF_HYBRID: the reference's whole approximate pipeline (baseline.cpp:
//                 ReadSortedBaseTimestamp, ReadSortedQuery, HybridGraph::Build*,
//                 the searchers, SortDataset and BatchSearch), with the graphs
//                 and base orders it used written out so the GPU router can be
//                 run on exactly the same inputs.
//   * REF_SQ8   : bruteforce / bruteforce_subgraph (bruteforce.h:244-289),
//                 L2SqrSQ8_sym (pyglass/glass/simd/distance.hpp:329-366) and
//                 SQ8SymmetricQuantizer (pyglass/glass/quant/sq8_sym_quant.hpp).
//                 Those intrinsics are AVX-512VL, so this object needs an
//                 AVX-512 host.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#ifdef REF_EXACT
#include "utils.h"
#endif

#ifdef REF_SQ8
#include "bruteforce.h"
#include "glass/quant/sq8_sym_quant.hpp"
#endif

extern "C" {

#ifdef REF_EXACT
// Runs the reference Bruteforce over contest-layout rows.
//   base_rows : N x 102 floats  [label, ts, 100 dims]   (utils.h:108-109)
//   query_rows: Q x 104 floats  [type, v, l, r, 100 dims] (utils.h:98-103)
//   gt        : Q x 100 u32, ascending (dist, id)       (utils.h:147-151)
// Returns 0, or -1 when the reference threw (a query with fewer than 100
// passing rows pops an empty heap, utils.h:44-47).  *seconds (nullable)
// receives the wall time of the Bruteforce call alone.
int ref_exact_bruteforce(const float *base_rows, uint32_t n, const float *query_rows,
                         uint32_t nq, uint32_t *gt, double *seconds) {
  std::vector<std::vector<float>> nodes(n), queries(nq);
  for (uint32_t i = 0; i < n; ++i) nodes[i].assign(base_rows + (size_t)i * 102, base_rows + (size_t)(i + 1) * 102);
  for (uint32_t i = 0; i < nq; ++i) queries[i].assign(query_rows + (size_t)i * 104, query_rows + (size_t)(i + 1) * 104);
  std::vector<std::vector<uint32_t>> out;
  auto t0 = std::chrono::steady_clock::now();
  try {
    Bruteforce(nodes, queries, out);
  } catch (const std::exception &) {
    return -1;
  }
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  for (uint32_t i = 0; i < nq; ++i) std::memcpy(gt + (size_t)i * 100, out[i].data(), 100 * sizeof(uint32_t));
  return 0;
}

// The reference's scalar distance (distance.h:62), exposed so the
// restatement's arithmetic can be compared value by value.
float ref_normal_l2(const float *a, const float *b, uint32_t dim) { return normal_l2(a, b, dim); }
#endif

#ifdef REF_SQ8
int ref_l2sqr_sq8_sym(const int8_t *x, const int8_t *y) { return glass::L2SqrSQ8_sym(x, y, 112); }

// SQ8SymmetricQuantizer::train + encode (sq8_sym_quant.hpp:32-74) over n x 100
// floats.  Writes alpha and n x 112 int8 codes (dims 100..111 are zero).
void ref_sq8_sym_train(const float *data, uint32_t n, float *alpha_out, int8_t *codes_out) {
  glass::SQ8SymmetricQuantizer<glass::Metric::L2> q(100);
  q.train(data, (int)n);
  *alpha_out = q.alpha;
  std::memcpy(codes_out, q.codes, (size_t)n * q.code_size);
}

// SQ8SymmetricQuantizer::encode with a given alpha (sq8_sym_quant.hpp:63-74).
void ref_sq8_sym_encode(const float *vec, float alpha, int8_t *code_out) {
  glass::SQ8SymmetricQuantizer<glass::Metric::L2> q(100);
  q.alpha = alpha;
  std::memset(code_out, 0, 112);
  q.encode(vec, (char *)code_out);
}

// bruteforce (bruteforce.h:244): one query, heap-array order output.
void ref_sq8_bruteforce(uint64_t k, int *closest, uint64_t npoints, const int8_t *codes, float alpha,
                        const int8_t *query) {
  bruteforce(100, k, closest, npoints, (char *)codes, alpha, 1, (int8_t *)query);
}

// bruteforce_subgraph (bruteforce.h:267): adds dist * alpha^2.
void ref_sq8_bruteforce_subgraph(uint64_t k, int *closest, float *dists, uint64_t npoints,
                                 const int8_t *codes, float alpha, const int8_t *query) {
  bruteforce_subgraph(100, k, closest, dists, npoints, (char *)codes, alpha, 1, (int8_t *)query);
}
#endif
}

#ifdef REF_GRAPH
#include "glass/hnsw/hnsw.hpp"
#include "glass/searcher.hpp"

extern "C" {
// HNSW::Build (pyglass/glass/hnsw/hnsw.hpp:33-89) with out-degree R = 2M and
// efConstruction efc over n x 100 vectors and their timestamps; the level-0
// graph, per-edge timestamps and the upper-layer initializer are written in
// Graph::save's format (graph.hpp:101-115) to path.  Returns 0.
int ref_hnsw_build(const float *data, const float *ts, int n, int R, int efc, const char *path) {
  glass::HNSW h(100, "L2", R, efc);
  h.Build((float *)data, (float *)ts, n, n, 0);
  h.final_graph.save(path);
  return 0;
}

// The reference Searcher (searcher.hpp) over a saved graph, with its own
// SQ8-sym quantizer trained on data (Searcher::SetData).  mode:
//   0 Search            1 SearchFilter        2 SearchFilterSubTime (dists)
//   3 SearchCategoryRange (bounds, id_bounds) 4 SearchRangeFilterSubTime (dists)
//   5 SearchRangeFilter
// K is the pool capacity argument ("k" of the reference calls), refine the
// number of ids written per query.
int ref_graph_search(const char *path, const float *data, const float *labels, const float *ts, int n,
                     const float *queries, int nq, int mode, int K, int refine, const float *bounds,
                     const int *id_bounds, int *out_ids, float *out_dists, double *seconds) {
  glass::Graph<int> g;
  g.load(path);
  auto s = glass::create_searcher(std::move(g), "L2");
  s->SetData(data, (float *)labels, (float *)ts, n, 100);
  const auto t0 = std::chrono::steady_clock::now();  // the query loop alone
  for (int i = 0; i < nq; ++i) {
    const float *q = queries + (size_t)i * 100;
    int *dst = out_ids + (size_t)i * refine;
    float *dd = out_dists ? out_dists + (size_t)i * refine : nullptr;
    std::pair<float, float> qb(bounds ? bounds[2 * i] : 0.f, bounds ? bounds[2 * i + 1] : 0.f);
    std::pair<int, int> ib(id_bounds ? id_bounds[2 * i] : 0, id_bounds ? id_bounds[2 * i + 1] : 0);
    switch (mode) {
      case 0: s->Search(q, K, dst); break;
      case 1: s->SearchFilter(q, K, refine, dst, nullptr); break;
      case 2: s->SearchFilterSubTime(q, K, refine, dst, dd, nullptr); break;
      case 3: s->SearchCategoryRange(q, K, refine, dst, qb, ib); break;
      case 4: s->SearchRangeFilterSubTime(q, K, refine, dst, dd, qb, ib); break;
      case 5: s->SearchRangeFilter(q, K, refine, dst, qb, ib); break;
      default: return -1;
    }
  }
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return 0;
}
}
#endif

#ifdef REF_HYBRID
#include <fstream>
#include <string>

#include "hybrid_graph.cpp"

extern "C" {
// baseline.cpp:45-147 as a function over the contest files at base_path and
// query_path, with BuildParams (M, efConstruction) given.  Before the
// sub-graphs move into their searchers they are saved in Graph::save's
// format to out_dir/c<category>.hnsw and out_dir/t<bucket>.hnsw; the three
// base orders go to out_dir/orders.bin (3 x N u32: sorted_base_ids,
// _by_time, _by_full_time) and the maps to out_dir/maps.txt ("c v start n",
// "t t start n", "m maxc_id max_count min_count").  ids: nq x 100 u32 as
// BatchSearch writes them; *seconds: the BatchSearch call alone.
int ref_hybrid_run(const char *base_path, const char *query_path, const char *out_dir, int M, int efc,
                   uint32_t *ids_out, double *seconds) {
  std::vector<float> base_vecs, base_vecs_by_time, base_vecs_by_full_time;
  std::vector<float> base_labels, base_labels_by_time, base_labels_by_full_time, base_timestamps,
      base_timestamps_by_time, base_timestamps_by_full_time;
  std::vector<float> query_vecs, query_metas;
  std::vector<uint32_t> sorted_ids;
  std::vector<uint32_t> sorted_base_ids, sorted_base_ids_by_time, sorted_base_ids_by_full_time;
  std::unordered_map<int32_t, std::pair<uint32_t, uint32_t>> category_map, timestamp_map;
  std::unordered_map<int32_t, std::vector<int>> category_query;
  uint32_t nb, nq;
  int maxc_id;
  int32_t max_count = 0, min_count = 1e9;
  ReadSortedBaseTimestamp(base_path, nb, base_vecs, base_labels, base_timestamps, sorted_base_ids, category_map,
                          base_vecs_by_time, base_labels_by_time, base_timestamps_by_time, sorted_base_ids_by_time,
                          maxc_id, base_vecs_by_full_time, base_labels_by_full_time, base_timestamps_by_full_time,
                          sorted_base_ids_by_full_time, timestamp_map, max_count, min_count);
  ReadSortedQuery(query_path, nq, query_vecs, query_metas, sorted_ids, category_query, category_map);
  const std::string dir(out_dir);
  {
    std::ofstream o(dir + "/orders.bin", std::ios::binary);
    o.write((const char *)sorted_base_ids.data(), (size_t)nb * 4);
    o.write((const char *)sorted_base_ids_by_time.data(), (size_t)nb * 4);
    o.write((const char *)sorted_base_ids_by_full_time.data(), (size_t)nb * 4);
    std::ofstream m(dir + "/maps.txt");
    for (auto &[v, p] : category_map) m << "c " << v << " " << p.first << " " << p.second << "\n";
    for (auto &[t, p] : timestamp_map) m << "t " << t << " " << p.first << " " << p.second << "\n";
    m << "m " << maxc_id << " " << max_count << " " << min_count << "\n";
  }
  HybridGraph h_graph;
  h_graph.sorted_ids = std::move(sorted_ids);
  h_graph.sorted_base_ids = std::move(sorted_base_ids);
  h_graph.category_map = std::move(category_map);
  h_graph.sorted_base_ids_by_time = std::move(sorted_base_ids_by_time);
  h_graph.bf_thr = 0.045;
  h_graph.cat_graph_thr = h_graph.bf_thr;
  h_graph.maxc_id = maxc_id;
  h_graph.timestamp_map = std::move(timestamp_map);
  h_graph.sorted_base_ids_by_full_time = std::move(sorted_base_ids_by_full_time);
  h_graph.maxc_size = max_count;
  h_graph.minc_size = min_count;
  h_graph.category_query = std::move(category_query);
  BuildParams build_params;
  build_params.M = M;
  build_params.efConstruction = efc;
  h_graph.Build(base_vecs_by_time.data(), base_labels_by_time.data(), base_timestamps_by_time.data(), nb,
                build_params);
  h_graph.BuildCategoryIndex(base_vecs.data(), base_labels.data(), base_timestamps.data(), nb, build_params);
  h_graph.BuildTimestampIndex(base_vecs_by_full_time.data(), base_labels_by_full_time.data(),
                              base_timestamps_by_full_time.data(), nb, build_params);
  const uint32_t dim = h_graph.dim;
  glass::Graph<int> graph;
  h_graph.searcher = std::unique_ptr<glass::SearcherBase>(glass::create_searcher(std::move(graph), h_graph.metric, 3));
  h_graph.searcher->SetData(base_vecs_by_time.data(), base_labels_by_time.data(), base_timestamps_by_time.data(), nb,
                            dim);
  std::vector<int> categories;
  for (auto &[category, p] : h_graph.category_map)
    if (p.second >= h_graph.cat_graph_thr * nb) categories.push_back(category);
  for (int v : categories) {
    auto &c_index = h_graph.category_index[v];
    auto &fg = ((glass::HNSW *)c_index.get())->final_graph;
    fg.save(dir + "/c" + std::to_string(v) + ".hnsw");
    h_graph.category_searcher[v] =
        std::unique_ptr<glass::SearcherBase>(glass::create_searcher(std::move(fg), h_graph.metric, 3));
    auto &[start_id, n] = h_graph.category_map[v];
    h_graph.category_searcher[v]->SetData(base_vecs.data() + (size_t)start_id * dim, base_labels.data() + start_id,
                                          base_timestamps.data() + start_id, n, dim);
  }
  std::vector<int> buckets;
  for (auto &[t, p] : h_graph.timestamp_map)
    if (p.second) buckets.push_back(t);
  for (int t : buckets) {
    auto &t_index = h_graph.timestamp_index[t];
    auto &fg = ((glass::HNSW *)t_index.get())->final_graph;
    fg.save(dir + "/t" + std::to_string(t) + ".hnsw");
    h_graph.timestamp_searcher[t] =
        std::unique_ptr<glass::SearcherBase>(glass::create_searcher(std::move(fg), h_graph.metric, 3));
    auto &[start_id, n] = h_graph.timestamp_map[t];
    h_graph.timestamp_searcher[t]->SetData(base_vecs_by_full_time.data() + (size_t)start_id * dim,
                                           base_labels_by_full_time.data() + start_id,
                                           base_timestamps_by_full_time.data() + start_id, n, dim);
  }
  auto &quant = ((glass::Searcher<glass::SQ8SymmetricQuantizer<glass::Metric::L2>> *)h_graph.searcher.get())->quant;
  h_graph.SortDataset(quant, base_labels_by_time.data(), base_timestamps_by_time.data(), nb);
  SearchParams search_params;
  std::vector<uint32_t> ids((size_t)nq * 100);
  auto t0 = std::chrono::steady_clock::now();
  h_graph.BatchSearch(base_vecs.data(), base_vecs_by_time.data(), base_vecs_by_full_time.data(), query_vecs.data(),
                      query_metas.data(), nq, ids.data(), search_params);
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  std::memcpy(ids_out, ids.data(), ids.size() * 4);
  return 0;
}
}
#endif
