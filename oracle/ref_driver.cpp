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
                     const int *id_bounds, int *out_ids, float *out_dists) {
  glass::Graph<int> g;
  g.load(path);
  auto s = glass::create_searcher(std::move(g), "L2");
  s->SetData(data, (float *)labels, (float *)ts, n, 100);
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
  return 0;
}
}
#endif
