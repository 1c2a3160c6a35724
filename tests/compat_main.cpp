// Exercises include/fknn_compat.hpp with the reference's call shapes:
// Bruteforce against a plain CPU restatement of utils.h:80 (sequential float
// sums, (distance, id) order), bruteforce against the k smallest SQ8
// distances, and HybridGraph::BatchSearch's sorted_ids placement.
// Prints "OK" and exits 0 when everything matches.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "fknn_compat.hpp"

static uint64_t g_state = 12345;
static float urand() {
  g_state = g_state * 6364136223846793005ull + 1442695040888963407ull;
  return (float)((g_state >> 40) & 0xffffff) / 16777216.0f;
}

static float seq_l2(const float *a, const float *b) {
  float r = 0.f;
  for (int d = 0; d < 100; ++d) {
    volatile float v = a[d] - b[d];
    volatile float s = v * v;
    r = r + s;
  }
  return r;
}

#define REQUIRE(c, msg)                    \
  do {                                     \
    if (!(c)) {                            \
      std::printf("FAIL: %s\n", msg);      \
      return 1;                            \
    }                                      \
  } while (0)

int main() {
  const int n = 20000, nq = 200;
  std::vector<std::vector<float>> nodes(n, std::vector<float>(102)), queries(nq, std::vector<float>(104));
  for (int i = 0; i < n; ++i) {
    nodes[i][0] = (float)(int)(urand() * 10);
    nodes[i][1] = urand();
    for (int d = 0; d < 100; ++d) nodes[i][2 + d] = urand() * 2 - 1;
  }
  for (int i = 0; i < nq; ++i) {
    const int t = i % 4;
    const float l = urand() * 0.5f;
    queries[i][0] = (float)t;
    queries[i][1] = (float)(int)(urand() * 10);
    queries[i][2] = l;
    queries[i][3] = l + 0.4f;
    for (int d = 0; d < 100; ++d) queries[i][4 + d] = urand() * 2 - 1;
  }
  // 1. Bruteforce (utils.h:80)
  std::vector<std::vector<uint32_t>> gt;
  fknn_compat::Bruteforce(nodes, queries, gt);
  REQUIRE((int)gt.size() == nq, "gt size");
  for (int i = 0; i < nq; ++i) {
    const float *m = queries[i].data();
    const uint32_t type = (uint32_t)m[0];
    std::vector<std::pair<float, uint32_t>> c;
    for (int r = 0; r < n; ++r) {
      const bool lab = (int32_t)nodes[r][0] == (int32_t)m[1];
      const bool win = nodes[r][1] >= m[2] && nodes[r][1] <= m[3];
      const bool pass = type == 0 || (type == 1 && lab) || (type == 2 && win) || (type == 3 && lab && win);
      if (pass) c.push_back({seq_l2(nodes[r].data() + 2, m + 4), (uint32_t)r});
    }
    std::sort(c.begin(), c.end());
    for (int j = 0; j < 100; ++j) {
      const uint32_t want = j < (int)c.size() ? c[j].second : 0xffffffffu;
      REQUIRE(gt[i][j] == want, "Bruteforce id differs from the CPU restatement");
    }
  }
  // 2. bruteforce (bruteforce.h:244) over one SQ8 slab
  std::vector<float> flat((size_t)n * 100);
  for (int i = 0; i < n; ++i) std::copy(nodes[i].begin() + 2, nodes[i].end(), flat.begin() + (size_t)i * 100);
  std::vector<int8_t> codes((size_t)n * 112), qc(112);
  float alpha = 0.f;
  fknn_compat::check(fknn_sq8_sym_train(flat.data(), n, &alpha, codes.data()));
  fknn_compat::check(fknn_sq8_sym_encode(queries[0].data() + 4, 1, alpha, qc.data()));
  std::vector<int> closest(140);
  fknn_compat::bruteforce(100, 140, closest.data(), n, (char *)codes.data(), alpha, 1, qc.data());
  std::vector<int> dist(n);
  for (int r = 0; r < n; ++r) {
    int s = 0;
    for (int d = 0; d < 112; ++d) {
      const int t = (int)codes[(size_t)r * 112 + d] - (int)qc[d];
      s += t * t;
    }
    dist[r] = s;
  }
  std::vector<int> sorted = dist;
  std::nth_element(sorted.begin(), sorted.begin() + 139, sorted.end());
  int worst = 0;
  for (int id : closest) {
    REQUIRE(id >= 0 && id < n, "bruteforce id out of range");
    worst = std::max(worst, dist[id]);
  }
  REQUIRE(worst <= sorted[139], "bruteforce did not return the 140 smallest SQ8 distances");
  // 3. HybridGraph::BatchSearch with sorted_ids (reverse order here)
  std::vector<float> labels(n), ts(n), qv((size_t)nq * 100), qm((size_t)nq * 4);
  for (int i = 0; i < n; ++i) {
    labels[i] = nodes[i][0];
    ts[i] = nodes[i][1];
  }
  fknn_compat::HybridGraph hg;
  hg.Build(flat.data(), labels.data(), ts.data(), n);
  hg.sorted_ids.resize(nq);
  for (int i = 0; i < nq; ++i) {
    const int orig = nq - 1 - i;
    hg.sorted_ids[i] = (uint32_t)orig;
    std::copy(queries[orig].begin() + 4, queries[orig].end(), qv.begin() + (size_t)i * 100);
    std::copy(queries[orig].begin(), queries[orig].begin() + 4, qm.begin() + (size_t)i * 4);
  }
  std::vector<uint32_t> ids((size_t)nq * 100);
  fknn_compat::SearchParams exact;
  exact.mode = FKNN_MODE_EXACT_FP32;
  hg.BatchSearch(nullptr, nullptr, nullptr, qv.data(), qm.data(), nq, ids.data(), exact);
  for (int q = 0; q < nq; ++q)
    for (int j = 0; j < 100; ++j) REQUIRE(ids[(size_t)q * 100 + j] == gt[q][j], "BatchSearch (exact) placement");
  struct ReferenceLikeParams {  // no mode / kprime members: the BF16 form with its default k'
    int ef1min = 1800;
  } rp;
  hg.BatchSearch(nullptr, nullptr, nullptr, qv.data(), qm.data(), nq, ids.data(), rp);
  double hit = 0, tot = 0;
  for (int q = 0; q < nq; ++q) {
    std::vector<uint32_t> a(gt[q]), b(ids.begin() + (size_t)q * 100, ids.begin() + (size_t)(q + 1) * 100);
    std::sort(a.begin(), a.end());
    std::sort(b.begin(), b.end());
    std::vector<uint32_t> in;
    std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(in));
    hit += (double)in.size();
    tot += 100;
  }
  REQUIRE(hit / tot >= 0.99, "BatchSearch (BF16) recall below 0.99");
  std::printf("OK recall %.6f\n", hit / tot);
  return 0;
}
