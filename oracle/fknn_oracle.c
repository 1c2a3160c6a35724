/*
 * fknn_oracle.c -- CPU restatement of the reference's filtered-kNN hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke
 * entry and bench.py's CPU-baseline leg may load it; the product library
 * (libfknn) never links, calls or falls back to it.
 *
 * Parity pins: every function here is checked against the reference's own
 * compiled code (oracle/_ref, built from the reference sources by
 * oracle/Makefile) and against the golden fixtures in tests/golden/, which
 * were produced by that compiled reference (tests/golden/make_golden.py).
 *
 * Must be compiled with -ffp-contract=off: the reference distance is a
 * sequential float sum with separate rounding of the difference, the square
 * and the running sum (distance.h:62-72), and a fused multiply-add would
 * change the last bits.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_DIM 100
#define SQ8_CODE 112

/* distance.h:62-72 normal_l2: r += (a-b)*(a-b), each step rounded to float,
 * in dimension order. */
float oracle_normal_l2(const float *a, const float *b, unsigned dim) {
  float r = 0.0f;
  for (unsigned i = 0; i < dim; ++i) {
    float v = a[i] - b[i];
    v = v * v;
    r = r + v;
  }
  return r;
}

/* The predicate of utils.h:98-137.  The query type is read as uint32 from a
 * float (utils.h:98), the category value and the row label as int32
 * (utils.h:99,109), the window bounds inclusive (utils.h:125). */
static inline int pass_row(uint32_t qtype, int32_t v, float l, float r, float label, float ts) {
  switch (qtype) {
  case 0: return 1;
  case 1: return (int32_t)label == v;
  case 2: return ts >= l && ts <= r;
  case 3: return (int32_t)label == v && ts >= l && ts <= r;
  default: return 0;
  }
}

/* Bounded max-heap on (dist, id): keeps the k lexicographically smallest.
 * Rows arrive in increasing id, so this keeps exactly what ResultMaxHeap
 * (utils.h:35-78) keeps with its strict `<` replacement: a later row with an
 * equal distance is never admitted over an earlier one. */
typedef struct { float d; uint32_t id; } dist_id;

static inline int di_greater(dist_id a, dist_id b) { return a.d > b.d || (a.d == b.d && a.id > b.id); }

static void heap_sift_down(dist_id *h, int n, int i) {
  for (;;) {
    int l = 2 * i + 1, r = l + 1, m = i;
    if (l < n && di_greater(h[l], h[m])) m = l;
    if (r < n && di_greater(h[r], h[m])) m = r;
    if (m == i) return;
    dist_id t = h[i]; h[i] = h[m]; h[m] = t; i = m;
  }
}

static void heap_push_bounded(dist_id *h, int *n, int k, dist_id x) {
  if (*n < k) {
    int i = (*n)++;
    h[i] = x;
    while (i > 0) {
      int p = (i - 1) / 2;
      if (!di_greater(h[i], h[p])) break;
      dist_id t = h[i]; h[i] = h[p]; h[p] = t; i = p;
    }
  } else if (x.d < h[0].d) { /* strict, as utils.h:62 */
    h[0] = x;
    heap_sift_down(h, k, 0);
  }
}

/* Pops the heap into ascending (dist, id) order (utils.h:147-151) and pads
 * the tail with UINT32_MAX / +inf when fewer than k rows passed.  The
 * reference throws in that case (utils.h:44-47); the padding is this
 * project's definition of the behaviour. */
static void heap_emit(dist_id *h, int n, int k, uint32_t *ids, float *dists) {
  for (int j = n; j < k; ++j) {
    ids[j] = UINT32_MAX;
    if (dists) dists[j] = INFINITY;
  }
  for (int j = n - 1; j >= 0; --j) {
    ids[j] = h[0].id;
    if (dists) dists[j] = h[0].d;
    h[0] = h[j];
    heap_sift_down(h, j, 0);
  }
}

/* ---- exact filtered kNN (utils.h:80-158) over SoA columns ---- */

typedef struct {
  const float *vecs, *labels, *ts;
  uint32_t n;
  const float *qvecs, *metas;
  uint32_t nq, k;
  uint32_t *ids;
  float *dists;
  int use_f64;
  double *dists64;
  volatile int next;
  int status;
} exact_job;

static void exact_one(exact_job *J, uint32_t qi, dist_id *heap) {
  const float *m = J->metas + (size_t)qi * 4;
  uint32_t qtype = (uint32_t)m[0];
  int32_t v = (int32_t)m[1];
  float l = m[2], r = m[3];
  const float *q = J->qvecs + (size_t)qi * ORACLE_DIM;
  int n = 0;
  for (uint32_t j = 0; j < J->n; ++j) {
    if (!pass_row(qtype, v, l, r, J->labels[j], J->ts[j])) continue;
    dist_id x;
    x.d = oracle_normal_l2(J->vecs + (size_t)j * ORACLE_DIM, q, ORACLE_DIM);
    x.id = j;
    heap_push_bounded(heap, &n, (int)J->k, x);
  }
  heap_emit(heap, n, (int)J->k, J->ids + (size_t)qi * J->k, J->dists ? J->dists + (size_t)qi * J->k : NULL);
}

/* FP64 variant: distances Σ (x-q)^2 in double, same predicate and (dist, id)
 * order.  Used as the accuracy yardstick for the reduced-precision forms. */
typedef struct { double d; uint32_t id; } dist_id64;
static inline int di64_greater(dist_id64 a, dist_id64 b) { return a.d > b.d || (a.d == b.d && a.id > b.id); }
static void heap64_sift_down(dist_id64 *h, int n, int i) {
  for (;;) {
    int l = 2 * i + 1, r = l + 1, m = i;
    if (l < n && di64_greater(h[l], h[m])) m = l;
    if (r < n && di64_greater(h[r], h[m])) m = r;
    if (m == i) return;
    dist_id64 t = h[i]; h[i] = h[m]; h[m] = t; i = m;
  }
}

static void exact_one_f64(exact_job *J, uint32_t qi, dist_id64 *h) {
  const float *m = J->metas + (size_t)qi * 4;
  uint32_t qtype = (uint32_t)m[0];
  int32_t v = (int32_t)m[1];
  float l = m[2], r = m[3];
  const float *q = J->qvecs + (size_t)qi * ORACLE_DIM;
  int n = 0, k = (int)J->k;
  for (uint32_t j = 0; j < J->n; ++j) {
    if (!pass_row(qtype, v, l, r, J->labels[j], J->ts[j])) continue;
    const float *x = J->vecs + (size_t)j * ORACLE_DIM;
    double s = 0.0;
    for (int i = 0; i < ORACLE_DIM; ++i) {
      double t = (double)x[i] - (double)q[i];
      s += t * t;
    }
    dist_id64 e = {s, j};
    if (n < k) {
      int i = n++;
      h[i] = e;
      while (i > 0) {
        int p = (i - 1) / 2;
        if (!di64_greater(h[i], h[p])) break;
        dist_id64 t = h[i]; h[i] = h[p]; h[p] = t; i = p;
      }
    } else if (e.d < h[0].d) {
      h[0] = e;
      heap64_sift_down(h, k, 0);
    }
  }
  uint32_t *ids = J->ids + (size_t)qi * k;
  double *d = J->dists64 ? J->dists64 + (size_t)qi * k : NULL;
  for (int j = n; j < k; ++j) {
    ids[j] = UINT32_MAX;
    if (d) d[j] = INFINITY;
  }
  for (int j = n - 1; j >= 0; --j) {
    ids[j] = h[0].id;
    if (d) d[j] = h[0].d;
    h[0] = h[j];
    heap64_sift_down(h, j, 0);
  }
}

static void *exact_worker(void *arg) {
  exact_job *J = (exact_job *)arg;
  void *heap = malloc((size_t)J->k * (J->use_f64 ? sizeof(dist_id64) : sizeof(dist_id)));
  if (!heap) { J->status = -2; return NULL; }
  for (;;) {
    int qi = __atomic_fetch_add(&J->next, 1, __ATOMIC_RELAXED);
    if (qi >= (int)J->nq) break;
    if (J->use_f64) exact_one_f64(J, (uint32_t)qi, (dist_id64 *)heap);
    else exact_one(J, (uint32_t)qi, (dist_id *)heap);
  }
  free(heap);
  return NULL;
}

static int run_exact(exact_job *J, int nthreads) {
  for (uint32_t i = 0; i < J->nq; ++i) {
    float t = J->metas[(size_t)i * 4];
    if (!(t == 0.0f || t == 1.0f || t == 2.0f || t == 3.0f)) return -1; /* searcher.hpp:39-42 rejects other types */
  }
  if (J->k == 0) return -1;
  if (nthreads < 1) nthreads = 1;
  J->next = 0;
  J->status = 0;
  if (nthreads == 1) {
    exact_worker(J);
    return J->status;
  }
  pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
  if (!th) return -2;
  for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, exact_worker, J);
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  free(th);
  return J->status;
}

/* Exact FP32 filtered kNN.  vecs: n x 100, labels/ts: n, qvecs: nq x 100,
 * metas: nq x 4 (type, v, l, r).  ids/dists: nq x k ascending (dist, id),
 * padded with UINT32_MAX / +inf.  dists may be NULL.  Returns 0, -1 on a
 * query type outside 0..3, -2 on allocation failure. */
int oracle_exact_knn(const float *vecs, const float *labels, const float *ts, uint32_t n,
                     const float *qvecs, const float *metas, uint32_t nq, uint32_t k,
                     uint32_t *ids, float *dists, int nthreads) {
  exact_job J;
  memset(&J, 0, sizeof(J));
  J.vecs = vecs; J.labels = labels; J.ts = ts; J.n = n;
  J.qvecs = qvecs; J.metas = metas; J.nq = nq; J.k = k;
  J.ids = ids; J.dists = dists;
  return run_exact(&J, nthreads);
}

/* FP64 oracle: same contract, double distances. */
int oracle_exact_knn_f64(const float *vecs, const float *labels, const float *ts, uint32_t n,
                         const float *qvecs, const float *metas, uint32_t nq, uint32_t k,
                         uint32_t *ids, double *dists, int nthreads) {
  exact_job J;
  memset(&J, 0, sizeof(J));
  J.vecs = vecs; J.labels = labels; J.ts = ts; J.n = n;
  J.qvecs = qvecs; J.metas = metas; J.nq = nq; J.k = k;
  J.ids = ids; J.use_f64 = 1; J.dists64 = dists;
  return run_exact(&J, nthreads);
}

/* Number of rows passing each query's predicate (utils.h:110-137). */
void oracle_count_matches(const float *labels, const float *ts, uint32_t n, const float *metas,
                          uint32_t nq, uint32_t *counts) {
  for (uint32_t i = 0; i < nq; ++i) {
    const float *m = metas + (size_t)i * 4;
    uint32_t qt = (uint32_t)m[0];
    int32_t v = (int32_t)m[1];
    uint32_t c = 0;
    for (uint32_t j = 0; j < n; ++j) c += (uint32_t)pass_row(qt, v, m[2], m[3], labels[j], ts[j]);
    counts[i] = c;
  }
}

/* ---- symmetric SQ8 (pyglass/glass/quant/sq8_sym_quant.hpp) ---- */

/* alpha = max |x| over the training rows (sq8_sym_quant.hpp:37-43). */
float oracle_sq8_sym_alpha(const float *data, uint64_t count) {
  float a = 0.0f;
  for (uint64_t i = 0; i < count; ++i) {
    float v = fabsf(data[i]);
    if (v > a) a = v; /* std::max(alpha, |x|) */
  }
  return a;
}

/* encode (sq8_sym_quant.hpp:63-74): round(clamp(x/alpha, -1, 1) * 127),
 * std::round = half away from zero; dims 100..111 are zero. */
void oracle_sq8_sym_encode(const float *vecs, uint64_t n, float alpha, int8_t *codes) {
  for (uint64_t r = 0; r < n; ++r) {
    const float *x = vecs + r * ORACLE_DIM;
    int8_t *c = codes + r * SQ8_CODE;
    for (int i = 0; i < ORACLE_DIM; ++i) {
      float y = x[i] / alpha;
      if (y > 1.0f) y = 1.0f;
      if (y < -1.0f) y = -1.0f;
      c[i] = (int8_t)roundf(y * 127.0f);
    }
    for (int i = ORACLE_DIM; i < SQ8_CODE; ++i) c[i] = 0;
  }
}

/* L2SqrSQ8_sym (simd/distance.hpp:329-366): exact int32 Σ (x-y)^2 over 112. */
int32_t oracle_l2sqr_sq8_sym(const int8_t *x, const int8_t *y) {
  int32_t s = 0;
  for (int i = 0; i < SQ8_CODE; ++i) {
    int32_t t = (int32_t)x[i] - (int32_t)y[i];
    s += t * t;
  }
  return s;
}

/* maxPQIFCS (bruteforce.h:57-117): 1-based array max-heap on distance only. */
typedef struct { int32_t d; int32_t id; } pq_node;

static void pq_push_down(pq_node *h, int cnt, int x) {
  while ((x << 1) <= cnt) {
    int t = x << 1;
    if ((t | 1) <= cnt && h[t | 1].d > h[t].d) t |= 1;
    if (h[t].d <= h[x].d) break;
    pq_node s = h[x]; h[x] = h[t]; h[t] = s;
    x = t;
  }
}

static void pq_emplace(pq_node *h, int *cnt, int32_t id, int32_t d) {
  int now = ++(*cnt);
  h[now].d = d;
  h[now].id = id;
  while (now != 1 && h[now].d > h[now >> 1].d) {
    pq_node s = h[now]; h[now] = h[now >> 1]; h[now >> 1] = s;
    now >>= 1;
  }
}

/* bruteforce / bruteforce_subgraph (bruteforce.h:244-289) for one query:
 * int32 distances for every slab code, the first k emplaced, then
 * must_pop_emplace (replace the root only when strictly smaller), output in
 * heap-array order reversed: closest[k-1-l] = heap[l+1].id.  Requires
 * k <= npoints (the caller guarantees it, hybrid_graph.cpp:206,406).
 * dists (nullable) receives heap distance * alpha * alpha as float. */
int oracle_sq8_bruteforce(uint64_t k, int32_t *closest, float *dists, uint64_t npoints,
                          const int8_t *codes, float alpha, const int8_t *query) {
  if (k == 0 || k > npoints) return -1;
  pq_node *h = (pq_node *)malloc(sizeof(pq_node) * (k + 5));
  if (!h) return -2;
  int cnt = 0;
  for (uint64_t p = 0; p < k; ++p) pq_emplace(h, &cnt, (int32_t)p, oracle_l2sqr_sq8_sym(query, codes + p * SQ8_CODE));
  for (uint64_t p = k; p < npoints; ++p) {
    int32_t d = oracle_l2sqr_sq8_sym(query, codes + p * SQ8_CODE);
    if (h[1].d <= d) continue;
    h[1].id = (int32_t)p;
    h[1].d = d;
    pq_push_down(h, cnt, 1);
  }
  for (uint64_t l = 0; l < k; ++l) {
    closest[k - l - 1] = h[l + 1].id;
    if (dists) dists[k - l - 1] = (float)h[l + 1].d * alpha * alpha;
  }
  free(h);
  return 0;
}

/* ---- Graph beam search: the pyglass Searcher (pyglass/glass/searcher.hpp) ----
 *
 * A sequential restatement over a graph in Graph::save's byte layout
 * (graph.hpp:101-115; initializer HNSWInitializer.hpp:73-82), with the
 * searcher's SQ8-sym codes (Searcher::SetData, searcher.hpp:94-101).
 * The visited sets are plain byte arrays, which answer exactly what the
 * lazily-cleared Bitset (neighbor.hpp:41-102) answers. */

typedef struct {
  int32_t nep, N, K, upK, ep;
  const int32_t *eps, *adj;
  const float *ets;
  int32_t *levels;
  const int32_t **lists; /* per node: levels * upK ids */
} og_graph;

static int og_parse(const uint8_t *b, size_t nbytes, og_graph *g) {
  size_t off = 0;
  memset(g, 0, sizeof(*g));
  g->ep = -1;
#define OG_NEED(x) do { if ((size_t)(x) > nbytes - off) return -1; } while (0)
  OG_NEED(4); memcpy(&g->nep, b + off, 4); off += 4;
  if (g->nep < 0) return -1;
  OG_NEED((size_t)g->nep * 4); g->eps = (const int32_t *)(b + off); off += (size_t)g->nep * 4;
  OG_NEED(8); memcpy(&g->N, b + off, 4); memcpy(&g->K, b + off + 4, 4); off += 8;
  if (g->N <= 0 || g->K <= 0) return -1;
  size_t nk = (size_t)g->N * g->K;
  OG_NEED(nk * 8);
  g->adj = (const int32_t *)(b + off); off += nk * 4;
  g->ets = (const float *)(b + off); off += nk * 4;
  if (off == nbytes) return g->nep > 0 ? 0 : -1;
  int32_t iN;
  OG_NEED(12); memcpy(&iN, b + off, 4); memcpy(&g->upK, b + off + 4, 4); memcpy(&g->ep, b + off + 8, 4); off += 12;
  if (iN != g->N || g->upK <= 0) return -1;
  g->levels = (int32_t *)calloc(g->N, 4);
  g->lists = (const int32_t **)calloc(g->N, sizeof(int32_t *));
  if (!g->levels || !g->lists) return -2;
  for (int32_t i = 0; i < g->N; ++i) {
    int32_t cur;
    OG_NEED(4); memcpy(&cur, b + off, 4); off += 4;
    if (cur < 0 || cur % g->upK) return -1;
    g->levels[i] = cur / g->upK;
    OG_NEED((size_t)cur * 4); g->lists[i] = (const int32_t *)(b + off); off += (size_t)cur * 4;
  }
#undef OG_NEED
  return off == nbytes ? 0 : -1;
}

/* LinearPool (neighbor.hpp:223-283). */
typedef struct {
  int size, cur, cap;
  pq_node *data; /* cap + 1 slots, zeroed */
  uint8_t *vis, *vis1;
} og_pool;

static int og_insert(og_pool *p, int32_t u, int32_t d) {
  if (p->size == p->cap && d >= p->data[p->size - 1].d) return 0;
  int lo = 0, hi = p->size;
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    if (p->data[mid].d > d) hi = mid; else lo = mid + 1;
  }
  memmove(&p->data[lo + 1], &p->data[lo], (size_t)(p->size - lo) * sizeof(pq_node));
  p->data[lo].d = d;
  p->data[lo].id = u;
  if (p->size < p->cap) p->size++;
  if (lo < p->cur) p->cur = lo;
  return 1;
}

static int32_t og_pop(og_pool *p) {
  p->data[p->cur].id |= (int32_t)0x80000000;
  int pre = p->cur;
  while (p->cur < p->size && (p->data[p->cur].id >> 31 & 1)) p->cur++;
  return p->data[pre].id & 0x7fffffff;
}

static inline int32_t og_dist(const int8_t *codes, const int8_t *q, int32_t u) {
  return oracle_l2sqr_sq8_sym(q, codes + (size_t)u * SQ8_CODE);
}

/* Graph::initialize_search (graph.hpp:90-99) + HNSWInitializer::initialize
 * (HNSWInitializer.hpp:36-58). */
static void og_initialize(const og_graph *g, og_pool *p, const int8_t *codes, const int8_t *q) {
  if (g->ep >= 0) {
    int32_t u = g->ep;
    int32_t cur_dist = og_dist(codes, q, u);
    for (int level = g->levels[u]; level > 0; --level) {
      int changed = 1;
      while (changed) {
        changed = 0;
        const int32_t *list = g->lists[u] + (size_t)(level - 1) * g->upK;
        for (int i = 0; i < g->upK && list[i] != -1; ++i) {
          int32_t v = list[i];
          int32_t d = og_dist(codes, q, v);
          if (d < cur_dist) { cur_dist = d; u = v; changed = 1; }
        }
      }
    }
    og_insert(p, u, cur_dist);
    p->vis[u] = 1;
  } else {
    for (int e = 0; e < g->nep; ++e) og_insert(p, g->eps[e], og_dist(codes, q, g->eps[e]));
  }
}

/* SearchImpl / SearchFilterImpl / SearchFilterSubTimeImpl expansion
 * (searcher.hpp:172-198, 271-299, 386-413). */
static void og_expand_plain(const og_graph *g, og_pool *p, const int8_t *codes, const int8_t *q, int32_t u) {
  for (int i = 0; i < g->K; ++i) {
    int32_t v = g->adj[(size_t)u * g->K + i];
    if (v == -1) break;
    if (p->vis[v]) continue;
    p->vis[v] = 1;
    og_insert(p, v, og_dist(codes, q, v));
  }
}

/* SearchCategoryRangeImpl (rf 1, searcher.hpp:320-374) and
 * SearchRangeFilter[SubTime]Impl (rf 2, searcher.hpp:438-491, 516-569). */
static void og_expand_filtered(const og_graph *g, og_pool *p, const int8_t *codes, const int8_t *q, int32_t u,
                               float l, float r, int rf) {
  int count1 = 0, count2 = 0;
  for (int i = 0; i < g->K; ++i) {
    int32_t v = g->adj[(size_t)u * g->K + i];
    if (v == -1) break;
    if (p->vis[v]) continue;
    count2++;
    p->vis[v] = 1;
    float t = g->ets[(size_t)u * g->K + i];
    if (t < l || t > r) continue;
    og_insert(p, v, og_dist(codes, q, v));
    count1++;
  }
  for (int i = 0; i < g->K; ++i) {
    if (count1 >= rf * count2) break;
    int32_t nei = g->adj[(size_t)u * g->K + i];
    if (nei == -1) break;
    if (p->vis1[nei]) continue;
    p->vis1[nei] = 1;
    for (int j = 0; j < g->K; ++j) {
      int32_t v = g->adj[(size_t)nei * g->K + j];
      if (v == -1) break;
      if (p->vis[v]) continue;
      p->vis[v] = 1;
      float t = g->ets[(size_t)nei * g->K + j];
      if (t < l || t > r) continue;
      og_insert(p, v, og_dist(codes, q, v));
      count1++;
      if (count1 >= rf * count2) break;
    }
  }
}

/* One batch of Searcher calls.  mode: 0 Search, 1 SearchFilter,
 * 2 SearchFilterSubTime, 3 SearchCategoryRange, 4 SearchRangeFilterSubTime,
 * 5 SearchRangeFilter.  k is the reference's pool argument (capacity
 * max(k, ef)), refine the ids written per query (slots 0..refine-1, as
 * reorder / reorder_dist write them, sq8_sym_quant.hpp:76-89); dists
 * (nullable) = slot distance * alpha_square.  codes: n x 112 searcher codes;
 * qcodes: nq x 112 query codes (Computer's encode).  Returns 0, or -1 for a
 * malformed graph / arguments, -3 for a seed outside [0, n). */
int oracle_graph_search(const uint8_t *gbytes, size_t nbytes, const int8_t *codes, float alpha,
                        const int8_t *qcodes, uint32_t nq, int mode, uint32_t k, uint32_t ef, uint32_t refine,
                        const float *bounds, const int32_t *id_bounds, int32_t *out_ids, float *out_dists) {
  og_graph g;
  int rc = og_parse(gbytes, nbytes, &g);
  if (rc) { free(g.levels); free((void *)g.lists); return -1; }
  int cap = (int)(k > ef ? k : ef);
  if (mode < 0 || mode > 5 || k == 0 || refine == 0 || refine > (uint32_t)cap + 1) {
    free(g.levels); free((void *)g.lists); return -1;
  }
  const float alpha_square = alpha * alpha;
  og_pool p;
  p.cap = cap;
  p.data = (pq_node *)malloc(sizeof(pq_node) * (cap + 1));
  p.vis = (uint8_t *)malloc(g.N);
  p.vis1 = (uint8_t *)malloc(g.N);
  rc = 0;
  for (uint32_t qi = 0; qi < nq && rc == 0; ++qi) {
    const int8_t *q = qcodes + (size_t)qi * SQ8_CODE;
    memset(p.data, 0, sizeof(pq_node) * (cap + 1));
    memset(p.vis, 0, g.N);
    memset(p.vis1, 0, g.N);
    p.size = p.cur = 0;
    float l = 0.f, r = 0.f;
    int lb = 0, ub = 0;
    if (mode >= 3) {
      l = bounds[2 * qi]; r = bounds[2 * qi + 1];
      lb = id_bounds[2 * qi]; ub = id_bounds[2 * qi + 1];
    }
    float sel = (float)(ub - lb) / (float)g.N;
    int seeded = mode == 3 || (mode >= 4 && sel < 1);
    if (seeded) {
      int interval = (ub - lb) / 10;
      for (int i = 0; i < 10; ++i) {
        int point = lb + interval * i;
        if (point < 0 || point >= g.N) { rc = -3; break; }
        og_insert(&p, point, og_dist(codes, q, point));
        p.vis[point] = 1;
      }
      if (rc) break;
    } else if (mode != 4) {
      og_initialize(&g, &p, codes, q);
    }
    while (p.cur < p.size) {
      int32_t u = og_pop(&p);
      if (mode == 3) og_expand_filtered(&g, &p, codes, q, u, l, r, 1);
      else if (mode >= 4) og_expand_filtered(&g, &p, codes, q, u, l, r, 2);
      else og_expand_plain(&g, &p, codes, q, u);
    }
    for (uint32_t i = 0; i < refine; ++i) {
      out_ids[(size_t)qi * refine + i] = p.data[i].id & 0x7fffffff;
      if (out_dists) out_dists[(size_t)qi * refine + i] = (float)p.data[i].d * alpha_square;
    }
  }
  free(p.data); free(p.vis); free(p.vis1);
  free(g.levels); free((void *)g.lists);
  return rc;
}
