// Reference-equivalent routing of HybridGraph::BatchSearch
// (hybrid_graph.cpp:147-503) on the GPU.
//
// Per query the selectivity sel = (e - s) / sel_rows of its predicate slab
// picks one route, as the reference's planner does:
//   brute force  sel < bf_thr, or type 3 and sel < bf_thr3 (:201-229): the
//                bf_refine_k smallest symmetric-SQ8 distances over the slab
//                (k_sq8_slab_topk, one block per query), then FP32 re-rank;
//   category     types 1 / 3 otherwise (:239-298): the category's graph,
//                SearchFilter / SearchCategoryRange with a pool of
//                ceil(ef_min + slope * category size), FP32 re-rank of the
//                graph_refine_k candidates;
//   type 0       (:303-333) SearchFilterSubTime on every time-bucket graph,
//                each bucket's candidates merged into one pool per query;
//   type 2       (:340-459) SplitInterval over the buckets the window
//                overlaps: FULL -> SearchFilterSubTime, MEDIUM ->
//                SearchRangeFilterSubTime, SMALL -> SQ8 brute force over the
//                bucket's codes; merged into the same kind of pool;
//   then the pools of types 0 and 2 are re-ranked in FP32 (:465-494).
// Graph searches run batched per (graph, form, pool size) through the
// warp-per-query beam search; the brute forces and re-ranks are batched
// kernels.  The pools follow maxPQIFCS<int> (bruteforce.h:57-117) on the
// host, so candidates enter them in the reference's order and with its tie
// rule.  The brute-force candidates are the k smallest by (distance,
// position) where the reference keeps a heap's survivors: the same rows
// except among equal distances at the k-th place.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_util.cuh"

namespace fknn {
namespace {

constexpr int ST_THREADS = 256;
constexpr int ST_CAP = 1024;   // keys one brute-force block holds
constexpr int ST_KMAX = 256;   // largest brute-force k
constexpr int CODE = 112;

// One block per work item: the kmax smallest (SQ8 distance, position) keys
// of query qi over rows [s, e) of codes (112-byte rows), ascending, padded
// with ~0.  item i: sel[3i] = query, sel[3i+1] = s, sel[3i+2] = e;
// codes_of[i] picks codes0 (0) or codes1 (1).
__global__ void __launch_bounds__(ST_THREADS)
    k_sq8_slab_topk(const int8_t *__restrict__ codes0, const int8_t *__restrict__ codes1,
                    const int8_t *__restrict__ qcodes, const uint32_t *__restrict__ sel,
                    const uint8_t *__restrict__ codes_of, uint32_t nitems, uint32_t kmax, uint64_t *__restrict__ out) {
  __shared__ uint64_t buf[ST_CAP];
  __shared__ int qws[CODE / 4];
  __shared__ int cnt, qq_s;
  __shared__ uint64_t thr;
  const int tid = threadIdx.x;
  for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
    const uint32_t qi = sel[3 * it], s = sel[3 * it + 1], e = sel[3 * it + 2];
    const int8_t *codes = (codes_of && codes_of[it]) ? codes1 : codes0;
    const uint32_t K = min(kmax, e > s ? e - s : 0u);
    if (tid < CODE / 4) qws[tid] = reinterpret_cast<const int *>(qcodes + (uint64_t)qi * CODE)[tid];
    if (tid == 0) {
      cnt = 0;
      thr = ~0ull;
    }
    __syncthreads();
    if (tid == 0) {
      int qq = 0;
      for (int w = 0; w < CODE / 4; ++w) qq = __dp4a(qws[w], qws[w], qq);
      qq_s = qq;
    }
    int qw[CODE / 4];
#pragma unroll
    for (int w = 0; w < CODE / 4; ++w) qw[w] = qws[w];
    __syncthreads();
    const int qq = qq_s;
    for (uint32_t base = s; base < e; base += ST_THREADS) {
      const uint32_t p = base + tid;
      if (p < e) {
        const int d = sq8_dist(qw, qq, codes + (uint64_t)p * CODE);
        const uint64_t key = ((uint64_t)(uint32_t)d << 32) | (p - s);
        if (key < thr) buf[atomicAdd(&cnt, 1)] = key;
      }
      __syncthreads();
      if (cnt > ST_CAP - ST_THREADS) {
        for (int i = cnt + tid; i < ST_CAP; i += ST_THREADS) buf[i] = ~0ull;
        __syncthreads();
        block_bitonic_sort(buf, ST_CAP);
        if (tid == 0) {
          cnt = (int)K;
          thr = buf[K - 1];
        }
        __syncthreads();
      }
    }
    const int c = cnt;
    int np2 = 32;
    while (np2 < c) np2 <<= 1;
    for (int i = c + tid; i < np2; i += ST_THREADS) buf[i] = ~0ull;
    __syncthreads();
    block_bitonic_sort(buf, np2);
    for (uint32_t j = tid; j < kmax; j += ST_THREADS)
      out[(uint64_t)it * kmax + j] = (j < K && (int)j < c) ? buf[j] : ~0ull;
    __syncthreads();
  }
}

// Brute-force keys -> row ids: id = map[s + position], map = map1 for the
// items with which[it] set, else map0 (NULL map: s + position); padding
// stays UINT32_MAX.  Optional dist_out: the key's distance times scale.
__global__ void k_keys_to_ids(const uint64_t *__restrict__ keys, uint32_t nitems, uint32_t kmax,
                              const uint32_t *__restrict__ sel, const uint8_t *__restrict__ which,
                              const uint32_t *__restrict__ map0, const uint32_t *__restrict__ map1,
                              uint32_t *__restrict__ ids) {
  const uint64_t total = (uint64_t)nitems * kmax;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    const uint32_t it = (uint32_t)(i / kmax);
    uint32_t id = 0xffffffffu;
    if (k != ~0ull) {
      const uint32_t p = sel[3 * it + 1] + (uint32_t)k;
      const uint32_t *map = (which && which[it]) ? map1 : map0;
      id = map ? map[p] : p;
    }
    ids[i] = id;
  }
}

// Graph-local ids -> row ids: map[start + local] (negative: UINT32_MAX).
__global__ void k_local_to_ids(const int32_t *__restrict__ local, uint64_t total, uint32_t start,
                               const uint32_t *__restrict__ map, uint32_t *__restrict__ ids) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const int32_t l = local[i];
    ids[i] = l < 0 ? 0xffffffffu : map[start + (uint32_t)l];
  }
}

__global__ void k_gather_rows(const float *__restrict__ src, const uint32_t *__restrict__ rows, uint32_t nrows,
                              uint32_t width, float *__restrict__ dst) {
  const uint64_t total = (uint64_t)nrows * width;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = i / width;
    dst[i] = src[(uint64_t)rows[r] * width + (i - r * width)];
  }
}

__global__ void k_scatter_rows_u32(const uint32_t *__restrict__ src, const uint32_t *__restrict__ rows,
                                   uint32_t nrows, uint32_t width, uint32_t *__restrict__ dst) {
  const uint64_t total = (uint64_t)nrows * width;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = i / width;
    dst[(uint64_t)rows[r] * width + (i - r * width)] = src[i];
  }
}

// SQ8 codes of the rows in a row order: out[p] = codes[perm[p]]
__global__ void k_gather_codes(const int8_t *__restrict__ codes, const uint32_t *__restrict__ perm, uint64_t n,
                               int8_t *__restrict__ out) {
  const uint64_t total = n * (CODE / 16);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = i / (CODE / 16), w = i - p * (CODE / 16);
    reinterpret_cast<int4 *>(out)[i] = reinterpret_cast<const int4 *>(codes)[(uint64_t)perm[p] * (CODE / 16) + w];
  }
}

unsigned grid_of(uint64_t work) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((work + 255) / 256, 148 * 16)); }

// maxPQIFCS<int> (bruteforce.h:57-117): a max-heap of (distance, id) in
// slots 1..cnt; emplace while not full, then replace the root only by a
// strictly smaller distance.
struct IntPool {
  int cap = 0, cnt = 0;
  std::vector<std::pair<int, int>> d;  // (distance, id)
  void reset(int c) {
    cap = c;
    cnt = 0;
    d.assign((size_t)c + 2, {0, 0});
  }
  void push_down(int x) {
    while ((x << 1) <= cnt) {
      int t = x << 1;
      if ((t | 1) <= cnt && d[t | 1].first > d[t].first) t |= 1;
      if (d[t].first <= d[x].first) break;
      std::swap(d[x], d[t]);
      x = t;
    }
  }
  void offer(int id, int dist) {
    if (cnt < cap) {
      d[++cnt] = {dist, id};
      int now = cnt;
      while (now != 1 && d[now].first > d[now >> 1].first) {
        std::swap(d[now], d[now >> 1]);
        now >>= 1;
      }
      return;
    }
    if (d[1].first <= dist) return;
    d[1] = {dist, id};
    push_down(1);
  }
};

template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t cap = 0;
  int get(size_t n) {
    if (n <= cap) return FKNN_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    FKNN_CUDA(cudaMalloc((void **)&p, std::max<size_t>(n, 1) * sizeof(T)));
    cap = n;
    return FKNN_OK;
  }
  ~DBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace
}  // namespace fknn

struct fknn_router {
  struct Sub {
    int32_t key;
    uint32_t start, count;
    fknn_graph *g;
  };
  int device = 0;
  fknn_index *idx = nullptr;
  cudaStream_t st = nullptr;
  float alpha = 0.f;                         // SQ8 scale over the whole base (the full searcher's)
  int8_t *codes[2] = {nullptr, nullptr};     // SQ8 codes in the index's ORDER_TIME / ORDER_CAT row orders
  uint32_t *d_cat_ids = nullptr, *d_full_ids = nullptr;
  std::vector<uint32_t> full_ids;            // host copy: timestamp order -> id
  std::vector<float> ts_full;                // timestamps in timestamp order (SplitInterval)
  std::vector<Sub> cats, bks;
  uint32_t maxc = 0, minc = 0;
  // per-call device scratch
  fknn::DBuf<float> q, meta, qsub, bounds;
  fknn::DBuf<int8_t> qcodes, qcodes_b;
  fknn::DBuf<uint32_t> sel, rows, cand, out, ids;
  fknn::DBuf<uint64_t> keys;
  fknn::DBuf<int32_t> lids, idb;
  fknn::DBuf<float> ldist;
  fknn::DBuf<uint8_t> which;
  fknn::DBuf<int> err;
};

using namespace fknn;

namespace {

void destroy_router(fknn_router *r) {
  if (!r) return;
  cudaSetDevice(r->device);
  cudaDeviceSynchronize();
  for (auto &s : r->cats)
    if (s.g) fknn_graph_destroy(s.g);
  for (auto &s : r->bks)
    if (s.g) fknn_graph_destroy(s.g);
  if (r->idx) fknn_index_destroy(r->idx);
  cudaFree(r->codes[0]);
  cudaFree(r->codes[1]);
  cudaFree(r->d_cat_ids);
  cudaFree(r->d_full_ids);
  if (r->st) cudaStreamDestroy(r->st);
  delete r;
}

int add_subgraphs(fknn_router *r, const fknn_router_subgraph *sg, uint32_t nsg, const uint32_t *order,
                  const float *vecs, uint64_t n, std::vector<fknn_router::Sub> &dst, const char *what) {
  std::vector<float> v;
  for (uint32_t i = 0; i < nsg; ++i) {
    const fknn_router_subgraph &s = sg[i];
    if (!s.graph_bytes || (uint64_t)s.start + s.count > n || s.count == 0) {
      set_error(std::string("fknn_router_create: bad ") + what + " subgraph");
      return FKNN_EINVAL;
    }
    // the graph's points are its rows in base order, as Searcher::SetData gets them
    v.resize((size_t)s.count * DIM);
    for (uint32_t j = 0; j < s.count; ++j) std::memcpy(&v[(size_t)j * DIM], vecs + (size_t)order[s.start + j] * DIM, DIM * 4);
    fknn_router::Sub sub{s.key, s.start, s.count, nullptr};
    int rc = fknn_graph_create(s.graph_bytes, s.nbytes, v.data(), r->device, &sub.g);
    if (rc) return rc;
    dst.push_back(sub);
    uint32_t gn = 0, deg = 0;
    float a = 0.f;
    fknn_graph_info(sub.g, &gn, &deg, &a);
    if (gn != s.count) {
      set_error(std::string("fknn_router_create: a ") + what + " graph's size differs from its row count");
      return FKNN_EINVAL;
    }
  }
  return FKNN_OK;
}

int launch_graph(fknn_router *r, const fknn_router::Sub &sub, int mode, const float *d_q, uint32_t nq, uint32_t K,
                 uint32_t refine, const float *d_bounds, const int32_t *d_idb, int32_t *d_ids, float *d_d) {
  return fknn_graph_search(sub.g, d_q, nq, mode, K, 0, refine, d_bounds, d_idb, d_ids, d_d, r->st);
}

}  // namespace

extern "C" {

int fknn_router_default_params(fknn_router_params *p) {
  if (!p) return FKNN_EINVAL;
  // hybrid_graph.h:14-34 and :70-77; baseline.cpp:77 sets bf_thr to 0.045
  p->ef0_full = 425;
  p->ef1min = 1800;
  p->ef1max = 2500;
  p->ef3min = 1800;
  p->ef3max = 2800;
  p->ef2_full_large = 480;
  p->ef2_full_medium = 630;
  p->ef2_full_small = 780;
  p->ef2_medium_large = 680;
  p->ef2_medium_medium = 780;
  p->ef2_medium_small = 1180;
  p->bf_thr = 0.045f;
  p->bf_thr3 = 0.08f;
  p->bf_refine_k = 140;
  p->graph_refine_k = 150;
  p->sel_rows = 10000000;
  return FKNN_OK;
}

int fknn_router_create(const fknn_router_desc *d, fknn_router **out) {
  if (!out || !d || !d->vecs || !d->labels || !d->ts || !d->sorted_base_ids || !d->sorted_base_ids_by_full_time ||
      (d->ncategories && !d->categories) || (d->nbuckets && !d->buckets)) {
    set_error("fknn_router_create: NULL argument");
    return FKNN_EINVAL;
  }
  *out = nullptr;
  const uint64_t n = d->n;
  fknn_router *r = new (std::nothrow) fknn_router();
  if (!r) return FKNN_ENOMEM;
  r->device = d->device;
  r->maxc = d->maxc_size;
  r->minc = d->minc_size;
  fknn_index_opts o{};
  o.device = d->device;
  int rc = fknn_index_create(d->vecs, d->labels, d->ts, n, DIM, &o, &r->idx);
  auto fail = [&](int code) {
    destroy_router(r);
    return code;
  };
  if (rc) return fail(rc);
  for (uint64_t i = 0; i < n; ++i)
    if (d->sorted_base_ids[i] >= n || d->sorted_base_ids_by_full_time[i] >= n) {
      set_error("fknn_router_create: a base order names a row outside the base");
      return fail(FKNN_EINVAL);
    }
  cudaError_t e = cudaSetDevice(r->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&r->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(cuda_fail(e, "fknn_router_create"));
  // the whole base's symmetric SQ8 codes (the full searcher's quantizer,
  // baseline.cpp:104-107 / :141), laid out in the index's two row orders
  {
    int8_t *c0 = nullptr;
    e = cudaMalloc(&c0, (size_t)n * CODE);
    if (e != cudaSuccess) return fail(cuda_fail(e, "fknn_router_create: codes"));
    rc = fknn_sq8_sym_train(r->idx->vecs, n, &r->alpha, c0);
    for (int k = 0; k < 2 && !rc; ++k) {
      e = cudaMalloc(&r->codes[k], (size_t)n * CODE);
      if (e != cudaSuccess) {
        rc = cuda_fail(e, "fknn_router_create: codes");
        break;
      }
      k_gather_codes<<<grid_of(n * (CODE / 16)), 256, 0, r->st>>>(c0, r->idx->ord[k].perm, n, r->codes[k]);
    }
    if (!rc) {
      e = cudaStreamSynchronize(r->st);
      if (e != cudaSuccess) rc = cuda_fail(e, "fknn_router_create: codes");
    }
    cudaFree(c0);
    if (rc) return fail(rc);
  }
  e = cudaMalloc(&r->d_cat_ids, n * 4);
  if (e == cudaSuccess) e = cudaMalloc(&r->d_full_ids, n * 4);
  if (e == cudaSuccess) e = cudaMemcpy(r->d_cat_ids, d->sorted_base_ids, n * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(r->d_full_ids, d->sorted_base_ids_by_full_time, n * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(cuda_fail(e, "fknn_router_create: base orders"));
  r->full_ids.assign(d->sorted_base_ids_by_full_time, d->sorted_base_ids_by_full_time + n);
  r->ts_full.resize(n);
  for (uint64_t i = 0; i < n; ++i) r->ts_full[i] = d->ts[r->full_ids[i]];
  if ((rc = add_subgraphs(r, d->categories, d->ncategories, d->sorted_base_ids, d->vecs, n, r->cats, "category")))
    return fail(rc);
  if ((rc = add_subgraphs(r, d->buckets, d->nbuckets, d->sorted_base_ids_by_full_time, d->vecs, n, r->bks,
                          "time-bucket")))
    return fail(rc);
  *out = r;
  return FKNN_OK;
}

int fknn_router_destroy(fknn_router *r) {
  destroy_router(r);
  return FKNN_OK;
}

int fknn_router_search(fknn_router *r, const float *qvecs, const float *metas, uint32_t nq,
                       const fknn_router_params *params, uint32_t *ids, fknn_router_stats *stats) {
  if (!r || !qvecs || !metas || !ids) {
    set_error("fknn_router_search: NULL argument");
    return FKNN_EINVAL;
  }
  fknn_router_params P;
  if (params) P = *params;
  else fknn_router_default_params(&P);
  if (P.bf_refine_k < 100 || P.bf_refine_k > (uint32_t)ST_KMAX || P.graph_refine_k < 100 ||
      P.graph_refine_k > 2048 || P.sel_rows == 0) {
    set_error("fknn_router_search: need 100 <= bf_refine_k <= 256, 100 <= graph_refine_k <= 2048, sel_rows > 0");
    return FKNN_EINVAL;
  }
  if (nq == 0) return FKNN_OK;
  const auto t0 = std::chrono::steady_clock::now();
  auto tl = t0;
  auto lap = [&tl]() {  // ms since the last lap (stage boundaries are host syncs)
    const auto t = std::chrono::steady_clock::now();
    const float ms = std::chrono::duration<float, std::milli>(t - tl).count();
    tl = t;
    return ms;
  };
  fknn_router_stats S{};
  FKNN_CUDA(cudaSetDevice(r->device));
  cudaStream_t st = r->st;
  constexpr uint32_t K = 100;
  const uint32_t R = P.graph_refine_k;
  int rc;
  if ((rc = r->q.get((size_t)nq * DIM)) || (rc = r->meta.get((size_t)nq * 4)) || (rc = r->out.get((size_t)nq * K)) ||
      (rc = r->err.get(1)))
    return rc;
  FKNN_CUDA(cudaMemcpyAsync(r->q.p, qvecs, (size_t)nq * DIM * 4, cudaMemcpyHostToDevice, st));
  FKNN_CUDA(cudaMemcpyAsync(r->meta.p, metas, (size_t)nq * 16, cudaMemcpyHostToDevice, st));
  FKNN_CUDA(cudaMemsetAsync(r->out.p, 0xff, (size_t)nq * K * 4, st));
  FKNN_CUDA(cudaMemsetAsync(r->err.p, 0, 4, st));
  QueryDesc *d_desc, *h_desc;
  float *h_meta;
  {
    std::lock_guard<std::mutex> lock(r->idx->mu);
    if ((rc = prepare_queries(r->idx, r->q.p, r->meta.p, nq, st, &d_desc, &h_desc, &h_meta))) return rc;
  }
  // the global-alpha query codes (hybrid_graph.cpp:155-160)
  if ((rc = r->qcodes.get((size_t)nq * CODE))) return rc;
  launch_sq8_encode(r->q.p, nq, r->alpha, r->qcodes.p, st);

  // ---- route of every query (hybrid_graph.cpp:168-200, 248-253, 350-356)
  const float slope1 = (r->maxc > r->minc) ? (float)((int)P.ef1max - (int)P.ef1min) / (float)(r->maxc - r->minc) : 0.f;
  const float slope3 = (r->maxc > r->minc) ? (float)((int)P.ef3max - (int)P.ef3min) / (float)(r->maxc - r->minc) : 0.f;
  std::vector<float> sel(nq);
  std::vector<uint32_t> bf, type0, type2;
  std::vector<std::vector<uint32_t>> cat1(r->cats.size()), cat3(r->cats.size());
  for (uint32_t i = 0; i < nq; ++i) {
    const float type = metas[(size_t)i * 4];
    const QueryDesc &dq = h_desc[i];
    float s = 1.f;
    if (type != 0.f) s = (float)(dq.e - dq.s) / (float)P.sel_rows;
    sel[i] = s;
    if (s < P.bf_thr || (type == 3.f && s < P.bf_thr3)) {
      bf.push_back(i);
    } else if (type == 0.f) {
      type0.push_back(i);
    } else if (type == 2.f) {
      type2.push_back(i);
    } else {
      const int32_t v = (int32_t)metas[(size_t)i * 4 + 1];
      size_t c = 0;
      while (c < r->cats.size() && r->cats[c].key != v) ++c;
      if (c == r->cats.size()) bf.push_back(i);  // no graph for the category: its slab is scanned
      else (type == 1.f ? cat1 : cat3)[c].push_back(i);
    }
  }
  S.n_bruteforce = (uint32_t)bf.size();
  S.ms_prepare = lap();
  S.n_type0 = (uint32_t)type0.size();
  S.n_type2 = (uint32_t)type2.size();

  // FP32 re-rank of the candidate lists in r->cand (one row of width nc per
  // query of `list`), written to those queries' rows of r->out
  auto rerank_rows = [&](const std::vector<uint32_t> &list, uint32_t nc) -> int {
    const uint32_t m = (uint32_t)list.size();
    if (!m) return FKNN_OK;
    int rc2;
    if ((rc2 = r->rows.get(m)) || (rc2 = r->qsub.get((size_t)m * DIM)) || (rc2 = r->ids.get((size_t)m * K))) return rc2;
    FKNN_CUDA(cudaMemcpyAsync(r->rows.p, list.data(), (size_t)m * 4, cudaMemcpyHostToDevice, st));
    k_gather_rows<<<grid_of((uint64_t)m * DIM), 256, 0, st>>>(r->q.p, r->rows.p, m, DIM, r->qsub.p);
    if ((rc2 = launch_rerank(r->idx, r->qsub.p, m, r->cand.p, nc, K, r->ids.p, nullptr, r->err.p, st))) return rc2;
    k_scatter_rows_u32<<<grid_of((uint64_t)m * K), 256, 0, st>>>(r->ids.p, r->rows.p, m, K, r->out.p);
    g_launches += 3;
    FKNN_CUDA(cudaStreamSynchronize(st));  // list and the staging buffers are reused next
    return FKNN_OK;
  };
  // the queries of `list` gathered into r->qsub (graph searches take them contiguous)
  auto gather_queries = [&](const std::vector<uint32_t> &list) -> int {
    const uint32_t m = (uint32_t)list.size();
    int rc2;
    if ((rc2 = r->rows.get(m)) || (rc2 = r->qsub.get((size_t)m * DIM))) return rc2;
    FKNN_CUDA(cudaMemcpyAsync(r->rows.p, list.data(), (size_t)m * 4, cudaMemcpyHostToDevice, st));
    k_gather_rows<<<grid_of((uint64_t)m * DIM), 256, 0, st>>>(r->q.p, r->rows.p, m, DIM, r->qsub.p);
    g_launches += 1;
    return FKNN_OK;
  };

  // 1. brute force over the slab with the global codes, FP32 re-rank of
  //    the bf_refine_k candidates (hybrid_graph.cpp:201-229)
  if (!bf.empty()) {
    const uint32_t m = (uint32_t)bf.size(), kb = P.bf_refine_k;
    std::vector<uint32_t> h_sel((size_t)m * 3);
    std::vector<uint8_t> h_which(m);
    for (uint32_t j = 0; j < m; ++j) {
      const QueryDesc &dq = h_desc[bf[j]];
      h_sel[3 * j] = bf[j];
      h_sel[3 * j + 1] = dq.s;
      h_sel[3 * j + 2] = dq.e;
      h_which[j] = dq.order == ORDER_CAT ? 1 : 0;
    }
    if ((rc = r->sel.get((size_t)m * 3)) || (rc = r->which.get(m)) || (rc = r->keys.get((size_t)m * kb)) ||
        (rc = r->cand.get((size_t)m * kb)))
      return rc;
    FKNN_CUDA(cudaMemcpyAsync(r->sel.p, h_sel.data(), (size_t)m * 12, cudaMemcpyHostToDevice, st));
    FKNN_CUDA(cudaMemcpyAsync(r->which.p, h_which.data(), m, cudaMemcpyHostToDevice, st));
    k_sq8_slab_topk<<<std::min<uint32_t>(m, 148 * 8), ST_THREADS, 0, st>>>(r->codes[0], r->codes[1], r->qcodes.p,
                                                                          r->sel.p, r->which.p, m, kb, r->keys.p);
    k_keys_to_ids<<<grid_of((uint64_t)m * kb), 256, 0, st>>>(r->keys.p, m, kb, r->sel.p, r->which.p,
                                                               r->idx->ord[ORDER_TIME].perm,
                                                               r->idx->ord[ORDER_CAT].perm, r->cand.p);
    g_launches += 2;
    if ((rc = rerank_rows(bf, kb))) return rc;
  }
  S.ms_bruteforce = lap();

  // 2. category graphs (hybrid_graph.cpp:239-298): pool ceil(ef_min +
  //    slope * category size), graph_refine_k candidates, FP32 re-rank
  for (size_t c = 0; c < r->cats.size(); ++c) {
    const fknn_router::Sub &sub = r->cats[c];
    for (int form = 0; form < 2; ++form) {
      const std::vector<uint32_t> &list = form == 0 ? cat1[c] : cat3[c];
      const uint32_t m = (uint32_t)list.size();
      if (!m) continue;
      const uint32_t Kp = form == 0 ? (uint32_t)std::ceil((float)P.ef1min + slope1 * (float)sub.count)
                                    : (uint32_t)std::ceil((float)P.ef3min + slope3 * (float)sub.count);
      if ((rc = gather_queries(list)) || (rc = r->lids.get((size_t)m * R)) || (rc = r->cand.get((size_t)m * R)))
        return rc;
      if (form == 0) {
        rc = launch_graph(r, sub, FKNN_GRAPH_FILTER, r->qsub.p, m, Kp, R, nullptr, nullptr, r->lids.p, nullptr);
      } else {
        // the window (l, r) and the slab's positions inside the category (:275-282)
        std::vector<float> hb((size_t)m * 2);
        std::vector<int32_t> hib((size_t)m * 2);
        for (uint32_t j = 0; j < m; ++j) {
          const float *mt = metas + (size_t)list[j] * 4;
          hb[2 * j] = mt[2];
          hb[2 * j + 1] = mt[3];
          hib[2 * j] = (int32_t)(h_desc[list[j]].s - sub.start);
          hib[2 * j + 1] = (int32_t)(h_desc[list[j]].e - sub.start);
        }
        rc = launch_graph(r, sub, FKNN_GRAPH_CATEGORY_RANGE, r->qsub.p, m, Kp, R, hb.data(), hib.data(), r->lids.p,
                          nullptr);
      }
      if (rc) return rc;
      ++S.n_graph_calls;
      S.n_category += m;
      k_local_to_ids<<<grid_of((uint64_t)m * R), 256, 0, st>>>(r->lids.p, (uint64_t)m * R, sub.start, r->d_cat_ids,
                                                               r->cand.p);
      g_launches += 1;
      if ((rc = rerank_rows(list, R))) return rc;
    }
  }

  S.ms_category = lap();

  // 3. types 0 and 2: candidates of several time buckets merged per query
  //    into a pool of graph_refine_k (maxPQIFCS<int>), then FP32 re-rank
  std::vector<fknn::IntPool> pool(nq);
  std::vector<int32_t> h_ids;
  std::vector<float> h_d;
  // one batched graph search of `list` on bucket b; candidates offered to
  // the pools in the searcher's slot order (ids in timestamp order)
  auto bucket_search = [&](const fknn_router::Sub &b, int mode, const std::vector<uint32_t> &list, uint32_t Kp,
                           const std::vector<float> *hb, const std::vector<int32_t> *hib) -> int {
    const uint32_t m = (uint32_t)list.size();
    if (!m) return FKNN_OK;
    int rc2;
    if ((rc2 = gather_queries(list)) || (rc2 = r->lids.get((size_t)m * R)) || (rc2 = r->ldist.get((size_t)m * R)))
      return rc2;
    if ((rc2 = launch_graph(r, b, mode, r->qsub.p, m, Kp, R, hb ? hb->data() : nullptr, hib ? hib->data() : nullptr,
                            r->lids.p, r->ldist.p)))
      return rc2;
    ++S.n_graph_calls;
    h_ids.resize((size_t)m * R);
    h_d.resize((size_t)m * R);
    FKNN_CUDA(cudaMemcpyAsync(h_ids.data(), r->lids.p, (size_t)m * R * 4, cudaMemcpyDeviceToHost, st));
    FKNN_CUDA(cudaMemcpyAsync(h_d.data(), r->ldist.p, (size_t)m * R * 4, cudaMemcpyDeviceToHost, st));
    FKNN_CUDA(cudaStreamSynchronize(st));
    for (uint32_t j = 0; j < m; ++j) {
      fknn::IntPool &pl = pool[list[j]];
      if (pl.cap == 0) pl.reset((int)R);
      for (uint32_t t = 0; t < R; ++t) pl.offer(h_ids[(size_t)j * R + t] + (int)b.start, (int)h_d[(size_t)j * R + t]);
    }
    return FKNN_OK;
  };
  // type 0: SearchFilterSubTime with ef0_full on every bucket (:303-333)
  for (const fknn_router::Sub &b : r->bks)
    if ((rc = bucket_search(b, FKNN_GRAPH_FILTER_SUBTIME, type0, P.ef0_full, nullptr, nullptr))) return rc;
  S.ms_type0 = lap();

  // type 2: SplitInterval (:91-134) with bf_thr 0.5 when sel < 0.2, else 0.2
  if (!type2.empty()) {
    std::vector<size_t> border(r->bks.size());
    for (size_t b = 0; b < border.size(); ++b) border[b] = b;
    std::sort(border.begin(), border.end(), [&](size_t a, size_t c) { return r->bks[a].key < r->bks[c].key; });
    for (size_t bi : border) {  // buckets in t order (:378)
      const fknn_router::Sub &b = r->bks[bi];
      const float tsb = (float)b.key / 10, teb = (float)(b.key + 1) / 10;
      const float *tb = r->ts_full.data() + b.start;
      // per query: FULL / MEDIUM / SMALL with its pool size
      std::vector<uint32_t> fl[3], md[3], sm_list;
      std::vector<uint32_t> sm_s, sm_n;
      std::vector<float> mdb[3];
      std::vector<int32_t> mdib[3];
      for (uint32_t i : type2) {
        const float l = metas[(size_t)i * 4 + 2], rr = metas[(size_t)i * 4 + 3], s = sel[i];
        if (rr < tsb || l > teb) continue;
        if (l <= tsb && rr >= teb) {
          const int ki = s < 0.3f ? 0 : s < 0.6f ? 1 : 2;
          fl[ki].push_back(i);
          continue;
        }
        const float lb = std::max(tsb, l), rb = std::min(teb, rr);
        const uint32_t s0 = (uint32_t)(std::lower_bound(tb, tb + b.count, lb) - tb);
        const uint32_t e0 = (uint32_t)(std::upper_bound(tb, tb + b.count, rb) - tb);
        const uint32_t np = e0 > s0 ? e0 - s0 : 0;
        const float lsel = (float)np / (float)b.count;
        const float thr = s < 0.2f ? 0.5f : 0.2f;
        if (lsel < thr) {
          if (np) {
            sm_list.push_back(i);
            sm_s.push_back(s0);
            sm_n.push_back(np);
          }
        } else {
          const int ki = s > 0.6f ? 0 : s > 0.3f ? 1 : 2;
          md[ki].push_back(i);
          mdb[ki].push_back(l);
          mdb[ki].push_back(rr);
          mdib[ki].push_back((int32_t)s0);
          mdib[ki].push_back((int32_t)(s0 + np - 1));
        }
      }
      // the reference visits a bucket's queries in query order, each with
      // its own form; forms are batched here, and a query meets a bucket
      // once, so its pool sees the same sequence of candidates
      const uint32_t kfull[3] = {P.ef2_full_small, P.ef2_full_medium, P.ef2_full_large};
      const uint32_t kmed[3] = {P.ef2_medium_large, P.ef2_medium_medium, P.ef2_medium_small};
      for (int ki = 0; ki < 3; ++ki) {
        S.n_split_full += (uint32_t)fl[ki].size();
        S.n_split_medium += (uint32_t)md[ki].size();
        if ((rc = bucket_search(b, FKNN_GRAPH_FILTER_SUBTIME, fl[ki], kfull[ki], nullptr, nullptr))) return rc;
        if ((rc = bucket_search(b, FKNN_GRAPH_RANGE_SUBTIME, md[ki], kmed[ki], &mdb[ki], &mdib[ki]))) return rc;
      }
      if (!sm_list.empty()) {
        // SQ8 brute force over the bucket's own codes (its searcher's
        // quantizer), distances times alpha^2 (:399-417, bruteforce.h:267)
        const uint32_t m = (uint32_t)sm_list.size(), kb = P.bf_refine_k;
        S.n_split_small += m;
        const int8_t *bcodes;
        float ba;
        uint32_t bn;
        graph_codes(b.g, &bcodes, &ba, &bn);
        std::vector<uint32_t> h_sel((size_t)m * 3);
        for (uint32_t j = 0; j < m; ++j) {
          h_sel[3 * j] = j;
          h_sel[3 * j + 1] = sm_s[j];
          h_sel[3 * j + 2] = sm_s[j] + sm_n[j];
        }
        if ((rc = gather_queries(sm_list)) || (rc = r->qcodes_b.get((size_t)m * CODE)) ||
            (rc = r->sel.get((size_t)m * 3)) || (rc = r->keys.get((size_t)m * kb)))
          return rc;
        launch_sq8_encode(r->qsub.p, m, ba, r->qcodes_b.p, st);
        FKNN_CUDA(cudaMemcpyAsync(r->sel.p, h_sel.data(), (size_t)m * 12, cudaMemcpyHostToDevice, st));
        k_sq8_slab_topk<<<std::min<uint32_t>(m, 148 * 8), ST_THREADS, 0, st>>>(bcodes, bcodes, r->qcodes_b.p, r->sel.p,
                                                                              nullptr, m, kb, r->keys.p);
        g_launches += 2;
        std::vector<uint64_t> hk((size_t)m * kb);
        FKNN_CUDA(cudaMemcpyAsync(hk.data(), r->keys.p, hk.size() * 8, cudaMemcpyDeviceToHost, st));
        FKNN_CUDA(cudaStreamSynchronize(st));
        const float a2 = ba * ba;
        for (uint32_t j = 0; j < m; ++j) {
          fknn::IntPool &pl = pool[sm_list[j]];
          if (pl.cap == 0) pl.reset((int)R);
          for (uint32_t t = 0; t < kb; ++t) {
            const uint64_t key = hk[(size_t)j * kb + t];
            if (key == ~0ull) break;
            const float dist = (float)(uint32_t)(key >> 32) * ba * ba;
            (void)a2;
            pl.offer((int)(b.start + sm_s[j] + (uint32_t)key), (int)dist);
          }
        }
      }
    }
  }
  S.ms_type2 = lap();
  // global re-rank of the pools (:465-494), ids through the timestamp order
  {
    std::vector<uint32_t> list;
    for (uint32_t i : type0) list.push_back(i);
    for (uint32_t i : type2) list.push_back(i);
    const uint32_t m = (uint32_t)list.size();
    if (m) {
      std::vector<uint32_t> hc((size_t)m * R, 0xffffffffu);
      for (uint32_t j = 0; j < m; ++j) {
        const fknn::IntPool &pl = pool[list[j]];
        for (int t = 1; t <= pl.cnt; ++t) hc[(size_t)j * R + t - 1] = r->full_ids[pl.d[t].second];
      }
      if ((rc = r->cand.get((size_t)m * R))) return rc;
      FKNN_CUDA(cudaMemcpyAsync(r->cand.p, hc.data(), hc.size() * 4, cudaMemcpyHostToDevice, st));
      if ((rc = rerank_rows(list, R))) return rc;
    }
  }
  FKNN_CUDA(cudaMemcpyAsync(ids, r->out.p, (size_t)nq * K * 4, cudaMemcpyDeviceToHost, st));
  int err = 0;
  FKNN_CUDA(cudaMemcpyAsync(&err, r->err.p, 4, cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  if (err) {
    set_error("fknn_router_search: a candidate named a row outside the base");
    return FKNN_EINVAL;
  }
  S.ms_final = lap();
  S.ms_total = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (stats) *stats = S;
  return FKNN_OK;
}

}  // extern "C"
