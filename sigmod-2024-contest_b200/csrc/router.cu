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
#include <deque>
#include <thread>
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
  std::vector<cudaStream_t> sst;             // one per sub-graph (categories, then buckets)
  std::vector<cudaEvent_t> sev;              // their joins
  cudaEvent_t ev_in = nullptr;               // a stage's inputs are staged
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
  for (cudaStream_t x : r->sst)
    if (x) cudaStreamDestroy(x);
  for (cudaEvent_t x : r->sev)
    if (x) cudaEventDestroy(x);
  if (r->ev_in) cudaEventDestroy(r->ev_in);
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
  // the sub-graphs' searches of a stage run side by side
  const size_t nsub = r->cats.size() + r->bks.size();
  r->sst.assign(nsub, nullptr);
  r->sev.assign(nsub, nullptr);
  cudaError_t e2 = cudaEventCreateWithFlags(&r->ev_in, cudaEventDisableTiming);
  for (size_t i = 0; i < nsub && e2 == cudaSuccess; ++i) {
    e2 = cudaStreamCreateWithFlags(&r->sst[i], cudaStreamNonBlocking);
    if (e2 == cudaSuccess) e2 = cudaEventCreateWithFlags(&r->sev[i], cudaEventDisableTiming);
  }
  if (e2 != cudaSuccess) return fail(cuda_fail(e2, "fknn_router_create"));
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

  // The graph searches of a stage, enqueued together: every sub-graph's
  // searches on that sub-graph's stream (one graph's scratch serves one
  // search at a time), all inputs staged by one copy each, all outputs read
  // back once.  Batches keep the reference's order, in which their
  // candidates are merged afterwards.
  struct GBatch {
    uint32_t sub;                         // index into subs()
    int mode;
    const std::vector<uint32_t> *list;
    uint32_t K;                           // pool argument of the search
    std::vector<float> hb;                // ranged forms: the windows ...
    std::vector<int32_t> hib;             // ... and their row ranges in the sub-graph
    bool dists;
    size_t q0 = 0, b0 = 0, o0 = 0;        // offsets: queries, windows, outputs
  };
  struct BBatch {                         // SQ8 brute force over a bucket's own codes (SplitInterval SMALL)
    uint32_t sub;
    std::vector<uint32_t> list, s, cnt;
    size_t q0 = 0, k0 = 0;
  };
  auto subs = [&](uint32_t i) -> const fknn_router::Sub & {
    return i < r->cats.size() ? r->cats[i] : r->bks[i - r->cats.size()];
  };
  std::vector<int32_t> h_ids;
  std::vector<float> h_d;
  std::vector<uint64_t> h_keys;
  auto run_stage = [&](std::vector<GBatch> &B, std::vector<BBatch> &BB, bool to_host) -> int {
    size_t nqs = 0, nb = 0, no = 0, nk = 0;
    const uint32_t kb = P.bf_refine_k;
    std::vector<uint32_t> rows;
    std::vector<float> hb;
    std::vector<int32_t> hib;
    std::vector<uint32_t> hsel;
    for (GBatch &b : B) {
      b.q0 = nqs;
      b.b0 = nb;
      b.o0 = no;
      rows.insert(rows.end(), b.list->begin(), b.list->end());
      nqs += b.list->size();
      no += b.list->size() * R;
      if (!b.hb.empty()) {
        hb.insert(hb.end(), b.hb.begin(), b.hb.end());
        hib.insert(hib.end(), b.hib.begin(), b.hib.end());
        nb += b.list->size();
      }
    }
    for (BBatch &b : BB) {
      b.q0 = nqs;
      b.k0 = nk;
      for (size_t j = 0; j < b.list.size(); ++j) {
        hsel.push_back((uint32_t)(b.q0 + j));  // the query's row in the staged queries
        hsel.push_back(b.s[j]);
        hsel.push_back(b.s[j] + b.cnt[j]);
      }
      rows.insert(rows.end(), b.list.begin(), b.list.end());
      nqs += b.list.size();
      nk += b.list.size() * kb;
    }
    if (!nqs) return FKNN_OK;
    int rc2;
    if ((rc2 = r->rows.get(nqs)) || (rc2 = r->qsub.get(nqs * DIM)) || (rc2 = r->bounds.get(std::max<size_t>(nb, 1) * 2)) ||
        (rc2 = r->idb.get(std::max<size_t>(nb, 1) * 2)) || (rc2 = r->lids.get(std::max<size_t>(no, 1))) ||
        (rc2 = r->ldist.get(std::max<size_t>(no, 1))) || (rc2 = r->qcodes_b.get(nqs * CODE)) ||
        (rc2 = r->sel.get(std::max<size_t>(hsel.size(), 3))) || (rc2 = r->keys.get(std::max<size_t>(nk, 1))))
      return rc2;
    // scratch of every graph at its largest search of the stage (nothing is
    // allocated once searches are in flight)
    std::vector<uint32_t> used;
    {
      std::vector<uint32_t> mq(r->cats.size() + r->bks.size(), 0), mc(mq.size(), 0);
      for (GBatch &b : B) {
        uint32_t cap = 0;
        if ((rc2 = graph_check_args(subs(b.sub).g, r->q.p, (uint32_t)b.list->size(), b.mode, b.K, 0, R, r->bounds.p,
                                    r->idb.p, r->lids.p, &cap)))
          return rc2;
        mq[b.sub] = std::max<uint32_t>(mq[b.sub], (uint32_t)b.list->size());
        mc[b.sub] = std::max(mc[b.sub], cap);
      }
      for (uint32_t i = 0; i < mq.size(); ++i)
        if (mq[i]) {
          used.push_back(i);
          if ((rc2 = graph_reserve(subs(i).g, mq[i], mc[i]))) return rc2;
        }
    }
    FKNN_CUDA(cudaMemcpyAsync(r->rows.p, rows.data(), nqs * 4, cudaMemcpyHostToDevice, st));
    if (nb) {
      FKNN_CUDA(cudaMemcpyAsync(r->bounds.p, hb.data(), nb * 8, cudaMemcpyHostToDevice, st));
      FKNN_CUDA(cudaMemcpyAsync(r->idb.p, hib.data(), nb * 8, cudaMemcpyHostToDevice, st));
    }
    if (!hsel.empty()) FKNN_CUDA(cudaMemcpyAsync(r->sel.p, hsel.data(), hsel.size() * 4, cudaMemcpyHostToDevice, st));
    k_gather_rows<<<grid_of((uint64_t)nqs * DIM), 256, 0, st>>>(r->q.p, r->rows.p, (uint32_t)nqs, DIM, r->qsub.p);
    g_launches += 1;
    FKNN_CUDA(cudaEventRecord(r->ev_in, st));
    std::vector<uint8_t> waiting(r->sst.size(), 0);
    auto join_in = [&](uint32_t i) -> int {
      if (!waiting[i]) {
        FKNN_CUDA(cudaStreamWaitEvent(r->sst[i], r->ev_in, 0));
        waiting[i] = 1;
      }
      return FKNN_OK;
    };
    for (uint32_t i : used) {
      if ((rc2 = join_in(i))) return rc2;
      if ((rc2 = graph_flag_reset(subs(i).g, r->sst[i]))) return rc2;
    }
    for (GBatch &b : B) {
      const uint32_t m = (uint32_t)b.list->size();
      if (!m) continue;
      uint32_t cap = 0;
      graph_check_args(subs(b.sub).g, r->q.p, m, b.mode, b.K, 0, R, r->bounds.p, r->idb.p, r->lids.p, &cap);
      const bool ranged = !b.hb.empty();
      if ((rc2 = graph_launch(subs(b.sub).g, r->qsub.p + b.q0 * DIM, m, b.mode, b.K, cap, R,
                              ranged ? r->bounds.p + 2 * b.b0 : nullptr, ranged ? r->idb.p + 2 * b.b0 : nullptr,
                              r->lids.p + b.o0, b.dists ? r->ldist.p + b.o0 : nullptr, r->sst[b.sub])))
        return rc2;
      ++S.n_graph_calls;
    }
    for (BBatch &b : BB) {
      const uint32_t m = (uint32_t)b.list.size();
      const int8_t *bcodes;
      float ba;
      uint32_t bn;
      graph_codes(subs(b.sub).g, &bcodes, &ba, &bn);
      if ((rc2 = join_in(b.sub))) return rc2;
      launch_sq8_encode(r->qsub.p + b.q0 * DIM, m, ba, r->qcodes_b.p + b.q0 * CODE, r->sst[b.sub]);
      // sel rows name the query's row in the staged queries, codes_b holds them at the same rows
      k_sq8_slab_topk<<<std::min<uint32_t>(m, 148 * 8), ST_THREADS, 0, r->sst[b.sub]>>>(
          bcodes, bcodes, r->qcodes_b.p, r->sel.p + 3 * (b.k0 / kb), nullptr, m, kb, r->keys.p + b.k0);
      g_launches += 2;
    }
    for (uint32_t i = 0; i < r->sst.size(); ++i)
      if (waiting[i]) {
        FKNN_CUDA(cudaEventRecord(r->sev[i], r->sst[i]));
        FKNN_CUDA(cudaStreamWaitEvent(st, r->sev[i], 0));
      }
    if (to_host) {
      h_ids.resize(no);
      h_d.resize(no);
      h_keys.resize(nk);
      if (no) {
        FKNN_CUDA(cudaMemcpyAsync(h_ids.data(), r->lids.p, no * 4, cudaMemcpyDeviceToHost, st));
        FKNN_CUDA(cudaMemcpyAsync(h_d.data(), r->ldist.p, no * 4, cudaMemcpyDeviceToHost, st));
      }
      if (nk) FKNN_CUDA(cudaMemcpyAsync(h_keys.data(), r->keys.p, nk * 8, cudaMemcpyDeviceToHost, st));
    }
    FKNN_CUDA(cudaStreamSynchronize(st));
    for (uint32_t i : used)
      if ((rc2 = graph_flag_check(subs(i).g))) return rc2;
    return FKNN_OK;
  };

  // 2. category graphs (hybrid_graph.cpp:239-298): pool ceil(ef_min +
  //    slope * category size), graph_refine_k candidates, FP32 re-rank
  {
    std::vector<GBatch> B;
    std::vector<BBatch> none;
    for (size_t c = 0; c < r->cats.size(); ++c) {
      const fknn_router::Sub &sub = r->cats[c];
      for (int form = 0; form < 2; ++form) {
        const std::vector<uint32_t> &list = form == 0 ? cat1[c] : cat3[c];
        const uint32_t m = (uint32_t)list.size();
        if (!m) continue;
        GBatch b;
        b.sub = (uint32_t)c;
        b.mode = form == 0 ? FKNN_GRAPH_FILTER : FKNN_GRAPH_CATEGORY_RANGE;
        b.list = &list;
        b.K = form == 0 ? (uint32_t)std::ceil((float)P.ef1min + slope1 * (float)sub.count)
                        : (uint32_t)std::ceil((float)P.ef3min + slope3 * (float)sub.count);
        b.dists = false;
        if (form == 1) {
          // the window (l, r) and the slab's positions inside the category (:275-282)
          b.hb.resize((size_t)m * 2);
          b.hib.resize((size_t)m * 2);
          for (uint32_t j = 0; j < m; ++j) {
            const float *mt = metas + (size_t)list[j] * 4;
            b.hb[2 * j] = mt[2];
            b.hb[2 * j + 1] = mt[3];
            b.hib[2 * j] = (int32_t)(h_desc[list[j]].s - sub.start);
            b.hib[2 * j + 1] = (int32_t)(h_desc[list[j]].e - sub.start);
          }
        }
        S.n_category += m;
        B.push_back(std::move(b));
      }
    }
    if ((rc = run_stage(B, none, false))) return rc;
    std::vector<uint32_t> all;
    for (GBatch &b : B) all.insert(all.end(), b.list->begin(), b.list->end());
    if (!all.empty()) {
      if ((rc = r->cand.get(all.size() * R))) return rc;
      for (GBatch &b : B) {
        const uint64_t tot = (uint64_t)b.list->size() * R;
        k_local_to_ids<<<grid_of(tot), 256, 0, st>>>(r->lids.p + b.o0, tot, subs(b.sub).start, r->d_cat_ids,
                                                     r->cand.p + b.o0);
        g_launches += 1;
      }
      if ((rc = rerank_rows(all, R))) return rc;
    }
  }
  S.ms_category = lap();

  // 3. types 0 and 2: candidates of several time buckets merged per query
  //    into a pool of graph_refine_k (maxPQIFCS<int>), then FP32 re-rank
  std::vector<fknn::IntPool> pool(nq);
  {
    const uint32_t nc = (uint32_t)r->cats.size();
    std::vector<GBatch> B;
    std::vector<BBatch> BB;
    std::deque<std::vector<uint32_t>> lists;  // FULL / MEDIUM lists (stable addresses)
    // type 0 (:303-333): SearchFilterSubTime with ef0_full on every bucket, in the map's order
    if (!type0.empty())
      for (uint32_t bi = 0; bi < r->bks.size(); ++bi) {
        GBatch b;
        b.sub = nc + bi;
        b.mode = FKNN_GRAPH_FILTER_SUBTIME;
        b.list = &type0;
        b.K = P.ef0_full;
        b.dists = true;
        B.push_back(std::move(b));
      }
    const size_t n0 = B.size();
    // type 2: SplitInterval (:91-134) with bf_thr 0.5 when sel < 0.2, else 0.2,
    // buckets in t order (:378); per bucket its batches, then its SMALL brute force
    std::vector<size_t> border(r->bks.size());
    for (size_t b = 0; b < border.size(); ++b) border[b] = b;
    std::sort(border.begin(), border.end(), [&](size_t a, size_t c) { return r->bks[a].key < r->bks[c].key; });
    std::vector<size_t> bk_b0, bk_b1, bk_bb;  // per bucket (t order): its range of B, its BB index (or SIZE_MAX)
    if (!type2.empty())
      for (size_t bi : border) {
        const fknn_router::Sub &b = r->bks[bi];
        const float tsb = (float)b.key / 10, teb = (float)(b.key + 1) / 10;
        const float *tb = r->ts_full.data() + b.start;
        std::vector<uint32_t> fl[3], md[3];
        std::vector<float> mdb[3];
        std::vector<int32_t> mdib[3];
        BBatch small;
        small.sub = nc + (uint32_t)bi;
        for (uint32_t i : type2) {
          const float l = metas[(size_t)i * 4 + 2], rr = metas[(size_t)i * 4 + 3], s = sel[i];
          if (rr < tsb || l > teb) continue;
          if (l <= tsb && rr >= teb) {
            fl[s < 0.3f ? 0 : s < 0.6f ? 1 : 2].push_back(i);
            continue;
          }
          const float lb = std::max(tsb, l), rb = std::min(teb, rr);
          const uint32_t s0 = (uint32_t)(std::lower_bound(tb, tb + b.count, lb) - tb);
          const uint32_t e0 = (uint32_t)(std::upper_bound(tb, tb + b.count, rb) - tb);
          const uint32_t np_ = e0 > s0 ? e0 - s0 : 0;
          const float lsel = (float)np_ / (float)b.count;
          const float thr = s < 0.2f ? 0.5f : 0.2f;
          if (lsel < thr) {
            if (np_) {
              small.list.push_back(i);
              small.s.push_back(s0);
              small.cnt.push_back(np_);
            }
          } else {
            const int ki = s > 0.6f ? 0 : s > 0.3f ? 1 : 2;
            md[ki].push_back(i);
            mdb[ki].push_back(l);
            mdb[ki].push_back(rr);
            mdib[ki].push_back((int32_t)s0);
            mdib[ki].push_back((int32_t)(s0 + np_ - 1));
          }
        }
        const uint32_t kfull[3] = {P.ef2_full_small, P.ef2_full_medium, P.ef2_full_large};
        const uint32_t kmed[3] = {P.ef2_medium_large, P.ef2_medium_medium, P.ef2_medium_small};
        bk_b0.push_back(B.size());
        for (int ki = 0; ki < 3; ++ki) {
          S.n_split_full += (uint32_t)fl[ki].size();
          S.n_split_medium += (uint32_t)md[ki].size();
          if (!fl[ki].empty()) {
            lists.push_back(std::move(fl[ki]));
            GBatch g;
            g.sub = nc + (uint32_t)bi;
            g.mode = FKNN_GRAPH_FILTER_SUBTIME;
            g.list = &lists.back();
            g.K = kfull[ki];
            g.dists = true;
            B.push_back(std::move(g));
          }
          if (!md[ki].empty()) {
            lists.push_back(std::move(md[ki]));
            GBatch g;
            g.sub = nc + (uint32_t)bi;
            g.mode = FKNN_GRAPH_RANGE_SUBTIME;
            g.list = &lists.back();
            g.K = kmed[ki];
            g.hb = std::move(mdb[ki]);
            g.hib = std::move(mdib[ki]);
            g.dists = true;
            B.push_back(std::move(g));
          }
        }
        bk_b1.push_back(B.size());
        S.n_split_small += (uint32_t)small.list.size();
        bk_bb.push_back(small.list.empty() ? SIZE_MAX : BB.size());
        if (!small.list.empty()) BB.push_back(std::move(small));
      }
    if ((rc = run_stage(B, BB, true))) return rc;
    S.ms_type0 = lap();
    // the pools, in the reference's order of offers (a query meets a bucket
    // once); the queries split over host threads, each running the whole
    // order for its own range of query ids (the lists are ascending)
    const uint32_t kb = P.bf_refine_k;
    auto merge_range = [&](uint32_t lo, uint32_t hi) {
      auto span = [&](const std::vector<uint32_t> &L, size_t &a, size_t &b) {
        a = (size_t)(std::lower_bound(L.begin(), L.end(), lo) - L.begin());
        b = (size_t)(std::lower_bound(L.begin(), L.end(), hi) - L.begin());
      };
      auto offer_graph = [&](const GBatch &b) {
        const fknn_router::Sub &sub = subs(b.sub);
        size_t a, e;
        span(*b.list, a, e);
        for (size_t j = a; j < e; ++j) {
          fknn::IntPool &pl = pool[(*b.list)[j]];
          if (pl.cap == 0) pl.reset((int)R);
          const size_t o = b.o0 + j * R;
          for (uint32_t t = 0; t < R; ++t) pl.offer(h_ids[o + t] + (int)sub.start, (int)h_d[o + t]);
        }
      };
      for (size_t i2 = 0; i2 < n0; ++i2) offer_graph(B[i2]);
      for (size_t k = 0; k < bk_b0.size(); ++k) {
        for (size_t i2 = bk_b0[k]; i2 < bk_b1[k]; ++i2) offer_graph(B[i2]);
        if (bk_bb[k] == SIZE_MAX) continue;
        // SQ8 distances over the bucket's own codes times alpha^2 (:399-417, bruteforce.h:267)
        const BBatch &b = BB[bk_bb[k]];
        const fknn_router::Sub &sub = subs(b.sub);
        const int8_t *bcodes;
        float ba;
        uint32_t bn;
        graph_codes(sub.g, &bcodes, &ba, &bn);
        size_t a, e;
        span(b.list, a, e);
        for (size_t j = a; j < e; ++j) {
          fknn::IntPool &pl = pool[b.list[j]];
          if (pl.cap == 0) pl.reset((int)R);
          for (uint32_t t = 0; t < kb; ++t) {
            const uint64_t key = h_keys[b.k0 + j * kb + t];
            if (key == ~0ull) break;
            const float dist = (float)(uint32_t)(key >> 32) * ba * ba;
            pl.offer((int)(sub.start + b.s[j] + (uint32_t)key), (int)dist);
          }
        }
      }
    };
    const uint32_t nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (uint32_t t = 1; t < nth; ++t)
      th.emplace_back(merge_range, (uint32_t)((uint64_t)nq * t / nth), (uint32_t)((uint64_t)nq * (t + 1) / nth));
    merge_range(0, (uint32_t)((uint64_t)nq / nth));
    for (std::thread &x : th) x.join();
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
