// Internal definitions shared by the fknn CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <initializer_list>
#include <mutex>
#include <string>
#include <vector>

#include "fknn.h"

namespace fknn {

constexpr int DIM = FKNN_DIM;     // 100, utils.h:255
constexpr int BLK = 64;           // rows per layout block
constexpr int BLK_ROWS_F = DIM + 1;            // 100 dims + the row norm
constexpr int BLK_FLOATS = BLK_ROWS_F * BLK;   // one block: [101][64] float
constexpr uint32_t BLK_BYTES = BLK_FLOATS * 4; // 25856, a multiple of 16
constexpr int TQ = 64;            // queries per contraction tile
constexpr int CAP = 256;          // candidate slots per (work item, query)
constexpr int KMAX_TILE = 128;    // largest k the contraction path serves
constexpr int SMALL_SLAB = 4096;  // slabs up to this size go to the row-by-row exact scan
constexpr int MERGE_CAP = 8192;   // candidates one merge block can hold
constexpr int MAX_ITEMS_PER_TILE = 32;  // so a tile's lists (<= 32 x 192) always fit one merge
constexpr int RESCORE_CAP = 512;  // survivors one merge block can re-score

enum Order : int { ORDER_TIME = 0, ORDER_CAT = 1 };

// ---- order-preserving integer images of floats and ints ----
__host__ __device__ __forceinline__ uint32_t f32_bits(float f) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(f);
#else
  uint32_t u;
  __builtin_memcpy(&u, &f, 4);
  return u;
#endif
}
__host__ __device__ __forceinline__ float bits_f32(uint32_t u) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  __builtin_memcpy(&f, &u, 4);
  return f;
#endif
}
// Monotone map float -> uint32 (total order, -0 < +0; callers canonicalise -0).
__host__ __device__ __forceinline__ uint32_t f32_sortable(float f) {
  uint32_t u = f32_bits(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float sortable_f32(uint32_t s) {
  uint32_t u = (s & 0x80000000u) ? (s & 0x7fffffffu) : ~s;
  return bits_f32(u);
}
__host__ __device__ __forceinline__ uint32_t i32_sortable(int32_t v) { return (uint32_t)v ^ 0x80000000u; }

// Screening error bound.  ds = ||x||^2 + ||q||^2 - 2 q.x, every sum a
// float FMA chain over 100 terms, differs from the exact real distance by at
// most gamma_101 (sqrt(xn)+sqrt(qn))^2 + u|ds|, and the reference's
// sequential float sum (distance.h:62-72) differs from it by at most
// gamma_102 * d.  With sqrt(xn) <= sqrt(d) + sqrt(qn) both are bounded by a
// function of ds and qn alone; the constants below carry a factor > 1.5 of
// slack over gamma_104 = 6.2e-6 (u = 2^-24).
__host__ __device__ __forceinline__ float screen_eps(float ds, float qn) {
  float D = fmaxf(ds, 0.f) * 1.0001f + 1e-4f * qn;
  float a = sqrtf(D) + 2.f * sqrtf(qn);
  return 2e-5f * a * a + 1e-5f * D + 1e-30f;
}
__host__ __device__ __forceinline__ float screen_lo(float ds, float qn) { return ds - screen_eps(ds, qn); }
__host__ __device__ __forceinline__ float screen_hi(float ds, float qn) {
  float h = ds + screen_eps(ds, qn);
  return h + fabsf(h) * 1e-6f + 1e-30f;
}
// Largest ds whose lower bound can still reach T (a safe over-estimate).
__host__ __device__ __forceinline__ float screen_push_limit(float T, float qn) {
  float e = screen_eps(T + 2.f * screen_eps(T, qn), qn);
  return T + e * 1.01f + fabsf(T) * 1e-6f;
}

// Per-query slab after predicate resolution.
struct QueryDesc {
  int32_t order;  // ORDER_TIME or ORDER_CAT
  uint32_t s, e;  // rows [s, e) of that order pass the predicate
  float qn;       // ||q||^2 as a float FMA chain
};

// One contraction work item: rows [blk0*64, blk1*64) of the tile's order.
struct WorkItem {
  uint32_t tile;
  uint32_t blk0, blk1;
  uint32_t pad;
};

struct Tile {
  int32_t order;
  uint32_t item0, item1;  // its work items
  uint32_t nq;
};

struct Candidate {
  float ds;
  uint32_t pos;
};

// Host plan of one search call: which queries take the row-by-row exact
// scan, and the query tiles / row-chunk work items of the contraction.
// Sort key of a query in the plan: (order, cls, bucket, e, s, qi).
struct PlanKey {
  uint32_t order, cls;
  uint64_t bucket;
  uint32_t s, e, qi;
};

struct PlanTile {
  uint32_t first, count, S, E, order;
};

// A search plan.  It lives in its index (or view) and is rebuilt by every
// call; the vectors keep their capacity between calls, so planning touches
// no fresh pages (first-touch faults of multi-MB vectors cost more than the
// planning itself).
struct Plan {
  std::vector<uint32_t> small;                 // query ids for the exact scan
  std::vector<uint32_t> big, big_tile, big_lane;
  std::vector<Tile> tiles;
  std::vector<WorkItem> items;
  std::vector<int32_t> lane_q;
  std::vector<uint32_t> lane_s, lane_e;
  uint64_t pairs_screened = 0, pairs_passing = 0, pairs_contraction = 0;
  // working storage; the sort of each query class has its own
  struct SortScratch {
    std::vector<uint32_t> ix, ix2, cnt;
    std::vector<uint64_t> hi, lo, hi2, lo2;
    std::vector<PlanKey> out;
  };
  SortScratch w_sort[4];
  std::vector<uint32_t> w_big, w_per_tile, w_slot, w_fill;
  std::vector<PlanKey> w_keys, w_keys2;
  std::vector<PlanTile> w_tiles;
  std::vector<WorkItem> w_items;
  void reset() {
    small.clear();
    big.clear();
    big_tile.clear();
    big_lane.clear();
    tiles.clear();
    items.clear();
    lane_q.clear();
    lane_s.clear();
    lane_e.clear();
    pairs_screened = pairs_passing = pairs_contraction = 0;
  }
};

struct PlanShape {
  int tq;                   // queries per tile
  int blk_rows;             // rows per layout block of the order
  uint32_t small_slab;      // slabs up to this size take the exact scan
  uint32_t max_items_per_tile;
  uint32_t min_chunk_blocks;
  uint32_t target_items;    // work items wanted in total (several per resident CTA slot)
};

void make_plan(const QueryDesc *desc, const float *meta_host, uint32_t nq, uint64_t n, const PlanShape &shape,
               Plan &P);

// A search plan built on the device (device_plan.cu), for captured searches:
// the same tiles / work items as Plan, laid out in one device buffer, with
// every count in device memory (cnt).
struct DevPlanSizes {
  uint64_t nb_all = 1;   // start buckets
  uint32_t bw = 1;       // bucket width in rows
  uint32_t ntile_max = 1, nitems_max = 1;
};
struct DevPlan {
  uint32_t nq = 0;
  DevPlanSizes z;
  uint32_t *cnt = nullptr;  // [0] big queries, [1] small, [2] tiles, [3] items, [8..15] 64-bit pair counts
  uint32_t *key_lo = nullptr, *key_hi = nullptr, *vals = nullptr, *ktmp = nullptr, *vtmp = nullptr;
  uint32_t *seg = nullptr, *lane = nullptr, *tflag = nullptr;
  uint32_t *big_q = nullptr, *big_tile = nullptr, *big_lane = nullptr, *small = nullptr;
  uint32_t *tile_first = nullptr, *tS = nullptr, *tE = nullptr, *nblk = nullptr, *chunk = nullptr, *nit = nullptr;
  uint32_t *bsum = nullptr;
  // the work items longest first (ord_val after the sort), for a work queue
  uint32_t *ord_key = nullptr, *ord_val = nullptr, *ord_k2 = nullptr, *ord_v2 = nullptr;
  uint32_t *queue = nullptr;  // two work-queue counters (pilot pass, main pass), cleared by the plan
  Tile *tiles = nullptr;
  WorkItem *items = nullptr;
};
constexpr int DP_NBIG = 0, DP_NSMALL = 1, DP_NTILE = 2, DP_NITEMS = 3;

// Device data of one row order.
struct OrderData {
  float *blocks = nullptr;     // [nblk][101][64]
  uint32_t *perm = nullptr;    // [n] position -> row id
  float *ts = nullptr;         // [n] timestamps in this order
  int32_t *label = nullptr;    // [n] int32 labels in this order
};

// A captured search (BF16 / FP8 with a device plan): replayed while the
// call's shape, pointers and scratch buffers stay the same.
struct GraphCache {
  cudaGraphExec_t exec = nullptr;
  std::vector<uint64_t> key;
  uint32_t launches = 0;   // kernels in the graph
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // screen / merge / scan boundaries
  cudaStream_t cap = nullptr;  // the capture runs here: the caller's stream may be the legacy one
  cudaStream_t side = nullptr;  // a second branch of the graph (the short-slab scans)
  cudaEvent_t fork = nullptr, join = nullptr;
  void release() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    key.clear();
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
    for (auto &e : ev) e = nullptr;
  }
};

// The predicate compaction's persistent state over its sync buffer (ws
// slot 16): the grid barrier counts arrivals on a counter that is never
// reset, and launches tag their failure flag with an epoch, so no launch
// clears anything.
struct FilterState {
  const void *status = nullptr;  // the buffer the state belongs to ...
  size_t bytes = 0;              // ... and its size (a regrown buffer may reuse the address)
  uint32_t epoch = 0;            // the last launch's epoch
  uint64_t arrivals = 0;         // barrier arrivals so far (the counter's value)
  uint32_t grid = 0;             // resident CTAs of the cooperative launch (0: not yet measured)
};

// Grow-only device arena for per-call scratch.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

struct HostBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

}  // namespace fknn

struct fknn_index {
  int device = 0;
  uint64_t n = 0;
  uint32_t nblk = 0;
  float *vecs = nullptr;    // [n][100] row-major, original order
  float *norms = nullptr;   // [n]
  float *labels_f = nullptr;
  float *ts_f = nullptr;
  fknn::OrderData ord[2];
  uint64_t bytes = 0;
  uint64_t hbm_budget = 0;
  // reduced-precision copies (built on request)
  void *bf16_blocks[2] = {nullptr, nullptr};
  void *fp8_blocks[2] = {nullptr, nullptr};
  float *fp8_scale = nullptr;
  // per-call scratch
  std::mutex mu;
  fknn::DevBuf ws[20];
  fknn::HostBuf hs[8];
  int *d_flag = nullptr;
  cudaStream_t own_stream = nullptr;
  // side stream of the short-slab scans, which overlap the host plan
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  fknn::Plan plan;  // rebuilt by every search; capacity kept
  // per-mode plan / kernel parameters (fknn_index_set_tuning) and the SM count
  fknn_tuning tuning[3] = {{0, 16, 16, 0, 0}, {256, 3, 8, 0, 16}, {256, 3, 8, 0, 16}};
  int num_sms = 148;
  uint32_t n_labels = 1;  // distinct category values (bounds a device plan's segments)
  // a view shares the device data of another index and owns only its
  // per-call scratch (ws, hs, d_flag), so views search concurrently
  bool is_view = false;
  // test hook: the next reduced-precision search withholds one row-block copy
  bool test_withhold = false;
  // captured searches (fknn_search_opts.flags & FKNN_SEARCH_CAPTURE)
  fknn::GraphCache graph;
  fknn::FilterState filter_state;
};

namespace fknn {

// error plumbing
void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
#define FKNN_CUDA(call)                                  \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return ::fknn::cuda_fail(_e, #call); \
  } while (0)

// Where a caller's buffer lives, for a call that runs on device dev.  This
// device's memory and managed memory are used in place, host memory is
// staged through a copy, and another GPU's memory is refused: the kernels
// here would read or write it as peer memory, which faults without peer
// access.
enum class MemLoc { Host, Here, Other };
MemLoc mem_loc(const void *p, int dev);
// FKNN_EINVAL (message "<fn>: ... another device") when any non-NULL buffer
// of bufs is another GPU's memory, else FKNN_OK.
int check_local_buffers(const char *fn, int dev, std::initializer_list<const void *> bufs);

int dev_alloc(fknn_index *idx, void **p, size_t bytes);
// index creation around a column builder (capi.cu)
int create_index(uint64_t n, const fknn_index_opts *opts,
                 const std::function<int(fknn_index *, cudaStream_t)> &build, fknn_index **out);
// search views of one index (capi.cu)
int make_index_view(fknn_index *base, fknn_index **out);
void destroy_index(fknn_index *idx);
uint64_t scratch_bytes(const fknn_index *idx);
void trim_scratch(fknn_index *idx);
int ws_get(fknn_index *idx, int slot, size_t bytes, void **p);
int hs_get(fknn_index *idx, int slot, size_t bytes, void **p);

// index build (index_build.cu)
int build_index(fknn_index *idx, const float *vecs, const float *labels, const float *ts, cudaStream_t st);
// the same after the columns (vecs, labels_f, ts_f) are on the device
int alloc_index_columns(fknn_index *idx);
int build_index_from_columns(fknn_index *idx, cudaStream_t st);
int radix_sort_pairs(fknn_index *idx, uint32_t *keys, uint32_t *vals, uint32_t *keys_tmp, uint32_t *vals_tmp,
                     uint64_t n, int begin_bit, int end_bit, cudaStream_t st);

// device-built plans (device_plan.cu)
DevPlanSizes device_plan_sizes(const fknn_index *idx, uint32_t nq, const PlanShape &shape);
size_t device_plan_bytes(uint32_t nq, const DevPlanSizes &z);
void device_plan_layout(DevPlan &P, void *mem, uint32_t nq, const DevPlanSizes &z);
int device_plan_build(fknn_index *idx, const QueryDesc *d_desc, const float *d_meta, DevPlan &P,
                      const PlanShape &shape, cudaStream_t st);

// exact search (exact_search.cu)
int search_exact(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k, uint32_t *d_ids,
                 float *d_dists, cudaStream_t st, fknn_search_stats *stats);
int count_matches(fknn_index *idx, const float *d_meta, uint32_t nq, uint32_t *d_counts, cudaStream_t st);
// graph search (graph_search.cu) without a host round trip: checked
// arguments, device inputs and outputs; the graph's error flag collects
// the searches enqueued since graph_flag_reset
int graph_check_args(const fknn_graph *g, const float *queries, uint32_t nq, int mode, uint32_t k, uint32_t ef,
                     uint32_t refine, const float *bounds, const int32_t *id_bounds, const int32_t *out_ids,
                     uint32_t *cap);
int graph_reserve(fknn_graph *g, uint32_t nq, uint32_t cap);
int graph_launch(fknn_graph *g, const float *d_q, uint32_t nq, int mode, uint32_t k, uint32_t cap, uint32_t refine,
                 const float *d_bounds, const int32_t *d_idb, int32_t *d_ids, float *d_dists, cudaStream_t st);
int graph_flag_reset(fknn_graph *g, cudaStream_t st);
int graph_flag_check(fknn_graph *g);

// predicate compaction (filter.cu): host predicates, device outputs
int filter_check_preds(const float *metas_host, uint32_t np, const char *who);
int filter_rows_batch(fknn_index *idx, const float *metas_host, uint32_t np, uint32_t *d_out, uint64_t *d_counts,
                      cudaStream_t st);
int filter_rows(fknn_index *idx, const float *meta4_host, uint32_t *d_out, uint64_t *count, cudaStream_t st);
int validate_queries(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, cudaStream_t st);
// validation flag cleared and set, and the query descriptors, enqueued only
int enqueue_query_prep(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, QueryDesc *d_desc,
                       cudaStream_t st);
int check_query_flag_value(int flag);
int prepare_queries(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, cudaStream_t st,
                    QueryDesc **d_desc, QueryDesc **h_desc, float **h_meta);
int launch_exact_scan(fknn_index *idx, const uint32_t *list, const uint32_t *d_count, uint32_t h_count, unsigned grid,
                      const QueryDesc *desc, const float *q, uint32_t k, uint32_t *ids, float *dists, cudaStream_t st);
int launch_fill_u32(uint32_t *p, uint32_t n, uint32_t v, cudaStream_t st);
int launch_small_scans(fknn_index *idx, const QueryDesc *h_desc, const QueryDesc *d_desc, uint32_t nq,
                       const float *d_q, uint32_t k, uint32_t *d_ids, float *d_dists, cudaStream_t st,
                       uint32_t *nsmall);
int join_small_scans(fknn_index *idx, cudaStream_t st);

// reduced-precision search (bf16_search.cu)
int build_bf16(fknn_index *idx, cudaStream_t st);
int build_fp8(fknn_index *idx, cudaStream_t st);
int search_fp8(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k, uint32_t kprime,
               uint32_t *d_ids, float *d_dists, cudaStream_t st, fknn_search_stats *stats);
int search_bf16(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k, uint32_t kprime,
                uint32_t *d_ids, float *d_dists, cudaStream_t st, fknn_search_stats *stats);
// the same with the plan built on the device and the whole search one captured CUDA graph
int search_bf16_graph(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k,
                      uint32_t kprime, uint32_t *d_ids, float *d_dists, cudaStream_t st, fknn_search_stats *stats);
int search_fp8_graph(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k,
                     uint32_t kprime, uint32_t *d_ids, float *d_dists, cudaStream_t st, fknn_search_stats *stats);

// FP32 re-rank of device candidate lists, no synchronisation (rerank.cu)
int launch_rerank(fknn_index *idx, const float *d_q, uint32_t nq, const uint32_t *d_cand, uint32_t nc, uint32_t k,
                  uint32_t *d_ids, float *d_dists, int *d_err, cudaStream_t st);

// a graph's device SQ8 codes (n x 112, its own points' order) and alpha (graph_search.cu)
int graph_codes(const fknn_graph *g, const int8_t **codes, float *alpha, uint32_t *n);

// symmetric SQ8 encoding of n x 100 device rows with a given alpha (sq8.cu)
void launch_sq8_encode(const float *d_x, uint64_t n, float alpha, int8_t *d_codes, cudaStream_t st);

// launch counter (kernels launched by this library in the current call)
extern thread_local uint32_t g_launches;

}  // namespace fknn
