/*
 * fknn.h -- C ABI of the B200 filtered k-nearest-neighbour engine.
 *
 * Plain pointers and sizes only.  Every entry point returns an int status
 * (FKNN_OK or a negative FKNN_E* code) and never aborts the process; the
 * text of the last failure on the calling thread is in fknn_last_error().
 *
 * Pointers passed to fknn_search / fknn_sq8_* may be host memory (pageable
 * or pinned) or device memory on the index's device; the library tells them
 * apart with cudaPointerGetAttributes and copies as needed.  Device memory
 * of another GPU is refused with FKNN_EINVAL by every entry point (the
 * SQ8 calls compare with the calling thread's current device).
 *
 * Reference interfaces replaced (paths inside KevinZeng08/sigmod-2024-contest):
 *   fknn_bruteforce_rows   <- Bruteforce(nodes, queries, gt)          utils.h:80
 *   fknn_index_create +
 *   fknn_search(EXACT)     <- the same exact filtered top-k, resident  utils.h:80-158
 *   fknn_search(BF16/FP8)  <- HybridGraph::BatchSearch's brute-force
 *                             + FP32 re-rank leg                       hybrid_graph.cpp:201-229
 *   fknn_sq8_bruteforce    <- bruteforce(dim, k, ...)                  bruteforce.h:244
 *   fknn_sq8_bruteforce_subgraph <- bruteforce_subgraph(...)           bruteforce.h:267
 *   fknn_sq8_sym_train     <- SQ8SymmetricQuantizer::train/encode      pyglass/glass/quant/sq8_sym_quant.hpp:32-74
 *   fknn_graph_create      <- Graph::load + create_searcher + SetData  pyglass/glass/graph.hpp:117-137,
 *                                                                      searcher.hpp:94-101,572-583
 *   fknn_graph_search      <- Searcher::Search / SearchFilter /
 *                             SearchFilterSubTime / SearchCategoryRange /
 *                             SearchRangeFilterSubTime / SearchRangeFilter
 *                                                                      pyglass/glass/searcher.hpp:162-569
 */
#ifndef FKNN_H_
#define FKNN_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FKNN_OK 0
#define FKNN_EINVAL (-1)      /* bad argument: shape, query type, non-finite value, k */
#define FKNN_ENOMEM (-2)      /* device or host allocation failed, or over the HBM budget */
#define FKNN_ECUDA (-3)       /* a CUDA runtime call failed */
#define FKNN_ETIMEOUT (-4)    /* a bounded device wait (about a second) gave up; fknn_search and
                                 fknn_sq8_bruteforce* still return complete results: the queries
                                 it touched were answered again by the exact row scan */
#define FKNN_EUNSUPPORTED (-5) /* mode not built into this index */
#define FKNN_ENODEV (-6)      /* no CUDA device */

/* Search modes. */
#define FKNN_MODE_EXACT_FP32 0 /* ids bit-identical to utils.h:80 Bruteforce */
#define FKNN_MODE_BF16_RERANK 1 /* BF16 tensor-core screen, FP32 re-rank, FP64 boundary fix-up */
#define FKNN_MODE_FP8_RERANK 2  /* FP8-e4m3 per-dimension-scaled screen, same re-rank */

#define FKNN_DIM 100 /* the contest's vector width (utils.h:255 vec_dim) */

typedef struct fknn_index fknn_index;

typedef struct fknn_index_opts {
  int device;           /* CUDA device ordinal */
  int build_bf16;       /* keep BF16 copies for FKNN_MODE_BF16_RERANK */
  int build_fp8;        /* keep FP8-e4m3 per-dim codes for FKNN_MODE_FP8_RERANK */
  uint64_t hbm_budget;  /* bytes the index may hold on the device; 0 = no limit */
} fknn_index_opts;

/* Plan and kernel parameters of one search mode, per index (the autotuner
 * in fknn/autotune.py picks them per device, base size and mode). */
typedef struct fknn_tuning {
  uint32_t list_slack;       /* BF16/FP8: candidate-list room beyond k' between trims, rows (>= 256) */
  uint32_t items_per_sm;     /* contraction work items per SM: load balance against candidate traffic */
  uint32_t min_chunk_blocks; /* shortest row chunk of a work item, in row blocks (64 rows exact, 128 BF16/FP8) */
  uint32_t bound_refresh;    /* BF16/FP8: sub-tiles between reloads of the shared per-query bound (0 = at trims) */
  uint32_t pilot_stride;     /* a pilot pass over every pilot_stride-th row block first seeds the bounds
                                (0 or 1 = no pilot).  BF16/FP8: an estimate of the k'-th, checked by the
                                merge; exact: the k-th of the sample, a valid upper bound */
} fknn_tuning;

/* fknn_search_opts.flags */
#define FKNN_SEARCH_GRAPH 1u /* reduced-precision modes: plan on the device and replay a captured CUDA graph */

typedef struct fknn_search_opts {
  int mode;             /* FKNN_MODE_* */
  uint32_t kprime;      /* candidate width for the reduced-precision modes (0 = default 400) */
  uint32_t flags;       /* FKNN_SEARCH_* bits, 0 = host-planned search.  FKNN_SEARCH_GRAPH:
                         * the query grouping, tile and work-item plan are built by
                         * kernels, every launch has a size fixed by (nq, index), and
                         * the whole search is captured once into a CUDA graph that
                         * later calls with the same nq, k, kprime, tuning and buffer
                         * addresses replay (one graph launch + one flag read-back).
                         * Results equal the host-planned search's up to the order of
                         * equal-distance candidates.  Exact mode ignores the flag. */
} fknn_search_opts;

/* Per-call statistics (optional out-parameter of fknn_search_ex). */
typedef struct fknn_search_stats {
  uint64_t pairs_screened;     /* (query, row) pairs the screening contraction evaluated, masked ones included */
  uint64_t pairs_passing;      /* pairs that pass the predicate (sum of slab sizes), all queries */
  uint64_t pairs_contraction;  /* passing pairs of the queries the contraction served */
  uint32_t n_tiles;            /* query tiles of the contraction */
  uint32_t n_work_items;       /* (tile, row chunk) work items */
  uint32_t n_small;            /* queries routed to the row-by-row exact scan */
  uint32_t n_overflow;         /* queries re-run by the exact scan after a candidate overflow */
  uint32_t n_boundary_f64;     /* candidates recomputed in FP64 at the k-th boundary */
  uint32_t kernel_launches;    /* kernels this call launched */
  float ms_plan;               /* host planning time */
  float ms_screen;             /* device time of the screening contraction (CUDA events, launching stream) */
  float ms_merge;              /* device time of the merge + exact re-score */
  float ms_scan;               /* device time of the row-by-row exact scans */
} fknn_search_stats;

/* Library version (major*10000 + minor*100 + patch). */
int fknn_version(void);

/* Text of the last failure on this thread ("" if none). */
const char *fknn_last_error(void);

/* Builds a resident index on opts->device from SoA columns in host memory:
 * vecs n x dim float32 (dim must be 100), labels n float32 (category, read
 * as int32 like utils.h:109), ts n float32 (timestamp).  Values must be
 * finite; |label| < 2^31; |vec| <= 1e15.  Rows keep their position as id. */
int fknn_index_create(const float *vecs, const float *labels, const float *ts, uint64_t n,
                      uint32_t dim, const fknn_index_opts *opts, fknn_index **out);

/* Builds a resident index straight from a contest base file (u32 N, then N
 * rows [label, ts, 100 floats], as ReadBase reads it, utils.h:257-276):
 * the rows stream through pinned buffers to the device, a kernel splits
 * them into the columns, and the row orders that ReadSortedBaseTimestamp
 * builds with host sorts (utils.h:352-479) are radix-sorted on the GPU.
 * Row position in the file is the id. */
int fknn_index_create_from_file(const char *path, const fknn_index_opts *opts, fknn_index **out);

int fknn_index_destroy(fknn_index *index);

/* ---- Contest file formats ----
 * fknn_read_base_file   <- ReadBase          utils.h:257-276: *n rows; vecs n x 100, labels n, ts n
 *                          (all three NULL: only *n is set)
 * fknn_read_query_file  <- ReadQuery         utils.h:550-566: *nq rows; qvecs nq x 100, metas nq x 4
 *                          (both NULL: only *nq is set)
 * fknn_sorted_query_order <- the order ReadSortedQuery sorts queries into, utils.h:513-533:
 *                          ascending (uint32 type, int32 v, l, r); equal keys keep their order
 * fknn_save_knn         <- SaveKNN           io.h:22-33: nq x k uint32, no header
 * fknn_read_groundtruth <- ReadGroundTruth   utils.h:194-221: u32 nq header, then nq x k uint32
 *                          (ids NULL: only *nq is set)
 * A file shorter than its header says is rejected with FKNN_EINVAL. */
int fknn_read_base_file(const char *path, uint64_t *n, float *vecs, float *labels, float *ts);
int fknn_read_query_file(const char *path, uint32_t *nq, float *qvecs, float *metas);
int fknn_sorted_query_order(const float *metas, uint32_t nq, uint32_t *sorted_ids);
int fknn_save_knn(const char *path, const uint32_t *ids, uint32_t nq, uint32_t k);
int fknn_read_groundtruth(const char *path, uint32_t k, uint32_t *nq, uint32_t *ids);

/* Device bytes held by the index. */
int fknn_index_bytes(const fknn_index *index, uint64_t *bytes);

/* Filtered top-k for nq queries.
 *   qvecs : nq x 100 float32
 *   metas : nq x 4 float32 (type, v, l, r) -- the contest query header
 *           (utils.h:98-101); type 0 none, 1 label==v, 2 l<=ts<=r, 3 both.
 *   ids   : nq x k uint32, ascending (distance, id); UINT32_MAX padding
 *           when fewer than k rows pass.
 *   dists : nq x k float32 or NULL; +inf padding.
 *   stream: cudaStream_t or NULL (the legacy default stream).
 * Returns when the results are in ids/dists (host or device). */
int fknn_search(fknn_index *index, const float *qvecs, const float *metas, uint32_t nq, uint32_t k,
                int mode, uint32_t *ids, float *dists, void *stream);

/* Sets / reads the tuning of one search mode (FKNN_MODE_*) of an index.
 * Zero list_slack / items_per_sm / min_chunk_blocks keep their current
 * value; bound_refresh and pilot_stride are always taken.  Exact-mode results do not depend
 * on the tuning; reduced-precision results depend on it only through which
 * equal-screening-distance candidates are kept. */
int fknn_index_set_tuning(fknn_index *index, int mode, const fknn_tuning *t);
int fknn_index_get_tuning(const fknn_index *index, int mode, fknn_tuning *t);

/* Test hook for the failure path (no reference counterpart): the next
 * BF16 / FP8 search on the index issues no row-block copy for its first
 * work item, so that item's bounded device waits run out after about a
 * second; the search returns FKNN_ETIMEOUT with complete results, and the
 * hook is off again for the search after it. */
int fknn_index_test_withhold_copy(fknn_index *index);

/* As fknn_search with options and statistics (stats may be NULL). */
int fknn_search_ex(fknn_index *index, const float *qvecs, const float *metas, uint32_t nq, uint32_t k,
                   const fknn_search_opts *opts, uint32_t *ids, float *dists, void *stream,
                   fknn_search_stats *stats);

/* Number of rows passing each query's predicate (the selectivity numerator of
 * hybrid_graph.cpp:168-200), from the index's sorted attribute columns. */
int fknn_count_matches(fknn_index *index, const float *metas, uint32_t nq, uint32_t *counts, void *stream);

/* Predicate evaluation + row compaction over the attribute columns for ONE
 * predicate (type, v, l, r): writes the ids of passing rows in increasing
 * order into out_ids (capacity n) and their number into *count. */
int fknn_filter_rows(fknn_index *index, const float *meta4, uint32_t *out_ids, uint64_t *count, void *stream);

/* As fknn_filter_rows for np predicates at once (metas np x 4 float32, host
 * memory), asynchronous: the columns are read once for up to 16 predicates
 * per pass, row p of out_ids (DEVICE memory, np x n uint32, row stride n)
 * receives predicate p's passing ids in increasing order and counts[p]
 * (DEVICE memory, np uint64) their number.  Nothing is read back; results
 * are complete when `stream` reaches the point of the call.  A count of
 * UINT64_MAX means the kernel's bounded wait gave up (its ids are then
 * incomplete); it does not happen in normal operation.  Calls on one index
 * share its scratch and continue its grid-barrier counter: issue them on
 * one stream, and do not capture them into a CUDA graph (each launch's
 * barrier target and epoch are set on the host).  One cooperative launch
 * per 16 predicates: it starts when all its CTAs (two per SM) fit. */
int fknn_filter_rows_batch(fknn_index *index, const float *metas, uint32_t np, uint32_t *out_ids,
                           uint64_t *counts, void *stream);

/* No counterpart in the reference: the predicate evaluation + row compaction
 * of fknn_filter_rows for callers that cannot allocate device memory -- code
 * that runs under a fixed, pre-reserved HBM budget or a foreign memory pool
 * where cudaMalloc is refused, and latency-critical paths where cudaMalloc's
 * implicit device synchronisation is not acceptable.  It allocates nothing:
 * no cudaMalloc, no cudaFree, no pinned staging, no index.
 *   labels, ts : n float32 each, DEVICE memory of the current device, in the
 *                caller's row order (the ids written are positions in them)
 *   meta4      : HOST pointer to one predicate (type, v, l, r)
 *   out_ids    : DEVICE memory of capacity n; passing row ids, increasing
 *   count      : HOST pointer; receives the number of passing rows
 * Limit: n <= 268,435,456 (65,536 tiles of 4,096 rows); larger n returns
 * FKNN_EINVAL.  The per-tile counters live in one fixed 256 KiB device array
 * that every GPU loading this library holds until the process exits; every
 * call shares it and it keeps the last call's contents (each call rewrites
 * all counters it reads).  Calls that overlap on the GPU (other streams,
 * other host threads, same device) race on that array: serialise them.  The
 * first call on a device looks up the array's device address (set-up once
 * per device).  Every call waits for its stream before returning (the count
 * is read back into host memory), so it cannot be issued on a stream that is
 * being captured into a CUDA graph. */
int fknn_filter_rows_noalloc(const float *labels, const float *ts, uint64_t n, const float *meta4,
                             uint32_t *out_ids, uint64_t *count, void *stream);

/* Drop-in for utils.h:80 Bruteforce on contest-layout rows: nodes n x 102
 * (label, ts, 100 dims), queries nq x 104 (type, v, l, r, 100 dims), gt
 * nq x 100 ascending (distance, id).  Builds a temporary index on device 0. */
int fknn_bruteforce_rows(const float *nodes, uint32_t n, const float *queries, uint32_t nq, uint32_t *gt);

/* Symmetric SQ8 (sq8_sym_quant.hpp:32-74): alpha = max|x| over n x 100
 * vectors; codes n x 112 int8 = round(clamp(x/alpha,-1,1)*127), zero-padded. */
int fknn_sq8_sym_train(const float *vecs, uint64_t n, float *alpha, int8_t *codes);
/* Encodes with a given alpha (sq8_sym_quant.hpp:63-74). */
int fknn_sq8_sym_encode(const float *vecs, uint64_t n, float alpha, int8_t *codes);

/* Drop-in for bruteforce (bruteforce.h:244).  Same arguments; codes_in is a
 * slab of npoints x 112 int8 codes, queries_in nqueries x 112 int8.  Unlike
 * the reference, nqueries is honoured: closest_points is nqueries x k, each
 * row in the reference's heap-array order.  dim and alpha are ignored, as in
 * the reference.  Requires 1 <= k <= 2048 and k <= npoints < 2^31.  Pointers
 * may be host or device memory (device codes and queries 16-byte aligned are
 * read in place, after the work queued on the legacy default stream; work
 * that produced them on a non-blocking stream or a per-thread default stream
 * must be synchronised by the caller first).  The call is synchronous and
 * reentrant: each calling host thread has its own device scratch and stream,
 * kept between calls and only grown.  That scratch holds about
 * npoints x 132 bytes (plus npoints x 112 when the codes are host memory)
 * and npoints x k / 512 bytes per query of a pass (up to 8,192 queries), so
 * it scales with the number of calling threads; release it with
 * fknn_sq8_release_thread_scratch. */
int fknn_sq8_bruteforce(size_t dim, size_t k, int *closest_points, size_t npoints, const char *codes_in,
                        float alpha, size_t nqueries, const int8_t *queries_in);

/* Drop-in for bruteforce_subgraph (bruteforce.h:267): also writes
 * distances[k] = heap distance * alpha * alpha. */
int fknn_sq8_bruteforce_subgraph(size_t dim, size_t k, int *closest_points, float *distances, size_t npoints,
                                 const char *codes_in, float alpha, size_t nqueries, const int8_t *queries_in);

/* Frees the calling thread's SQ8 brute-force scratch (device memory, stream
 * and event; no reference counterpart: the reference holds no device
 * state).  The next call on the thread sets them up again. */
int fknn_sq8_release_thread_scratch(void);

/* FP32 re-rank of candidate lists (hybrid_graph.cpp:216-228, 284-296,
 * 481-492: approximate candidates re-scored in FP32, the k best kept).
 * cand is nq x nc ids of index rows in the caller's original numbering
 * (UINT32_MAX = empty slot; repeats allowed); per query the k smallest
 * exact distances (normal_l2 arithmetic, distance.h:62-72) are written
 * ascending by (distance, id), padded with UINT32_MAX / +inf.  The
 * reference keeps them in heap-array order; the set is the same.  Requires
 * 1 <= k <= nc <= 2048. */
int fknn_rerank(fknn_index *index, const float *qvecs, uint32_t nq, const uint32_t *cand, uint32_t nc, uint32_t k,
                uint32_t *ids, float *dists, void *stream);

/* ---- Graph beam search (pyglass Searcher over an HNSW level-0 graph) ---- */

/* Search forms, numbered as the reference's Searcher methods. */
#define FKNN_GRAPH_SEARCH 0            /* Search(q, k, dst)                         searcher.hpp:162 */
#define FKNN_GRAPH_FILTER 1            /* SearchFilter(q, k, refine, dst, f)         searcher.hpp:262 */
#define FKNN_GRAPH_FILTER_SUBTIME 2    /* SearchFilterSubTime (+ dists)              searcher.hpp:377 */
#define FKNN_GRAPH_CATEGORY_RANGE 3    /* SearchCategoryRange (bounds, id_bounds)    searcher.hpp:301 */
#define FKNN_GRAPH_RANGE_SUBTIME 4     /* SearchRangeFilterSubTime (+ dists)         searcher.hpp:415 */
#define FKNN_GRAPH_RANGE 5             /* SearchRangeFilter                          searcher.hpp:493 */

typedef struct fknn_graph fknn_graph;

/* Loads a graph from the bytes Graph::save writes (graph.hpp:101-115: nep,
 * eps, N, K, N x K neighbour ids with -1 padding, N x K edge timestamps, and
 * optionally the HNSW upper layers, HNSWInitializer.hpp:73-82) and trains
 * the searcher's symmetric SQ8 codes on vecs (N x 100 host or device
 * floats, the graph's own points), as Searcher::SetData does.  The graph
 * lives on `device`. */
int fknn_graph_create(const void *graph_bytes, size_t nbytes, const float *vecs, int device, fknn_graph **out);
int fknn_graph_destroy(fknn_graph *g);
/* n = points, degree = K of the level-0 graph, alpha = the SQ8 scale. */
int fknn_graph_info(const fknn_graph *g, uint32_t *n, uint32_t *degree, float *alpha);

/* nq searches of the Searcher form `mode`, one per query, with the
 * reference's pool (capacity max(k, ef); ef = 0 means the reference's 32),
 * visiting order and tie rules, so ids equal the reference's on the same
 * graph.  queries nq x 100; out_ids nq x refine (pool slots 0..refine-1,
 * as reorder writes them); out_dists nq x refine (slot distance x alpha^2,
 * as reorder_dist writes them; may be NULL).  bounds (nq x 2 floats, the
 * timestamp window [l, r]) and id_bounds (nq x 2 ints, the range whose ten
 * evenly spaced ids seed the pool) are read by modes 3-5 and may be NULL
 * otherwise.  Mode 0 writes k ids (refine must equal k).  Requires
 * 1 <= k <= 4096 and 1 <= refine <= max(k, ef) + 1.  Pointers may be host or
 * device memory; the call waits for `stream`.  A graph handle serves one
 * call at a time. */
int fknn_graph_search(fknn_graph *g, const float *queries, uint32_t nq, int mode, uint32_t k, uint32_t ef,
                      uint32_t refine, const float *bounds, const int32_t *id_bounds, int32_t *out_ids,
                      float *out_dists, void *stream);

/* ---- Reference-equivalent routing of HybridGraph::BatchSearch ----
 *
 * The reference answers its batch through a planner (hybrid_graph.cpp:
 * 147-503): per query the selectivity sel = matches / sel_rows picks a
 * route -- an SQ8 brute force over the query's slab (sel < bf_thr, or type 3
 * and sel < bf_thr3), the category's graph (types 1 and 3, SearchFilter /
 * SearchCategoryRange with a pool growing with the category's size), the
 * ten time-bucket graphs (type 0, SearchFilterSubTime on each), or the
 * buckets a window overlaps (type 2, SplitInterval: FULL / MEDIUM graph
 * searches, SMALL brute force) -- and every route ends in an FP32 re-rank
 * to the top 100.  fknn_router runs the same routes with the same
 * thresholds, pools and merge rules on the GPU, over the reference's own
 * subgraphs (Graph::save bytes) and base orders, so its recall can be
 * compared with the reference pipeline's; the exact and BF16 forms of
 * fknn_search need none of it. */
typedef struct fknn_router fknn_router;

typedef struct fknn_router_subgraph {
  int32_t key;             /* category value, or time bucket t (timestamps in [t/10, (t+1)/10]) */
  uint32_t start, count;   /* its rows: positions start .. start+count-1 of its base order */
  const void *graph_bytes; /* Graph::save bytes of its graph (graph.hpp:101-115) */
  size_t nbytes;
} fknn_router_subgraph;

typedef struct fknn_router_desc {
  const float *vecs, *labels, *ts;           /* n x 100, n, n host floats, original row order (ids) */
  uint64_t n;
  const uint32_t *sorted_base_ids;           /* n: category order (label, ts) -> id   (utils.h:395-425) */
  const uint32_t *sorted_base_ids_by_full_time; /* n: timestamp order -> id            (utils.h:420-425) */
  const fknn_router_subgraph *categories;    /* graphs of the categories with their own (hybrid_graph.cpp:52-75) */
  uint32_t ncategories;
  const fknn_router_subgraph *buckets;       /* time-bucket graphs, in the order type 0 visits them
                                                (hybrid_graph.cpp:303) */
  uint32_t nbuckets;
  uint32_t maxc_size, minc_size;             /* largest / smallest category size (utils.h:375-385) */
  int device;
} fknn_router_desc;

/* SearchParams (hybrid_graph.h:14-34) and HybridGraph's thresholds
 * (hybrid_graph.h:70-77, baseline.cpp:77-78); fknn_router_default_params
 * fills the reference's values. */
typedef struct fknn_router_params {
  uint32_t ef0_full, ef1min, ef1max, ef3min, ef3max;
  uint32_t ef2_full_large, ef2_full_medium, ef2_full_small;
  uint32_t ef2_medium_large, ef2_medium_medium, ef2_medium_small;
  float bf_thr, bf_thr3;
  uint32_t bf_refine_k;      /* SQ8 brute-force candidates (140) */
  uint32_t graph_refine_k;   /* graph candidates and merged pool size (150) */
  uint32_t sel_rows;         /* selectivity denominator: the reference's 10,000,000 (hybrid_graph.cpp:151) */
} fknn_router_params;

typedef struct fknn_router_stats {
  uint32_t n_bruteforce, n_category, n_type0, n_type2;  /* queries per route */
  uint32_t n_graph_calls, n_split_small, n_split_medium, n_split_full;
  float ms_total;            /* wall time of the call */
  /* wall time of each stage (each ends with its results on the host or in
   * the output): query upload + slabs, SQ8 brute force + re-rank, category
   * graphs + re-rank, the type-0 and type-2 bucket searches (all sub-graphs
   * side by side), their pool merge on the host, pooled re-rank + copy-out */
  float ms_prepare, ms_bruteforce, ms_category, ms_type0, ms_type2, ms_final;
} fknn_router_stats;

int fknn_router_default_params(fknn_router_params *p);
int fknn_router_create(const fknn_router_desc *desc, fknn_router **out);
/* qvecs nq x 100 and metas nq x 4 (type, v, l, r) host floats; ids nq x 100
 * host, ascending by FP32 distance, UINT32_MAX where a route found fewer
 * rows.  params NULL = the reference's.  stats may be NULL. */
int fknn_router_search(fknn_router *r, const float *qvecs, const float *metas, uint32_t nq,
                       const fknn_router_params *params, uint32_t *ids, fknn_router_stats *stats);
int fknn_router_destroy(fknn_router *r);

/* ---- Request loop (continuous batching over one resident index) ----
 *
 * No reference counterpart: the reference answers one offline batch
 * (baseline.cpp:150 -> HybridGraph::BatchSearch).  Requests (one query
 * each) are queued per query type; whenever one of `slots` search slots is
 * free, the oldest type's waiting requests -- up to max_batch -- are
 * searched together on that slot's stream while the other slots' batches
 * run.  A batch starts only while the device scratch the slots hold fits in
 * hbm_budget; a batch that runs over it releases its slot's scratch and
 * lowers the batch size for its query type.  Each result equals what
 * fknn_search returns for that query alone. */

typedef struct fknn_server fknn_server;

typedef struct fknn_server_opts {
  int mode;              /* FKNN_MODE_* for every request */
  uint32_t kprime;       /* candidate width of the reduced-precision modes (0 = default) */
  uint32_t k;            /* neighbours per request, <= 128 (0 = 100) */
  uint32_t max_batch;    /* queries per batch (0 = 4096) */
  uint32_t slots;        /* batches in flight (0 = 3, max 16) */
  uint32_t max_wait_us;  /* a partial batch may wait this long for more requests while other
                            slots keep the device busy (0 = dispatch at once) */
  uint64_t hbm_budget;   /* device bytes the slots' scratch may hold (0 = half the free HBM) */
} fknn_server_opts;

typedef struct fknn_server_stats {
  uint64_t submitted, completed, failed, batches;
  uint64_t admission_waits; /* times a free slot waited because the held scratch exceeded the budget */
  uint64_t budget_trims;    /* batches that ran over the budget (their slot released its scratch and
                               the type's batch size was lowered) */
  uint64_t scratch_bytes;   /* device bytes held by the slots' scratch */
  uint64_t budget_bytes;
  uint32_t max_batch_seen;
  float mean_batch;
  float p50_ms, p99_ms, max_ms, mean_ms; /* arrival -> result, requests completed since the last reset */
  double span_s;            /* first arrival -> last result of those requests */
  double qps;               /* their count / span_s */
} fknn_server_stats;

/* The index must outlive the server.  The server holds one search view of
 * the index per slot; direct fknn_search calls on the index stay valid. */
int fknn_server_create(fknn_index *index, const fknn_server_opts *opts, fknn_server **out);
/* The clock arrival stamps are read against (steady, nanoseconds). */
int64_t fknn_server_now_ns(void);
/* Enqueues nreq requests: qvecs nreq x 100 and metas nreq x 4 (type, v, l,
 * r) host memory, copied before returning; arrival_ns (nullable = now) the
 * time each request arrived, from which its latency counts.  ids (nreq x k)
 * and dists (nullable, nreq x k) are host memory written when each request
 * completes and must stay valid until then.  Tickets are first_ticket ..
 * first_ticket + nreq - 1.  A request that fails validation rejects the call
 * (nothing is enqueued). */
int fknn_server_submit(fknn_server *s, const float *qvecs, const float *metas, uint32_t nreq,
                       const int64_t *arrival_ns, uint32_t *ids, float *dists, uint64_t *first_ticket);
/* Waits for one request (timeout_ms < 0: forever); returns its status. */
int fknn_server_wait(fknn_server *s, uint64_t ticket, int timeout_ms);
/* Waits for every submitted request; returns the first failure's status. */
int fknn_server_drain(fknn_server *s, int timeout_ms);
int fknn_server_get_stats(fknn_server *s, fknn_server_stats *out, int reset);
/* Drains, then stops the threads and frees the slots. */
int fknn_server_destroy(fknn_server *s);

#ifdef __cplusplus
}
#endif

#endif /* FKNN_H_ */
