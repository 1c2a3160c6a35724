// Search plan built on the device, so a whole search is a fixed sequence of
// launches (no host round trip, grids that do not depend on the data) that
// can be captured into one CUDA graph and replayed.
//
// It makes the same kind of plan as make_plan (exact_search.cu), from the
// query slabs k_query_prep leaves in device memory:
//   1. k_dp_keys     per query: slabs of at most small_slab rows go to the
//                    row-by-row scan list; the others get a sort key
//                    (order, class, start bucket | end)
//   2. two stable LSD radix sorts (low word, then high word) order them
//   3. k_dp_segments a segment starts where (order, class, bucket) changes,
//                    or for category predicates where the slab changes; a
//                    max-scan gives every position its segment start
//   4. k_dp_lanes    tiles are runs of up to `tq` consecutive queries of one
//                    segment; a sum-scan numbers them
//   5. k_dp_tiles    per tile: first position, query count, row range
//   6. k_dp_chunk    the row-chunk length that gives every resident CTA
//                    slot several work items (as make_plan's)
//   7. k_dp_items    per tile its work items, numbered by a sum-scan
// The greedy tile closing of make_plan (a tile ends when its union range
// grows by a third) becomes the segment rule here: within a segment the
// slabs already overlap (same category slab, or starts within one bucket
// and ends sorted), so consecutive queries pack without it.
#include <algorithm>
#include <cmath>

#include "device_util.cuh"

namespace fknn {

namespace {

constexpr int DP_THREADS = 256;
constexpr int SC_ITEMS = 16;
constexpr int SC_TILE = DP_THREADS * SC_ITEMS;  // elements per scan block

unsigned grid_for(uint64_t work, int threads = DP_THREADS) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((work + threads - 1) / threads, 148 * 32));
}

// ---- multi-block inclusive scan (sum or max) of n u32 values in place ----

struct OpSum {
  __device__ __forceinline__ static uint32_t id() { return 0u; }
  __device__ __forceinline__ static uint32_t op(uint32_t a, uint32_t b) { return a + b; }
};
struct OpMax {
  __device__ __forceinline__ static uint32_t id() { return 0u; }
  __device__ __forceinline__ static uint32_t op(uint32_t a, uint32_t b) { return a > b ? a : b; }
};

template <class Op>
__device__ __forceinline__ uint32_t warp_incl(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t x = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = Op::op(v, x);
  }
  return v;
}

// Block-exclusive scan of one value per thread (all threads of the block,
// a multiple of 32, at most 1024); *total = the block's combination.
template <class Op>
__device__ __forceinline__ uint32_t block_excl(uint32_t v, uint32_t *ws, uint32_t *total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t inc = warp_incl<Op>(v);
  uint32_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) ex = Op::id();
  if (lane == 31) ws[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint32_t x = lane < nw ? ws[lane] : Op::id();
    x = warp_incl<Op>(x);
    ws[lane] = x;
  }
  __syncthreads();
  const uint32_t before = w ? ws[w - 1] : Op::id();
  *total = ws[nw - 1];
  __syncthreads();
  return Op::op(before, ex);
}

// pass 1: each block scans SC_TILE elements in place; bsum[b] = its total
template <class Op>
__global__ void __launch_bounds__(DP_THREADS) k_scan_tiles(uint32_t *__restrict__ data, uint64_t n,
                                                         uint32_t *__restrict__ bsum) {
  __shared__ uint32_t ws[32];
  const uint64_t base = (uint64_t)blockIdx.x * SC_TILE + (uint64_t)threadIdx.x * SC_ITEMS;
  uint32_t v[SC_ITEMS];
  uint32_t acc = Op::id();
#pragma unroll
  for (int i = 0; i < SC_ITEMS; ++i) {
    acc = Op::op(acc, base + i < n ? data[base + i] : Op::id());
    v[i] = acc;
  }
  uint32_t total;
  const uint32_t ex = block_excl<Op>(acc, ws, &total);
#pragma unroll
  for (int i = 0; i < SC_ITEMS; ++i)
    if (base + i < n) data[base + i] = Op::op(ex, v[i]);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// pass 2: one block, exclusive scan of the block totals in place
template <class Op>
__global__ void __launch_bounds__(1024) k_scan_top(uint32_t *__restrict__ bsum, uint32_t nb) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = Op::id();
  __syncthreads();
  for (uint32_t b0 = 0; b0 < nb; b0 += blockDim.x) {
    const uint32_t i = b0 + threadIdx.x;
    const uint32_t v = i < nb ? bsum[i] : Op::id();
    uint32_t total;
    const uint32_t ex = block_excl<Op>(v, ws, &total);
    const uint32_t c = carry;
    if (i < nb) bsum[i] = Op::op(c, ex);
    __syncthreads();
    if (threadIdx.x == 0) carry = Op::op(c, total);
    __syncthreads();
  }
}

// pass 3: every element combined with the prefix of the blocks before it
template <class Op>
__global__ void k_scan_add(uint32_t *__restrict__ data, uint64_t n, const uint32_t *__restrict__ bsum) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t b = (uint32_t)(i / SC_TILE);
    if (b) data[i] = Op::op(bsum[b], data[i]);
  }
}

template <class Op>
void scan_incl(uint32_t *data, uint64_t n, uint32_t *bsum, cudaStream_t st) {
  const uint32_t nb = (uint32_t)((n + SC_TILE - 1) / SC_TILE);
  k_scan_tiles<Op><<<nb, DP_THREADS, 0, st>>>(data, n, bsum);
  k_scan_top<Op><<<1, 1024, 0, st>>>(bsum, nb);
  k_scan_add<Op><<<grid_for(n), DP_THREADS, 0, st>>>(data, n, bsum);
  g_launches += 3;
}

// ---- plan kernels ----

enum : int { C_NBIG = 0, C_NSMALL = 1, C_NTILE = 2, C_NITEMS = 3, C_CB = 4, C_TOTBLK = 8, C_PAIRS_SCR = 10,
             C_PAIRS_PASS = 12, C_PAIRS_CONTR = 14 };

__device__ __forceinline__ void add_u64(uint32_t *c, uint64_t v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(c), (unsigned long long)v);
}

__global__ void k_dp_keys(const QueryDesc *__restrict__ desc, const float *__restrict__ meta, uint32_t nq,
                          uint32_t bw, uint32_t small_slab, uint32_t *__restrict__ key_lo,
                          uint32_t *__restrict__ key_hi, uint32_t *__restrict__ vals, uint32_t *__restrict__ small,
                          uint32_t *__restrict__ cnt) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
    const QueryDesc d = desc[i];
    const uint32_t len = d.e - d.s;
    add_u64(cnt + C_PAIRS_PASS, len);
    vals[i] = i;
    if (len <= small_slab) {
      small[atomicAdd(cnt + C_NSMALL, 1u)] = i;
      key_hi[i] = 0xffffffffu;
      key_lo[i] = 0xffffffffu;
    } else {
      atomicAdd(cnt + C_NBIG, 1u);
      add_u64(cnt + C_PAIRS_CONTR, len);
      // an invalid type is reported by k_validate_queries; clamped here so the
      // key stays inside its two bits and the segment bound holds
      const uint32_t cls = min((uint32_t)meta[(uint64_t)i * 4], 3u);
      const uint32_t bucket = (cls == 2 || cls == 3) ? min(d.s / bw, 0x1fffffffu) : 0u;
      key_hi[i] = ((uint32_t)d.order << 31) | (cls << 29) | bucket;
      key_lo[i] = d.e;
    }
  }
}

__global__ void k_gather_u32(const uint32_t *__restrict__ src, const uint32_t *__restrict__ idx, uint32_t n,
                             uint32_t *__restrict__ dst) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

// seg[i] = i where a segment starts, else 0 (max-scanned next into the start)
__global__ void k_dp_segments(const uint32_t *__restrict__ key_hi, const uint32_t *__restrict__ vals,
                              const QueryDesc *__restrict__ desc, uint32_t nq, const uint32_t *__restrict__ cnt,
                              uint32_t *__restrict__ seg) {
  const uint32_t nbig = cnt[C_NBIG];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
    uint32_t v = 0;
    if (i < nbig) {
      bool start = i == 0 || key_hi[i] != key_hi[i - 1];
      if (!start && ((key_hi[i] >> 29) & 3u) == 1u) start = desc[vals[i]].e != desc[vals[i - 1]].e;
      v = start ? i : 0u;
    }
    seg[i] = v;
  }
}

// lane of every big query inside its tile, and the tile-start flags (sum-scanned next)
__global__ void k_dp_lanes(const uint32_t *__restrict__ seg, uint32_t nq, uint32_t tq,
                           const uint32_t *__restrict__ cnt, uint32_t *__restrict__ lane,
                           uint32_t *__restrict__ tflag) {
  const uint32_t nbig = cnt[C_NBIG];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
    const uint32_t l = i < nbig ? (i - seg[i]) % tq : 0u;
    lane[i] = l;
    tflag[i] = (i < nbig && l == 0) ? 1u : 0u;
  }
}

__global__ void k_dp_tile_init(Tile *__restrict__ tiles, uint32_t *__restrict__ ts_, uint32_t *__restrict__ te_,
                               uint32_t ntile_max, uint32_t *__restrict__ ord_key, uint32_t nitems_max) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntile_max; t += gridDim.x * blockDim.x) {
    tiles[t] = Tile{0, 0, 0, 0};
    ts_[t] = 0xffffffffu;
    te_[t] = 0u;
  }
  // item slots past the item count sort last
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nitems_max; i += gridDim.x * blockDim.x)
    ord_key[i] = 0xffffffffu;
}

// per big query: its tile's first position, count, row range and order;
// the merge's per-query arrays; the tile count
__global__ void k_dp_tiles(const uint32_t *__restrict__ vals, const uint32_t *__restrict__ key_hi,
                           const QueryDesc *__restrict__ desc, const uint32_t *__restrict__ tile_incl,
                           const uint32_t *__restrict__ lane, uint32_t nq, uint32_t ntile_max,
                           uint32_t *__restrict__ cnt, uint32_t *__restrict__ tile_first, Tile *__restrict__ tiles,
                           uint32_t *__restrict__ tS, uint32_t *__restrict__ tE, uint32_t *__restrict__ big_q,
                           uint32_t *__restrict__ big_tile, uint32_t *__restrict__ big_lane, int *__restrict__ err) {
  const uint32_t nbig = cnt[C_NBIG];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nbig; i += gridDim.x * blockDim.x) {
    const uint32_t t = tile_incl[i] - 1, l = lane[i], qi = vals[i];
    if (t >= ntile_max) {  // cannot happen by the bound of device_plan_sizes; never written past
      atomicOr(err, ERR_PLAN_BOUND);
      if (i == nbig - 1) cnt[C_NTILE] = ntile_max;
      continue;
    }
    const QueryDesc d = desc[qi];
    if (l == 0) {
      tile_first[t] = i;
      tiles[t].order = (int32_t)(key_hi[i] >> 31);
    }
    atomicAdd(&tiles[t].nq, 1u);
    atomicMin(&tS[t], d.s);
    atomicMax(&tE[t], d.e);
    big_q[i] = qi;
    big_tile[i] = t;
    big_lane[i] = l;
    if (i == nbig - 1) cnt[C_NTILE] = t + 1;
  }
}

// per tile: its row blocks; their total
__global__ void k_dp_blocks(const uint32_t *__restrict__ tS, const uint32_t *__restrict__ tE, uint32_t blk_rows,
                            uint32_t ntile_max, uint32_t *__restrict__ cnt, uint32_t *__restrict__ nblk) {
  const uint32_t ntile = cnt[C_NTILE];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntile_max; t += gridDim.x * blockDim.x) {
    uint32_t b = 0;
    if (t < ntile) {
      b = (tE[t] + blk_rows - 1) / blk_rows - tS[t] / blk_rows;
      add_u64(cnt + C_TOTBLK, b);
    }
    nblk[t] = b;
  }
}

__global__ void k_dp_chunk(uint32_t *__restrict__ cnt, uint32_t target_items, uint32_t min_chunk) {
  const unsigned long long tot = *reinterpret_cast<const unsigned long long *>(cnt + C_TOTBLK);
  // rounded up, so that sum over tiles of ceil(blocks / chunk) <= target + tiles
  const uint64_t tgt = target_items ? target_items : 1u;
  uint64_t cb = (tot + tgt - 1) / tgt;
  if (cb < min_chunk) cb = min_chunk;
  if (cb < 1) cb = 1;
  cnt[C_CB] = (uint32_t)(cb < 0xffffffffull ? cb : 0xffffffffull);
}

// per tile: chunk length and item count (sum-scanned next into item ranges)
__global__ void k_dp_item_counts(const uint32_t *__restrict__ nblk, uint32_t ntile_max, uint32_t max_items,
                                 const uint32_t *__restrict__ cnt, uint32_t *__restrict__ chunk,
                                 uint32_t *__restrict__ nit) {
  const uint32_t ntile = cnt[C_NTILE], cb = cnt[C_CB];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntile_max; t += gridDim.x * blockDim.x) {
    uint32_t n_ = 0, c = 1;
    if (t < ntile && nblk[t]) {
      c = max(cb, (nblk[t] + max_items - 1) / max_items);
      n_ = (nblk[t] + c - 1) / c;
    }
    chunk[t] = c;
    nit[t] = n_;
  }
}

__global__ void k_dp_items(const uint32_t *__restrict__ tS, const uint32_t *__restrict__ nblk,
                           const uint32_t *__restrict__ chunk, const uint32_t *__restrict__ nit_incl,
                           uint32_t blk_rows, uint32_t tq, uint32_t ntile_max, uint32_t nitems_max,
                           uint32_t *__restrict__ cnt, Tile *__restrict__ tiles, WorkItem *__restrict__ items,
                           uint32_t *__restrict__ ord_key, uint32_t *__restrict__ ord_val, int *__restrict__ err) {
  const uint32_t ntile = cnt[C_NTILE];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntile; t += gridDim.x * blockDim.x) {
    const uint32_t c = chunk[t], b0 = tS[t] / blk_rows, b1 = b0 + nblk[t];
    uint32_t end = nit_incl[t];
    uint32_t n_ = (nblk[t] + c - 1) / c;
    if (end > nitems_max) {  // cannot happen by the bound of device_plan_sizes; never written past
      atomicOr(err, ERR_PLAN_BOUND);
      n_ = end - n_ >= nitems_max ? 0u : n_ - (end - nitems_max);
      end = nitems_max;
    }
    const uint32_t first = end - n_;
    tiles[t].item0 = first;
    tiles[t].item1 = end;
    for (uint32_t j = 0; j < n_; ++j) {
      WorkItem w;
      w.tile = t;
      w.blk0 = b0 + j * c;
      w.blk1 = min(b1, w.blk0 + c);
      w.pad = 0;
      items[first + j] = w;
      // longest first after the sort (ties keep the item order: the sort is stable)
      ord_key[first + j] = 0xfffffffeu - (w.blk1 - w.blk0);
      ord_val[first + j] = first + j;
      add_u64(cnt + C_PAIRS_SCR, (uint64_t)(w.blk1 - w.blk0) * blk_rows * tq);
    }
    if (t == ntile - 1) cnt[C_NITEMS] = min(nit_incl[t], nitems_max);
  }
}

}  // namespace

// Bounds of a device plan for nq queries (the buffers are sized for them):
// tiles <= nq/tq + segments, segments <= 1 + labels + 2 (buckets + 1);
// items <= target_items + tiles.
DevPlanSizes device_plan_sizes(const fknn_index *idx, uint32_t nq, const PlanShape &shape) {
  DevPlanSizes z;
  z.nb_all = std::max<uint64_t>(1, (uint64_t)std::sqrt((double)nq / 64.0));
  z.bw = (uint32_t)std::max<uint64_t>(shape.blk_rows, (idx->n + z.nb_all - 1) / z.nb_all);
  const uint64_t buckets = (idx->n + z.bw - 1) / z.bw + 1;
  z.ntile_max = (uint32_t)std::min<uint64_t>(nq, (nq + shape.tq - 1) / shape.tq + 1 + idx->n_labels + 2 * buckets);
  z.ntile_max = std::max<uint32_t>(z.ntile_max, 1);
  z.nitems_max = z.ntile_max + shape.target_items + 1;
  return z;
}

size_t device_plan_bytes(uint32_t nq, const DevPlanSizes &z) {
  const size_t q = (size_t)nq + 1, t = (size_t)z.ntile_max + 1;
  const size_t nb = ((size_t)nq + SC_TILE - 1) / SC_TILE + ((size_t)z.ntile_max + SC_TILE - 1) / SC_TILE + 2;
  const size_t it = (size_t)z.nitems_max + 1;
  return 256 * 28 + 4 * (12 * q + 6 * t + 4 * it + nb) + sizeof(Tile) * t + sizeof(WorkItem) * it + 64 * 4 + 64;
}

// Lays a DevPlan out in one device buffer of device_plan_bytes bytes.
void device_plan_layout(DevPlan &P, void *mem, uint32_t nq, const DevPlanSizes &z) {
  unsigned char *b = static_cast<unsigned char *>(mem);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    void *p = b + off;
    off = (off + bytes + 255) & ~(size_t)255;
    return p;
  };
  const size_t q = (size_t)nq + 1, t = (size_t)z.ntile_max + 1;
  P.nq = nq;
  P.z = z;
  P.cnt = (uint32_t *)take(64 * 4);
  P.key_lo = (uint32_t *)take(q * 4);
  P.key_hi = (uint32_t *)take(q * 4);
  P.vals = (uint32_t *)take(q * 4);
  P.ktmp = (uint32_t *)take(q * 4);
  P.vtmp = (uint32_t *)take(q * 4);
  P.seg = (uint32_t *)take(q * 4);
  P.lane = (uint32_t *)take(q * 4);
  P.big_q = (uint32_t *)take(q * 4);
  P.big_tile = (uint32_t *)take(q * 4);
  P.big_lane = (uint32_t *)take(q * 4);
  P.small = (uint32_t *)take(q * 4);
  P.tflag = (uint32_t *)take(q * 4);
  P.tile_first = (uint32_t *)take(t * 4);
  P.tS = (uint32_t *)take(t * 4);
  P.tE = (uint32_t *)take(t * 4);
  P.nblk = (uint32_t *)take(t * 4);
  P.chunk = (uint32_t *)take(t * 4);
  P.nit = (uint32_t *)take(t * 4);
  const size_t it = (size_t)z.nitems_max + 1;
  P.ord_key = (uint32_t *)take(it * 4);
  P.ord_val = (uint32_t *)take(it * 4);
  P.ord_k2 = (uint32_t *)take(it * 4);
  P.ord_v2 = (uint32_t *)take(it * 4);
  P.queue = (uint32_t *)take(64);
  P.bsum = (uint32_t *)take((((size_t)nq + SC_TILE - 1) / SC_TILE + ((size_t)z.ntile_max + SC_TILE - 1) / SC_TILE + 2) * 4);
  P.tiles = (Tile *)take(sizeof(Tile) * t);
  P.items = (WorkItem *)take(sizeof(WorkItem) * (z.nitems_max + 1));
}

// Enqueues the plan kernels on st (no host synchronisation, no allocation).
int device_plan_build(fknn_index *idx, const QueryDesc *d_desc, const float *d_meta, DevPlan &P,
                      const PlanShape &shape, cudaStream_t st) {
  const uint32_t nq = P.nq;
  const DevPlanSizes &z = P.z;
  FKNN_CUDA(cudaMemsetAsync(P.cnt, 0, 64 * 4, st));
  k_dp_keys<<<grid_for(nq), DP_THREADS, 0, st>>>(d_desc, d_meta, nq, z.bw, shape.small_slab, P.key_lo, P.key_hi,
                                                 P.vals, P.small, P.cnt);
  g_launches += 1;
  int rc;
  // (high word, low word) order, stable: sort by the low word, carry the high word along, sort by it
  if ((rc = radix_sort_pairs(idx, P.key_lo, P.vals, P.ktmp, P.vtmp, nq, 0, 32, st))) return rc;
  k_gather_u32<<<grid_for(nq), DP_THREADS, 0, st>>>(P.key_hi, P.vals, nq, P.ktmp);
  FKNN_CUDA(cudaMemcpyAsync(P.key_hi, P.ktmp, (size_t)nq * 4, cudaMemcpyDeviceToDevice, st));
  g_launches += 1;
  if ((rc = radix_sort_pairs(idx, P.key_hi, P.vals, P.ktmp, P.vtmp, nq, 0, 32, st))) return rc;
  k_dp_segments<<<grid_for(nq), DP_THREADS, 0, st>>>(P.key_hi, P.vals, d_desc, nq, P.cnt, P.seg);
  scan_incl<OpMax>(P.seg, nq, P.bsum, st);
  k_dp_lanes<<<grid_for(nq), DP_THREADS, 0, st>>>(P.seg, nq, (uint32_t)shape.tq, P.cnt, P.lane, P.tflag);
  scan_incl<OpSum>(P.tflag, nq, P.bsum, st);
  k_dp_tile_init<<<grid_for(std::max(z.ntile_max, z.nitems_max)), DP_THREADS, 0, st>>>(P.tiles, P.tS, P.tE,
                                                                                      z.ntile_max, P.ord_key,
                                                                                      z.nitems_max);
  k_dp_tiles<<<grid_for(nq), DP_THREADS, 0, st>>>(P.vals, P.key_hi, d_desc, P.tflag, P.lane, nq, z.ntile_max, P.cnt,
                                                  P.tile_first, P.tiles, P.tS, P.tE, P.big_q, P.big_tile, P.big_lane,
                                                  idx->d_flag);
  k_dp_blocks<<<grid_for(z.ntile_max), DP_THREADS, 0, st>>>(P.tS, P.tE, (uint32_t)shape.blk_rows, z.ntile_max, P.cnt,
                                                            P.nblk);
  k_dp_chunk<<<1, 1, 0, st>>>(P.cnt, shape.target_items, shape.min_chunk_blocks);
  k_dp_item_counts<<<grid_for(z.ntile_max), DP_THREADS, 0, st>>>(P.nblk, z.ntile_max, shape.max_items_per_tile,
                                                                 P.cnt, P.chunk, P.nit);
  scan_incl<OpSum>(P.nit, z.ntile_max, P.bsum, st);
  k_dp_items<<<grid_for(z.ntile_max), DP_THREADS, 0, st>>>(P.tS, P.nblk, P.chunk, P.nit, (uint32_t)shape.blk_rows,
                                                           (uint32_t)shape.tq, z.ntile_max, z.nitems_max, P.cnt,
                                                           P.tiles, P.items, P.ord_key, P.ord_val, idx->d_flag);
  g_launches += 9;
  // processing order of the work items (longest first) and the queues
  if ((rc = radix_sort_pairs(idx, P.ord_key, P.ord_val, P.ord_k2, P.ord_v2, z.nitems_max, 0, 32, st))) return rc;
  FKNN_CUDA(cudaMemsetAsync(P.queue, 0, 64, st));
  FKNN_CUDA(cudaGetLastError());
  return FKNN_OK;
}

}  // namespace fknn
