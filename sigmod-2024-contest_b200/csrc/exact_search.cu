// Exact FP32 filtered top-k (the B200 form of utils.h:80-158 Bruteforce).
//
// Pipeline for one batch of queries:
//   1. k_query_prep   predicate -> contiguous slab [s, e) of one row order
//                     (binary search on the sorted attribute columns), ||q||^2
//   2. host planner   slabs <= SMALL_SLAB -> row-by-row exact scan; others
//                     sorted and grouped into 64-query tiles, split into
//                     (tile, row chunk) work items
//   3. k_tile_stage   query tiles in the [101][64] layout of the base blocks
//   4. k_screen       FP32 FFMA contraction q.x over 64-row blocks streamed by
//                     the TMA bulk engine; ds = |x|^2+|q|^2-2q.x; rows whose
//                     ds can still reach the running k-th bound are kept in a
//                     per-(item, query) candidate list that a warp bitonic
//                     sort compacts; the bound is shared across CTAs.
//   5. k_merge        per query: union of its items' lists, k-th bound, then
//                     exact re-score of the survivors with the reference's
//                     sequential arithmetic, (dist, id) sort, top-k out.
//   6. k_exact_scan   small slabs and any query whose candidates overflowed:
//                     exact distances row by row, block select on (dist, id).
// Ids and distances equal the reference's bit for bit: every row that can
// be in the top k (screening error bound in screen_eps) is re-scored with
// normal_l2's exact operation sequence and ordered by (dist, id) like the
// ResultMaxHeap of utils.h:35-78.
#include <algorithm>
#include <functional>
#include <thread>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>

#include "device_util.cuh"

namespace fknn {

namespace {

// ---------------------------------------------------------------- prep --

__device__ __forceinline__ uint32_t lower_bound_i32(const int32_t *a, uint32_t lo, uint32_t hi, int32_t v) {
  while (lo < hi) {
    uint32_t m = lo + ((hi - lo) >> 1);
    if (a[m] < v) lo = m + 1; else hi = m;
  }
  return lo;
}
__device__ __forceinline__ uint32_t upper_bound_i32(const int32_t *a, uint32_t lo, uint32_t hi, int32_t v) {
  while (lo < hi) {
    uint32_t m = lo + ((hi - lo) >> 1);
    if (a[m] <= v) lo = m + 1; else hi = m;
  }
  return lo;
}
// first position with ts >= v
__device__ __forceinline__ uint32_t lower_bound_f32(const float *a, uint32_t lo, uint32_t hi, float v) {
  while (lo < hi) {
    uint32_t m = lo + ((hi - lo) >> 1);
    if (a[m] < v) lo = m + 1; else hi = m;
  }
  return lo;
}
// first position with ts > v
__device__ __forceinline__ uint32_t upper_bound_f32(const float *a, uint32_t lo, uint32_t hi, float v) {
  while (lo < hi) {
    uint32_t m = lo + ((hi - lo) >> 1);
    if (a[m] <= v) lo = m + 1; else hi = m;
  }
  return lo;
}

// Query checks: type in {0,1,2,3} (searcher.hpp:39-42 rejects the rest),
// v inside int32 for types 1/3 (read as int32, utils.h:99), window bounds
// not NaN for types 2/3, vector values finite and <= 1e15.
__global__ void k_validate_queries(const float *__restrict__ q, const float *__restrict__ meta, uint32_t nq,
                                   int *flag) {
  const uint64_t total = (uint64_t)nq * DIM;
  int bad = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (!(fabsf(q[i]) <= 1e15f)) bad |= ERR_BAD_QUERY_VEC;
    if (i < nq) {
      const float *m = meta + i * 4;
      float t = m[0];
      if (!(t == 0.f || t == 1.f || t == 2.f || t == 3.f)) bad |= ERR_BAD_QUERY_TYPE;
      if ((t == 1.f || t == 3.f) && !(fabsf(m[1]) < 2147483648.f)) bad |= ERR_BAD_QUERY_VALUE;
      if ((t == 2.f || t == 3.f) && (m[2] != m[2] || m[3] != m[3])) bad |= ERR_BAD_QUERY_VALUE;
    }
  }
  if (bad) atomicOr(flag, bad);
}

// Predicate -> slab.  type 0: all rows (time order); 1: label == v (category
// order); 2: l <= ts <= r (time order); 3: both (category order, the window
// inside the label's slab).  The semantics are utils.h:110-137's.
__device__ __forceinline__ void resolve_slab(const float *m, uint32_t n, const float *ts_t, const int32_t *lab_c,
                                             const float *ts_c, int32_t &order, uint32_t &s, uint32_t &e) {
  const uint32_t type = (uint32_t)m[0];
  if (type == 0) {
    order = ORDER_TIME; s = 0; e = n;
  } else if (type == 2) {
    order = ORDER_TIME;
    s = lower_bound_f32(ts_t, 0, n, m[2]);
    e = upper_bound_f32(ts_t, 0, n, m[3]);
  } else {
    order = ORDER_CAT;
    const int32_t v = (int32_t)m[1];
    s = lower_bound_i32(lab_c, 0, n, v);
    e = upper_bound_i32(lab_c, s, n, v);
    if (type == 3) {
      uint32_t cs = s, ce = e;
      s = lower_bound_f32(ts_c, cs, ce, m[2]);
      e = upper_bound_f32(ts_c, cs, ce, m[3]);
    }
  }
  if (e < s) e = s;
}

__global__ void k_query_prep(const float *__restrict__ q, const float *__restrict__ meta, uint32_t nq, uint32_t n,
                             const float *__restrict__ ts_t, const int32_t *__restrict__ lab_c,
                             const float *__restrict__ ts_c, QueryDesc *__restrict__ desc) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  QueryDesc dsc;
  resolve_slab(meta + (uint64_t)i * 4, n, ts_t, lab_c, ts_c, dsc.order, dsc.s, dsc.e);
  const float *v = q + (uint64_t)i * DIM;
  float s = 0.f;
#pragma unroll 10
  for (int d = 0; d < DIM; ++d) s = fmaf(v[d], v[d], s);
  dsc.qn = s;
  desc[i] = dsc;
}

__global__ void k_count(const float *__restrict__ meta, uint32_t nq, uint32_t n, const float *__restrict__ ts_t,
                        const int32_t *__restrict__ lab_c, const float *__restrict__ ts_c,
                        uint32_t *__restrict__ counts) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  int32_t o;
  uint32_t s, e;
  resolve_slab(meta + (uint64_t)i * 4, n, ts_t, lab_c, ts_c, o, s, e);
  counts[i] = e - s;
}

// Query tiles in the base-block layout: [101][64] (dims, then |q|^2).
__global__ void k_tile_stage(const float *__restrict__ q, const QueryDesc *__restrict__ desc,
                             const int32_t *__restrict__ lane_q, float *__restrict__ qtiles) {
  const uint32_t t = blockIdx.x;
  __shared__ float tile[TQ][DIM + 1];
  for (int i = threadIdx.x; i < TQ * DIM; i += blockDim.x) {
    int l = i / DIM, d = i % DIM;
    int32_t qi = lane_q[t * TQ + l];
    tile[l][d] = qi >= 0 ? q[(uint64_t)qi * DIM + d] : 0.f;
  }
  __syncthreads();
  float *out = qtiles + (uint64_t)t * BLK_FLOATS;
  for (int i = threadIdx.x; i < TQ * DIM; i += blockDim.x) {
    int d = i / TQ, l = i % TQ;
    out[d * TQ + l] = tile[l][d];
  }
  for (int l = threadIdx.x; l < TQ; l += blockDim.x) {
    int32_t qi = lane_q[t * TQ + l];
    out[DIM * TQ + l] = qi >= 0 ? desc[qi].qn : 0.f;
  }
}

// -------------------------------------------------------------- screen --

constexpr int SC_CONSUMERS = 4;                   // compute warps
constexpr int SC_THREADS = (SC_CONSUMERS + 1) * 32;  // + one producer warp
constexpr int SC_STAGES = 3;
constexpr int SC_REFRESH = 16;  // sub-tiles between reads of the shared bound

// Each consumer warp w owns the candidate lists of queries [16w, 16w+16) of
// the tile: with the thread mapping below (rows ty*4.., queries tx*8..,
// tx = tid/16) only warp w ever pushes into them, so lists are compacted by
// their owner with no CTA-wide barrier.  Row blocks stream through a ring of
// SC_STAGES buffers: the producer warp issues one bulk copy per 64-row block
// after the four consumer warps released the slot (empty barrier).
struct ScreenSmem {
  float qs[BLK_FLOATS];
  float xs[SC_STAGES][BLK_FLOATS];
  float push[TQ];     // largest ds worth keeping
  float thr[TQ];      // current upper bound T on the k-th distance
  float qn[TQ];
  int cnt[TQ];
  uint32_t ls[TQ], le[TQ];
  int32_t lq[TQ];
  uint64_t full[SC_STAGES], empty[SC_STAGES], qbar;
};

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Sort, bound and trim one (item, query) candidate list.  Whole warp.
__device__ __noinline__ void compact_list(Candidate *list, ScreenSmem &sm, int L, uint32_t k, uint32_t *T_global,
                                          uint32_t *ovf) {
  const int lane = threadIdx.x & 31;
  const int n = sm.cnt[L];
  float key[CAP / 32];
  uint32_t val[CAP / 32];
#pragma unroll
  for (int j = 0; j < CAP / 32; ++j) {
    int e = j * 32 + lane;
    if (e < n) {
      Candidate c = list[e];
      key[j] = c.ds;
      val[j] = c.pos;
    } else {
      key[j] = INFINITY;
      val[j] = 0xffffffffu;
    }
  }
  warp_bitonic_sort<CAP / 32>(key, val);
  const float qn = sm.qn[L];
  const int32_t qi = sm.lq[L];
  float T = sm.thr[L];
  if (n >= (int)k) {
    const int e = (int)k - 1;
    float mine = key[0];
#pragma unroll
    for (int j = 1; j < CAP / 32; ++j)
      if (j == (e >> 5)) mine = key[j];
    const float kth = __shfl_sync(0xffffffffu, mine, e & 31);
    T = fminf(T, screen_hi(kth, qn));
  }
  const float Tg = sortable_f32(ld_volatile_u32(T_global + qi));
  if (Tg < T) T = Tg;
  if (lane == 0 && T < Tg) atomicMin(T_global + qi, f32_sortable(T));
  int kept = 0;
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < CAP / 32; ++j) {
    const bool keep = (j * 32 + lane) < n && screen_lo(key[j], qn) <= T;
    const uint32_t b = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      Candidate c;
      c.ds = key[j];
      c.pos = val[j];
      list[kept + __popc(b & lt)] = c;
    }
    kept += __popc(b);
  }
  __syncwarp();
  if (lane == 0) {
    if (kept > CAP - BLK) {
      // More near-ties than the list can hold: hand the query to the exact scan.
      ovf[qi] = 1u;
      sm.cnt[L] = 0;
      sm.thr[L] = -INFINITY;
      sm.push[L] = -INFINITY;
    } else {
      sm.cnt[L] = kept;
      sm.thr[L] = T;
      sm.push[L] = (T == INFINITY) ? INFINITY : screen_push_limit(T, qn);
    }
  }
  __syncwarp();
}

__global__ void __launch_bounds__(SC_THREADS, 2)
    k_screen(const WorkItem *__restrict__ items, const Tile *__restrict__ tiles, const float *__restrict__ qtiles,
             const int32_t *__restrict__ lane_q, const uint32_t *__restrict__ lane_s,
             const uint32_t *__restrict__ lane_e, const float *__restrict__ blocks_t,
             const float *__restrict__ blocks_c, uint32_t *__restrict__ T_global, uint32_t *__restrict__ ovf,
             Candidate *__restrict__ out, uint32_t *__restrict__ out_cnt, uint32_t k, uint32_t stride, int *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  ScreenSmem &sm = *reinterpret_cast<ScreenSmem *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t item_id = blockIdx.x;
  const WorkItem it = items[item_id];
  const Tile tl = tiles[it.tile];
  const float *blocks = tl.order == ORDER_TIME ? blocks_t : blocks_c;
  // every stride-th row block of the item (stride 1: all of them)
  const uint32_t nsub = (it.blk1 - it.blk0 + stride - 1) / stride;
  Candidate *out_item = out + (uint64_t)item_id * TQ * CAP;

  if (tid == 0) {
    for (int s = 0; s < SC_STAGES; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], SC_CONSUMERS);
    }
    mbar_init(&sm.qbar, 1);
    fence_mbar_init();
  }
  __syncthreads();  // the only CTA-wide barrier

  if (warp == SC_CONSUMERS) {
    // ---------------- producer: one lane issues every bulk copy
    if (lane == 0) {
      mbar_arrive_expect_tx(&sm.qbar, BLK_BYTES);
      bulk_g2s(sm.qs, qtiles + (uint64_t)it.tile * BLK_FLOATS, BLK_BYTES, &sm.qbar);
      uint32_t issued = 0;
      for (uint32_t sub = 0; sub < nsub; ++sub) {
        const int st = sub % SC_STAGES;
        if (sub >= SC_STAGES && !mbar_wait_bounded(&sm.empty[st], ((sub / SC_STAGES) - 1) & 1, err)) break;
        mbar_arrive_expect_tx(&sm.full[st], BLK_BYTES);
        bulk_g2s(sm.xs[st], blocks + (uint64_t)(it.blk0 + sub * stride) * BLK_FLOATS, BLK_BYTES, &sm.full[st]);
        ++issued;
      }
      // every issued copy must have landed before the CTA may exit
      mbar_wait_bounded(&sm.qbar, 0, err);
      for (uint32_t i = issued > SC_STAGES ? issued - SC_STAGES : 0; i < issued; ++i)
        mbar_wait_bounded(&sm.full[i % SC_STAGES], (i / SC_STAGES) & 1, err);
    }
    return;
  }

  // ---------------- consumers
  // waits are warp-uniform: the lanes' timers may disagree at the deadline
  bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&sm.qbar, 0, err));
  if (lane < 16) {
    const int L = 16 * warp + lane;
    const int32_t qi = lane_q[it.tile * TQ + L];
    sm.lq[L] = qi;
    sm.cnt[L] = 0;
    sm.qn[L] = sm.qs[DIM * TQ + L];
    if (qi >= 0) {
      sm.ls[L] = lane_s[it.tile * TQ + L];
      sm.le[L] = lane_e[it.tile * TQ + L];
      const float T = sortable_f32(ld_volatile_u32(T_global + qi));
      sm.thr[L] = T;
      sm.push[L] = (T == INFINITY) ? INFINITY : screen_push_limit(T, sm.qn[L]);
      if (ld_volatile_u32(ovf + qi)) sm.push[L] = -INFINITY;
    } else {
      sm.ls[L] = sm.le[L] = 0;
      sm.thr[L] = -INFINITY;
      sm.push[L] = -INFINITY;
    }
  }
  __syncwarp();

  const int ty = tid & 15;  // rows ty*4 .. ty*4+3 of the 64-row block
  const int tx = tid >> 4;  // queries tx*8 .. tx*8+7 of the tile (owned by this warp)
  for (uint32_t sub = 0; sub < nsub && ok; ++sub) {
    const int st = sub % SC_STAGES;
    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&sm.full[st], (sub / SC_STAGES) & 1, err))) {
      ok = false;
      break;
    }
    const float *xs = sm.xs[st];
    float acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
    const float4 *xr = reinterpret_cast<const float4 *>(xs) + ty;
    const float4 *qr = reinterpret_cast<const float4 *>(sm.qs) + tx * 2;
#pragma unroll 10
    for (int d = 0; d < DIM; ++d) {
      const float4 a = xr[d * (BLK / 4)];
      const float4 b0 = qr[d * (TQ / 4)];
      const float4 b1 = qr[d * (TQ / 4) + 1];
      const float av[4] = {a.x, a.y, a.z, a.w};
      const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    const float4 xn4 = reinterpret_cast<const float4 *>(xs + DIM * BLK)[ty];
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[st]);  // this warp is done with the slot
    // epilogue: ds = (|x|^2 + |q|^2) - 2 q.x; keep rows that can reach the bound
    const float xn[4] = {xn4.x, xn4.y, xn4.z, xn4.w};
    const uint32_t row0 = (it.blk0 + sub * stride) * BLK + ty * 4;
    uint32_t pass = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int L = tx * 8 + j;
      const float pl = sm.push[L];
      const float qn = sm.qn[L];
      const uint32_t s = sm.ls[L], e = sm.le[L];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float ds = fmaf(-2.f, acc[i][j], xn[i] + qn);
        acc[i][j] = ds;
        const uint32_t p = row0 + i;
        pass |= (uint32_t)(ds <= pl && p >= s && p < e) << (j * 4 + i);
      }
    }
    if (__any_sync(0xffffffffu, pass != 0)) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (pass & (1u << (j * 4 + i))) {
            const int L = tx * 8 + j;
            const int idx = atomicAdd(&sm.cnt[L], 1);
            Candidate c;
            c.ds = acc[i][j];
            c.pos = row0 + i;
            out_item[(uint64_t)L * CAP + idx] = c;
          }
        }
      }
      __syncwarp();
    }
    // own lists near capacity are compacted; bounds refreshed from other CTAs
    {
      const int L = 16 * warp + (lane & 15);
      const bool need = lane < 16 && sm.cnt[L] > CAP - BLK;
      uint32_t m = __ballot_sync(0xffffffffu, need);
      while (m) {
        const int b = __ffs(m) - 1;
        m &= m - 1;
        compact_list(out_item + (uint64_t)(16 * warp + b) * CAP, sm, 16 * warp + b, k, T_global, ovf);
      }
      if ((sub % SC_REFRESH) == SC_REFRESH - 1 && lane < 16 && !need) {
        const int32_t qi = sm.lq[L];
        if (qi >= 0 && sm.push[L] != -INFINITY) {
          const float Tg = sortable_f32(ld_volatile_u32(T_global + qi));
          if (Tg < sm.thr[L]) {
            sm.thr[L] = Tg;
            sm.push[L] = screen_push_limit(Tg, sm.qn[L]);
          }
        }
      }
      __syncwarp();
    }
  }
  if (!ok) {
    // A bulk copy never landed (bounded wait gave up): this warp's queries
    // are answered by the exact scan instead.
    if (lane < 16) {
      const int L = 16 * warp + lane;
      if (sm.lq[L] >= 0) ovf[sm.lq[L]] = 1u;
      out_cnt[(uint64_t)item_id * TQ + L] = 0;
    }
    return;
  }
  // final trim of this warp's non-empty lists
  for (int b = 0; b < 16; ++b) {
    const int L = 16 * warp + b;
    if (sm.cnt[L] > 0) compact_list(out_item + (uint64_t)L * CAP, sm, L, k, T_global, ovf);
  }
  if (lane < 16) out_cnt[(uint64_t)item_id * TQ + 16 * warp + lane] = (uint32_t)sm.cnt[16 * warp + lane];
}

// --------------------------------------------------------------- merge --

constexpr int MG_THREADS = 256;

struct MergeSmem {
  float key[MERGE_CAP];
  uint32_t val[MERGE_CAP];
  uint64_t ekey[RESCORE_CAP];
  float qv[DIM];
  uint32_t cnt_prefix[MG_THREADS + 1];
  int total, surv, status;
};

__global__ void __launch_bounds__(MG_THREADS)
    k_merge(const uint32_t *__restrict__ big_q, const uint32_t *__restrict__ big_tile,
            const uint32_t *__restrict__ big_lane, const Tile *__restrict__ tiles, const uint32_t *__restrict__ item_slot,
            const Candidate *__restrict__ out,
            const uint32_t *__restrict__ out_cnt, const QueryDesc *__restrict__ desc, const float *__restrict__ q,
            const float *__restrict__ vecs, const uint32_t *__restrict__ perm_t, const uint32_t *__restrict__ perm_c,
            const uint32_t *__restrict__ T_global, const uint32_t *__restrict__ ovf, uint32_t *__restrict__ ovf_list,
            uint32_t *__restrict__ ovf_count, uint32_t k, uint32_t *__restrict__ ids, float *__restrict__ dists) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  MergeSmem &sm = *reinterpret_cast<MergeSmem *>(smem_raw);
  const int tid = threadIdx.x;
  const uint32_t qi = big_q[blockIdx.x];
  if (ovf[qi]) {
    if (tid == 0) ovf_list[atomicAdd(ovf_count, 1u)] = qi;
    return;
  }
  const Tile tl = tiles[big_tile[blockIdx.x]];
  const uint32_t L = big_lane[blockIdx.x];
  const uint32_t nitems = tl.item1 - tl.item0;
  const QueryDesc dsc = desc[qi];
  const float qn = dsc.qn;
  for (int d = tid; d < DIM; d += MG_THREADS) sm.qv[d] = q[(uint64_t)qi * DIM + d];
  // 1. gather the lists: item offsets (a tile has at most a few dozen
  // items), then the whole block copies each list
  // more items than offset slots: the exact scan answers the query
  list_offsets(item_slot, tl.item0, nitems, out_cnt, L, TQ, sm.cnt_prefix, &sm.total, MG_THREADS, MERGE_CAP + 1);
  __syncthreads();
  const int M = sm.total;
  if (M > MERGE_CAP) {
    if (tid == 0) ovf_list[atomicAdd(ovf_count, 1u)] = qi;
    return;
  }
  for (uint32_t i = 0; i < nitems; ++i) {
    const uint64_t item = item_slot[tl.item0 + i];
    const uint32_t base = sm.cnt_prefix[i];
    const uint32_t c = (i + 1 < nitems ? sm.cnt_prefix[i + 1] : (uint32_t)M) - base;
    const Candidate *src = out + (item * TQ + L) * CAP;
    for (uint32_t j = tid; j < c; j += MG_THREADS) {
      const Candidate cd = src[j];
      sm.key[base + j] = cd.ds;
      sm.val[base + j] = cd.pos;
    }
  }
  int np2 = 32;
  while (np2 < M) np2 <<= 1;
  for (int i = M + tid; i < np2; i += MG_THREADS) {
    sm.key[i] = INFINITY;
    sm.val[i] = 0xffffffffu;
  }
  __syncthreads();
  // 2. k-th bound over the union
  block_bitonic_sort_kv(sm.key, sm.val, np2);
  float T = sortable_f32(T_global[qi]);
  if (M >= (int)k) T = fminf(T, screen_hi(sm.key[k - 1], qn));
  // 3. survivors (a prefix of the sorted list up to rounding; scan anyway)
  if (tid == 0) sm.surv = 0;
  __syncthreads();
  for (int i = tid; i < M; i += MG_THREADS) {
    if (screen_lo(sm.key[i], qn) <= T) {
      int slot = atomicAdd(&sm.surv, 1);
      if (slot < RESCORE_CAP) {
        const uint32_t pos = sm.val[i];
        const uint32_t id = (dsc.order == ORDER_TIME ? perm_t : perm_c)[pos];
        sm.ekey[slot] = (uint64_t)id;  // re-scored below
      }
    }
  }
  __syncthreads();
  const int S = sm.surv;
  if (S > RESCORE_CAP) {
    if (tid == 0) ovf_list[atomicAdd(ovf_count, 1u)] = qi;
    return;
  }
  // 4. exact re-score (distance.h:62-72 order of operations)
  for (int i = tid; i < S; i += MG_THREADS) {
    const uint32_t id = (uint32_t)sm.ekey[i];
    const float d = seq_l2_strided(vecs + (uint64_t)id * DIM, 1, sm.qv);
    sm.ekey[i] = exact_key(d, id);
  }
  int sp2 = 32;
  while (sp2 < S) sp2 <<= 1;
  for (int i = S + tid; i < sp2; i += MG_THREADS) sm.ekey[i] = ~0ull;
  __syncthreads();
  block_bitonic_sort(sm.ekey, sp2);
  for (uint32_t j = tid; j < k; j += MG_THREADS) {
    uint32_t id = 0xffffffffu;
    float d = INFINITY;
    if ((int)j < S) {
      id = (uint32_t)sm.ekey[j];
      d = sortable_f32((uint32_t)(sm.ekey[j] >> 32));
    }
    ids[(uint64_t)qi * k + j] = id;
    if (dists) dists[(uint64_t)qi * k + j] = d;
  }
}

// ----------------------------------------------------------- exact scan --

constexpr int ES_THREADS = 256;
constexpr int ES_CAP = 1024;

__global__ void __launch_bounds__(ES_THREADS)
    k_exact_scan(const uint32_t *__restrict__ list, const uint32_t *__restrict__ d_count, uint32_t h_count,
                 const QueryDesc *__restrict__ desc, const float *__restrict__ q, const float *__restrict__ blocks_t,
                 const float *__restrict__ blocks_c, const uint32_t *__restrict__ perm_t,
                 const uint32_t *__restrict__ perm_c, uint32_t k, uint32_t *__restrict__ ids,
                 float *__restrict__ dists) {
  __shared__ uint64_t buf[ES_CAP];
  __shared__ float qv[DIM];
  __shared__ int cnt;
  __shared__ uint64_t thr;
  const uint32_t count = d_count ? *d_count : h_count;
  const int tid = threadIdx.x;
  for (uint32_t li = blockIdx.x; li < count; li += gridDim.x) {
    const uint32_t qi = list[li];
    const QueryDesc dsc = desc[qi];
    const float *blocks = dsc.order == ORDER_TIME ? blocks_t : blocks_c;
    const uint32_t *perm = dsc.order == ORDER_TIME ? perm_t : perm_c;
    for (int d = tid; d < DIM; d += ES_THREADS) qv[d] = q[(uint64_t)qi * DIM + d];
    if (tid == 0) {
      cnt = 0;
      thr = ~0ull;
    }
    __syncthreads();
    for (uint64_t base = dsc.s; base < dsc.e; base += ES_THREADS) {
      const uint64_t p = base + tid;
      if (p < dsc.e) {
        const float *x = blocks + (p / BLK) * BLK_FLOATS + (p % BLK);
        const float d = seq_l2_strided(x, BLK, qv);
        const uint64_t key = exact_key(d, perm[p]);
        if (key < thr) buf[atomicAdd(&cnt, 1)] = key;
      }
      __syncthreads();
      if (cnt > ES_CAP - ES_THREADS) {
        for (int i = cnt + tid; i < ES_CAP; i += ES_THREADS) buf[i] = ~0ull;
        __syncthreads();
        block_bitonic_sort(buf, ES_CAP);
        if (tid == 0) {
          cnt = (int)k;
          thr = buf[k - 1];
        }
        __syncthreads();
      }
    }
    int c = cnt;
    int np2 = 32;
    while (np2 < c) np2 <<= 1;
    for (int i = c + tid; i < np2; i += ES_THREADS) buf[i] = ~0ull;
    __syncthreads();
    block_bitonic_sort(buf, np2);
    for (uint32_t j = tid; j < k; j += ES_THREADS) {
      uint32_t id = 0xffffffffu;
      float d = INFINITY;
      if ((int)j < c) {
        id = (uint32_t)buf[j];
        d = sortable_f32((uint32_t)(buf[j] >> 32));
      }
      ids[(uint64_t)qi * k + j] = id;
      if (dists) dists[(uint64_t)qi * k + j] = d;
    }
    __syncthreads();
  }
}

// ------------------------------------ predicate compaction (no-alloc form) --
//
// Count -> scan -> write over 4,096-row tiles: its only scratch is one
// counter per tile, which fits the fixed array of fknn_filter_rows_noalloc.
// The index's fknn_filter_rows / fknn_filter_rows_batch use filter.cu.

constexpr int FC_THREADS = 256;
constexpr int FC_ITEMS = 16;
constexpr int FC_TILE = FC_THREADS * FC_ITEMS;

__device__ __forceinline__ bool row_passes(uint32_t type, int32_t v, float l, float r, float label, float ts) {
  switch (type) {
    case 0: return true;
    case 1: return (int32_t)label == v;
    case 2: return ts >= l && ts <= r;
    default: return (int32_t)label == v && ts >= l && ts <= r;
  }
}

// Pass 1: passing rows per 4096-row tile (warp ballots, coalesced columns).
__global__ void k_filter_count(const float *__restrict__ labels, const float *__restrict__ ts, uint64_t n,
                               float4 m, uint32_t *__restrict__ tile_cnt) {
  __shared__ uint32_t wsum[FC_THREADS / 32];
  const uint32_t type = (uint32_t)m.x;
  const int32_t v = (int32_t)m.y;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * FC_TILE;
  uint32_t c = 0;
  for (int i = 0; i < FC_ITEMS; ++i) {
    const uint64_t idx = base + (uint64_t)i * FC_THREADS + threadIdx.x;
    const bool p = idx < n && row_passes(type, v, m.z, m.w, labels[idx], ts[idx]);
    c += __popc(__ballot_sync(0xffffffffu, p));
  }
  if (lane == 0) wsum[w] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int i = 0; i < FC_THREADS / 32; ++i) s += wsum[i];
    tile_cnt[blockIdx.x] = s;
  }
}

// Pass 2 (after an exclusive scan of tile_cnt): write passing ids in order.
// Each thread keeps its 16 predicates as a bit mask; one block scan over the
// (item, warp) counts gives every ballot its output offset.
__global__ void k_filter_write(const float *__restrict__ labels, const float *__restrict__ ts, uint64_t n, float4 m,
                               const uint32_t *__restrict__ tile_off, uint32_t *__restrict__ out) {
  constexpr int NW = FC_THREADS / 32;
  __shared__ uint32_t cnt[FC_ITEMS * NW + 1];
  const uint32_t type = (uint32_t)m.x;
  const int32_t v = (int32_t)m.y;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * FC_TILE;
  uint32_t bits = 0, ballots[FC_ITEMS];
#pragma unroll
  for (int i = 0; i < FC_ITEMS; ++i) {
    const uint64_t idx = base + (uint64_t)i * FC_THREADS + threadIdx.x;
    const bool p = idx < n && row_passes(type, v, m.z, m.w, labels[idx], ts[idx]);
    ballots[i] = __ballot_sync(0xffffffffu, p);
    bits |= (p ? 1u : 0u) << i;
  }
  // counts in output order: item-major, then warp
  if (lane < FC_ITEMS) {
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < FC_ITEMS; ++i)
      if (i == lane) c = __popc(ballots[i]);
    cnt[lane * NW + w] = c;
  }
  __syncthreads();
  if (threadIdx.x < 32) {  // exclusive scan of the FC_ITEMS * NW = 128 counts, 4 per lane
    constexpr int PER = FC_ITEMS * NW / 32;
    uint32_t loc[PER], sum = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      loc[j] = cnt[lane * PER + j];
      sum += loc[j];
    }
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    uint32_t run = tile_off[blockIdx.x] + inc - sum;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      cnt[lane * PER + j] = run;
      run += loc[j];
    }
  }
  __syncthreads();
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int i = 0; i < FC_ITEMS; ++i)
    if ((bits >> i) & 1u)
      out[cnt[i * NW + w] + __popc(ballots[i] & lt)] = (uint32_t)(base + (uint64_t)i * FC_THREADS + threadIdx.x);
}

// Exclusive scan of the tile counts in place, one block; *total = their sum.
__global__ void __launch_bounds__(1024) k_exclusive_scan_small(uint32_t *data, uint32_t len, uint32_t *total) {
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t carry;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < len; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < len ? data[i] : 0u;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
      const uint32_t x = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0u;
      uint32_t y = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= o) y += t;
      }
      wsum[lane] = y - x;  // exclusive sum of the warps before
    }
    __syncthreads();
    const uint32_t c = carry;
    if (i < len) data[i] = c + wsum[w] + inc - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = c + wsum[w] + inc;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_fill_u32(uint32_t *__restrict__ p, uint32_t n, uint32_t v) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

// ============================================================== host side

int validate_queries(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, cudaStream_t st) {
  int *flag = idx->d_flag;
  FKNN_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
  unsigned grid = (unsigned)std::min<uint64_t>(((uint64_t)nq * DIM + 255) / 256, 148 * 8);
  if (grid == 0) grid = 1;
  k_validate_queries<<<grid, 256, 0, st>>>(d_q, d_meta, nq, flag);
  g_launches += 1;
  return FKNN_OK;
}

static int check_query_flag(int flag) {
  if (!flag) return FKNN_OK;
  if (flag == ERR_PLAN_BOUND) {
    set_error("fknn_search: the device-built plan met a buffer bound (internal error; no output was written past it)");
    return FKNN_ECUDA;
  }
  std::string m = "fknn_search: ";
  if (flag & ERR_BAD_QUERY_TYPE) m += "query type not in {0,1,2,3}; ";
  if (flag & ERR_BAD_QUERY_VALUE) m += "query category outside int32 or NaN window bound; ";
  if (flag & ERR_BAD_QUERY_VEC) m += "query vector value not finite or above 1e15; ";
  set_error(m);
  return FKNN_EINVAL;
}

int count_matches(fknn_index *idx, const float *d_meta, uint32_t nq, uint32_t *d_counts, cudaStream_t st) {
  if (nq == 0) return FKNN_OK;
  k_count<<<(nq + 255) / 256, 256, 0, st>>>(d_meta, nq, (uint32_t)idx->n, idx->ord[ORDER_TIME].ts,
                                           idx->ord[ORDER_CAT].label, idx->ord[ORDER_CAT].ts, d_counts);
  g_launches += 1;
  FKNN_CUDA(cudaGetLastError());
  return FKNN_OK;
}

// Groups queries into 64-query tiles whose slabs overlap (same order and
// predicate class, start bucket, then end), and cuts each tile's union
// range into row chunks.
namespace {

inline int bits_for(uint64_t v) {
  int b = 0;
  while (b < 64 && (v >> b)) ++b;
  return b;
}

// Sorts keys[0..m) of one query class by (bucket, e, s, qi).  The keys
// arrive in increasing qi and the LSD radix sort is stable, so qi needs no
// key bits; bucket, e and s are packed into one 64-bit key at their actual
// widths (under 49 bits at n = 1e6) and sorted with 11-bit digits, passes
// whose digit is constant skipped.  Wider packings use two 64-bit words.
void sort_class(PlanKey *keys, size_t m, Plan::SortScratch &W) {
  if (m < 2) return;
  uint32_t max_e = 0, max_s = 0, max_b = 0;
  for (size_t i = 0; i < m; ++i) {
    max_e = std::max(max_e, keys[i].e);
    max_s = std::max(max_s, keys[i].s);
    max_b = std::max<uint32_t>(max_b, (uint32_t)std::min<uint64_t>(keys[i].bucket, 0xffffffffu));
  }
  const int be = bits_for(max_e), bs = bits_for(max_s), bb = bits_for(max_b);
  const bool one_word = bb + be + bs <= 64;
  auto &hi = W.hi, &lo = W.lo, &hi2 = W.hi2, &lo2 = W.lo2;
  auto &ix = W.ix, &ix2 = W.ix2, &cnt = W.cnt;
  lo.resize(m);
  lo2.resize(m);
  ix.resize(m);
  ix2.resize(m);
  if (!one_word) {
    hi.resize(m);
    hi2.resize(m);
  }
  for (size_t i = 0; i < m; ++i) {
    const PlanKey &k = keys[i];
    if (one_word) {
      lo[i] = ((((uint64_t)k.bucket << be) | k.e) << bs) | k.s;
    } else {
      hi[i] = ((k.bucket & 0xffffffffull) << 32) | k.e;
      lo[i] = k.s;
    }
    ix[i] = (uint32_t)i;
  }
  constexpr int DB = 11, NB = 1 << DB;
  cnt.resize(NB + 1);
  const int words = one_word ? 1 : 2;
  for (int w = 0; w < words; ++w) {
    const int width = w == 0 ? (one_word ? bb + be + bs : 32) : 64;
    for (int shift = 0; shift < width; shift += DB) {
      std::vector<uint64_t> &src = w == 0 ? lo : hi;
      std::vector<uint64_t> &dst = w == 0 ? lo2 : hi2;
      std::fill(cnt.begin(), cnt.end(), 0u);
      for (size_t i = 0; i < m; ++i) ++cnt[((src[i] >> shift) & (NB - 1)) + 1];
      if (cnt[((src[0] >> shift) & (NB - 1)) + 1] == m) continue;  // one digit value: order unchanged
      for (int d = 0; d < NB; ++d) cnt[d + 1] += cnt[d];
      for (size_t i = 0; i < m; ++i) {
        const uint32_t pos = cnt[(src[i] >> shift) & (NB - 1)]++;
        dst[pos] = src[i];
        ix2[pos] = ix[i];
        if (w == 0 && !one_word) hi2[pos] = hi[i];
        if (w == 1) lo2[pos] = lo[i];
      }
      src.swap(dst);
      if (w == 0 && !one_word) hi.swap(hi2);
      if (w == 1) lo.swap(lo2);
      ix.swap(ix2);
    }
  }
  auto &out = W.out;
  out.resize(m);
  for (size_t i = 0; i < m; ++i) out[i] = keys[ix[i]];
  std::copy(out.begin(), out.end(), keys);
}

// Sorts plan keys by (order, cls, bucket, e, s, qi): a stable partition by
// class in (order, cls) order -- classes 0 and 2 on the time order, then 1
// and 3 on the category order -- and the classes' own sorts side by side
// on host threads.  Class 0 (no predicate) needs none: its keys are equal.
void sort_keys(std::vector<PlanKey> &keys, Plan &P) {
  const size_t m = keys.size();
  if (m < 2) return;
  static const int rank_of_cls[4] = {0, 2, 1, 3};  // (order, cls) order of the classes
  size_t start[5] = {0, 0, 0, 0, 0};
  for (const PlanKey &k : keys) ++start[rank_of_cls[k.cls & 3] + 1];
  for (int r = 0; r < 4; ++r) start[r + 1] += start[r];
  auto &part = P.w_keys2;
  part.resize(m);
  size_t fill[4] = {start[0], start[1], start[2], start[3]};
  for (const PlanKey &k : keys) part[fill[rank_of_cls[k.cls & 3]]++] = k;
  keys.swap(part);
  std::vector<std::thread> pool;
  for (int r = 1; r < 4; ++r) {
    const size_t len = start[r + 1] - start[r];
    if (len < 2) continue;
    if (len < 4096 || pool.size() == 2) {
      sort_class(keys.data() + start[r], len, P.w_sort[r]);
    } else {
      pool.emplace_back(sort_class, keys.data() + start[r], len, std::ref(P.w_sort[r]));
    }
  }
  for (auto &t : pool) t.join();
}

}  // namespace

void make_plan(const QueryDesc *desc, const float *meta_host, uint32_t nq, uint64_t n, const PlanShape &shape,
               Plan &P) {
  const int TQ = shape.tq, BLK = shape.blk_rows;
  P.reset();
  std::vector<uint32_t> &big = P.w_big;
  big.clear();
  for (uint32_t i = 0; i < nq; ++i) {
    const uint32_t len = desc[i].e - desc[i].s;
    P.pairs_passing += len;
    if (len <= (uint32_t)shape.small_slab) {
      P.small.push_back(i);
    } else {
      big.push_back(i);
      P.pairs_contraction += len;
    }
  }
  if (big.empty()) return;
  // start buckets: about sqrt(#queries/64) per class so a tile spans little
  const uint64_t nb_all = std::max<uint64_t>(1, (uint64_t)std::sqrt((double)big.size() / 64.0));
  const uint64_t bw = std::max<uint64_t>(BLK, (n + nb_all - 1) / nb_all);
  using Key = PlanKey;
  std::vector<Key> &keys = P.w_keys;
  keys.resize(big.size());
  for (size_t j = 0; j < big.size(); ++j) {
    const uint32_t i = big[j];
    const QueryDesc &d = desc[i];
    Key kk;
    kk.order = (uint32_t)d.order;
    kk.cls = (uint32_t)meta_host[(size_t)i * 4];
    kk.bucket = (kk.cls == 2 || kk.cls == 3) ? d.s / bw : 0;
    kk.s = d.s;
    kk.e = d.e;
    kk.qi = i;
    keys[j] = kk;
  }
  sort_keys(keys, P);
  // greedy tiles
  using TileTmp = PlanTile;
  std::vector<TileTmp> &tt = P.w_tiles;
  tt.clear();
  size_t i = 0;
  while (i < keys.size()) {
    TileTmp t{(uint32_t)i, 1, keys[i].s, keys[i].e, keys[i].order};
    uint32_t maxlen = keys[i].e - keys[i].s;
    size_t j = i + 1;
    while (j < keys.size() && t.count < TQ && keys[j].order == keys[i].order && keys[j].cls == keys[i].cls &&
           keys[j].bucket == keys[i].bucket) {
      const uint32_t S = std::min(t.S, keys[j].s), E = std::max(t.E, keys[j].e);
      const uint32_t ml = std::max(maxlen, keys[j].e - keys[j].s);
      if ((uint64_t)(E - S) > (uint64_t)ml + std::max<uint64_t>(ml / 3, 8192)) break;
      t.S = S;
      t.E = E;
      maxlen = ml;
      ++t.count;
      ++j;
    }
    tt.push_back(t);
    i = j;
  }
  // Row chunks per tile.  Every chunk restarts its candidate bound from the
  // shared one, so fewer, longer chunks mean fewer candidate pushes; a tile
  // is split only as far as needed to give every resident CTA slot several
  // work items (shape.target_items in total), and never below
  // min_chunk_blocks blocks or above max_items_per_tile chunks.
  uint64_t total_blk = 0;
  for (auto &t : tt) total_blk += (t.E + BLK - 1) / BLK - t.S / BLK;
  uint64_t cb = std::max<uint64_t>(1, total_blk / std::max<uint32_t>(1, shape.target_items));
  cb = std::max<uint64_t>(cb, shape.min_chunk_blocks);
  const size_t ntile = tt.size();
  P.tiles.resize(ntile);
  P.lane_q.assign(ntile * TQ, -1);
  P.lane_s.assign(ntile * TQ, 0);
  P.lane_e.assign(ntile * TQ, 0);
  P.big.reserve(big.size());
  P.big_tile.reserve(big.size());
  P.big_lane.reserve(big.size());
  std::vector<WorkItem> &items = P.w_items;
  items.clear();
  for (size_t t = 0; t < ntile; ++t) {
    const TileTmp &T = tt[t];
    for (uint32_t l = 0; l < T.count; ++l) {
      const Key &kk = keys[T.first + l];
      P.lane_q[t * TQ + l] = (int32_t)kk.qi;
      P.lane_s[t * TQ + l] = kk.s;
      P.lane_e[t * TQ + l] = kk.e;
      P.big.push_back(kk.qi);
      P.big_tile.push_back((uint32_t)t);
      P.big_lane.push_back(l);
    }
    const uint32_t b0 = T.S / BLK, b1 = (T.E + BLK - 1) / BLK;
    P.tiles[t].order = (int32_t)T.order;
    P.tiles[t].nq = T.count;
    const uint32_t cbt = std::max<uint32_t>((uint32_t)cb, (b1 - b0 + shape.max_items_per_tile - 1) / shape.max_items_per_tile);
    for (uint32_t b = b0; b < b1; b += cbt) {
      WorkItem w;
      w.tile = (uint32_t)t;
      w.blk0 = b;
      w.blk1 = std::min<uint32_t>(b1, b + cbt);
      w.pad = 0;
      items.push_back(w);
      P.pairs_screened += (uint64_t)(w.blk1 - w.blk0) * BLK * TQ;
    }
  }
  // Launch order: longest items first (the grid drains evenly), equal
  // lengths side by side by row range (L2 reuse of the row blocks).  A
  // tile's items are then spread out; the merge finds them through the
  // per-tile slot table built by the caller.
  std::stable_sort(items.begin(), items.end(), [&](const WorkItem &a, const WorkItem &b) {
    const uint32_t la = a.blk1 - a.blk0, lb = b.blk1 - b.blk0;
    if (la != lb) return la > lb;
    if (P.tiles[a.tile].order != P.tiles[b.tile].order) return P.tiles[a.tile].order < P.tiles[b.tile].order;
    return a.blk0 < b.blk0;
  });
  std::vector<uint32_t> &per_tile = P.w_per_tile;
  per_tile.assign(ntile + 1, 0);
  for (auto &w : items) per_tile[w.tile + 1]++;
  for (size_t t = 0; t < ntile; ++t) per_tile[t + 1] += per_tile[t];
  for (size_t t = 0; t < ntile; ++t) {
    P.tiles[t].item0 = per_tile[t];
    P.tiles[t].item1 = per_tile[t + 1];
  }
  P.items.swap(items);
}

int enqueue_query_prep(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, QueryDesc *d_desc,
                       cudaStream_t st) {
  int rc;
  if ((rc = validate_queries(idx, d_q, d_meta, nq, st))) return rc;
  k_query_prep<<<(nq + 255) / 256, 256, 0, st>>>(d_q, d_meta, nq, (uint32_t)idx->n, idx->ord[ORDER_TIME].ts,
                                                 idx->ord[ORDER_CAT].label, idx->ord[ORDER_CAT].ts, d_desc);
  g_launches += 1;
  FKNN_CUDA(cudaGetLastError());
  return FKNN_OK;
}

int check_query_flag_value(int flag) { return check_query_flag(flag); }

int prepare_queries(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, cudaStream_t st,
                    QueryDesc **d_desc_out, QueryDesc **h_desc_out, float **h_meta_out) {
  const uint64_t n = idx->n;
  int rc;
  QueryDesc *d_desc;
  if ((rc = ws_get(idx, 2, (size_t)nq * sizeof(QueryDesc), (void **)&d_desc))) return rc;
  if ((rc = validate_queries(idx, d_q, d_meta, nq, st))) return rc;
  k_query_prep<<<(nq + 255) / 256, 256, 0, st>>>(d_q, d_meta, nq, (uint32_t)n, idx->ord[ORDER_TIME].ts,
                                                 idx->ord[ORDER_CAT].label, idx->ord[ORDER_CAT].ts, d_desc);
  g_launches += 1;
  QueryDesc *h_desc;
  float *h_meta;
  int *h_flag;
  if ((rc = hs_get(idx, 0, (size_t)nq * sizeof(QueryDesc), (void **)&h_desc))) return rc;
  if ((rc = hs_get(idx, 1, (size_t)nq * 16, (void **)&h_meta))) return rc;
  if ((rc = hs_get(idx, 2, 64, (void **)&h_flag))) return rc;
  FKNN_CUDA(cudaMemcpyAsync(h_flag, idx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaMemcpyAsync(h_desc, d_desc, (size_t)nq * sizeof(QueryDesc), cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaMemcpyAsync(h_meta, d_meta, (size_t)nq * 16, cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  if ((rc = check_query_flag(*h_flag))) return rc;
  *d_desc_out = d_desc;
  *h_desc_out = h_desc;
  *h_meta_out = h_meta;
  return FKNN_OK;
}

int launch_exact_scan(fknn_index *idx, const uint32_t *list, const uint32_t *d_count, uint32_t h_count, unsigned grid,
                      const QueryDesc *desc, const float *q, uint32_t k, uint32_t *ids, float *dists, cudaStream_t st) {
  const OrderData &OT = idx->ord[ORDER_TIME], &OC = idx->ord[ORDER_CAT];
  k_exact_scan<<<grid, ES_THREADS, 0, st>>>(list, d_count, h_count, desc, q, OT.blocks, OC.blocks, OT.perm, OC.perm, k,
                                            ids, dists);
  g_launches += 1;
  FKNN_CUDA(cudaGetLastError());
  return FKNN_OK;
}

// The row-by-row exact scan of every query whose slab has at most
// SMALL_SLAB rows needs only the slabs, so it starts before the host plan,
// on the index's side stream (ordered after everything already on st), and
// runs while the host plans the rest.  Its rows of ids / dists are disjoint
// from the contraction's.  join_small_scans orders st after it.
int launch_small_scans(fknn_index *idx, const QueryDesc *h_desc, const QueryDesc *d_desc, uint32_t nq,
                       const float *d_q, uint32_t k, uint32_t *d_ids, float *d_dists, cudaStream_t st,
                       uint32_t *nsmall) {
  int rc;
  *nsmall = 0;
  uint32_t *h_list, *d_list;
  if ((rc = hs_get(idx, 4, (size_t)nq * 4 + 64, (void **)&h_list))) return rc;
  uint32_t m = 0;
  for (uint32_t i = 0; i < nq; ++i)
    if (h_desc[i].e - h_desc[i].s <= (uint32_t)SMALL_SLAB) h_list[m++] = i;
  *nsmall = m;
  if (!m) return FKNN_OK;
  if ((rc = ws_get(idx, 12, (size_t)m * 4 + 64, (void **)&d_list))) return rc;
  if (!idx->side_stream) FKNN_CUDA(cudaStreamCreateWithFlags(&idx->side_stream, cudaStreamNonBlocking));
  if (!idx->ev_fork) FKNN_CUDA(cudaEventCreateWithFlags(&idx->ev_fork, cudaEventDisableTiming));
  if (!idx->ev_join) FKNN_CUDA(cudaEventCreateWithFlags(&idx->ev_join, cudaEventDisableTiming));
  FKNN_CUDA(cudaEventRecord(idx->ev_fork, st));
  FKNN_CUDA(cudaStreamWaitEvent(idx->side_stream, idx->ev_fork, 0));
  FKNN_CUDA(cudaMemcpyAsync(d_list, h_list, (size_t)m * 4, cudaMemcpyHostToDevice, idx->side_stream));
  if ((rc = launch_exact_scan(idx, d_list, nullptr, m, std::min<uint32_t>(m, 148 * 8), d_desc, d_q, k, d_ids,
                              d_dists, idx->side_stream)))
    return rc;
  FKNN_CUDA(cudaEventRecord(idx->ev_join, idx->side_stream));
  return FKNN_OK;
}

int join_small_scans(fknn_index *idx, cudaStream_t st) {
  if (idx->ev_join) FKNN_CUDA(cudaStreamWaitEvent(st, idx->ev_join, 0));
  return FKNN_OK;
}

int launch_fill_u32(uint32_t *p, uint32_t n, uint32_t v, cudaStream_t st) {
  k_fill_u32<<<std::min<uint32_t>((n + 255) / 256, 1024), 256, 0, st>>>(p, n, v);
  g_launches += 1;
  FKNN_CUDA(cudaGetLastError());
  return FKNN_OK;
}

int search_exact(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k, uint32_t *d_ids,
                 float *d_dists, cudaStream_t st, fknn_search_stats *stats) {
  const uint64_t n = idx->n;
  int rc;
  // 1. validate + resolve slabs
  QueryDesc *d_desc, *h_desc;
  float *h_meta;
  if ((rc = prepare_queries(idx, d_q, d_meta, nq, st, &d_desc, &h_desc, &h_meta))) return rc;
  uint32_t nsmall_early = 0;
  if ((rc = launch_small_scans(idx, h_desc, d_desc, nq, d_q, k, d_ids, d_dists, st, &nsmall_early))) return rc;

  // 2. plan
  auto t0 = std::chrono::steady_clock::now();
  Plan &P = idx->plan;
  PlanShape shape;
  shape.tq = TQ;
  shape.blk_rows = BLK;
  shape.small_slab = SMALL_SLAB;
  shape.max_items_per_tile = MAX_ITEMS_PER_TILE;
  shape.min_chunk_blocks = idx->tuning[FKNN_MODE_EXACT_FP32].min_chunk_blocks;
  shape.target_items = idx->num_sms * idx->tuning[FKNN_MODE_EXACT_FP32].items_per_sm;
  make_plan(h_desc, h_meta, nq, n, shape, P);
  auto t1 = std::chrono::steady_clock::now();
  const uint32_t ntile = (uint32_t)P.tiles.size(), nitems = (uint32_t)P.items.size();
  const uint32_t nbig = (uint32_t)P.big.size(), nsmall = (uint32_t)P.small.size();

  // item slots: the merge reads a tile's lists through tile.item0..item1 of
  // a slot table, the screen writes each item's lists at its launch slot.
  std::vector<uint32_t> &slot_of_tile_item = P.w_slot;
  slot_of_tile_item.resize(nitems);
  {
    std::vector<uint32_t> &fill = P.w_fill;
    fill.resize(ntile);
    for (uint32_t t = 0; t < ntile; ++t) fill[t] = P.tiles[t].item0;
    for (uint32_t s = 0; s < nitems; ++s) slot_of_tile_item[fill[P.items[s].tile]++] = s;
  }

  // 3. upload the plan as one blob
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = align_up(off + bytes, 256);
    return o;
  };
  const size_t o_small = take(nsmall * 4), o_big = take(nbig * 4), o_btile = take(nbig * 4),
               o_blane = take(nbig * 4), o_tiles = take(ntile * sizeof(Tile)), o_items = take(nitems * sizeof(WorkItem)),
               o_lq = take((size_t)ntile * TQ * 4), o_ls = take((size_t)ntile * TQ * 4),
               o_le = take((size_t)ntile * TQ * 4), o_slot = take(nitems * 4);
  const size_t blob = off;
  unsigned char *h_blob, *d_blob;
  if ((rc = hs_get(idx, 3, blob + 256, (void **)&h_blob))) return rc;
  if ((rc = ws_get(idx, 3, blob + 256, (void **)&d_blob))) return rc;
  auto put = [&](size_t o, const void *src, size_t bytes) {
    if (bytes) std::memcpy(h_blob + o, src, bytes);
  };
  put(o_small, P.small.data(), nsmall * 4);
  put(o_big, P.big.data(), nbig * 4);
  put(o_btile, P.big_tile.data(), nbig * 4);
  put(o_blane, P.big_lane.data(), nbig * 4);
  put(o_tiles, P.tiles.data(), ntile * sizeof(Tile));
  put(o_items, P.items.data(), nitems * sizeof(WorkItem));
  put(o_lq, P.lane_q.data(), (size_t)ntile * TQ * 4);
  put(o_ls, P.lane_s.data(), (size_t)ntile * TQ * 4);
  put(o_le, P.lane_e.data(), (size_t)ntile * TQ * 4);
  put(o_slot, slot_of_tile_item.data(), nitems * 4);
  if (blob) FKNN_CUDA(cudaMemcpyAsync(d_blob, h_blob, blob, cudaMemcpyHostToDevice, st));

  // per-query state: bound, overflow flag, overflow list + count
  uint32_t *d_state;
  if ((rc = ws_get(idx, 5, (size_t)nq * 12 + 64, (void **)&d_state))) return rc;
  uint32_t *T_global = d_state, *ovf = d_state + nq, *ovf_list = d_state + 2 * (size_t)nq,
           *ovf_count = d_state + 3 * (size_t)nq;
  // bounds start at +inf (as an order-preserving integer image)
  k_fill_u32<<<std::min<uint32_t>((nq + 255) / 256, 1024), 256, 0, st>>>(T_global, nq, f32_sortable(INFINITY));
  g_launches += 1;
  FKNN_CUDA(cudaMemsetAsync(ovf, 0, (size_t)nq * 4, st));
  FKNN_CUDA(cudaMemsetAsync(ovf_count, 0, 4, st));

  const OrderData &OT = idx->ord[ORDER_TIME], &OC = idx->ord[ORDER_CAT];
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  if (stats) {
    for (auto &e : ev) FKNN_CUDA(cudaEventCreate(&e));
  }
  if (nitems) {
    float *d_qt;
    Candidate *d_out;
    uint32_t *d_ocnt;
    if ((rc = ws_get(idx, 4, (size_t)ntile * BLK_BYTES, (void **)&d_qt))) return rc;
    if ((rc = ws_get(idx, 6, (size_t)nitems * TQ * CAP * sizeof(Candidate), (void **)&d_out))) return rc;
    if ((rc = ws_get(idx, 7, (size_t)nitems * TQ * 4, (void **)&d_ocnt))) return rc;
    k_tile_stage<<<ntile, 256, 0, st>>>(d_q, d_desc, (const int32_t *)(d_blob + o_lq), d_qt);
    const size_t smem = sizeof(ScreenSmem);
    // per device context, so set on every call (cheap)
    FKNN_CUDA(cudaFuncSetAttribute(k_screen, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    FKNN_CUDA(cudaFuncSetAttribute(k_merge, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MergeSmem)));
    if (stats) FKNN_CUDA(cudaEventRecord(ev[0], st));
    const uint32_t pstride = idx->tuning[FKNN_MODE_EXACT_FP32].pilot_stride;
    if (pstride > 1) {
      // Pilot: the same screen over every pstride-th row block.  Each list's
      // k-th screening distance (widened by screen_hi) bounds the k-th
      // reference distance of its query from above -- the k-th smallest of
      // a subset is never below the k-th smallest of the whole slab -- so the
      // bounds it leaves in T_global are valid seeds and the main pass keeps
      // every row that can be in the top k.  Its overflow marks are its own.
      uint32_t *ovf_p;
      if ((rc = ws_get(idx, 13, (size_t)nq * 4, (void **)&ovf_p))) return rc;
      FKNN_CUDA(cudaMemsetAsync(ovf_p, 0, (size_t)nq * 4, st));
      k_screen<<<nitems, SC_THREADS, smem, st>>>(
          (const WorkItem *)(d_blob + o_items), (const Tile *)(d_blob + o_tiles), d_qt,
          (const int32_t *)(d_blob + o_lq), (const uint32_t *)(d_blob + o_ls), (const uint32_t *)(d_blob + o_le),
          OT.blocks, OC.blocks, T_global, ovf_p, d_out, d_ocnt, k, pstride, idx->d_flag);
      g_launches += 1;
    }
    k_screen<<<nitems, SC_THREADS, smem, st>>>(
        (const WorkItem *)(d_blob + o_items), (const Tile *)(d_blob + o_tiles), d_qt, (const int32_t *)(d_blob + o_lq),
        (const uint32_t *)(d_blob + o_ls), (const uint32_t *)(d_blob + o_le), OT.blocks, OC.blocks, T_global, ovf,
        d_out, d_ocnt, k, 1u, idx->d_flag);
    if (stats) FKNN_CUDA(cudaEventRecord(ev[1], st));
    k_merge<<<nbig, MG_THREADS, sizeof(MergeSmem), st>>>(
        (const uint32_t *)(d_blob + o_big), (const uint32_t *)(d_blob + o_btile), (const uint32_t *)(d_blob + o_blane),
        (const Tile *)(d_blob + o_tiles), (const uint32_t *)(d_blob + o_slot), d_out, d_ocnt, d_desc, d_q, idx->vecs,
        OT.perm, OC.perm, T_global, ovf, ovf_list, ovf_count, k, d_ids, d_dists);
    g_launches += 3;
  }
  if (stats) FKNN_CUDA(cudaEventRecord(ev[2], st));
  if (nbig) {
    k_exact_scan<<<148 * 2, ES_THREADS, 0, st>>>(ovf_list, ovf_count, 0, d_desc, d_q, OT.blocks, OC.blocks, OT.perm,
                                                 OC.perm, k, d_ids, d_dists);
    g_launches += 1;
  }
  if (nsmall_early && (rc = join_small_scans(idx, st))) return rc;
  FKNN_CUDA(cudaGetLastError());
  if (stats) {
    FKNN_CUDA(cudaEventRecord(ev[3], st));
    FKNN_CUDA(cudaEventSynchronize(ev[3]));
    float ms = 0.f;
    if (nitems) {
      FKNN_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
      stats->ms_screen = ms;
      FKNN_CUDA(cudaEventElapsedTime(&ms, ev[1], ev[2]));
      stats->ms_merge = ms;
    }
    FKNN_CUDA(cudaEventElapsedTime(&ms, ev[2], ev[3]));
    stats->ms_scan = ms;
    for (auto &e : ev) cudaEventDestroy(e);
    stats->pairs_screened = P.pairs_screened;
    stats->pairs_passing = P.pairs_passing;
    stats->pairs_contraction = P.pairs_contraction;
    stats->n_tiles = ntile;
    stats->n_work_items = nitems;
    stats->n_small = nsmall;
    stats->ms_plan = std::chrono::duration<float, std::milli>(t1 - t0).count();
    uint32_t h_ovf = 0;
    FKNN_CUDA(cudaMemcpyAsync(&h_ovf, ovf_count, 4, cudaMemcpyDeviceToHost, st));
    FKNN_CUDA(cudaStreamSynchronize(st));
    stats->n_overflow = h_ovf;
  }
  return FKNN_OK;
}

}  // namespace fknn

// ===================================================== no-allocation form
//
// fknn_filter_rows_noalloc: the predicate-compaction kernels above, for
// callers that must not allocate device memory.  Their only scratch (one
// counter per 4096-row tile plus the total) lives in the fixed array below,
// which the module holds on every GPU that loads this library until the
// process exits.

namespace fknn {

constexpr uint32_t NOALLOC_FILTER_MAX_TILES = 1u << 16;  // 65,536 tiles x 4,096 rows = 268,435,456 rows
constexpr uint64_t NOALLOC_FILTER_MAX_ROWS = (uint64_t)NOALLOC_FILTER_MAX_TILES * FC_TILE;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) uint32_t g_noalloc_filter_scratch[NOALLOC_FILTER_MAX_TILES + 1];

static std::mutex g_noalloc_mu;
static uint32_t *g_noalloc_ptr[NOALLOC_MAX_DEVICES];

// Device address of the scratch array on the current device.  The array's
// name in host code is only a host-side handle, so the address is looked up
// once per device (with that device current) and cached.
static int noalloc_scratch(uint32_t **out) {
  int dev = 0;
  FKNN_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
    set_error("fknn_filter_rows_noalloc: device ordinal above 63");
    return FKNN_EINVAL;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_filter_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_filter_scratch)");
    g_noalloc_ptr[dev] = static_cast<uint32_t *>(p);
  }
  *out = g_noalloc_ptr[dev];
  return FKNN_OK;
}

// True for device memory of device `dev` and for managed memory; false for
// host memory and for another GPU's memory (its kernels would read a peer's
// memory, which faults without peer access).
static bool on_device(const void *p, int dev) { return mem_loc(p, dev) == MemLoc::Here; }

}  // namespace fknn

extern "C" int fknn_filter_rows_noalloc(const float *labels, const float *ts, uint64_t n, const float *meta4,
                                        uint32_t *out_ids, uint64_t *count, void *stream) {
  using namespace fknn;
  g_launches = 0;
  if (!labels || !ts || !meta4 || !out_ids || !count) {
    set_error("fknn_filter_rows_noalloc: NULL argument");
    return FKNN_EINVAL;
  }
  if (n > NOALLOC_FILTER_MAX_ROWS) {
    set_error("fknn_filter_rows_noalloc: n = " + std::to_string(n) + " exceeds the fixed scratch limit of " +
              std::to_string(NOALLOC_FILTER_MAX_ROWS) + " rows (65,536 tiles of 4,096)");
    return FKNN_EINVAL;
  }
  const float t = meta4[0];
  if (!(t == 0.f || t == 1.f || t == 2.f || t == 3.f)) {
    set_error("fknn_filter_rows_noalloc: query type not in {0,1,2,3}");
    return FKNN_EINVAL;
  }
  if ((t == 1.f || t == 3.f) && !(fabsf(meta4[1]) < 2147483648.f)) {
    set_error("fknn_filter_rows_noalloc: category outside int32");
    return FKNN_EINVAL;
  }
  *count = 0;
  if (n == 0) return FKNN_OK;
  int cur = 0;
  FKNN_CUDA(cudaGetDevice(&cur));
  if (!on_device(labels, cur) || !on_device(ts, cur) || !on_device(out_ids, cur)) {
    set_error("fknn_filter_rows_noalloc: labels, ts and out_ids must be device memory of the current device");
    return FKNN_EINVAL;
  }
  uint32_t *tc = nullptr;
  int rc = noalloc_scratch(&tc);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t ntiles = (uint32_t)((n + FC_TILE - 1) / FC_TILE);
  const float4 m = make_float4(meta4[0], meta4[1], meta4[2], meta4[3]);
  // every tile counter and the total are rewritten by this call, so nothing
  // left in the array by an earlier call is read
  k_filter_count<<<ntiles, FC_THREADS, 0, st>>>(labels, ts, n, m, tc);
  k_exclusive_scan_small<<<1, 1024, 0, st>>>(tc, ntiles, tc + ntiles);
  k_filter_write<<<ntiles, FC_THREADS, 0, st>>>(labels, ts, n, m, tc, out_ids);
  g_launches += 3;
  FKNN_CUDA(cudaGetLastError());
  uint32_t tot = 0;
  FKNN_CUDA(cudaMemcpyAsync(&tot, tc + ntiles, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  *count = tot;
  return FKNN_OK;
}
