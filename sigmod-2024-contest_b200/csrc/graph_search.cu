// Batched graph beam search: the B200 form of the pyglass Searcher
// (pyglass/glass/searcher.hpp:162-569) over the reference's saved graphs.
//
// One warp runs one query at a time and replays the reference step for step,
// so on the same graph it returns the same ids:
//   * LinearPool (pyglass/glass/neighbor.hpp:223-283): a sorted array of
//     capacity max(k, ef) plus one overflow slot, zero-initialised; insertion
//     after equal distances (upper bound) with a shift of the tail; bit 31 of
//     the id is the checked flag and `cur` the first unchecked slot.  It
//     lives in shared memory.
//   * Bitset vis / vis1 (neighbor.hpp:41-102): lazily cleared 512-bit blocks;
//     the block flags are in shared memory, the bits in a per-warp global
//     bitmap read through L2.
//   * HNSWInitializer::initialize (HNSWInitializer.hpp:36-58): greedy descent
//     through the upper layers, the scanned list fixed for each pass.
//   * Distances: L2SqrSQ8_sym on the searcher's symmetric SQ8 codes, exact
//     int32.  The neighbours of a node are screened lane-parallel (visited
//     test, edge timestamp, distance) and then inserted one by one in
//     adjacency order, which is the order the reference inserts them in.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "device_util.cuh"

struct fknn_graph {
  int device = 0;
  uint32_t n = 0, K = 0, upK = 1, nep = 0;
  int32_t ep = -1;
  int32_t *adj = nullptr;     // [n][K] neighbour ids, -1 padded
  float *ets = nullptr;       // [n][K] edge timestamps
  int32_t *levels = nullptr;  // [n] upper-layer count per node
  int64_t *up_off = nullptr;  // [n + 1] offsets into up
  int32_t *up = nullptr;      // per node levels * upK ids, level 1 first
  int32_t *eps = nullptr;     // [nep] entry points (graphs without upper layers)
  int8_t *codes = nullptr;    // [n][112] symmetric SQ8 codes
  float alpha = 0.f;
  // per-call scratch, grown on demand
  float *io = nullptr;        // staged queries, bounds, outputs
  size_t io_cap = 0;
  int8_t *qcodes = nullptr;
  size_t qcodes_cap = 0;
  uint64_t *vis = nullptr;    // per warp slot: two bitmaps of nwords words
  size_t vis_cap = 0;
  int *dflag = nullptr;
};

namespace fknn {
namespace {

constexpr int GS_WARPS = 4;  // warps per block, one query in flight each
constexpr int CODE = 112;    // SQ8 code bytes per point (100 dims aligned to 16)
constexpr int EF_DEFAULT = 32;
constexpr uint32_t CAP_MAX = 4096;
constexpr int GS_OCC_BLOCKS = 8;                 // blocks per SM of the register-capped variant
constexpr int GS_BASE_BLOCKS = 6;                // ... and of the default one (the registers it needs)
constexpr size_t GS_SMEM_PER_SM = 228 * 1024;    // shared memory of an SM
constexpr size_t VIS_BUDGET = 4ull << 30;  // bytes of visited bitmaps across all warp slots

struct Slot {  // one LinearPool entry; bit 31 of id = checked
  int d;
  int id;
};

struct GParams {
  const int32_t *adj;
  const float *ets;
  const int32_t *levels;
  const int64_t *up_off;
  const int32_t *up;
  const int32_t *eps;
  const int8_t *codes;
  uint32_t n, K, upK, nep;
  int32_t ep;
  float alpha2;
  const int8_t *qcodes;
  uint32_t nq;
  int mode;
  uint32_t cap, refine;
  bool batch;  // refine <= cap: the overflow slot is never read, inserts may be batched
  const float *bounds;
  const int32_t *id_bounds;
  int32_t *out_ids;
  float *out_dists;
  uint64_t *vis;
  uint32_t nwords;  // 64-bit words per bitmap: whole 512-bit blocks
  uint32_t nblkw;   // 32-bit words of block flags per bitmap
  int *err;
};

struct Warp {
  Slot *pool;
  uint32_t *chg;   // block flags [2][nblkw]
  int *qw;         // query code as 28 words
  int *cand;       // sorted candidate distances of a batch insert (32)
  uint64_t *mass;  // bitmaps [2][nwords]
  int qq;
  uint32_t size, cur;
};

__host__ __device__ inline size_t pool_bytes(uint32_t cap) {
  return ((size_t)(cap + 1) * sizeof(Slot) + 15) & ~(size_t)15;
}

__host__ __device__ inline size_t warp_smem_bytes(uint32_t cap, uint32_t nblkw) {
  return pool_bytes(cap) + 2 * (size_t)nblkw * 4 + CODE + 32 * sizeof(int);
}

__device__ __forceinline__ int gdist(const GParams &P, const Warp &W, uint32_t v) {
  return sq8_dist(W.qw, W.qq, P.codes + (uint64_t)v * CODE);
}

// Bitset::get (neighbor.hpp:88-92) of set b (0 = vis, 1 = vis1).
__device__ __forceinline__ bool vis_get(const GParams &P, const Warp &W, int b, uint32_t v) {
  const uint32_t blk = v >> 9;
  if (!((W.chg[b * P.nblkw + (blk >> 5)] >> (blk & 31)) & 1u)) return false;
  return (__ldcg(reinterpret_cast<const unsigned long long *>(W.mass + (uint64_t)b * P.nwords + (v >> 6))) >>
          (v & 63)) & 1ull;
}

// Bitset::set (neighbor.hpp:80-87) for the lanes with `on`, whole warp: a
// block seen for the first time is cleared, then (after the warp barrier
// that orders the clears) the bits are set.
__device__ __forceinline__ void vis_set(const GParams &P, const Warp &W, int b, uint32_t v, bool on) {
  uint64_t *m = W.mass + (uint64_t)b * P.nwords;
  if (on) {
    const uint32_t blk = v >> 9, bit = 1u << (blk & 31);
    if (!(atomicOr(&W.chg[b * P.nblkw + (blk >> 5)], bit) & bit)) {
#pragma unroll
      for (int w = 0; w < 8; ++w) __stcg(reinterpret_cast<unsigned long long *>(m + (uint64_t)blk * 8 + w), 0ull);
    }
  }
  __syncwarp();
  if (on) atomicOr(reinterpret_cast<unsigned long long *>(m + (v >> 6)), 1ull << (v & 63));
  __syncwarp();
}

// LinearPool::insert (neighbor.hpp:240-255), whole warp, warp-uniform arguments.
__device__ void pool_insert(Warp &W, uint32_t cap, int u, int d) {
  const int lane = threadIdx.x & 31;
  if (W.size == cap && d >= W.pool[W.size - 1].d) return;
  uint32_t lo = 0, hi = W.size;  // first slot whose distance exceeds d
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (W.pool[mid].d > d) hi = mid;
    else lo = mid + 1;
  }
  // move [lo, size) up one slot, top chunk first (slot `size` may be the overflow slot)
  for (int top = (int)W.size - 1; top >= (int)lo; top -= 32) {
    const int idx = top - lane;
    Slot t;
    if (idx >= (int)lo) t = W.pool[idx];
    __syncwarp();
    if (idx >= (int)lo) W.pool[idx + 1] = t;
    __syncwarp();
  }
  if (lane == 0) {
    Slot s;
    s.d = d;
    s.id = u;
    W.pool[lo] = s;
  }
  __syncwarp();
  if (W.size < cap) ++W.size;
  if (lo < W.cur) W.cur = lo;
}

// LinearPool::pop (neighbor.hpp:259-266), whole warp.
__device__ int pool_pop(Warp &W) {
  const int lane = threadIdx.x & 31;
  const uint32_t pre = W.cur;
  const int raw = W.pool[pre].id;
  __syncwarp();
  if (lane == 0) W.pool[pre].id = raw | (int)0x80000000;
  __syncwarp();
  uint32_t c = pre;
  while (c < W.size) {
    const uint32_t idx = c + lane;
    const uint32_t b = __ballot_sync(0xffffffffu, idx < W.size && W.pool[idx].id >= 0);
    if (b) {
      c += __ffs(b) - 1;
      break;
    }
    c = min(c + 32, W.size);
  }
  W.cur = c;
  return raw & 0x7fffffff;
}

// Lanes of one 32-wide chunk of an adjacency list: `valid` up to the first
// -1, `first` for the earliest lane holding each id (a later copy is already
// visited when the reference reaches it).
struct Chunk {
  int v;
  bool valid, first, end;
};

__device__ __forceinline__ Chunk load_chunk(const int32_t *list, uint32_t len, uint32_t base) {
  const int lane = threadIdx.x & 31;
  Chunk c;
  const uint32_t i = base + lane;
  c.v = i < len ? list[i] : -1;
  const uint32_t endb = __ballot_sync(0xffffffffu, c.v == -1);
  c.end = endb != 0;
  c.valid = endb ? lane < __ffs(endb) - 1 : true;
  const uint32_t same = __match_any_sync(0xffffffffu, c.v);
  c.first = (__ffs(same) - 1) == lane;
  return c;
}

// The lanes of mask m inserted one after another in lane order, in one
// pass over the pool.  Equal distances keep insertion order (the pool's
// upper-bound rule: old entries first, then candidates by lane), so the
// pool's first cap slots, its size and its cursor end as after the one-by-one
// inserts: the pool is the first cap entries of the stable merge, and the
// cursor moves to the first candidate's final slot.  Only the overflow slot
// (slot cap) is not kept, so this is used when it is never read.
__device__ void pool_insert_batch(Warp &W, uint32_t cap, uint32_t m, int v, int d) {
  const int lane = threadIdx.x & 31;
  const int n = __popc(m);
  // warp bitonic sort of the keys (distance, lane); empty lanes sort last
  uint32_t key = (m >> lane) & 1u ? ((uint32_t)d << 5) | (uint32_t)lane : 0xffffffffu;
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1)
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const uint32_t other = __shfl_xor_sync(0xffffffffu, key, stride);
      const bool asc = (lane & size) == 0, lower = (lane & stride) == 0;
      key = (lower == asc) ? min(key, other) : max(key, other);
    }
  const int cd = (int)(key >> 5);
  const int cv = __shfl_sync(0xffffffffu, v, (int)(key & 31));
  if (lane < n) W.cand[lane] = cd;
  __syncwarp();
  // candidate j's final slot: j + pool entries with distance <= d_j
  uint32_t pos = 0xffffffffu;
  if (lane < n) {
    uint32_t lo = 0, hi = W.size;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (W.pool[mid].d > cd) hi = mid;
      else lo = mid + 1;
    }
    pos = (uint32_t)lane + lo;
  }
  const uint32_t first = __shfl_sync(0xffffffffu, pos, 0);  // entries below it do not move
  // old entry i moves up by the number of candidates strictly closer, top chunk first
  for (int top = (int)W.size - 1; top >= (int)first; top -= 32) {
    const int i = top - lane;
    Slot t;
    int ni = (int)cap;
    if (i >= (int)first) {
      t = W.pool[i];
      int a = 0, b = n;
      while (a < b) {
        const int mid = (a + b) >> 1;
        if (W.cand[mid] < t.d) a = mid + 1;
        else b = mid;
      }
      ni = i + a;
    }
    __syncwarp();
    if (ni < (int)cap) W.pool[ni] = t;
    __syncwarp();
  }
  if (pos < cap) {
    Slot sl;
    sl.d = cd;
    sl.id = cv;
    W.pool[pos] = sl;
  }
  __syncwarp();
  W.size = min(W.size + (uint32_t)n, cap);
  if (first < cap && first < W.cur) W.cur = first;
}

// Inserts the lanes of mask m in lane order (the adjacency order).
__device__ __forceinline__ int insert_lanes(const GParams &P, Warp &W, uint32_t m, int v, int d) {
  const int count = __popc(m);
  if (P.batch && count > 1) {
    pool_insert_batch(W, P.cap, m, v, d);
    return count;
  }
  while (m) {
    const int b = __ffs(m) - 1;
    m &= m - 1;
    pool_insert(W, P.cap, __shfl_sync(0xffffffffu, v, b), __shfl_sync(0xffffffffu, d, b));
  }
  return count;
}

// SearchImpl / SearchFilterImpl / SearchFilterSubTimeImpl (searcher.hpp:172-198,
// 271-299, 386-413): every unvisited neighbour is marked and inserted.
// (SearchFilterImpl's `count1 > count2` exit can never fire: both counts
// grow together.)
__device__ void expand_plain(const GParams &P, Warp &W, uint32_t u) {
  const int32_t *list = P.adj + (uint64_t)u * P.K;
  for (uint32_t base = 0; base < P.K; base += 32) {
    const Chunk c = load_chunk(list, P.K, base);
    const bool fresh = c.valid && c.first && !vis_get(P, W, 0, (uint32_t)c.v);
    const int d = fresh ? gdist(P, W, (uint32_t)c.v) : 0;
    vis_set(P, W, 0, (uint32_t)c.v, fresh);
    insert_lanes(P, W, __ballot_sync(0xffffffffu, fresh), c.v, d);
    if (c.end) break;
  }
}

// SearchCategoryRangeImpl (rf = 1, searcher.hpp:320-374) and
// SearchRangeFilter[SubTime]Impl (rf = 2, searcher.hpp:438-491, 516-569): an
// unvisited neighbour is always marked, but inserted only when the edge's
// timestamp lies in [l, r]; while inserts < rf x (unvisited 1-hop
// neighbours), the neighbours' own lists are scanned the same way, stopping
// right after the insert that reaches the bound.
__device__ void expand_filtered(const GParams &P, Warp &W, uint32_t u, float l, float r, int rf) {
  const int lane = threadIdx.x & 31;
  const int32_t *list = P.adj + (uint64_t)u * P.K;
  const float *tlist = P.ets + (uint64_t)u * P.K;
  int count1 = 0, count2 = 0;
  for (uint32_t base = 0; base < P.K; base += 32) {
    const Chunk c = load_chunk(list, P.K, base);
    const bool fresh = c.valid && c.first && !vis_get(P, W, 0, (uint32_t)c.v);
    const float t = fresh ? tlist[base + lane] : 0.f;
    const bool pass = fresh && !(t < l || t > r);
    const int d = pass ? gdist(P, W, (uint32_t)c.v) : 0;
    vis_set(P, W, 0, (uint32_t)c.v, fresh);
    count2 += __popc(__ballot_sync(0xffffffffu, fresh));
    count1 += insert_lanes(P, W, __ballot_sync(0xffffffffu, pass), c.v, d);
    if (c.end) break;
  }
  for (uint32_t i = 0; i < P.K; ++i) {
    if (count1 >= rf * count2) break;
    const int nei = list[i];
    if (nei == -1) break;
    if (vis_get(P, W, 1, (uint32_t)nei)) continue;
    vis_set(P, W, 1, (uint32_t)nei, lane == 0);
    const int32_t *list2 = P.adj + (uint64_t)nei * P.K;
    const float *tlist2 = P.ets + (uint64_t)nei * P.K;
    for (uint32_t base = 0; base < P.K; base += 32) {
      const Chunk c = load_chunk(list2, P.K, base);
      const bool fresh = c.valid && c.first && !vis_get(P, W, 0, (uint32_t)c.v);
      const float t = fresh ? tlist2[base + lane] : 0.f;
      const bool pass = fresh && !(t < l || t > r);
      const uint32_t passm = __ballot_sync(0xffffffffu, pass);
      // the scan stops after the need-th insert: lanes past it are untouched
      const int need = rf * count2 - count1;
      uint32_t upto = 0xffffffffu;
      bool stop = false;
      if (__popc(passm) >= need) {
        uint32_t mm = passm;
        for (int j = 1; j < need; ++j) mm &= mm - 1;
        const int last = __ffs(mm) - 1;
        upto = last == 31 ? 0xffffffffu : ((2u << last) - 1u);
        stop = true;
      }
      const bool mine = (upto >> lane) & 1u;
      const int d = (pass && mine) ? gdist(P, W, (uint32_t)c.v) : 0;
      vis_set(P, W, 0, (uint32_t)c.v, fresh && mine);
      count1 += insert_lanes(P, W, passm & upto, c.v, d);
      if (stop || c.end) break;
    }
  }
}

// Graph::initialize_search (graph.hpp:90-99): HNSWInitializer::initialize
// when the graph has upper layers (insert the descent's end, then mark it),
// else every entry point inserted, unmarked.
__device__ void initialize_search(const GParams &P, Warp &W) {
  const int lane = threadIdx.x & 31;
  if (P.ep >= 0) {
    int u = P.ep;
    int cur_dist = gdist(P, W, (uint32_t)u);
    for (int level = P.levels[u]; level > 0; --level) {
      bool changed = true;
      while (changed) {
        changed = false;
        const int32_t *list = P.up + P.up_off[u] + (int64_t)(level - 1) * P.upK;
        for (uint32_t base = 0; base < P.upK; base += 32) {
          const uint32_t i = base + lane;
          const int v = i < P.upK ? list[i] : -1;
          const uint32_t endb = __ballot_sync(0xffffffffu, v == -1);
          const bool valid = endb ? lane < __ffs(endb) - 1 : true;
          const int d = valid ? gdist(P, W, (uint32_t)v) : 0;
          uint32_t m = __ballot_sync(0xffffffffu, valid);
          while (m) {  // the reference's sequential scan: a strictly closer point moves u
            const int b = __ffs(m) - 1;
            m &= m - 1;
            const int db = __shfl_sync(0xffffffffu, d, b);
            const int vb = __shfl_sync(0xffffffffu, v, b);
            if (db < cur_dist) {
              cur_dist = db;
              u = vb;
              changed = true;
            }
          }
          if (endb) break;
        }
      }
    }
    pool_insert(W, P.cap, u, cur_dist);
    vis_set(P, W, 0, (uint32_t)u, lane == 0);
  } else {
    for (uint32_t e = 0; e < P.nep; ++e) {
      const int v = P.eps[e];
      pool_insert(W, P.cap, v, gdist(P, W, (uint32_t)v));
    }
  }
}

// Ten evenly spaced seeds of the id range (searcher.hpp:306-313, 421-430,
// 499-508): insert, then mark; a range narrower than ten repeats its start.
__device__ void range_seeds(const GParams &P, Warp &W, int lb, int ub) {
  const int lane = threadIdx.x & 31;
  const int interval = (ub - lb) / 10;
  for (int i = 0; i < 10; ++i) {
    const int point = lb + interval * i;
    pool_insert(W, P.cap, point, gdist(P, W, (uint32_t)point));
    vis_set(P, W, 0, (uint32_t)point, lane == 0);
  }
}

// Registers capped so that MINB blocks fit an SM: GS_OCC_BLOCKS when the
// pools are small enough for that many blocks' shared memory, else
// GS_BASE_BLOCKS (no spills).
template <int MINB>
__global__ void __launch_bounds__(GS_WARPS * 32, MINB) k_graph_search(GParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  unsigned char *mine = smem_raw + wib * warp_smem_bytes(P.cap, P.nblkw);
  Warp W;
  W.pool = reinterpret_cast<Slot *>(mine);
  W.chg = reinterpret_cast<uint32_t *>(mine + pool_bytes(P.cap));
  W.qw = reinterpret_cast<int *>(W.chg + 2 * P.nblkw);
  W.cand = W.qw + 28;
  const uint32_t slot = blockIdx.x * GS_WARPS + wib;
  W.mass = P.vis + (uint64_t)slot * 2 * P.nwords;
  for (uint32_t qi = slot; qi < P.nq; qi += gridDim.x * GS_WARPS) {
    for (uint32_t i = lane; i <= P.cap; i += 32) {
      Slot z;
      z.d = 0;
      z.id = 0;
      W.pool[i] = z;
    }
    for (uint32_t i = lane; i < 2 * P.nblkw; i += 32) W.chg[i] = 0;
    if (lane < 28) W.qw[lane] = reinterpret_cast<const int *>(P.qcodes + (uint64_t)qi * CODE)[lane];
    __syncwarp();
    int qq = 0;
    for (int w = 0; w < 28; ++w) qq = __dp4a(W.qw[w], W.qw[w], qq);
    W.qq = qq;
    W.size = 0;
    W.cur = 0;
    const bool ranged = P.mode >= FKNN_GRAPH_CATEGORY_RANGE;
    const float l = ranged ? P.bounds[2 * (uint64_t)qi] : 0.f;
    const float r = ranged ? P.bounds[2 * (uint64_t)qi + 1] : 0.f;
    const int lb = ranged ? P.id_bounds[2 * (uint64_t)qi] : 0;
    const int ub = ranged ? P.id_bounds[2 * (uint64_t)qi + 1] : 0;
    // float sel = (float)(ub - lb) / nb; seeds only when sel < 1
    const bool partial = __fdiv_rn((float)(ub - lb), (float)P.n) < 1.f;
    const bool seeded = P.mode == FKNN_GRAPH_CATEGORY_RANGE || (P.mode >= FKNN_GRAPH_RANGE_SUBTIME && partial);
    bool bad = false;
    if (seeded) {  // every seed lb + i * ((ub - lb) / 10), i < 10, must be a point
      const long long last = (long long)lb + 9ll * ((ub - lb) / 10);
      bad = lb < 0 || (uint32_t)lb >= P.n || last < 0 || last >= (long long)P.n;
    }
    if (bad) {
      if (lane == 0) atomicOr(P.err, ERR_BAD_QUERY_VALUE);
      for (uint32_t i = lane; i < P.refine; i += 32) {
        P.out_ids[(uint64_t)qi * P.refine + i] = -1;
        if (P.out_dists) P.out_dists[(uint64_t)qi * P.refine + i] = __int_as_float(0x7fc00000);
      }
      __syncwarp();
      continue;
    }
    if (seeded) range_seeds(P, W, lb, ub);
    else if (P.mode != FKNN_GRAPH_RANGE_SUBTIME) initialize_search(P, W);
    // each pop checks one slot; an expansion inserts each point at most once
    // (vis), besides at most ten seeds and the unmarked entry points, so
    // n + nep + 16 pops is a hard bound
    uint32_t pops = 0;
    while (W.cur < W.size) {
      if (++pops > P.n + P.nep + 16) {
        if (lane == 0) atomicOr(P.err, ERR_WAIT_TIMEOUT);
        break;
      }
      const int u = pool_pop(W);
      if (P.mode == FKNN_GRAPH_CATEGORY_RANGE) expand_filtered(P, W, (uint32_t)u, l, r, 1);
      else if (P.mode >= FKNN_GRAPH_RANGE_SUBTIME) expand_filtered(P, W, (uint32_t)u, l, r, 2);
      else expand_plain(P, W, (uint32_t)u);
    }
    // reorder / reorder_dist (sq8_sym_quant.hpp:76-89): slots 0..refine-1 as
    // they stand, ids unmasked, distances times alpha^2
    for (uint32_t i = lane; i < P.refine; i += 32) {
      const Slot s = W.pool[i];
      P.out_ids[(uint64_t)qi * P.refine + i] = s.id & 0x7fffffff;
      if (P.out_dists) P.out_dists[(uint64_t)qi * P.refine + i] = __fmul_rn((float)s.d, P.alpha2);
    }
    __syncwarp();
  }
}

}  // namespace

int graph_codes(const fknn_graph *g, const int8_t **codes, float *alpha, uint32_t *n) {
  *codes = g->codes;
  *alpha = g->alpha;
  *n = g->n;
  return FKNN_OK;
}

namespace {

template <typename T>
int grow(T **p, size_t *cap, size_t want) {
  if (*cap >= want) return FKNN_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  FKNN_CUDA(cudaMalloc((void **)p, want * sizeof(T)));
  *cap = want;
  return FKNN_OK;
}

bool on_device(const void *p, int dev) { return mem_loc(p, dev) == MemLoc::Here; }

void free_graph(fknn_graph *g) {
  if (!g) return;
  cudaSetDevice(g->device);
  cudaDeviceSynchronize();
  cudaFree(g->adj);
  cudaFree(g->ets);
  cudaFree(g->levels);
  cudaFree(g->up_off);
  cudaFree(g->up);
  cudaFree(g->eps);
  cudaFree(g->codes);
  cudaFree(g->io);
  cudaFree(g->qcodes);
  cudaFree(g->vis);
  cudaFree(g->dflag);
  delete g;
}

int upload(void **dst, const void *src, size_t bytes) {
  FKNN_CUDA(cudaMalloc(dst, bytes ? bytes : 16));
  if (bytes) FKNN_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
  return FKNN_OK;
}

// Parsed Graph::save bytes (graph.hpp:101-115, HNSWInitializer.hpp:73-82).
struct HostGraph {
  std::vector<int32_t> eps, adj, levels, up;
  std::vector<float> ets;
  std::vector<int64_t> up_off;
  int32_t N = 0, K = 0, upK = 0, ep = -1;
};

bool parse_graph(const unsigned char *b, size_t nbytes, HostGraph &h) {
  size_t off = 0;
  auto rd = [&](void *dst, size_t bytes) {
    if (bytes > nbytes - off) return false;
    std::memcpy(dst, b + off, bytes);
    off += bytes;
    return true;
  };
  int32_t nep = 0;
  if (!rd(&nep, 4) || nep < 0 || (size_t)nep > nbytes / 4) return false;
  h.eps.resize(nep);
  if (nep && !rd(h.eps.data(), (size_t)nep * 4)) return false;
  if (!rd(&h.N, 4) || !rd(&h.K, 4) || h.N <= 0 || h.K <= 0 || h.K > 1024) return false;
  const size_t nk = (size_t)h.N * h.K;
  if (nk > (nbytes - off) / 8) return false;
  h.adj.resize(nk);
  h.ets.resize(nk);
  rd(h.adj.data(), nk * 4);
  rd(h.ets.data(), nk * 4);
  for (int32_t v : h.adj)
    if (v < -1 || v >= h.N) return false;
  for (int32_t v : h.eps)
    if (v < 0 || v >= h.N) return false;
  if (off == nbytes) return nep > 0;  // no initializer: the entry points seed the search
  int32_t iN = 0;
  if (!rd(&iN, 4) || !rd(&h.upK, 4) || !rd(&h.ep, 4)) return false;
  if (iN != h.N || h.upK <= 0 || h.upK > 1024 || h.ep < 0 || h.ep >= h.N) return false;
  h.levels.resize(h.N);
  h.up_off.resize((size_t)h.N + 1);
  h.up_off[0] = 0;
  for (int32_t i = 0; i < h.N; ++i) {
    int32_t cur = 0;
    if (!rd(&cur, 4) || cur < 0 || cur % h.upK) return false;
    h.levels[i] = cur / h.upK;
    const size_t at = h.up.size();
    if ((size_t)cur > (nbytes - off) / 4) return false;
    h.up.resize(at + cur);
    if (cur) rd(h.up.data() + at, (size_t)cur * 4);
    h.up_off[i + 1] = (int64_t)h.up.size();
  }
  // a level-L list may only name points that exist at level L (the descent
  // reads the named point's own level-L list next)
  for (int32_t i = 0; i < h.N; ++i)
    for (int64_t j = h.up_off[i]; j < h.up_off[i + 1]; ++j) {
      const int32_t v = h.up[j];
      const int32_t level = (int32_t)((j - h.up_off[i]) / h.upK) + 1;
      if (v < -1 || v >= h.N || (v >= 0 && h.levels[v] < level)) return false;
    }
  return off == nbytes;
}

}  // namespace
}  // namespace fknn

using namespace fknn;

namespace fknn {

// The argument checks of fknn_graph_search; *cap = the pool capacity.
int graph_check_args(const fknn_graph *g, const float *queries, uint32_t nq, int mode, uint32_t k, uint32_t ef,
                     uint32_t refine, const float *bounds, const int32_t *id_bounds, const int32_t *out_ids,
                     uint32_t *cap) {
  (void)nq;
  if (!g || !queries || !out_ids) {
    set_error("fknn_graph_search: NULL argument");
    return FKNN_EINVAL;
  }
  if (mode < FKNN_GRAPH_SEARCH || mode > FKNN_GRAPH_RANGE) {
    set_error("fknn_graph_search: unknown mode");
    return FKNN_EINVAL;
  }
  if (ef == 0) ef = EF_DEFAULT;
  *cap = std::max(k, ef);  // LinearPool(nb, max(k, ef), k)
  if (k == 0 || *cap > CAP_MAX || refine == 0 || refine > *cap + 1) {
    set_error("fknn_graph_search: need 1 <= k, max(k, ef) <= 4096 and 1 <= refine <= max(k, ef) + 1");
    return FKNN_EINVAL;
  }
  if (mode == FKNN_GRAPH_SEARCH && refine != k) {
    set_error("fknn_graph_search: mode 0 (Search) writes k ids; refine must equal k");
    return FKNN_EINVAL;
  }
  if (mode >= FKNN_GRAPH_CATEGORY_RANGE && (!bounds || !id_bounds)) {
    set_error("fknn_graph_search: modes 3-5 need bounds and id_bounds");
    return FKNN_EINVAL;
  }
  return FKNN_OK;
}

// Launch geometry of a search of nq queries at pool capacity cap.
using GraphKernel = void (*)(GParams);

static int graph_geometry(const fknn_graph *g, uint32_t nq, uint32_t cap, size_t *smem, size_t *grid,
                          uint32_t *nwords, uint32_t *nblkw, GraphKernel *kern = nullptr) {
  const uint32_t nblocks512 = (g->n + 511) / 512;
  *nwords = nblocks512 * 8;
  *nblkw = (nblocks512 + 31) / 32;
  *smem = warp_smem_bytes(cap, *nblkw) * GS_WARPS;
  if (*smem > 200 * 1024) {
    set_error("fknn_graph_search: pool and visited flags exceed shared memory (max(k, ef) or n too large)");
    return FKNN_EINVAL;
  }
  // small pools: eight blocks of four warps fit an SM's shared memory, so
  // the register-capped variant raises occupancy (measured: beam 256 up to
  // 23 % faster); larger pools are limited by shared memory, where the cap
  // only adds spills (beam 1024: 4 % slower)
  const GraphKernel k = (*smem + 1024) * GS_OCC_BLOCKS <= GS_SMEM_PER_SM ? k_graph_search<GS_OCC_BLOCKS>
                                                                          : k_graph_search<GS_BASE_BLOCKS>;
  if (kern) *kern = k;
  FKNN_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem));
  int per_sm = 0;
  FKNN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, GS_WARPS * 32, *smem));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
  const size_t slot_bytes = (size_t)*nwords * 16;
  const size_t max_slots = std::max<size_t>(GS_WARPS, VIS_BUDGET / slot_bytes);
  size_t gr = (size_t)sms * std::max(per_sm, 1);
  gr = std::min(gr, std::max<size_t>(1, max_slots / GS_WARPS));
  *grid = std::min(gr, ((size_t)nq + GS_WARPS - 1) / GS_WARPS);
  return FKNN_OK;
}

// Grows the graph's per-call scratch for searches of up to nq queries at
// pool capacity up to cap, so that graph_launch allocates nothing.
int graph_reserve(fknn_graph *g, uint32_t nq, uint32_t cap) {
  size_t smem, grid;
  uint32_t nwords, nblkw;
  int rc;
  if ((rc = graph_geometry(g, nq, cap, &smem, &grid, &nwords, &nblkw))) return rc;
  if ((rc = grow(&g->qcodes, &g->qcodes_cap, (size_t)nq * CODE))) return rc;
  return grow(&g->vis, &g->vis_cap, grid * GS_WARPS * 2 * (size_t)nwords);
}

// Enqueues one search on st (device inputs and outputs, checked arguments);
// the graph's error flag accumulates until graph_flag_reset.
int graph_launch(fknn_graph *g, const float *q_use, uint32_t nq, int mode, uint32_t k, uint32_t cap,
                 uint32_t refine, const float *b_use, const int32_t *ib_use, int32_t *ids_use, float *d_use,
                 cudaStream_t st) {
  int rc;
  if ((rc = grow(&g->qcodes, &g->qcodes_cap, (size_t)nq * CODE))) return rc;
  launch_sq8_encode(q_use, nq, g->alpha, g->qcodes, st);
  size_t smem, grid;
  uint32_t nwords, nblkw;
  GraphKernel kern = nullptr;
  if ((rc = graph_geometry(g, nq, cap, &smem, &grid, &nwords, &nblkw, &kern))) return rc;
  if ((rc = grow(&g->vis, &g->vis_cap, grid * GS_WARPS * 2 * (size_t)nwords))) return rc;
  const bool ranged = mode >= FKNN_GRAPH_CATEGORY_RANGE;
  GParams P;
  P.adj = g->adj;
  P.ets = g->ets;
  P.levels = g->levels;
  P.up_off = g->up_off;
  P.up = g->up;
  P.eps = g->eps;
  P.codes = g->codes;
  P.n = g->n;
  P.K = g->K;
  P.upK = g->upK;
  P.nep = g->nep;
  P.ep = g->ep;
  P.alpha2 = g->alpha * g->alpha;
  P.qcodes = g->qcodes;
  P.nq = nq;
  P.mode = mode;
  P.cap = cap;
  P.refine = refine;
  P.batch = refine <= cap;
  P.bounds = ranged ? b_use : nullptr;
  P.id_bounds = ranged ? ib_use : nullptr;
  P.out_ids = ids_use;
  P.out_dists = d_use;
  P.vis = g->vis;
  P.nwords = nwords;
  P.nblkw = nblkw;
  P.err = g->dflag;
  kern<<<(unsigned)grid, GS_WARPS * 32, smem, st>>>(P);
  g_launches += 1;
  FKNN_CUDA(cudaGetLastError());
  return FKNN_OK;
}

int graph_flag_reset(fknn_graph *g, cudaStream_t st) {
  FKNN_CUDA(cudaMemsetAsync(g->dflag, 0, 4, st));
  return FKNN_OK;
}

// The searches enqueued since the last reset (call after they finished).
int graph_flag_check(fknn_graph *g) {
  int flag = 0;
  FKNN_CUDA(cudaMemcpy(&flag, g->dflag, 4, cudaMemcpyDeviceToHost));
  if (flag & ERR_BAD_QUERY_VALUE) {
    set_error("fknn_graph_search: id_bounds seed a point outside [0, n)");
    return FKNN_EINVAL;
  }
  if (flag) {
    set_error("fknn_graph_search: a search exceeded its pop bound");
    return FKNN_ETIMEOUT;
  }
  return FKNN_OK;
}

}  // namespace fknn

extern "C" {

int fknn_graph_create(const void *graph_bytes, size_t nbytes, const float *vecs, int device, fknn_graph **out) {
  g_launches = 0;
  if (!graph_bytes || !vecs || !out) {
    set_error("fknn_graph_create: NULL argument");
    return FKNN_EINVAL;
  }
  *out = nullptr;
  HostGraph h;
  if (!parse_graph(static_cast<const unsigned char *>(graph_bytes), nbytes, h)) {
    set_error("fknn_graph_create: malformed graph bytes (expected the Graph::save layout)");
    return FKNN_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("fknn_graph_create: no CUDA device");
    return FKNN_ENODEV;
  }
  if (device < 0 || device >= ndev) {
    set_error("fknn_graph_create: bad device ordinal");
    return FKNN_EINVAL;
  }
  FKNN_CUDA(cudaSetDevice(device));
  fknn_graph *g = new (std::nothrow) fknn_graph();
  if (!g) {
    set_error("fknn_graph_create: out of host memory");
    return FKNN_ENOMEM;
  }
  g->device = device;
  g->n = (uint32_t)h.N;
  g->K = (uint32_t)h.K;
  g->nep = (uint32_t)h.eps.size();
  g->ep = h.ep;
  g->upK = h.upK > 0 ? (uint32_t)h.upK : 1u;
  const size_t nk = (size_t)h.N * h.K;
  int rc = upload((void **)&g->adj, h.adj.data(), nk * 4);
  if (!rc) rc = upload((void **)&g->ets, h.ets.data(), nk * 4);
  if (!rc) rc = upload((void **)&g->eps, h.eps.data(), h.eps.size() * 4);
  if (!rc && h.ep >= 0) {
    rc = upload((void **)&g->levels, h.levels.data(), h.levels.size() * 4);
    if (!rc) rc = upload((void **)&g->up_off, h.up_off.data(), h.up_off.size() * 8);
    if (!rc) rc = upload((void **)&g->up, h.up.data(), h.up.size() * 4);
  }
  if (!rc) {
    const cudaError_t e = cudaMalloc((void **)&g->dflag, 64);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc");
  }
  if (!rc) {
    const cudaError_t e = cudaMalloc((void **)&g->codes, (size_t)h.N * CODE);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc");
  }
  // Searcher::SetData: the searcher's own quantizer, trained on the graph's points
  if (!rc) rc = fknn_sq8_sym_train(vecs, (uint64_t)h.N, &g->alpha, g->codes);
  if (rc) {
    free_graph(g);
    return rc;
  }
  *out = g;
  return FKNN_OK;
}

int fknn_graph_destroy(fknn_graph *g) {
  free_graph(g);
  return FKNN_OK;
}

int fknn_graph_info(const fknn_graph *g, uint32_t *n, uint32_t *degree, float *alpha) {
  if (!g) {
    set_error("fknn_graph_info: NULL graph");
    return FKNN_EINVAL;
  }
  if (n) *n = g->n;
  if (degree) *degree = g->K;
  if (alpha) *alpha = g->alpha;
  return FKNN_OK;
}

int fknn_graph_search(fknn_graph *g, const float *queries, uint32_t nq, int mode, uint32_t k, uint32_t ef,
                      uint32_t refine, const float *bounds, const int32_t *id_bounds, int32_t *out_ids,
                      float *out_dists, void *stream) {
  g_launches = 0;
  uint32_t cap = 0;
  int rc;
  if ((rc = fknn::graph_check_args(g, queries, nq, mode, k, ef, refine, bounds, id_bounds, out_ids, &cap))) return rc;
  if (nq == 0) return FKNN_OK;
  FKNN_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  const bool ranged = mode >= FKNN_GRAPH_CATEGORY_RANGE;

  // staging: [queries | bounds | id_bounds | ids | dists], 4-byte words
  const size_t qf = (size_t)nq * DIM, bf = ranged ? (size_t)nq * 2 : 0, of = (size_t)nq * refine;
  if ((rc = grow(&g->io, &g->io_cap, qf + 2 * bf + 2 * of))) return rc;
  float *s_q = g->io, *s_b = s_q + qf;
  int32_t *s_ib = reinterpret_cast<int32_t *>(s_b + bf);
  int32_t *s_ids = s_ib + bf;
  float *s_d = reinterpret_cast<float *>(s_ids + of);
  const int dev = g->device;
  if ((rc = fknn::check_local_buffers("fknn_graph_search", dev,
                                      {queries, ranged ? bounds : nullptr, ranged ? id_bounds : nullptr, out_ids,
                                       out_dists})))
    return rc;
  const float *q_use = queries;
  if (!on_device(queries, dev)) {
    FKNN_CUDA(cudaMemcpyAsync(s_q, queries, qf * 4, cudaMemcpyHostToDevice, st));
    q_use = s_q;
  }
  const float *b_use = bounds;
  const int32_t *ib_use = id_bounds;
  if (ranged && !on_device(bounds, dev)) {
    FKNN_CUDA(cudaMemcpyAsync(s_b, bounds, bf * 4, cudaMemcpyHostToDevice, st));
    b_use = s_b;
  }
  if (ranged && !on_device(id_bounds, dev)) {
    FKNN_CUDA(cudaMemcpyAsync(s_ib, id_bounds, bf * 4, cudaMemcpyHostToDevice, st));
    ib_use = s_ib;
  }
  int32_t *ids_use = on_device(out_ids, dev) ? out_ids : s_ids;
  float *d_use = out_dists ? (on_device(out_dists, dev) ? out_dists : s_d) : nullptr;
  FKNN_CUDA(cudaMemsetAsync(g->dflag, 0, 4, st));
  if ((rc = fknn::graph_launch(g, q_use, nq, mode, k, cap, refine, b_use, ib_use, ids_use, d_use, st))) return rc;
  if (ids_use != out_ids) FKNN_CUDA(cudaMemcpyAsync(out_ids, ids_use, of * 4, cudaMemcpyDeviceToHost, st));
  if (out_dists && d_use != out_dists)
    FKNN_CUDA(cudaMemcpyAsync(out_dists, d_use, of * 4, cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  return fknn::graph_flag_check(g);
}

}  // extern "C"
