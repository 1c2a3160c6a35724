// Symmetric SQ8 (pyglass/glass/quant/sq8_sym_quant.hpp) and the SQ8 slab
// brute force (bruteforce.h:244-289) on the GPU.
//
// bruteforce() returns the reference's maxPQIFCS heap array, which depends
// on the exact insertion history (ties on the int distance are frequent).
// The kernels below reproduce that history (the three steps are described
// above k_sq8_prefix).  Every distance is an exact int32 L2SqrSQ8_sym value:
// |q-c|^2 = |q|^2 + |c|^2 - 2 q.c, from dp4a or from the int8 tensor cores.
#include <climits>

#include "tc_util.cuh"

namespace fknn {

namespace {

constexpr int SQ8_CODE = 112;
constexpr int BF_KMAX = 2048;

__global__ void k_absmax(const float *__restrict__ x, uint64_t count, uint32_t *__restrict__ out) {
  float m = 0.f;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(x[i]));
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));  // non-negative floats order as uints
}

// sq8_sym_quant.hpp:63-74: x / alpha (IEEE division), clamp to [-1, 1],
// std::round(x * 127) (half away from zero), dims 100..111 zero.
__global__ void k_sq8_encode(const float *__restrict__ x, uint64_t n, float alpha, int8_t *__restrict__ codes) {
  const uint64_t total = n * SQ8_CODE;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = i / SQ8_CODE;
    const int d = (int)(i % SQ8_CODE);
    int8_t c = 0;
    if (d < DIM) {
      float y = __fdiv_rn(x[r * DIM + d], alpha);
      if (y > 1.0f) y = 1.0f;
      if (y < -1.0f) y = -1.0f;
      c = (int8_t)roundf(__fmul_rn(y, 127.0f));
    }
    codes[i] = c;
  }
}

struct HeapNode {
  int d;
  int id;
};

// ------------------------------------------------------------------------
// The slab brute force as three steps per batch of queries:
//
//  1. k_sq8_prefix (one warp per query): the first SQ_PREFIX codes replayed
//     exactly -- emplace of the first k, then must_pop_emplace -- with a
//     warp-wide filter in front of the serial heap steps.  The heap root
//     afterwards, T_q, bounds every later root (the root only falls), so a
//     later code can enter only if its distance is below T_q.
//  2. k_sq8_screen (tcgen05, kind::i8): the int32 inner products of a tile of
//     128 queries with the code tiles of one slab segment, exact in the
//     accumulator; an epilogue thread per query writes every code of the
//     segment with d = |q|^2 + |c|^2 - 2 q.c < T_q, in slab order, to the
//     query's list for that segment.  A list that fills up marks the query.
//  3. k_sq8_tail (one warp per query): the heap from step 1, the segment lists
//     in order through the same filter and serial steps, the heap array out.
//     A marked query scans the codes itself instead, with the step-1 code.
//
// Every distance is the exact int32 L2SqrSQ8_sym value and every code that
// can enter the heap reaches the serial steps in slab order, so the heap
// array is the reference's.
constexpr uint32_t SQ_PREFIX = 8192;    // codes replayed before the screen (multiple of 128)
constexpr int SQ_WARPS = 4;             // queries per block of the replay kernels
constexpr int SQ_SCAN = 128;            // codes per warp step of the replay kernels
constexpr uint32_t SQ_TILE = TC_ROWS * 128;  // 128 rows x 128 bytes (112 code bytes, 16 zero)
constexpr int SQ_BS = 4;                // shared-memory stages of code tiles
constexpr int SQ_EPI_WARPS = 4;
constexpr int SQ_THREADS = (2 + SQ_EPI_WARPS) * 32;  // producer, MMA issuer, epilogue
constexpr uint32_t SQ_TMEM_COLS = 2 * TC_ROWS;       // double-buffered accumulator
constexpr int SQ_MMAS = 128 / 32;       // kind::i8: K = 32 bytes per MMA
constexpr int SQ_NCC_PAD = INT_MIN / 2;  // -|c|^2 of rows past the slab: no candidate test passes
constexpr uint32_t SQ_QBATCH = 8192;    // queries per pass (bounds the candidate lists)
// S32 accumulate, signed 8-bit A and B, K-major, N = 128, M = 128
constexpr uint32_t SQ_IDESC =
    (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_ROWS >> 3) << 17) | ((uint32_t)(TC_ROWS >> 4) << 24);

// code p (row p of 112 bytes; row 0 when p >= bound) as seven 16-byte words
__device__ __forceinline__ void load_code(const int8_t *__restrict__ codes, uint64_t p, uint64_t bound,
                                          int4 (&c)[7]) {
  const int4 *src = reinterpret_cast<const int4 *>(codes + (p < bound ? p : 0) * SQ8_CODE);
#pragma unroll
  for (int w = 0; w < 7; ++w) c[w] = __ldg(src + w);
}

__device__ __forceinline__ int dot112(const int4 (&c)[7], const int4 (&q)[7]) {
  int s = 0;
#pragma unroll
  for (int w = 0; w < 7; ++w) {
    s = __dp4a(q[w].x, c[w].x, s);
    s = __dp4a(q[w].y, c[w].y, s);
    s = __dp4a(q[w].z, c[w].z, s);
    s = __dp4a(q[w].w, c[w].w, s);
  }
  return s;
}

// Heap steps of maxPQIFCS on a 1-based array, with a hole moved in place of
// the reference's swaps (the same comparisons, so the same array).

// emplace (bruteforce.h:106-113) at position now (1-based, = new size)
__device__ __forceinline__ void heap_emplace(HeapNode *h, int now, HeapNode nd) {
  while (now != 1) {
    const HeapNode p = h[now >> 1];
    if (!(nd.d > p.d)) break;
    h[now] = p;
    now >>= 1;
  }
  h[now] = nd;
}

// must_pop_emplace (bruteforce.h:99-105) behind the root test
// bruteforce.h:258-260 makes; push_down (bruteforce.h:78-87) reads both
// children of a level with one 16-byte load (h is 16-byte aligned and the
// pair h[2x], h[2x+1] lies inside the heap's region even when 2x = cnt).
__device__ __forceinline__ void heap_offer(HeapNode *h, int cnt, HeapNode nd) {
  if (h[1].d <= nd.d) return;
  int x = 1;
  while ((x << 1) <= cnt) {
    const int t0 = x << 1;
    const int4 pr = *reinterpret_cast<const int4 *>(h + t0);
    const bool r = t0 < cnt && pr.z > pr.x;
    HeapNode c;
    c.d = r ? pr.z : pr.x;
    c.id = r ? pr.w : pr.y;
    if (c.d <= nd.d) break;
    h[x] = c;
    x = t0 + (r ? 1 : 0);
  }
  h[x] = nd;
}

// nodes of one warp's shared-memory region: the heap (1-based, k + 1 nodes,
// rounded up to an even count past k + 1 for the pair loads), then the stage
__host__ __device__ __forceinline__ uint32_t sq_region(uint32_t k) { return ((k + 2u + 1u) & ~1u) + SQ_SCAN; }

// list[0..n) (shared memory) offered in order by lane 0
__device__ __forceinline__ void offer_list(HeapNode *h, int cnt, const HeapNode *list, int n, int lane) {
  if (lane == 0)
    for (int j = 0; j < n; ++j) heap_offer(h, cnt, list[j]);
  __syncwarp();
}

// Codes [p0, p1) of the slab through one query's heap, in order: positions
// below k are emplaced, the rest offered.  The warp scores SQ_SCAN codes per
// step; lane 0 runs the heap steps for the ones that can enter: all of a step
// that starts before the heap holds k nodes, else those below the root at the
// start of the step (the root only falls).  cc[p] = |c_p|^2 = -ncc[p].
__device__ void scan_codes(HeapNode *heap, HeapNode *stage, const int4 (&qv)[7], int qq,
                           const int8_t *__restrict__ codes, const int *__restrict__ ncc, uint64_t p0, uint64_t p1,
                           uint32_t k, int lane) {
  const uint32_t below = (1u << lane) - 1u;
  for (uint64_t base = p0; base < p1; base += SQ_SCAN) {
    int d[SQ_SCAN / 32];
    int4 c[SQ_SCAN / 32][7];
#pragma unroll
    for (int i = 0; i < SQ_SCAN / 32; ++i) load_code(codes, base + 32 * i + lane, p1, c[i]);
#pragma unroll
    for (int i = 0; i < SQ_SCAN / 32; ++i) {
      const uint64_t p = base + 32 * i + lane;
      d[i] = p < p1 ? qq - ncc[p] - 2 * dot112(c[i], qv) : INT_MAX;
    }
    const bool full = base >= k;  // the heap holds k nodes from here on
    const int root = heap[1].d;
    int off = 0;
#pragma unroll
    for (int i = 0; i < SQ_SCAN / 32; ++i) {
      const uint64_t p = base + 32 * i + lane;
      const uint32_t m = __ballot_sync(0xffffffffu, p < p1 && (!full || d[i] < root));
      if ((m >> lane) & 1u) {
        HeapNode nd;
        nd.d = d[i];
        nd.id = (int)p;
        stage[off + __popc(m & below)] = nd;
      }
      off += __popc(m);
    }
    __syncwarp();
    if (full) {
      offer_list(heap, (int)k, stage, off, lane);
    } else {
      if (lane == 0)
        for (int j = 0; j < off; ++j) {
          const HeapNode nd = stage[j];
          if ((uint32_t)nd.id < k) heap_emplace(heap, nd.id + 1, nd);
          else heap_offer(heap, (int)k, nd);
        }
      __syncwarp();
    }
  }
}

__device__ __forceinline__ void load_query(const int8_t *__restrict__ queries, uint32_t q, int4 (&qv)[7], int &qq) {
  const int4 *src = reinterpret_cast<const int4 *>(queries + (uint64_t)q * SQ8_CODE);
#pragma unroll
  for (int w = 0; w < 7; ++w) qv[w] = __ldg(src + w);
  qq = dot112(qv, qv);
}

// closest_points[k - l - 1] = data_[l + 1].id (bruteforce.h:262-264), and for
// bruteforce_subgraph distances[k - l - 1] = data_[l + 1].dist * alpha^2
__device__ __forceinline__ void write_heap(const HeapNode *heap, uint32_t k, uint64_t q, int *__restrict__ closest,
                                           float *__restrict__ dists, float alpha, int lane) {
  for (uint32_t l = lane; l < k; l += 32) {
    closest[q * k + (k - l - 1)] = heap[l + 1].id;
    if (dists) dists[q * k + (k - l - 1)] = (float)heap[l + 1].d * alpha * alpha;
  }
}

// The screen's accumulator carries most of -|c|^2/2: bytes 112..127 of a
// row (zero padding in every SQ8 code, so the dot product is unchanged) hold
// base-127 digits of f = min(ceil(|c|^2 / 2), SQ_FOLD_MAX) on the code side --
// fifteen digits of weight 127 and one of weight 1 -- and the multipliers
// -127 / -1 on the query side, so the MMA returns z = q.c - f.
constexpr int SQ_FOLD_MAX = 127 * (15 * 127) + 126;

__host__ __device__ __forceinline__ int sq_fold(int cc) { return min((cc + 1) >> 1, SQ_FOLD_MAX); }

// Rows [row0, row0 + 128 * ntiles) of n rows of 112 bytes as 128-row
// core-matrix tiles of 128 bytes per row (rows past n zero), bytes 112..127
// the fold digits (side 0, codes) or multipliers (side 1, queries), and
// ncc[r] = -|row r|^2 (SQ_NCC_PAD past n).  One block per tile.
__global__ void __launch_bounds__(256) k_sq8_tiles(const int8_t *__restrict__ rows, uint64_t n, uint64_t row0,
                                                   int side, unsigned char *__restrict__ tiles,
                                                   int *__restrict__ ncc) {
  const uint64_t t = blockIdx.x;
  unsigned char *o = tiles + t * SQ_TILE;
  for (uint32_t c = threadIdx.x; c < TC_ROWS * 8; c += blockDim.x) {
    const uint32_t r = c >> 3, kc = c & 7;
    const uint64_t p = row0 + t * TC_ROWS + r;
    int4 v = make_int4(0, 0, 0, 0);
    if (p < n) {
      if (kc < 7) {
        v = __ldg(reinterpret_cast<const int4 *>(rows + p * SQ8_CODE) + kc);
      } else {
        int4 cw[7];
        load_code(rows, p, n, cw);
        const int cc = dot112(cw, cw);
        ncc[t * TC_ROWS + r] = -cc;
        int8_t b[16];
        if (side == 0) {
          const int f = sq_fold(cc);
          int e = f / 127;
          for (int i = 0; i < 15; ++i) {
            const int di = e > 127 ? 127 : e;
            b[i] = (int8_t)di;
            e -= di;
          }
          b[15] = (int8_t)(f % 127);
        } else {
          for (int i = 0; i < 15; ++i) b[i] = (int8_t)-127;
          b[15] = (int8_t)-1;
        }
        memcpy(&v, b, 16);
      }
    } else if (kc == 7) {
      ncc[t * TC_ROWS + r] = SQ_NCC_PAD;
    }
    *reinterpret_cast<int4 *>(o + cm_byte(r, kc * 16)) = v;
  }
}

// Step 1.  With final set (the whole slab is the prefix) it writes the
// answer; else the heap and its root T_q.
__global__ void __launch_bounds__(SQ_WARPS * 32, 4)
    k_sq8_prefix(const int8_t *__restrict__ codes, const int *__restrict__ ncc, uint64_t prefix,
                 const int8_t *__restrict__ queries, uint32_t nq, uint32_t k, int final, HeapNode *__restrict__ heaps,
                 int *__restrict__ T, int *__restrict__ closest, float *__restrict__ dists, float alpha) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t q = blockIdx.x * SQ_WARPS + warp;
  if (q >= nq) return;  // warp-uniform; the kernel has no block barrier
  HeapNode *heap = reinterpret_cast<HeapNode *>(smem_raw) + (size_t)warp * sq_region(k);
  HeapNode *stage = heap + (sq_region(k) - SQ_SCAN);
  int4 qv[7];
  int qq;
  load_query(queries, q, qv, qq);
  scan_codes(heap, stage, qv, qq, codes, ncc, 0, prefix, k, lane);
  if (final) {
    write_heap(heap, k, q, closest, dists, alpha, lane);
  } else {
    for (uint32_t l = lane; l <= k; l += 32) heaps[(uint64_t)q * (k + 1) + l] = heap[l];
    if (lane == 0) T[q] = heap[1].d;
  }
}

constexpr int SQ_STAGE_ROW = 36;  // ints per lane row of the candidate staging area

struct SqScreenSmem {
  unsigned char a[SQ_TILE];
  unsigned char b[SQ_BS][SQ_TILE];
  // per epilogue lane, the 32 values y of a chunk that holds candidates
  // (rows padded to 36 ints: conflict-free 16-byte stores)
  int stage[SQ_EPI_WARPS][32 * SQ_STAGE_ROW];
  uint64_t full[SQ_BS], empty[SQ_BS], accfull[2], accempty[2], abar;
  uint32_t tmem_base;
};
static_assert(sizeof(SqScreenSmem) <= 113 * 1024, "two screen CTAs per SM");

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(SQ_IDESC), "r"(accumulate));
}

// Step 2.  Block (query tile, segment); the segment is code tiles
// [seg * tps, min(nct, (seg + 1) * tps)) of the screened part, whose tile t
// holds slab rows row0 + 128 t ...  The list of query q for segment seg is
// cand[(q * nseg + seg) * cap ...], its length counts[q * nseg + seg].
__global__ void __launch_bounds__(SQ_THREADS, 2)
    k_sq8_screen(const unsigned char *__restrict__ qtiles, const int *__restrict__ qncc, uint32_t nq,
                 const unsigned char *__restrict__ ctiles, const int *__restrict__ cncc, uint32_t nct, uint32_t tps,
                 uint32_t nseg, uint32_t row0, uint64_t npoints, const int *__restrict__ T, int2 *__restrict__ cand,
                 uint32_t cap, uint32_t *__restrict__ counts, uint32_t *__restrict__ mark, int *err) {
  extern __shared__ __align__(1024) unsigned char screen_smem[];
  SqScreenSmem &sm = *reinterpret_cast<SqScreenSmem *>(screen_smem);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t qt = blockIdx.x, seg = blockIdx.y;
  const uint32_t t0 = seg * tps;
  const uint32_t ntile = t0 < nct ? min(tps, nct - t0) : 0u;

  if (tid == 0) {
    for (int s = 0; s < SQ_BS; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&sm.accfull[a], 1);
      mbar_init(&sm.accempty[a], SQ_EPI_WARPS);
    }
    mbar_init(&sm.abar, 1);
    fence_mbar_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                 "r"(SQ_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;

  if (warp == 0) {
    // ------------------------------------------------ producer
    if (lane == 0) {
      mbar_arrive_expect_tx(&sm.abar, SQ_TILE);
      bulk_g2s(sm.a, qtiles + (uint64_t)qt * SQ_TILE, SQ_TILE, &sm.abar);
      uint32_t issued = 0;
      for (uint32_t sub = 0; sub < ntile; ++sub) {
        const int st = sub % SQ_BS;
        if (sub >= SQ_BS && !mbar_wait_bounded(&sm.empty[st], ((sub / SQ_BS) - 1) & 1, err)) break;
        mbar_arrive_expect_tx(&sm.full[st], SQ_TILE);
        bulk_g2s(sm.b[st], ctiles + (uint64_t)(t0 + sub) * SQ_TILE, SQ_TILE, &sm.full[st]);
        ++issued;
      }
      // no copy may still be landing when the block exits
      mbar_wait_bounded(&sm.abar, 0, err);
      for (uint32_t i = issued > SQ_BS ? issued - SQ_BS : 0; i < issued; ++i)
        mbar_wait_bounded(&sm.full[i % SQ_BS], (i / SQ_BS) & 1, err);
    }
  } else if (warp == 1) {
    // ------------------------------------------------ MMA issuer
    if (lane == 0) {
      uint32_t done = 0;
      if (mbar_wait_bounded(&sm.abar, 0, err)) {
        const uint32_t a0 = smem_u32(sm.a);
        for (uint32_t sub = 0; sub < ntile; ++sub) {
          const int st = sub % SQ_BS, ab = sub & 1;
          if (!mbar_wait_bounded(&sm.full[st], (sub / SQ_BS) & 1, err)) break;
          if (sub >= 2 && !mbar_wait_bounded(&sm.accempty[ab], ((sub >> 1) - 1) & 1, err)) break;
          tc_fence_after();
          const uint32_t b0 = smem_u32(sm.b[st]);
#pragma unroll
          for (int kk = 0; kk < SQ_MMAS; ++kk) {
            const uint64_t da = umma_desc(a0 + kk * 2 * (TC_ROWS / 8) * 128, (TC_ROWS / 8) * 128, 128);
            const uint64_t db = umma_desc(b0 + kk * 2 * (TC_ROWS / 8) * 128, (TC_ROWS / 8) * 128, 128);
            umma_i8(tmem + ab * TC_ROWS, da, db, kk > 0);
          }
          umma_commit(&sm.empty[st]);
          umma_commit(&sm.accfull[ab]);
          ++done;
        }
      }
      // no MMA may be in flight when TMEM is released
      if (done) mbar_wait_bounded(&sm.accfull[(done - 1) & 1], ((done - 1) >> 1) & 1, err);
    }
  } else {
    // ------------------------------------------------ epilogue: thread = query
    const int wg = warp & 3;  // TMEM lanes 32*wg .. 32*wg+31 are reachable from this warp
    const uint32_t q = qt * TC_ROWS + wg * 32 + lane;
    const bool valid = q < nq;
    // The accumulator is z = q.c - f with f = sq_fold(|c|^2) <= (|c|^2 + 1) / 2,
    // so d = qq + |c|^2 - 2 q.c < T implies 2 z > qq - T - 1: the test
    // z > floor((qq - T - 1) / 2) keeps every code that can enter the heap
    // (and a few more), and d = qq + cc - 2 (z + f) is exact.
    const int qq = valid ? -qncc[q] : 0;
    const int thr = valid ? ((qq - T[q] - 1) >> 1) : INT_MAX;
    int2 *list = cand + ((uint64_t)(valid ? q : 0) * nseg + seg) * cap;
    int *row = &sm.stage[wg][lane * SQ_STAGE_ROW];
    uint32_t cnt = 0;
    bool ok = true;
    for (uint32_t sub = 0; sub < ntile; ++sub) {
      const int ab = sub & 1;
      // warp-uniform: the lanes' timers may disagree at the deadline
      if (!__all_sync(0xffffffffu, mbar_wait_bounded(&sm.accfull[ab], (sub >> 1) & 1, err))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t tile = t0 + sub;
      const int *nc = cncc + (uint64_t)tile * TC_ROWS;
      const int id0 = (int)(row0 + tile * TC_ROWS);
      const int ncols = (int)min((uint64_t)TC_ROWS, npoints - (uint64_t)id0);  // the slab's last tile is short
#pragma unroll 1
      for (int c2 = 0; c2 < TC_ROWS; c2 += 64) {
        float v[64];
        tmem_ld64(tmem + ((uint32_t)(wg * 32) << 16) + ab * TC_ROWS + c2, v);
#pragma unroll
        for (int h = 0; h < 64; h += 32) {
          // candidate bits of 32 columns, four independent chains
          uint32_t mk[4] = {0u, 0u, 0u, 0u};
#pragma unroll
          for (int j = 0; j < 32; ++j) mk[j & 3] |= (__float_as_int(v[h + j]) > thr ? 1u : 0u) << j;
          uint32_t mask = (mk[0] | mk[1]) | (mk[2] | mk[3]);
          const int lim = ncols - (c2 + h);
          if (lim < 32) mask &= lim > 0 ? (1u << lim) - 1u : 0u;
          if (mask) {
            // the lane's candidates in column order, z read back from its
            // staging row (the loop runs once per candidate)
#pragma unroll
            for (int j = 0; j < 32; j += 4)
              *reinterpret_cast<int4 *>(row + j) =
                  make_int4(__float_as_int(v[h + j]), __float_as_int(v[h + j + 1]), __float_as_int(v[h + j + 2]),
                            __float_as_int(v[h + j + 3]));
            do {
              const int j = __ffs(mask) - 1;
              mask &= mask - 1;
              const int cc = -__ldg(nc + c2 + h + j);
              if (cnt < cap) list[cnt] = make_int2(qq + cc - 2 * (row[j] + sq_fold(cc)), id0 + c2 + h + j);
              ++cnt;
            } while (mask);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive1(&sm.accempty[ab]);
    }
    if (valid) {
      counts[(uint64_t)q * nseg + seg] = min(cnt, cap);
      if (!ok || cnt > cap) mark[q] = 1u;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(SQ_TMEM_COLS));
  }
}

// Step 3.
__global__ void __launch_bounds__(SQ_WARPS * 32, 4)
    k_sq8_tail(const int8_t *__restrict__ codes, const int *__restrict__ ncc, uint64_t prefix, uint64_t npoints,
               const int8_t *__restrict__ queries, uint32_t nq, uint32_t k, const HeapNode *__restrict__ heaps,
               const int2 *__restrict__ cand, uint32_t cap, const uint32_t *__restrict__ counts, uint32_t nseg,
               const uint32_t *__restrict__ mark, int *__restrict__ closest, float *__restrict__ dists, float alpha) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t q = blockIdx.x * SQ_WARPS + warp;
  if (q >= nq) return;  // warp-uniform; the kernel has no block barrier
  HeapNode *heap = reinterpret_cast<HeapNode *>(smem_raw) + (size_t)warp * sq_region(k);
  HeapNode *stage = heap + (sq_region(k) - SQ_SCAN);
  for (uint32_t l = lane; l <= k; l += 32) heap[l] = heaps[(uint64_t)q * (k + 1) + l];
  __syncwarp();
  if (mark[q]) {
    int4 qv[7];
    int qq;
    load_query(queries, q, qv, qq);
    scan_codes(heap, stage, qv, qq, codes, ncc, prefix, npoints, k, lane);
  } else {
    const uint32_t below = (1u << lane) - 1u;
    for (uint32_t s = 0; s < nseg; ++s) {
      const uint32_t cnt = counts[(uint64_t)q * nseg + s];
      const int2 *list = cand + ((uint64_t)q * nseg + s) * cap;
      for (uint32_t j0 = 0; j0 < cnt; j0 += SQ_SCAN) {
        int2 cd[SQ_SCAN / 32];
#pragma unroll
        for (int i = 0; i < SQ_SCAN / 32; ++i) {
          const uint32_t j = j0 + 32 * i + lane;
          cd[i] = j < cnt ? list[j] : make_int2(INT_MAX, 0);
        }
        const int root = heap[1].d;
        int off = 0;
#pragma unroll
        for (int i = 0; i < SQ_SCAN / 32; ++i) {
          const uint32_t m = __ballot_sync(0xffffffffu, cd[i].x < root);
          if ((m >> lane) & 1u) {
            HeapNode nd;
            nd.d = cd[i].x;
            nd.id = cd[i].y;
            stage[off + __popc(m & below)] = nd;
          }
          off += __popc(m);
        }
        __syncwarp();
        offer_list(heap, (int)k, stage, off, lane);
      }
    }
  }
  __syncwarp();
  write_heap(heap, k, q, closest, dists, alpha, lane);
}

// Device memory of the current device (or managed memory).
bool is_dev(const void *p) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return mem_loc(p, dev) == MemLoc::Here;
}

struct Scoped {
  void *p = nullptr;
  ~Scoped() {
    if (p) cudaFree(p);
  }
};

// Device copy of a host buffer (or the pointer itself when it is already a
// 16-byte aligned device pointer; the code rows are read as int4).
int stage_in(const void *src, size_t bytes, Scoped &s, const void **out, cudaStream_t st) {
  if (is_dev(src) && ((uintptr_t)src & 15) == 0) {
    *out = src;
    return FKNN_OK;
  }
  FKNN_CUDA(cudaMalloc(&s.p, bytes ? bytes : 16));
  FKNN_CUDA(cudaMemcpyAsync(s.p, src, bytes, cudaMemcpyDefault, st));
  *out = s.p;
  return FKNN_OK;
}

int stage_out(void *dst, size_t bytes, Scoped &s, void **out) {
  if (is_dev(dst)) {
    *out = dst;
    return FKNN_OK;
  }
  FKNN_CUDA(cudaMalloc(&s.p, bytes ? bytes : 16));
  *out = s.p;
  return FKNN_OK;
}

int ensure_device() {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return FKNN_ENODEV;
  }
  return FKNN_OK;
}

int sq8_encode_impl(const float *vecs, uint64_t n, float alpha, int8_t *codes, bool train, float *alpha_out) {
  if (!vecs || !codes || n == 0) {
    set_error("fknn_sq8: bad arguments");
    return FKNN_EINVAL;
  }
  int rc = ensure_device();
  if (rc) return rc;
  int dev = 0;
  FKNN_CUDA(cudaGetDevice(&dev));
  if ((rc = check_local_buffers("fknn_sq8", dev, {vecs, codes}))) return rc;
  cudaStream_t st = 0;
  Scoped sin, sout, sa;
  const float *d_x;
  int8_t *d_c;
  if ((rc = stage_in(vecs, n * DIM * 4, sin, (const void **)&d_x, st))) return rc;
  if ((rc = stage_out(codes, n * SQ8_CODE, sout, (void **)&d_c))) return rc;
  if (train) {
    FKNN_CUDA(cudaMalloc(&sa.p, 4));
    FKNN_CUDA(cudaMemsetAsync(sa.p, 0, 4, st));
    k_absmax<<<148 * 4, 256, 0, st>>>(d_x, n * DIM, (uint32_t *)sa.p);
    g_launches += 1;
    uint32_t bits = 0;
    FKNN_CUDA(cudaMemcpyAsync(&bits, sa.p, 4, cudaMemcpyDeviceToHost, st));
    FKNN_CUDA(cudaStreamSynchronize(st));
    alpha = bits_f32(bits);
    if (alpha_out) *alpha_out = alpha;
  }
  if (!(alpha > 0.f) || !(alpha <= 3.0e38f)) {
    set_error("fknn_sq8: alpha must be positive and finite (all-zero or non-finite training data?)");
    return FKNN_EINVAL;
  }
  k_sq8_encode<<<148 * 8, 256, 0, st>>>(d_x, n, alpha, d_c);
  g_launches += 1;
  FKNN_CUDA(cudaGetLastError());
  if (d_c != codes) FKNN_CUDA(cudaMemcpyAsync(codes, d_c, n * SQ8_CODE, cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  return FKNN_OK;
}

// Device scratch of the slab brute force: one per calling host thread, with
// its own non-blocking stream, kept between calls (it only grows).  The
// reference calls bruteforce() from concurrent OpenMP workers
// (hybrid_graph.cpp:168,380); with a scratch and a stream each, their calls
// run side by side on the GPU, and after the first call of a thread at a
// given size none of them allocates (cudaFree would wait for the device).
struct Sq8Scratch {
  void *p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;  // orders the call after the legacy default stream
  int device = -1;
  int num_sms = 0;
  void release() {
    if (p) cudaFree(p);
    if (ev) cudaEventDestroy(ev);
    if (st) cudaStreamDestroy(st);
    p = nullptr;
    ev = nullptr;
    st = nullptr;
    bytes = 0;
    device = -1;
  }
  ~Sq8Scratch() { release(); }
};

Sq8Scratch &sq8_scratch() {
  thread_local Sq8Scratch s;
  return s;
}

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

// segments and list capacity for a pass of nqb queries over nct code tiles
struct Sq8Pass {
  uint32_t nqt, tps, nseg, cap;
  size_t bytes;  // query tiles, norms, heaps, bounds, lists, counts, marks
};

Sq8Pass sq8_pass(uint32_t nqb, uint32_t nct, size_t k, int num_sms) {
  Sq8Pass p{};
  p.nqt = (nqb + TC_ROWS - 1) / TC_ROWS;
  // about four screen CTAs per SM (two resident, two waves)
  uint32_t nseg = std::max(1u, std::min(nct, (uint32_t)((4u * num_sms + p.nqt - 1) / p.nqt)));
  p.tps = (nct + nseg - 1) / nseg;
  p.nseg = (nct + p.tps - 1) / p.tps;
  // a code of the screened part is a candidate iff it is below the k-th
  // smallest of the prefix: about k / SQ_PREFIX of them; the lists hold twice
  // that, and a query whose list fills up takes the exact scan
  const double expect = (double)p.tps * TC_ROWS * (double)k / SQ_PREFIX;
  p.cap = (uint32_t)std::min<double>((double)p.tps * TC_ROWS, ((uint32_t)(2.0 * expect) + 64 + 31) & ~31u);
  p.bytes = al256((size_t)p.nqt * SQ_TILE) + al256((size_t)p.nqt * TC_ROWS * 4) +
            al256((size_t)nqb * (k + 1) * sizeof(HeapNode)) + al256((size_t)nqb * 4) +
            al256((size_t)nqb * p.nseg * p.cap * sizeof(int2)) + al256((size_t)nqb * p.nseg * 4) +
            al256((size_t)nqb * 4) + 256;
  return p;
}

int sq8_bf_impl(size_t k, int *closest, float *dists, size_t npoints, const char *codes_in, float alpha,
                size_t nqueries, const int8_t *queries_in) {
  if (!closest || !codes_in || !queries_in || k == 0 || k > npoints || k > (size_t)BF_KMAX || nqueries == 0 ||
      npoints >= (1ull << 31) || nqueries >= (1ull << 31)) {
    set_error("fknn_sq8_bruteforce: need 1 <= k <= npoints, k <= 2048, 1 <= nqueries < 2^31, npoints < 2^31");
    return FKNN_EINVAL;
  }
  int rc = ensure_device();
  if (rc) return rc;
  int dev = 0;
  FKNN_CUDA(cudaGetDevice(&dev));
  if ((rc = check_local_buffers("fknn_sq8_bruteforce", dev, {closest, dists, codes_in, queries_in}))) return rc;
  Sq8Scratch &scr = sq8_scratch();
  if (scr.device != dev) {
    // once per thread and device: stream, event, SM count, and the kernels'
    // dynamic shared-memory limits at their largest (k = BF_KMAX)
    scr.release();
    FKNN_CUDA(cudaStreamCreateWithFlags(&scr.st, cudaStreamNonBlocking));
    FKNN_CUDA(cudaEventCreateWithFlags(&scr.ev, cudaEventDisableTiming));
    FKNN_CUDA(cudaDeviceGetAttribute(&scr.num_sms, cudaDevAttrMultiProcessorCount, dev));
    const int rmax = (int)((size_t)SQ_WARPS * sq_region(BF_KMAX) * sizeof(HeapNode));
    FKNN_CUDA(cudaFuncSetAttribute(k_sq8_prefix, cudaFuncAttributeMaxDynamicSharedMemorySize, rmax));
    FKNN_CUDA(cudaFuncSetAttribute(k_sq8_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, rmax));
    FKNN_CUDA(cudaFuncSetAttribute(k_sq8_screen, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sizeof(SqScreenSmem)));
    scr.device = dev;
  }
  const int num_sms = scr.num_sms;
  const uint32_t nq = (uint32_t)nqueries, K = (uint32_t)k;
  const bool screened = npoints > SQ_PREFIX;
  const uint64_t prefix = screened ? SQ_PREFIX : npoints;
  const uint32_t nct_all = (uint32_t)((npoints + TC_ROWS - 1) / TC_ROWS);
  const uint32_t nct = screened ? nct_all - SQ_PREFIX / TC_ROWS : 0;
  const uint32_t qbatch = std::min(nq, SQ_QBATCH);
  const uint32_t qlast = nq - (nq - 1) / qbatch * qbatch;
  const Sq8Pass pa = sq8_pass(qbatch, std::max(nct, 1u), k, num_sms);
  const Sq8Pass pb = sq8_pass(qlast, std::max(nct, 1u), k, num_sms);

  // inputs already on the device (16-byte aligned) are used in place, the
  // rest staged through the scratch, as are outputs that live on the host
  const bool codes_dev = is_dev(codes_in) && ((uintptr_t)codes_in & 15) == 0;
  const bool q_dev = is_dev(queries_in) && ((uintptr_t)queries_in & 15) == 0;
  const bool ids_dev = is_dev(closest);
  const bool d_dev = dists && is_dev(dists);
  const size_t b_codes = codes_dev ? 0 : al256(npoints * SQ8_CODE);
  const size_t b_q = q_dev ? 0 : al256(nqueries * SQ8_CODE);
  const size_t b_ids = ids_dev ? 0 : al256(nqueries * k * 4);
  const size_t b_d = (!dists || d_dev) ? 0 : al256(nqueries * k * 4);
  const size_t codes_bytes = al256((size_t)nct_all * SQ_TILE) + al256((size_t)nct_all * TC_ROWS * 4);
  const size_t need = b_codes + b_q + b_ids + b_d + codes_bytes + std::max(pa.bytes, pb.bytes) + 256;

  if (scr.bytes < need) {
    if (scr.p) cudaFree(scr.p);
    scr.p = nullptr;
    scr.bytes = 0;
    FKNN_CUDA(cudaMalloc(&scr.p, need));
    scr.bytes = need;
  }
  const cudaStream_t st = scr.st;
  // device inputs are read in place: whatever the legacy default stream (and
  // the blocking streams it orders) has queued so far comes first
  FKNN_CUDA(cudaEventRecord(scr.ev, 0));
  FKNN_CUDA(cudaStreamWaitEvent(st, scr.ev, 0));
  unsigned char *base = static_cast<unsigned char *>(scr.p);
  const int8_t *d_codes = codes_dev ? reinterpret_cast<const int8_t *>(codes_in) : reinterpret_cast<int8_t *>(base);
  base += b_codes;
  const int8_t *d_q = q_dev ? queries_in : reinterpret_cast<int8_t *>(base);
  base += b_q;
  int *d_ids = ids_dev ? closest : reinterpret_cast<int *>(base);
  base += b_ids;
  float *d_d = !dists ? nullptr : d_dev ? dists : reinterpret_cast<float *>(base);
  base += b_d;
  if (!codes_dev)
    FKNN_CUDA(cudaMemcpyAsync(const_cast<int8_t *>(d_codes), codes_in, npoints * SQ8_CODE, cudaMemcpyDefault, st));
  if (!q_dev)
    FKNN_CUDA(cudaMemcpyAsync(const_cast<int8_t *>(d_q), queries_in, nqueries * SQ8_CODE, cudaMemcpyDefault, st));
  unsigned char *ctiles = base;
  int *cncc = reinterpret_cast<int *>(base + al256((size_t)nct_all * SQ_TILE));
  unsigned char *pass_base = base + codes_bytes;
  int *d_err = reinterpret_cast<int *>(base + codes_bytes + std::max(pa.bytes, pb.bytes));

  const size_t rsmem = (size_t)SQ_WARPS * sq_region(K) * sizeof(HeapNode);
  FKNN_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
  // |c|^2 of every code (the replay kernels use it too) and the tiles
  k_sq8_tiles<<<nct_all, 256, 0, st>>>(d_codes, npoints, 0, 0, ctiles, cncc);
  g_launches += 2;
  for (uint32_t q0 = 0; q0 < nq; q0 += qbatch) {
    const uint32_t nqb = std::min(qbatch, nq - q0);
    const Sq8Pass ps = sq8_pass(nqb, std::max(nct, 1u), k, num_sms);
    size_t off = 0;
    auto take = [&](size_t b) {
      unsigned char *p = pass_base + off;
      off += al256(b);
      return p;
    };
    unsigned char *qtiles = take((size_t)ps.nqt * SQ_TILE);
    int *qncc = reinterpret_cast<int *>(take((size_t)ps.nqt * TC_ROWS * 4));
    HeapNode *heaps = reinterpret_cast<HeapNode *>(take((size_t)nqb * (k + 1) * sizeof(HeapNode)));
    int *T = reinterpret_cast<int *>(take((size_t)nqb * 4));
    int2 *cand = reinterpret_cast<int2 *>(take((size_t)nqb * ps.nseg * ps.cap * sizeof(int2)));
    uint32_t *counts = reinterpret_cast<uint32_t *>(take((size_t)nqb * ps.nseg * 4));
    uint32_t *mark = reinterpret_cast<uint32_t *>(take((size_t)nqb * 4));
    const int8_t *qs = d_q + (uint64_t)q0 * SQ8_CODE;
    int *ids = d_ids + (uint64_t)q0 * k;
    float *dd = d_d ? d_d + (uint64_t)q0 * k : nullptr;
    const unsigned rblocks = (nqb + SQ_WARPS - 1) / SQ_WARPS;
    k_sq8_prefix<<<rblocks, SQ_WARPS * 32, rsmem, st>>>(d_codes, cncc, prefix, qs, nqb, K, screened ? 0 : 1, heaps,
                                                        T, ids, dd, alpha);
    g_launches += 1;
    if (screened) {
      FKNN_CUDA(cudaMemsetAsync(mark, 0, (size_t)nqb * 4, st));
      k_sq8_tiles<<<ps.nqt, 256, 0, st>>>(qs, nqb, 0, 1, qtiles, qncc);
      k_sq8_screen<<<dim3(ps.nqt, ps.nseg), SQ_THREADS, sizeof(SqScreenSmem), st>>>(
          qtiles, qncc, nqb, ctiles + (size_t)(SQ_PREFIX / TC_ROWS) * SQ_TILE, cncc + SQ_PREFIX, nct, ps.tps, ps.nseg,
          SQ_PREFIX, npoints, T, cand, ps.cap, counts, mark, d_err);
      k_sq8_tail<<<rblocks, SQ_WARPS * 32, rsmem, st>>>(d_codes, cncc, SQ_PREFIX, npoints, qs, nqb, K, heaps, cand,
                                                        ps.cap, counts, ps.nseg, mark, ids, dd, alpha);
      g_launches += 3;
    }
    FKNN_CUDA(cudaGetLastError());
  }
  // the kernels finish before any copy to (pageable) host memory is queued,
  // so those copies do not wait on the GPU inside the driver's copy path,
  // where concurrent callers' copies would queue behind them
  FKNN_CUDA(cudaStreamSynchronize(st));
  if (!ids_dev) FKNN_CUDA(cudaMemcpyAsync(closest, d_ids, nqueries * k * 4, cudaMemcpyDeviceToHost, st));
  if (dists && !d_dev) FKNN_CUDA(cudaMemcpyAsync(dists, d_d, nqueries * k * 4, cudaMemcpyDeviceToHost, st));
  int err = 0;
  FKNN_CUDA(cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  if (err & ERR_WAIT_TIMEOUT) {
    // outputs are complete (the affected queries took the exact scan)
    set_error("fknn_sq8_bruteforce: a bounded device wait gave up; affected queries were answered by the exact scan");
    return FKNN_ETIMEOUT;
  }
  return FKNN_OK;
}

}  // namespace

void launch_sq8_encode(const float *d_x, uint64_t n, float alpha, int8_t *d_codes, cudaStream_t st) {
  k_sq8_encode<<<148 * 8, 256, 0, st>>>(d_x, n, alpha, d_codes);
  g_launches += 1;
}

}  // namespace fknn

using namespace fknn;

extern "C" {

int fknn_sq8_sym_train(const float *vecs, uint64_t n, float *alpha, int8_t *codes) {
  g_launches = 0;
  if (!alpha) {
    set_error("fknn_sq8_sym_train: alpha is NULL");
    return FKNN_EINVAL;
  }
  return sq8_encode_impl(vecs, n, 0.f, codes, true, alpha);
}

int fknn_sq8_sym_encode(const float *vecs, uint64_t n, float alpha, int8_t *codes) {
  g_launches = 0;
  return sq8_encode_impl(vecs, n, alpha, codes, false, nullptr);
}

int fknn_sq8_bruteforce(size_t dim, size_t k, int *closest_points, size_t npoints, const char *codes_in, float alpha,
                        size_t nqueries, const int8_t *queries_in) {
  (void)dim;
  g_launches = 0;
  return sq8_bf_impl(k, closest_points, nullptr, npoints, codes_in, alpha, nqueries, queries_in);
}

int fknn_sq8_bruteforce_subgraph(size_t dim, size_t k, int *closest_points, float *distances, size_t npoints,
                                 const char *codes_in, float alpha, size_t nqueries, const int8_t *queries_in) {
  (void)dim;
  g_launches = 0;
  if (!distances) {
    set_error("fknn_sq8_bruteforce_subgraph: distances is NULL");
    return FKNN_EINVAL;
  }
  return sq8_bf_impl(k, closest_points, distances, npoints, codes_in, alpha, nqueries, queries_in);
}

int fknn_sq8_release_thread_scratch(void) {
  // the thread's stream has no work left: every SQ8 call waits for it
  sq8_scratch().release();
  return FKNN_OK;
}

}  // extern "C"
